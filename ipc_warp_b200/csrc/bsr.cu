// 3x3-block CSR assembly from triplets (the contract of warp.sparse
// bsr_from_triplets as used at dynamic_contacts.py:290-297 and
// time_integrator_base.py:413-426): key = (row, col), device radix sort,
// segment heads, prefix sum, then one thread per unique block sums its
// segment in sorted (= input) order, so the result is deterministic.
#include "common.cuh"
#include "sort.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr int kScanBlock = 1024;

inline int bits_for(int v) {  // bits to represent 0..v
  int b = 1;
  while ((1LL << b) <= (long long)v) ++b;
  return b;
}
inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

// Triplets with an all-zero block or an index outside the matrix get the
// sentinel key (sorted last, dropped).
template <class S>
__global__ void k_keys(int n, const int* __restrict__ rows, const int* __restrict__ cols, const S* __restrict__ vals,
                       int nrow, int ncol, int colbits, unsigned long long sentinel,
                       unsigned long long* __restrict__ keys, int* __restrict__ idx) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  bool nz = false;
#pragma unroll
  for (int k = 0; k < 9; ++k) nz |= vals[9LL * t + k] != S(0);
  int r = rows[t], c = cols[t];
  bool inside = r >= 0 && r < nrow && c >= 0 && c < ncol;
  keys[t] = (nz && inside) ? (((unsigned long long)r << colbits) | (unsigned long long)c) : sentinel;
  idx[t] = t;
}

// heads[t] = 1 at the first element of each non-sentinel key run
__global__ void k_heads(int n, const unsigned long long* __restrict__ keys, unsigned long long sentinel,
                        int* __restrict__ heads) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  unsigned long long k = keys[t];
  heads[t] = (k != sentinel && (t == 0 || keys[t - 1] != k)) ? 1 : 0;
}

// block-local exclusive scan; block totals to sums[]
__global__ void __launch_bounds__(kScanBlock) k_scan_local(int n, int* __restrict__ a, unsigned* __restrict__ sums) {
  __shared__ int s[kScanBlock / 32];
  int t = blockIdx.x * kScanBlock + threadIdx.x;
  int v = t < n ? a[t] : 0;
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = s[lane];
    for (int o = 1; o < 32; o <<= 1) {
      int z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    s[lane] = y;
  }
  __syncthreads();
  int excl = x - v + (w > 0 ? s[w - 1] : 0);
  if (t < n) a[t] = excl;
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = (unsigned)(excl + v);
}

__global__ void k_scan_add(int n, int* __restrict__ a, const unsigned* __restrict__ sums) {
  int t = blockIdx.x * kScanBlock + threadIdx.x;
  if (t < n) a[t] += (int)sums[blockIdx.x];
}

__global__ void k_segments(int n, const unsigned long long* __restrict__ keys, unsigned long long sentinel,
                           const int* __restrict__ heads_scanned, int colbits, int* __restrict__ seg_start,
                           int* __restrict__ seg_row, int* __restrict__ columns, int* __restrict__ nnz) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  unsigned long long k = keys[t];
  bool head = k != sentinel && (t == 0 || keys[t - 1] != k);
  int u = heads_scanned[t];
  if (head) {
    seg_start[u] = t;
    seg_row[u] = (int)(k >> colbits);
    columns[u] = (int)(k & ((1ULL << colbits) - 1ULL));
  }
  bool last_valid = k != sentinel && (t == n - 1 || keys[t + 1] == sentinel);
  if (last_valid) *nnz = u + 1;
  if (t == 0 && k == sentinel) *nnz = 0;
}

template <class S>
__global__ void k_reduce(int n, const unsigned long long* __restrict__ keys, const int* __restrict__ perm,
                         const int* __restrict__ seg_start, const int* __restrict__ nnz, const S* __restrict__ vals,
                         S* __restrict__ values) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= *nnz) return;
  int t = seg_start[u];
  unsigned long long k = keys[t];
  S acc[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) acc[q] = S(0);
  for (; t < n && keys[t] == k; ++t) {
    const S* v = vals + 9LL * perm[t];
#pragma unroll
    for (int q = 0; q < 9; ++q) acc[q] += v[q];
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) values[9LL * u + q] = acc[q];
}

__global__ void k_offsets(int cap, int nrow, const int* __restrict__ seg_row, const int* __restrict__ nnz,
                          int* __restrict__ offsets) {
  int u = blockIdx.x * blockDim.x + threadIdx.x;
  int m = *nnz;
  if (m == 0) {
    for (int r = u; r <= nrow; r += gridDim.x * blockDim.x) offsets[r] = 0;
    return;
  }
  if (u >= m) return;
  int r = seg_row[u];
  int rp = u == 0 ? -1 : seg_row[u - 1];
  for (int rr = rp + 1; rr <= r; ++rr) offsets[rr] = u;
  if (u == m - 1)
    for (int rr = r + 1; rr <= nrow; ++rr) offsets[rr] = m;
  (void)cap;
}

template <class S>
__global__ void k_bsr_mv(int nrow, const int* __restrict__ off, const int* __restrict__ colsi,
                         const S* __restrict__ val, const S* __restrict__ x, S* __restrict__ y, S alpha, S beta) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrow) return;
  S a0 = 0, a1 = 0, a2 = 0;
  for (int k = off[r]; k < off[r + 1]; ++k) {
    int c = colsi[k];
    const S* b = val + 9LL * k;
    S x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
    a0 += b[0] * x0 + b[1] * x1 + b[2] * x2;
    a1 += b[3] * x0 + b[4] * x1 + b[5] * x2;
    a2 += b[6] * x0 + b[7] * x1 + b[8] * x2;
  }
  if (beta == S(0)) {
    y[3 * r] = alpha * a0;
    y[3 * r + 1] = alpha * a1;
    y[3 * r + 2] = alpha * a2;
  } else {
    y[3 * r] = alpha * a0 + beta * y[3 * r];
    y[3 * r + 1] = alpha * a1 + beta * y[3 * r + 1];
    y[3 * r + 2] = alpha * a2 + beta * y[3 * r + 2];
  }
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

size_t ipcb_bsr_workspace(int n_trip, int nrow, int ncol) {
  (void)nrow;
  (void)ncol;
  size_t n = (size_t)(n_trip > 0 ? n_trip : 1);
  size_t nb = (n + kScanBlock - 1) / kScanBlock;
  return al(n * 8) + al(n * 4) * 4 + al(nb * 4) + 256 + sort::workspace_bytes<unsigned long long>((int)n);
}

int ipcb_bsr_from_triplets(int nrow, int ncol, int n_trip, const int* rows, const int* cols, const void* vals,
                           int fp64, int* offsets, int* columns, void* values, int* nnz, void* ws, size_t ws_bytes,
                           ipcb_stream s) {
  if (nrow < 0 || ncol < 0 || n_trip < 0 || !offsets || !nnz) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (n_trip == 0) {
    cudaMemsetAsync(offsets, 0, (size_t)(nrow + 1) * sizeof(int), st);
    cudaMemsetAsync(nnz, 0, sizeof(int), st);
    return check_launch("ipcb_bsr_from_triplets");
  }
  if (!rows || !cols || !vals || !columns || !values || !ws || ws_bytes < ipcb_bsr_workspace(n_trip, nrow, ncol))
    return IPCB_E_ARG;
  int colbits = bits_for(ncol > 0 ? ncol - 1 : 0);
  int rowbits = bits_for(nrow);
  if (colbits + rowbits > 62) return IPCB_E_ARG;
  unsigned long long sentinel = (unsigned long long)nrow << colbits;
  size_t n = (size_t)n_trip, nb = (n + kScanBlock - 1) / kScanBlock;
  char* p = (char*)ws;
  unsigned long long* keys = (unsigned long long*)p; p += al(n * 8);
  int* perm = (int*)p; p += al(n * 4);
  int* heads = (int*)p; p += al(n * 4);
  int* seg_start = (int*)p; p += al(n * 4);
  int* seg_row = (int*)p; p += al(n * 4);
  unsigned* sums = (unsigned*)p; p += al(nb * 4);
  p += 256;
  void* sws = p;
  size_t sws_bytes = ws_bytes - (size_t)(p - (char*)ws);
  int g = div_up(n_trip, 256);
  if (fp64)
    k_keys<double><<<g, 256, 0, st>>>(n_trip, rows, cols, (const double*)vals, nrow, ncol, colbits, sentinel, keys, perm);
  else
    k_keys<float><<<g, 256, 0, st>>>(n_trip, rows, cols, (const float*)vals, nrow, ncol, colbits, sentinel, keys, perm);
  sort::sort_pairs<unsigned long long>(keys, perm, n_trip, colbits + rowbits, sws, sws_bytes, st);
  k_heads<<<g, 256, 0, st>>>(n_trip, keys, sentinel, heads);
  k_scan_local<<<(int)nb, kScanBlock, 0, st>>>(n_trip, heads, sums);
  if (nb > 1) {
    sort::k_scan<<<1, 1024, 0, st>>>(sums, (int)nb);
    k_scan_add<<<(int)nb, kScanBlock, 0, st>>>(n_trip, heads, sums);
  }
  k_segments<<<g, 256, 0, st>>>(n_trip, keys, sentinel, heads, colbits, seg_start, seg_row, columns, nnz);
  if (fp64)
    k_reduce<double><<<g, 256, 0, st>>>(n_trip, keys, perm, seg_start, nnz, (const double*)vals, (double*)values);
  else
    k_reduce<float><<<g, 256, 0, st>>>(n_trip, keys, perm, seg_start, nnz, (const float*)vals, (float*)values);
  k_offsets<<<g, 256, 0, st>>>(n_trip, nrow, seg_row, nnz, offsets);
  return check_launch("ipcb_bsr_from_triplets");
}

int ipcb_bsr_mv(int nrow, const int* offsets, const int* columns, const void* values, int fp64, const void* x,
                void* y, double alpha, double beta, ipcb_stream s) {
  if (nrow < 0 || !offsets || !x || !y) return IPCB_E_ARG;
  if (nrow == 0) return IPCB_OK;
  int g = div_up(nrow, 128);
  if (fp64)
    k_bsr_mv<double><<<g, 128, 0, (cudaStream_t)s>>>(nrow, offsets, columns, (const double*)values,
                                                     (const double*)x, (double*)y, alpha, beta);
  else
    k_bsr_mv<float><<<g, 128, 0, (cudaStream_t)s>>>(nrow, offsets, columns, (const float*)values, (const float*)x,
                                                    (float*)y, (float)alpha, (float)beta);
  return check_launch("ipcb_bsr_mv");
}

}  // extern "C"
