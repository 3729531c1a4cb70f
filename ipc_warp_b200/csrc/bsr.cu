// 3x3-block CSR assembly from triplets (the contract of warp.sparse
// bsr_from_triplets as used at dynamic_contacts.py:290-297 and
// time_integrator_base.py:413-426).
//
// Row buckets instead of a global (row, col) key sort:
//   1. count valid triplets per row (atomics), exclusive scan -> row starts
//   2. scatter triplet ids into their row bucket
//   3. one warp per row: rank its entries by (col, triplet id) -- the id
//      breaks ties, so duplicates are summed in input order and the result is
//      deterministic -- and count the distinct columns
//   4. scan the per-row distinct counts -> offsets, nnz
//   5. one warp per row: write sorted columns and the summed 3x3 blocks
// Triplets whose block is all zero or whose index is outside the matrix are
// dropped (warp's prune_numerical_zeros behaviour for the former).
#include "common.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr int kScanBlock = 1024;
constexpr int kWarpsPerBlock = 8;

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

template <class S>
IPCB_D bool valid_triplet(int t, const int* __restrict__ rows, const int* __restrict__ cols,
                          const S* __restrict__ vals, int nrow, int ncol) {
  int r = rows[t], c = cols[t];
  if (r < 0 || r >= nrow || c < 0 || c >= ncol) return false;
  bool nz = false;
#pragma unroll
  for (int k = 0; k < 9; ++k) nz |= vals[9LL * t + k] != S(0);
  return nz;
}

template <class S>
__global__ void k_row_count(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                            const S* __restrict__ vals, int nrow, int ncol, int* __restrict__ row_cnt) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (valid_triplet(t, rows, cols, vals, nrow, ncol)) atomicAdd(row_cnt + rows[t], 1);
}

// Exclusive scan, phase 1: per-block scan in place, block totals to sums.
__global__ void __launch_bounds__(kScanBlock) k_scan_local(int n, int* __restrict__ a, int* __restrict__ sums) {
  __shared__ int s[kScanBlock / 32];
  int t = blockIdx.x * kScanBlock + threadIdx.x;
  int v = t < n ? a[t] : 0;
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s[w] = x;
  __syncthreads();
  if (w == 0) {
    int y = s[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int z = __shfl_up_sync(0xffffffffu, y, o);
      if (lane >= o) y += z;
    }
    s[lane] = y;
  }
  __syncthreads();
  int excl = x - v + (w > 0 ? s[w - 1] : 0);
  if (t < n) a[t] = excl;
  if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = excl + v;
}

// phase 2: exclusive scan of the block totals (one block, looping)
__global__ void __launch_bounds__(kScanBlock) k_scan_sums(int nb, int* __restrict__ sums, int* __restrict__ total) {
  __shared__ int s[kScanBlock / 32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nb; base += kScanBlock) {
    int t = base + threadIdx.x;
    int v = t < nb ? sums[t] : 0;
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s[w] = x;
    __syncthreads();
    if (w == 0) {
      int y = s[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int z = __shfl_up_sync(0xffffffffu, y, o);
        if (lane >= o) y += z;
      }
      s[lane] = y;
    }
    __syncthreads();
    int excl = x - v + (w > 0 ? s[w - 1] : 0) + carry;
    if (t < nb) sums[t] = excl;
    __syncthreads();
    if (threadIdx.x == kScanBlock - 1) carry = excl + v;
    __syncthreads();
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

// phase 3: add the scanned block totals
__global__ void k_scan_add(int n, int* __restrict__ a, const int* __restrict__ sums) {
  int t = blockIdx.x * kScanBlock + threadIdx.x;
  if (t < n) a[t] += sums[blockIdx.x];
}

// exclusive scan of a[0..n) in place; *total = sum (device)
void exclusive_scan(int* a, int n, int* sums, int* total, cudaStream_t st) {
  int nb = div_up(n, kScanBlock);
  k_scan_local<<<nb, kScanBlock, 0, st>>>(n, a, sums);
  k_scan_sums<<<1, kScanBlock, 0, st>>>(nb, sums, total);
  k_scan_add<<<nb, kScanBlock, 0, st>>>(n, a, sums);
}

template <class S>
__global__ void k_row_scatter(int n, const int* __restrict__ rows, const int* __restrict__ cols,
                              const S* __restrict__ vals, int nrow, int ncol, const int* __restrict__ row_start,
                              int* __restrict__ cursor, int* __restrict__ bucket) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (!valid_triplet(t, rows, cols, vals, nrow, ncol)) return;
  int r = rows[t];
  int pos = row_start[r] + atomicAdd(cursor + r, 1);
  bucket[pos] = t;
}

// (col, id) as one 64-bit ordering key
IPCB_D unsigned long long ckey(const int* __restrict__ cols, int t) {
  return ((unsigned long long)(unsigned)cols[t] << 32) | (unsigned)t;
}

constexpr int kRowCap = 256;  // entries a warp ranks from shared memory

// Warp per row: sort the row's bucket by (col, id) by ranking (rank = number
// of smaller keys; keys are distinct because ids are) and count the distinct
// columns.  Rows longer than kRowCap rank from global memory.
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_row_sort(int nrow, const int* __restrict__ cols,
                                                                  const int* __restrict__ row_start,
                                                                  int* __restrict__ bucket, int* __restrict__ tmp,
                                                                  int* __restrict__ row_nnz) {
  __shared__ unsigned long long sk[kWarpsPerBlock][kRowCap];
  const int wib = threadIdx.x >> 5;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nrow) return;
  int b = row_start[warp], e = row_start[warp + 1], L = e - b;
  if (L <= kRowCap) {
    for (int i = lane; i < L; i += 32) sk[wib][i] = ckey(cols, bucket[b + i]);
    __syncwarp();
    for (int i = lane; i < L; i += 32) {
      unsigned long long ki = sk[wib][i];
      int rank = 0;
      for (int j = 0; j < L; ++j) rank += sk[wib][j] < ki;
      tmp[b + rank] = (int)(unsigned)(ki & 0xffffffffULL);
    }
  } else {
    for (int i = lane; i < L; i += 32) {
      unsigned long long ki = ckey(cols, bucket[b + i]);
      int rank = 0;
      for (int j = 0; j < L; ++j) rank += ckey(cols, bucket[b + j]) < ki;
      tmp[b + rank] = bucket[b + i];
    }
  }
  __syncwarp();
  int distinct = 0;
  for (int i = lane; i < L; i += 32) {
    int t = tmp[b + i];
    bucket[b + i] = t;
    distinct += (i == 0 || cols[tmp[b + i - 1]] != cols[t]) ? 1 : 0;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) distinct += __shfl_xor_sync(0xffffffffu, distinct, o);
  if (lane == 0) row_nnz[warp] = distinct;
}

// Warp per row over the sorted bucket: the first entry of each run of equal
// columns sums the run in order (deterministic) and writes one block; the
// run's output slot is the number of run heads before it (ballot prefix).
template <class S>
__global__ void __launch_bounds__(kWarpsPerBlock * 32) k_row_emit(int nrow, const int* __restrict__ cols,
                                                                  const S* __restrict__ vals,
                                                                  const int* __restrict__ row_start,
                                                                  const int* __restrict__ bucket,
                                                                  const int* __restrict__ offsets,
                                                                  int* __restrict__ columns, S* __restrict__ values) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nrow) return;
  int b = row_start[warp], e = row_start[warp + 1], L = e - b;
  int out = offsets[warp];
  const unsigned le = 0xffffffffu >> (31 - lane);
  int carry = 0;
  for (int base = 0; base < L; base += 32) {
    int i = base + lane;
    bool in = i < L;
    int t = in ? bucket[b + i] : 0;
    int c = in ? cols[t] : 0;
    bool head = in && (i == 0 || cols[bucket[b + i - 1]] != c);
    unsigned m = __ballot_sync(0xffffffffu, head);
    if (head) {
      int u = carry + __popc(m & le) - 1;
      S acc[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) acc[q] = S(0);
      for (int j = i; j < L; ++j) {
        int tj = bucket[b + j];
        if (cols[tj] != c) break;
        const S* v = vals + 9LL * tj;
#pragma unroll
        for (int q = 0; q < 9; ++q) acc[q] += v[q];
      }
      columns[out + u] = c;
#pragma unroll
      for (int q = 0; q < 9; ++q) values[9LL * (out + u) + q] = acc[q];
    }
    carry += __popc(m);
  }
}

__global__ void k_finish_offsets(int nrow, int* __restrict__ offsets, const int* __restrict__ total,
                                 int* __restrict__ nnz) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    offsets[nrow] = *total;
    *nnz = *total;
  }
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

template <class S>
int assemble(int nrow, int ncol, int n, const int* rows, const int* cols, const S* vals, int* offsets, int* columns,
             S* values, int* nnz, void* ws, cudaStream_t st) {
  size_t R = (size_t)nrow + 1, N = (size_t)n;
  size_t nbr = (size_t)div_up((int)R, kScanBlock);
  char* p = (char*)ws;
  int* row_start = (int*)p; p += al(R * 4);
  int* cursor = (int*)p; p += al(R * 4);
  int* sums = (int*)p; p += al((nbr + 1) * 4);
  int* total = (int*)p; p += 256;
  int* bucket = (int*)p; p += al(N * 4);
  int* tmp = (int*)p;
  cudaMemsetAsync(row_start, 0, R * sizeof(int), st);
  cudaMemsetAsync(cursor, 0, R * sizeof(int), st);
  int g = div_up(n, 256);
  k_row_count<S><<<g, 256, 0, st>>>(n, rows, cols, vals, nrow, ncol, row_start);
  exclusive_scan(row_start, (int)R, sums, total, st);  // row_start[nrow] = valid count
  k_row_scatter<S><<<g, 256, 0, st>>>(n, rows, cols, vals, nrow, ncol, row_start, cursor, bucket);
  int gw = div_up(nrow, kWarpsPerBlock);
  k_row_sort<<<gw, kWarpsPerBlock * 32, 0, st>>>(nrow, cols, row_start, bucket, tmp, offsets);
  exclusive_scan(offsets, nrow, sums, total, st);
  k_finish_offsets<<<1, 32, 0, st>>>(nrow, offsets, total, nnz);
  k_row_emit<S><<<gw, kWarpsPerBlock * 32, 0, st>>>(nrow, cols, vals, row_start, bucket, offsets, columns, values);
  return check_launch("ipcb_bsr_from_triplets");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

size_t ipcb_bsr_workspace(int n_trip, int nrow, int ncol) {
  (void)ncol;
  size_t R = (size_t)(nrow > 0 ? nrow : 0) + 1, N = (size_t)(n_trip > 0 ? n_trip : 1);
  size_t nbr = (R + kScanBlock - 1) / kScanBlock;
  return 2 * al(R * 4) + al((nbr + 1) * 4) + 256 + 2 * al(N * 4);
}

int ipcb_bsr_from_triplets(int nrow, int ncol, int n_trip, const int* rows, const int* cols, const void* vals,
                           int fp64, int* offsets, int* columns, void* values, int* nnz, void* ws, size_t ws_bytes,
                           ipcb_stream s) {
  if (nrow < 0 || ncol < 0 || n_trip < 0 || !offsets || !nnz) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (n_trip == 0 || nrow == 0) {
    cudaMemsetAsync(offsets, 0, (size_t)(nrow + 1) * sizeof(int), st);
    cudaMemsetAsync(nnz, 0, sizeof(int), st);
    return check_launch("ipcb_bsr_from_triplets");
  }
  if (!rows || !cols || !vals || !columns || !values || !ws || ws_bytes < ipcb_bsr_workspace(n_trip, nrow, ncol))
    return IPCB_E_ARG;
  if (fp64)
    return assemble<double>(nrow, ncol, n_trip, rows, cols, (const double*)vals, offsets, columns, (double*)values,
                            nnz, ws, st);
  return assemble<float>(nrow, ncol, n_trip, rows, cols, (const float*)vals, offsets, columns, (float*)values, nnz,
                         ws, st);
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
