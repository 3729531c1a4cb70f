// 3x3-block CSR assembly from triplets (the contract of warp.sparse
// bsr_from_triplets as used at dynamic_contacts.py:290-297 and
// time_integrator_base.py:413-426).
//
// Row buckets instead of a global (row, col) key sort:
//   1. count valid triplets per row (atomics), exclusive scan -> row starts
//   2. scatter triplet ids into their row bucket
//   3. one warp per row: bitonic-sort its entries by (col, triplet id) in
//      shared memory -- the id breaks ties, so the order, and with it every
//      sum, is fixed by the input -- and count the distinct columns
//   4. scan the per-row distinct counts -> offsets, nnz
//   5. one warp per row: segmented reduction over the sorted entries, one
//      3x3 block per distinct column
// Rows longer than a warp's shared-memory sort (the 12 DOF rows of an affine
// body collect every contact of the body: 1e4..1e5 entries) are listed by
// step 3 and handled by one 1024-thread CTA each: a bitonic sort whose
// stages below 4096 run on shared-memory chunks and whose longer strides
// run in global memory, and an emit step whose 32 warps take equal slices of
// the row (a warp owns the runs whose first entry lies in its slice).
// Triplets whose block is all zero or whose index is outside the matrix are
// dropped (warp's prune_numerical_zeros behaviour for the former).
#include "common.cuh"
#include "scan.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

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

constexpr int kRowCap = 1024;      // entries a warp sorts in shared memory
constexpr int kSortWarps = 4;      // warps (rows) per block in k_row_sort

// Warp per row: sort the row's bucket by (col, id), keys distinct, then count
// distinct columns.  Rows up to kRowCap entries use a bitonic network in
// shared memory; longer rows are appended to long_rows for k_row_sort_long.
__global__ void __launch_bounds__(kSortWarps * 32) k_row_sort(int nrow, const int* __restrict__ cols,
                                                              const int* __restrict__ row_start,
                                                              int* __restrict__ bucket, int* __restrict__ tmp,
                                                              int* __restrict__ row_nnz, int* __restrict__ long_rows,
                                                              int* __restrict__ n_long) {
  __shared__ unsigned long long sk[kSortWarps][kRowCap];
  const int wib = threadIdx.x >> 5;
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nrow) return;
  int b = row_start[warp], e = row_start[warp + 1], L = e - b;
  if (L <= kRowCap) {
    int P = 1;
    while (P < L) P <<= 1;
    unsigned long long* k = sk[wib];
    for (int i = lane; i < P; i += 32) k[i] = i < L ? ckey(cols, bucket[b + i]) : ~0ULL;
    __syncwarp();
    for (int sz = 2; sz <= P; sz <<= 1) {
      for (int st = sz >> 1; st > 0; st >>= 1) {
        for (int i = lane; i < P; i += 32) {
          int l = i ^ st;
          if (l > i) {
            unsigned long long a = k[i], c = k[l];
            bool up = (i & sz) == 0;
            if ((a > c) == up) {
              k[i] = c;
              k[l] = a;
            }
          }
        }
        __syncwarp();
      }
    }
    for (int i = lane; i < L; i += 32) tmp[b + i] = (int)(unsigned)(k[i] & 0xffffffffULL);
  } else {  // a long row: sorted and counted by k_row_sort_long
    if (lane == 0) {
      long_rows[atomicAdd(n_long, 1)] = warp;
      row_nnz[warp] = 0;
    }
    return;
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

// Warp per row over the sorted bucket, 32 entries at a time: a segmented
// inclusive scan (segments = runs of equal column) of the 9 block values;
// the last entry of each run writes the block.  A run that crosses a chunk
// boundary is carried into the next chunk.  The combination order is fixed
// by the sorted order, so results are deterministic.
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
  if (L > kRowCap) return;  // k_row_emit_long
  int out = offsets[warp];
  const unsigned le = 0xffffffffu >> (31 - lane);
  int runs_before = 0;  // heads in earlier chunks
  int prev_col = -1;    // column of the last entry of the previous chunk
  S carry[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) carry[q] = S(0);
  for (int base = 0; base < L; base += 32) {
    int i = base + lane;
    bool in = i < L;
    int t = in ? bucket[b + i] : 0;
    int c = in ? cols[t] : -1;
    int cprev = __shfl_up_sync(0xffffffffu, c, 1);
    if (lane == 0) cprev = prev_col;
    bool head = in && (i == 0 || c != cprev);
    int cnext = __shfl_down_sync(0xffffffffu, c, 1);
    if (lane == 31) cnext = (i + 1 < L) ? cols[bucket[b + i + 1]] : -2;
    bool tail = in && (i == L - 1 || cnext != c);
    S v[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) v[q] = in ? vals[9LL * t + q] : S(0);
    if (lane == 0 && in && !head) {
#pragma unroll
      for (int q = 0; q < 9; ++q) v[q] = carry[q] + v[q];
    }
    int f = head ? 1 : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int nf = __shfl_up_sync(0xffffffffu, f, o);
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        S nv = __shfl_up_sync(0xffffffffu, v[q], o);
        if (lane >= o && !f) v[q] = nv + v[q];
      }
      if (lane >= o) f |= nf;
    }
    unsigned hm = __ballot_sync(0xffffffffu, head);
    int u = runs_before + __popc(hm & le) - 1;
    if (tail) {
      columns[out + u] = c;
#pragma unroll
      for (int q = 0; q < 9; ++q) values[9LL * (out + u) + q] = v[q];
    }
#pragma unroll
    for (int q = 0; q < 9; ++q) carry[q] = __shfl_sync(0xffffffffu, v[q], 31);
    prev_col = __shfl_sync(0xffffffffu, c, 31);
    runs_before += __popc(hm);
  }
}

constexpr int kLongThreads = 1024;
constexpr int kLongChunk = 4096;  // keys a CTA sorts in shared memory (32 KB)
constexpr int kLongGrid = 148;    // CTAs over the long-row list (one per SM)

IPCB_D void cas(unsigned long long* k, int i, int l, bool up) {
  const unsigned long long a = k[i], c = k[l];
  if ((a > c) == up) {
    k[i] = c;
    k[l] = a;
  }
}

// the stages of stride < C of the bitonic merge sizes sz_lo..sz_hi, on each
// C-key chunk of the row in shared memory (C = min(P, kLongChunk))
IPCB_D void chunk_stages(unsigned long long* __restrict__ g, unsigned long long* __restrict__ sk, int P, int C,
                         int sz_lo, int sz_hi) {
  for (int c0 = 0; c0 < P; c0 += C) {
    for (int i = threadIdx.x; i < C; i += kLongThreads) sk[i] = g[c0 + i];
    __syncthreads();
    for (int sz = sz_lo; sz <= sz_hi; sz <<= 1) {
      for (int st = min(sz, C) >> 1; st > 0; st >>= 1) {
        for (int i = threadIdx.x; i < C; i += kLongThreads) {
          const int l = i ^ st;
          if (l > i) cas(sk, i, l, ((c0 + i) & sz) == 0);
        }
        __syncthreads();
      }
    }
    for (int i = threadIdx.x; i < C; i += kLongThreads) g[c0 + i] = sk[i];
    __syncthreads();
  }
}

// One CTA per long row (grid-stride over the list): bitonic sort of the
// (col, id) keys padded to the power of two P >= L in lkeys (the row's region
// [2 b, 2 b + P) lies inside [2 b, 2 b + 2 L), its own), then the sorted ids
// back into the bucket and the distinct-column count into row_nnz.
__global__ void __launch_bounds__(kLongThreads) k_row_sort_long(const int* __restrict__ long_rows,
                                                                const int* __restrict__ n_long,
                                                                const int* __restrict__ cols,
                                                                const int* __restrict__ row_start,
                                                                int* __restrict__ bucket,
                                                                unsigned long long* __restrict__ lkeys,
                                                                int* __restrict__ row_nnz) {
  __shared__ unsigned long long sk[kLongChunk];
  __shared__ int s_distinct;
  const int n = *n_long;
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    const int r = long_rows[li];
    const int b = row_start[r], L = row_start[r + 1] - b;
    int P = 1;
    while (P < L) P <<= 1;
    const int C = P < kLongChunk ? P : kLongChunk;
    unsigned long long* g = lkeys + 2LL * b;
    for (int i = threadIdx.x; i < P; i += kLongThreads) g[i] = i < L ? ckey(cols, bucket[b + i]) : ~0ULL;
    if (threadIdx.x == 0) s_distinct = 0;
    __syncthreads();
    chunk_stages(g, sk, P, C, 2, C);
    for (int sz = 2 * C; sz <= P; sz <<= 1) {
      for (int st = sz >> 1; st >= C; st >>= 1) {
        for (int i = threadIdx.x; i < P; i += kLongThreads) {
          const int l = i ^ st;
          if (l > i) cas(g, i, l, (i & sz) == 0);
        }
        __syncthreads();
      }
      chunk_stages(g, sk, P, C, sz, sz);
    }
    int d = 0;
    for (int i = threadIdx.x; i < L; i += kLongThreads) {
      const unsigned long long k = g[i];
      bucket[b + i] = (int)(unsigned)(k & 0xffffffffULL);
      d += (i == 0 || (g[i - 1] >> 32) != (k >> 32)) ? 1 : 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    if ((threadIdx.x & 31) == 0 && d) atomicAdd(&s_distinct, d);
    __syncthreads();
    if (threadIdx.x == 0) row_nnz[r] = s_distinct;
    __syncthreads();
  }
}

// One CTA per long row: warp w owns the runs whose first entry lies in its
// slice [w L / 32, (w + 1) L / 32) and reduces them with the same segmented
// scan as k_row_emit, reading past its slice end to finish its last run; a
// block scan of the warps' run counts gives each warp's output position.
template <class S>
__global__ void __launch_bounds__(kLongThreads) k_row_emit_long(const int* __restrict__ long_rows,
                                                                const int* __restrict__ n_long,
                                                                const int* __restrict__ cols,
                                                                const S* __restrict__ vals,
                                                                const int* __restrict__ row_start,
                                                                const int* __restrict__ bucket,
                                                                const int* __restrict__ offsets,
                                                                int* __restrict__ columns, S* __restrict__ values) {
  __shared__ int s_runs[kLongThreads / 32];
  const int n = *n_long;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nw = kLongThreads / 32;
  for (int li = blockIdx.x; li < n; li += gridDim.x) {
    const int r = long_rows[li];
    const int b = row_start[r], L = row_start[r + 1] - b;
    auto col_at = [&](int i) { return cols[bucket[b + i]]; };
    auto is_head = [&](int i) { return i == 0 || col_at(i) != col_at(i - 1); };
    // first head at or after the slice start (warp-parallel search)
    auto first_head = [&](int from) {
      for (int base = from; base < L; base += 32) {
        const int i = base + lane;
        const unsigned m = __ballot_sync(0xffffffffu, i < L && is_head(i));
        if (m) return base + __ffs(m) - 1;
      }
      return L;
    };
    const int s0 = (int)((long long)L * w / nw), s1 = (int)((long long)L * (w + 1) / nw);
    const int start = first_head(s0);
    const int end = s1 >= L ? L : first_head(s1);
    int heads = 0;
    for (int base = start; base < end; base += 32) {
      const int i = base + lane;
      heads += __popc(__ballot_sync(0xffffffffu, i < end && is_head(i)));
    }
    if (lane == 0) s_runs[w] = heads;
    __syncthreads();
    int runs_before = 0;
    for (int k = 0; k < w; ++k) runs_before += s_runs[k];
    __syncthreads();
    const int out = offsets[r];
    const unsigned le = 0xffffffffu >> (31 - lane);
    int prev_col = -1;
    S carry[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) carry[q] = S(0);
    for (int base = start; base < end; base += 32) {
      const int i = base + lane;
      const bool in = i < end;
      const int t = in ? bucket[b + i] : 0;
      const int c = in ? cols[t] : -1;
      int cprev = __shfl_up_sync(0xffffffffu, c, 1);
      if (lane == 0) cprev = base == start ? -1 : prev_col;
      const bool head = in && (i == start || c != cprev);
      int cnext = __shfl_down_sync(0xffffffffu, c, 1);
      if (lane == 31) cnext = (i + 1 < end) ? cols[bucket[b + i + 1]] : -2;
      const bool tail = in && (i == end - 1 || cnext != c);
      S v[9];
#pragma unroll
      for (int q = 0; q < 9; ++q) v[q] = in ? vals[9LL * t + q] : S(0);
      if (lane == 0 && in && !head) {
#pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = carry[q] + v[q];
      }
      int f = head ? 1 : 0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int nf = __shfl_up_sync(0xffffffffu, f, o);
#pragma unroll
        for (int q = 0; q < 9; ++q) {
          const S nv = __shfl_up_sync(0xffffffffu, v[q], o);
          if (lane >= o && !f) v[q] = nv + v[q];
        }
        if (lane >= o) f |= nf;
      }
      const unsigned hm = __ballot_sync(0xffffffffu, head);
      const int u = runs_before + __popc(hm & le) - 1;
      if (tail) {
        columns[out + u] = c;
#pragma unroll
        for (int q = 0; q < 9; ++q) values[9LL * (out + u) + q] = v[q];
      }
#pragma unroll
      for (int q = 0; q < 9; ++q) carry[q] = __shfl_sync(0xffffffffu, v[q], 31);
      prev_col = __shfl_sync(0xffffffffu, c, 31);
      runs_before += __popc(hm);
    }
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
  char* p = (char*)ws;
  int* row_start = (int*)p; p += al(R * 4);
  int* cursor = (int*)p; p += al(R * 4);
  int* total = (int*)p; p += 256;
  int* bucket = (int*)p; p += al(N * 4);
  int* tmp = (int*)p; p += al(N * 4);
  int* long_rows = (int*)p; p += al(R * 4);
  int* n_long = (int*)p; p += 256;
  unsigned long long* lkeys = (unsigned long long*)p; p += al(2 * N * 8);
  void* scratch = p;
  cudaMemsetAsync(n_long, 0, sizeof(int), st);
  cudaMemsetAsync(row_start, 0, R * sizeof(int), st);
  cudaMemsetAsync(cursor, 0, R * sizeof(int), st);
  int g = div_up(n, 256);
  k_row_count<S><<<g, 256, 0, st>>>(n, rows, cols, vals, nrow, ncol, row_start);
  scan::exclusive<int>(row_start, (int)R, scratch, total, st);  // row_start[nrow] = valid count
  k_row_scatter<S><<<g, 256, 0, st>>>(n, rows, cols, vals, nrow, ncol, row_start, cursor, bucket);
  k_row_sort<<<div_up(nrow, kSortWarps), kSortWarps * 32, 0, st>>>(nrow, cols, row_start, bucket, tmp, offsets,
                                                                     long_rows, n_long);
  const int g_long = nrow < kLongGrid ? nrow : kLongGrid;
  k_row_sort_long<<<g_long, kLongThreads, 0, st>>>(long_rows, n_long, cols, row_start, bucket, lkeys, offsets);
  scan::exclusive<int>(offsets, nrow, scratch, total, st);
  int gw = div_up(nrow, kWarpsPerBlock);
  k_finish_offsets<<<1, 32, 0, st>>>(nrow, offsets, total, nnz);
  k_row_emit<S><<<gw, kWarpsPerBlock * 32, 0, st>>>(nrow, cols, vals, row_start, bucket, offsets, columns, values);
  k_row_emit_long<S><<<g_long, kLongThreads, 0, st>>>(long_rows, n_long, cols, vals, row_start, bucket, offsets,
                                                      columns, values);
  return check_launch("ipcb_bsr_from_triplets");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

size_t ipcb_bsr_workspace(int n_trip, int nrow, int ncol) {
  (void)ncol;
  size_t R = (size_t)(nrow > 0 ? nrow : 0) + 1, N = (size_t)(n_trip > 0 ? n_trip : 1);
  return 3 * al(R * 4) + 512 + 2 * al(N * 4) + al(2 * N * 8) + scan::scratch_bytes((int)R);
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
