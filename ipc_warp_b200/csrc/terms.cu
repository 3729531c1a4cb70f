// Batched per-iteration terms of the Newton system and its fixed-pattern
// assembly.
//
// k_terms is one persistent launch over every term of an iteration, in the
// order EE contact records | PT contact records | tets: a warp takes a tile of
// consecutive items from a global counter (one atomic per tile) and its lanes
// run the items' device functions (narrow_impl.cuh contact_hessian_item,
// fem_impl.cuh tet_hessian_item); a 32-item chunk of tets only goes through a
// shared-memory stage so its 576-byte block records are stored coalesced.  Contact counts are read on the device, so
// the launch needs no host synchronisation and can be graph-captured.  Grid,
// block and tile sizes are picked by the host autotuner.
//
// The elastic part of the Newton matrix has a fixed pattern (the mesh
// connectivity plus the diagonal): it is computed once, together with a map
// from every pattern slot to the tet blocks that land on it.  Per iteration
// the matrix is the union of that pattern with the contact matrix's
// (ipcb_bsr_union: one sequential merge per row, counts, scan, fill) and its
// values are gathered slot by slot (ipcb_newton_values: diagonal term + h^2
// sum of tet blocks + h^2 contact block), with no sort of the ~16 blocks per
// tet and contact record that the generic assembly needs.
#include "fem_impl.cuh"
#include "narrow_impl.cuh"
#include "scan.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

IPCB_D int device_count(const ipcb_contacts& L) {
  if (!L.cnt) return 0;
  const int c = *L.cnt;
  return c < L.capacity ? c : L.capacity;
}

// dynamic shared memory: one 32-tet stage per warp
template <class S>
__global__ void __launch_bounds__(128) k_terms(ipcb_terms T, int tile) {
  extern __shared__ __align__(16) unsigned char dsm[];
  S* stage = reinterpret_cast<S*>(dsm) + (threadIdx.x >> 5) * 32 * kTetStage;
  const int lane = threadIdx.x & 31;
  const int n_ee = device_count(T.ee);
  const int n_pt = device_count(T.pt);
  const long long n_c = (long long)n_ee + n_pt;
  const long long total = n_c + T.n_tets;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(T.queue, tile);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    for (int k0 = 0; k0 < tile; k0 += 32) {
      const long long c0 = (long long)base + k0;
      if (c0 >= total) break;
      if (c0 >= n_c) {  // a chunk of tets only: staged, coalesced block stores
        tet_hessian_warp<S>(T.material, (const S*)T.x, (const int4*)T.tets, (int)(c0 - n_c), T.n_tets,
                            (const S*)T.Bm, (const S*)T.W, S(T.mu), S(T.lam), T.t_rows, T.t_cols, (S*)T.t_vals,
                            (S*)T.force, stage);
        continue;
      }
      const long long it = c0 + lane;
      if (it >= total) continue;
      if (it < n_ee)
        contact_hessian_item<S, 0>((const S*)T.x, (const S*)T.xcs, T.ee, (int)it, 0, T.kappa, T.c_rows, T.c_cols,
                                   (S*)T.c_vals, (S*)T.force, T.c_mask);
      else if (it < n_c)
        contact_hessian_item<S, 1>((const S*)T.x, (const S*)T.xcs, T.pt, (int)(it - n_ee), n_ee, T.kappa, T.c_rows,
                                   T.c_cols, (S*)T.c_vals, (S*)T.force, T.c_mask);
      else
        tet_hessian_item<S>(T.material, (const S*)T.x, (const int4*)T.tets, (int)(it - n_c), (const S*)T.Bm,
                            (const S*)T.W, S(T.mu), S(T.lam), T.t_rows, T.t_cols, (S*)T.t_vals, (S*)T.force);
    }
  }
}

// slot of (row, col) in a BSR pattern, -1 if absent
IPCB_D int find_slot(const int* __restrict__ off, const int* __restrict__ cols, int r, int c) {
  int lo = __ldg(off + r), hi = __ldg(off + r + 1) - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = __ldg(cols + mid);
    if (v == c) return mid;
    if (v < c) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

__global__ void k_slots(int n, const int* __restrict__ off, const int* __restrict__ cols, const int* __restrict__ rows,
                        const int* __restrict__ tcols, int* __restrict__ slots) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) slots[i] = find_slot(off, cols, __ldg(rows + i), __ldg(tcols + i));
}

// one thread per row: size of the union of the two sorted column lists
__global__ void k_union_count(int nrow, const int* __restrict__ a_off, const int* __restrict__ a_cols,
                              const int* __restrict__ b_off, const int* __restrict__ b_cols, int* __restrict__ cnt) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrow) return;
  int i = a_off[r], ie = a_off[r + 1], j = b_off[r], je = b_off[r + 1], n = 0;
  while (i < ie && j < je) {
    const int ca = a_cols[i], cb = b_cols[j];
    i += ca <= cb;
    j += cb <= ca;
    ++n;
  }
  cnt[r] = n + (ie - i) + (je - j);
}

__global__ void k_union_fill(int nrow, const int* __restrict__ a_off, const int* __restrict__ a_cols,
                             const int* __restrict__ b_off, const int* __restrict__ b_cols,
                             const int* __restrict__ c_off, int capacity, int* __restrict__ c_rows,
                             int* __restrict__ c_cols, int* __restrict__ src_a, int* __restrict__ src_b,
                             int* __restrict__ nnz, int* status) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r == nrow) {
    *nnz = c_off[nrow];
    if (c_off[nrow] > capacity) atomicOr(status, IPCB_STATUS_PATTERN);
  }
  if (r >= nrow) return;
  if (c_off[nrow] > capacity) return;
  int i = a_off[r], ie = a_off[r + 1], j = b_off[r], je = b_off[r + 1], p = c_off[r];
  while (i < ie || j < je) {
    const int ca = i < ie ? a_cols[i] : 0x7fffffff, cb = j < je ? b_cols[j] : 0x7fffffff;
    const int c = ca < cb ? ca : cb;
    c_rows[p] = r;
    c_cols[p] = c;
    src_a[p] = ca == c ? i++ : -1;
    src_b[p] = cb == c ? j++ : -1;
    ++p;
  }
}

// one thread per (slot, component)
template <class S>
__global__ void k_newton_values(const int* __restrict__ nnz, int capacity, const int* __restrict__ c_rows,
                                const int* __restrict__ c_cols, const int* __restrict__ src_a,
                                const int* __restrict__ src_b, const int* __restrict__ g_off,
                                const int* __restrict__ g_idx, const S* __restrict__ t_vals, S t_scale,
                                const S* __restrict__ diag, const S* __restrict__ b_vals, S b_scale,
                                S* __restrict__ vals) {
  const long long n = 9LL * min(*nnz, capacity);
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const int p = (int)(t / 9), c = (int)(t - 9LL * p);
    S v = S(0);
    const int sa = __ldg(src_a + p);
    if (sa >= 0) {
      S acc = S(0);
      const int k1 = __ldg(g_off + sa + 1);
      for (int k = __ldg(g_off + sa); k < k1; ++k) acc += __ldg(t_vals + 9LL * __ldg(g_idx + k) + c);
      v = t_scale * acc;
      const int r = __ldg(c_rows + p);
      if (diag && c % 4 == 0 && __ldg(c_cols + p) == r) v += __ldg(diag + r);
    }
    const int sb = __ldg(src_b + p);
    if (sb >= 0) v += b_scale * __ldg(b_vals + 9LL * sb + c);
    vals[t] = v;
  }
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_terms_launch(const ipcb_terms* T, int blocks, int threads, int tile, ipcb_stream s) {
  if (!T || blocks <= 0 || threads <= 0 || threads > 128 || threads % 32 || tile <= 0 || !T->x || !T->queue ||
      !T->force || T->n_tets < 0)
    return IPCB_E_ARG;
  if (T->n_tets && (!T->tets || !T->Bm || !T->W || !T->t_vals)) return IPCB_E_ARG;
  if ((T->ee.capacity > 0 || T->pt.capacity > 0) && (!T->c_rows || !T->c_cols || !T->c_vals || !T->xcs))
    return IPCB_E_ARG;
  if (T->material < 0 || T->material > 2) return IPCB_E_ARG;
  if (tile % 32) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(T->queue, 0, sizeof(int), st);
  const size_t smem = (size_t)(threads / 32) * 32 * kTetStage * (T->fp64 ? sizeof(double) : sizeof(float));
  if (T->fp64) {
    cudaFuncSetAttribute(k_terms<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_terms<double><<<blocks, threads, smem, st>>>(*T, tile);
  } else {
    cudaFuncSetAttribute(k_terms<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_terms<float><<<blocks, threads, smem, st>>>(*T, tile);
  }
  return check_launch("ipcb_terms_launch");
}

int ipcb_bsr_slots(int nrow, const int* offsets, const int* columns, int n, const int* rows, const int* cols,
                   int* slots, ipcb_stream s) {
  if (nrow < 0 || n < 0) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  if (!offsets || !columns || !rows || !cols || !slots) return IPCB_E_ARG;
  k_slots<<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>(n, offsets, columns, rows, cols, slots);
  return check_launch("ipcb_bsr_slots");
}

size_t ipcb_bsr_union_workspace(int nrow) { return scan::scratch_bytes(nrow + 1); }

int ipcb_bsr_union(int nrow, const int* a_off, const int* a_cols, const int* b_off, const int* b_cols, int* c_off,
                   int* c_rows, int* c_cols, int* src_a, int* src_b, int capacity, int* c_nnz, int* status, void* ws,
                   size_t ws_bytes, ipcb_stream s) {
  if (nrow <= 0 || capacity < 0 || !a_off || !a_cols || !b_off || !b_cols || !c_off || !c_rows || !c_cols || !src_a ||
      !src_b || !c_nnz || !status || !ws || ws_bytes < ipcb_bsr_union_workspace(nrow))
    return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  k_union_count<<<div_up(nrow, 256), 256, 0, st>>>(nrow, a_off, a_cols, b_off, b_cols, c_off);
  cudaMemsetAsync(c_off + nrow, 0, sizeof(int), st);
  scan::exclusive<int>(c_off, nrow + 1, ws, nullptr, st);
  k_union_fill<<<div_up(nrow + 1, 256), 256, 0, st>>>(nrow, a_off, a_cols, b_off, b_cols, c_off, capacity, c_rows,
                                                     c_cols, src_a, src_b, c_nnz, status);
  return check_launch("ipcb_bsr_union");
}

int ipcb_newton_values(int fp64, const int* nnz, int capacity, const int* c_rows, const int* c_cols, const int* src_a,
                       const int* src_b, const int* gather_off, const int* gather_idx, const void* tet_vals,
                       double tet_scale, const void* diag, const void* contact_vals, double contact_scale,
                       void* values, ipcb_stream s) {
  if (!nnz || capacity < 0 || !c_rows || !c_cols || !src_a || !src_b || !gather_off || !gather_idx || !values)
    return IPCB_E_ARG;
  if (capacity == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  const int grid = 148 * 8;
  if (fp64)
    k_newton_values<double><<<grid, 256, 0, st>>>(nnz, capacity, c_rows, c_cols, src_a, src_b, gather_off,
                                                  gather_idx, (const double*)tet_vals, tet_scale,
                                                  (const double*)diag, (const double*)contact_vals, contact_scale,
                                                  (double*)values);
  else
    k_newton_values<float><<<grid, 256, 0, st>>>(nnz, capacity, c_rows, c_cols, src_a, src_b, gather_off, gather_idx,
                                                 (const float*)tet_vals, (float)tet_scale, (const float*)diag,
                                                 (const float*)contact_vals, (float)contact_scale, (float*)values);
  return check_launch("ipcb_newton_values");
}

}  // extern "C"
