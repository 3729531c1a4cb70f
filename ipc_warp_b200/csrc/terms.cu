// Batched per-iteration terms of the Newton system and its fixed-pattern
// assembly.
//
// k_terms is one persistent launch over every term of an iteration, in the
// order EE contact records | PT contact records | tets | affine-body items:
// a warp takes a tile of consecutive items from a global counter (one
// atomic per tile) and runs them 32 at a time.  The contact records run in
// the cost-class order of the class-sorted narrow phase (the two ordering
// passes run first, in the same call) with the warp-cooperative block
// stores of hessian_from_warp; a 32-item chunk of tets goes through a
// shared-memory stage so its 576-byte block records are stored coalesced;
// an affine-body item is one (body, i, j) block of inertia + orthogonality
// (and the body gradient row when j = 0).  Each kind runs in its own
// non-inlined device function, so the kernel's register budget is the
// largest kind's, not their union.  Contact counts are read on the device,
// so the launch needs no host synchronisation and can be graph-captured.
// Grid, block and tile sizes are picked by the host autotuner.
//
// The elastic part of the Newton matrix has a fixed pattern (the mesh
// connectivity plus the diagonal): it is computed once, together with a map
// from every pattern slot to the tet blocks that land on it.  Per iteration
// the matrix is the union of that pattern with the contact matrix's
// (ipcb_bsr_union: one sequential merge per row, counts, scan, fill) and its
// values are gathered slot by slot (ipcb_newton_values: diagonal term + h^2
// sum of tet blocks + h^2 contact block), with no sort of the ~16 blocks per
// tet and contact record that the generic assembly needs.
#include "abd_impl.cuh"
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

// one sorted contact position t per lane (active lanes), all 32 lanes call
template <class S, int KIND>
__device__ __noinline__ void contact_chunk(const S* __restrict__ x, const S* __restrict__ xcs, const Sorted<S>& W,
                                           int t, bool active, int offset, double kappa, int* __restrict__ rows,
                                           int* __restrict__ cols, S* __restrict__ vals, S* __restrict__ force,
                                           unsigned short* __restrict__ mask, S* __restrict__ stage) {
  int i = 0;
  int4 id = make_int4(0, 0, 0, 0);
  S l0 = S(0);
  Pre p{0.f, 0.f, 0.f, 0};
  if (active) {
    i = __ldg(W.order + t);
    id = __ldg(W.sids + t);
    l0 = __ldg(W.sl0 + t);
    p = unpack(__ldg(W.spre + t));
  }
  hessian_from_warp<S, KIND>(x, xcs, id, l0, i, offset, kappa, p, active, rows, cols, vals, force, mask, stage);
}

template <class S>
__device__ __noinline__ void tet_chunk(const ipcb_terms& T, int e0, S* __restrict__ stage) {
  tet_hessian_warp<S>(T.material, (const S*)T.x, (const int4*)T.tets, e0, T.n_tets, (const S*)T.Bm, (const S*)T.W,
                      S(T.mu), S(T.lam), T.t_rows, T.t_cols, (S*)T.t_vals, (S*)T.force, stage);
}

template <class S>
__device__ __noinline__ void tet_one(const ipcb_terms& T, int e) {
  tet_hessian_item<S>(T.material, (const S*)T.x, (const int4*)T.tets, e, (const S*)T.Bm, (const S*)T.W, S(T.mu),
                      S(T.lam), T.t_rows, T.t_cols, (S*)T.t_vals, (S*)T.force);
}

// affine-body item t = 16 b + 4 i + j: the block at (row0 + 4 b + i,
// row0 + 4 b + j) and, for j = 0, gradient row 4 b + i
template <class S>
__device__ __noinline__ void body_one(const ipcb_terms& T, int t) {
  const Abd<S> A = view<S>(&T.abd);
  const int b = t >> 4, i = (t >> 2) & 3, j = t & 3;
  S blk[9];
  body_block(A, b, i, j, S(T.h2), blk);
  T.a_rows[t] = T.body_row0 + 4 * b + i;
  T.a_cols[t] = T.body_row0 + 4 * b + j;
  S* dst = (S*)T.a_vals + 9LL * t;
#pragma unroll
  for (int k = 0; k < 9; ++k) dst[k] = blk[k];
  if (j == 0) st3((S*)T.a_grad, 4 * b + i, body_gradient(A, b, i, S(T.h2)));
}

// dynamic shared memory: one 32-tet stage per warp (also holds a contact
// chunk's 32 block rows)
// MINB: resident CTAs of 128 per SM the register budget is sized for (3:
// 168 registers, the contact chunks spill a little; 2: 255, no spills)
template <class S, int MINB>
__global__ void __launch_bounds__(128, MINB) k_terms(ipcb_terms T, Sorted<S> We, Sorted<S> Wp, int tile) {
  extern __shared__ __align__(16) unsigned char dsm[];
  S* stage = reinterpret_cast<S*>(dsm) + (threadIdx.x >> 5) * 32 * kTetStage;
  const int lane = threadIdx.x & 31;
  const int n_ee = device_count(T.ee);
  const int n_pt = device_count(T.pt);
  const long long n_c = (long long)n_ee + n_pt;
  const long long n_t = n_c + T.n_tets;
  const long long total = n_t + 16LL * T.abd.n_bodies;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(T.queue, tile);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= total) break;
    for (int k0 = 0; k0 < tile; k0 += 32) {
      const long long c0 = (long long)base + k0;
      if (c0 >= total) break;
      const long long it = c0 + lane;
      if (c0 < n_ee)  // warp-uniform: the chunk holds EE records
        contact_chunk<S, 0>((const S*)T.x, (const S*)T.xcs, We, (int)it, it < n_ee, 0, T.kappa, T.c_rows, T.c_cols,
                            (S*)T.c_vals, (S*)T.force, T.c_mask, stage);
      if (c0 < n_c && c0 + 32 > n_ee)
        contact_chunk<S, 1>((const S*)T.x, (const S*)T.xcs, Wp, (int)(it - n_ee), it >= n_ee && it < n_c, n_ee,
                            T.kappa, T.c_rows, T.c_cols, (S*)T.c_vals, (S*)T.force, T.c_mask, stage);
      if (c0 < n_t && c0 + 32 > n_c) {
        if (c0 >= n_c && c0 + 32 <= n_t) tet_chunk<S>(T, (int)(c0 - n_c), stage);  // a chunk of tets only
        else if (it >= n_c && it < n_t) tet_one<S>(T, (int)(it - n_c));
      }
      if (c0 + 32 > n_t && it >= n_t && it < total) body_one<S>(T, (int)(it - n_t));
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

int ipcb_terms_launch(const ipcb_terms* T, int blocks, int threads, int tile, int variant, ipcb_stream s) {
  if (!T || blocks <= 0 || threads <= 0 || threads > 128 || threads % 32 || tile <= 0 || !T->x || !T->queue ||
      (variant != 0 && variant != 1) ||
      !T->force || T->n_tets < 0 || T->abd.n_bodies < 0)
    return IPCB_E_ARG;
  if (T->n_tets && (!T->tets || !T->Bm || !T->W || !T->t_vals)) return IPCB_E_ARG;
  if ((T->ee.capacity > 0 || T->pt.capacity > 0) && (!T->c_rows || !T->c_cols || !T->c_vals || !T->xcs))
    return IPCB_E_ARG;
  if ((T->ee.capacity > 0 && !T->ee_ws) || (T->pt.capacity > 0 && !T->pt_ws)) return IPCB_E_ARG;
  if (T->abd.n_bodies && (!T->abd.q || !T->abd.q_tilde || !T->abd.mass || !T->abd.volume || !T->abd.stiffness ||
                          !T->abd.fixed || !T->a_rows || !T->a_cols || !T->a_vals || !T->a_grad ||
                          T->abd.fp64 != T->fp64))
    return IPCB_E_ARG;
  if (T->material < 0 || T->material > 2) return IPCB_E_ARG;
  if (tile % 32) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  cudaMemsetAsync(T->queue, 0, sizeof(int), st);
  const size_t smem = (size_t)(threads / 32) * 32 * kTetStage * (T->fp64 ? sizeof(double) : sizeof(float));
  auto run = [&](auto zero) {
    using S = decltype(zero);
    const S* x = (const S*)T->x;
    const S* xcs = (const S*)T->xcs;
    Sorted<S> W[2] = {};
    const ipcb_contacts* L[2] = {&T->ee, &T->pt};
    void* ws[2] = {T->ee_ws, T->pt_ws};
    for (int k = 0; k < 2; ++k) {
      if (L[k]->capacity <= 0) continue;
      int* counts = (int*)ws[k];
      W[k] = sorted_ws<S>(ws[k], L[k]->capacity);
      cudaMemsetAsync(counts, 0, 8 * sizeof(int), st);
      const int g = div_up(L[k]->capacity, 256);
      if (k == 0) k_classify<S, 0><<<g, 256, 0, st>>>(x, xcs, *L[k], -1, W[k].pre, counts);
      else k_classify<S, 1><<<g, 256, 0, st>>>(x, xcs, *L[k], -1, W[k].pre, counts);
      k_class_order<S><<<g, 256, 0, st>>>(*L[k], -1, counts, counts + 4, W[k]);
    }
    if (variant == 0) {
      cudaFuncSetAttribute(k_terms<S, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_terms<S, 3><<<blocks, threads, smem, st>>>(*T, W[0], W[1], tile);
    } else {
      cudaFuncSetAttribute(k_terms<S, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      k_terms<S, 2><<<blocks, threads, smem, st>>>(*T, W[0], W[1], tile);
    }
  };
  if (T->fp64) run(0.0);
  else run(0.0f);
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
