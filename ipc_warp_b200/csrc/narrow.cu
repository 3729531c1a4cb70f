// Narrow phase: barrier energy, force and PSD-filtered 12x12 Hessian per
// EE / PT record (dynamic_contacts.py:49-246, 375-398).
//
// Per record (one thread):
//   1. float32 closest distance and feature (exact ops)  -> gate dist < l0
//   2. feature geometry in double: weights c (r = sum_k c_k x_k), the edge
//      vectors E_j of its 0..2 parameters, unit normal n, signed distance rho
//   3. grad(d^2) = 2 c (x) r; the negative spectral part of hess(d^2) from the
//      3x3 (point-edge) or 5x5 (point-triangle, edge-edge) restriction of the
//      Hessian to span{c^ (x) frame, f_a (x) n}, diagonalised by Jacobi
//   4. IPC barrier b(d^2) and derivatives in double; EE mollifier when the
//      edges are near parallel
//   5. H = sum_m w_m h_m h_m^T (h_0 = grad, h_e = negative eigenvectors),
//      written as 16 3x3 triplets; force atomically added to b.
#include <cstddef>

#include "narrow_impl.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

// T: arithmetic type of the eigen-solve and of H (float for S=float).
template <class S, int KIND>
__global__ void __launch_bounds__(128, 3) k_contact_hessian(const S* __restrict__ x, const S* __restrict__ xcs,
                                                         ipcb_contacts L, int n, int offset,
                                                         const int* __restrict__ offset_dev, double kappa,
                                                         int* __restrict__ rows, int* __restrict__ cols,
                                                         S* __restrict__ vals, S* __restrict__ bforce,
                                                         unsigned short* __restrict__ block_mask) {
  // The CTA's 128 records are classified (their float32 part, kept in shared
  // memory) and handed to the threads in class order, so most warps run one
  // path of hessian_from instead of the union of their records' paths (a
  // record's outputs go to its own slots; only the order of the force
  // atomics changes).
  __shared__ int s_count[4], s_cursor[4], s_order[128];
  __shared__ float4 s_pre[128];
  const int cnt = list_count<S>(L, n);
  const int base = blockIdx.x * 128;
  if (base >= cnt) return;  // the whole CTA
  const int tid = threadIdx.x, m = min(128, cnt - base);
  if (tid < 4) s_count[tid] = 0;
  __syncthreads();
  int cls = -1;
  if (tid < m) {
    const int i = base + tid;
    const int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
    const S l0 = static_cast<const S*>(L.l0)[i];
    const v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
    const Pre p = predicate<S, KIND>(xcs, id, l0, xs);
    s_pre[tid] = pack(p);
    cls = p.cls();
    atomicAdd(&s_count[cls], 1);
  }
  __syncthreads();
  if (tid == 0) {
    int run = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      s_cursor[k] = run;
      run += s_count[k];
    }
  }
  __syncthreads();
  if (cls >= 0) s_order[atomicAdd(&s_cursor[cls], 1)] = tid;
  __syncthreads();
  if (tid >= m) return;
  // offset_dev: the records follow another list's min(count, offset) records
  const int off = offset_dev ? min(*offset_dev, offset) : offset;
  const int t = s_order[tid], i = base + t;
  const int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
  const S l0 = static_cast<const S*>(L.l0)[i];
  hessian_from<S, KIND>(x, xcs, id, l0, i, off, kappa, unpack(s_pre[t]), rows, cols, vals, bforce, block_mask);
}

// After the ordering pass, one thread per position of the sorted order; a
// warp's lanes store their records' blocks together (hessian_from_warp).
template <class S, int KIND>
__global__ void __launch_bounds__(128, 3) k_contact_hessian_sorted(const S* __restrict__ x,
                                                                const S* __restrict__ xcs, ipcb_contacts L, int n,
                                                                int offset, const int* __restrict__ offset_dev,
                                                                double kappa, Sorted<S> W,
                                                                int* __restrict__ rows, int* __restrict__ cols,
                                                                S* __restrict__ vals, S* __restrict__ bforce,
                                                                unsigned short* __restrict__ block_mask) {
  __shared__ __align__(16) S stage[4][32 * 36];
  const int cnt = list_count<S>(L, n);
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int warp_first = t & ~31;
  if (warp_first >= cnt) return;  // the whole warp
  const bool active = t < cnt;
  const int off = offset_dev ? min(*offset_dev, offset) : offset;
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
  hessian_from_warp<S, KIND>(x, xcs, id, l0, i, off, kappa, p, active, rows, cols, vals, bforce, block_mask,
                             stage[threadIdx.x >> 5]);
}


template <class S, int KIND>
__global__ void __launch_bounds__(256) k_contact_energy(const S* __restrict__ x, const S* __restrict__ xcs,
                                                        ipcb_contacts L, int n, double kappa,
                                                        double* __restrict__ energy) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int cnt = list_count<S>(L, n);
  double e = 0.0;
  if (i < cnt) {
    int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
    S l0 = static_cast<const S*>(L.l0)[i];
    v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
    f3 xf[4] = {to_f(xs[0]), to_f(xs[1]), to_f(xs[2]), to_f(xs[3])};
    float dist;
    if (KIND == 0) dist = closest_point_edge_edge(xf[0], xf[1], xf[2], xf[3], 1.0e-6f).d;
    else dist = closest_point_triangle(xf[0], xf[1], xf[2], xf[3]).d;
    if (S(dist) < l0) {
      double d2 = (double)dist * (double)dist, d02 = (double)l0 * (double)l0;
      e = barrier(d2, d02, kappa).b;
      if (KIND == 0) {
        S eps_x = ee_eps_x(xcs, id);
        v3<S> ea = esub(xs[1], xs[0]), eb = esub(xs[3], xs[2]);
        v3<S> cr = ecross(ea, eb);
        if (eps_x > S(0) && edot(cr, cr) < eps_x) {
          d3 xd[4] = {to_d(xs[0]), to_d(xs[1]), to_d(xs[2]), to_d(xs[3])};
          double mv, gm[12];
          mollifier(xd, (double)eps_x, mv, gm);
          e *= mv;
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  __shared__ double s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s[k];
    if (t != 0.0) atomicAdd(energy, t);
  }
}

template <class S>
int launch_hessian(int kind, const ipcb_soup* soup, const ipcb_contacts* L, int n, int offset, const int* offset_dev,
                   double kappa, int* rows, int* cols, void* vals, void* b, unsigned short* mask, cudaStream_t st) {
  int threads = n >= 0 ? n : L->capacity;
  if (threads == 0) return IPCB_OK;
  dim3 grid(div_up(threads, 128));
  const S* x = (const S*)soup->x;
  const S* xcs = (const S*)soup->xcs;
  if (kind == 0)
    k_contact_hessian<S, 0><<<grid, 128, 0, st>>>(x, xcs, *L, n, offset, offset_dev, kappa, rows, cols, (S*)vals,
                                                  (S*)b, mask);
  else
    k_contact_hessian<S, 1><<<grid, 128, 0, st>>>(x, xcs, *L, n, offset, offset_dev, kappa, rows, cols, (S*)vals,
                                                  (S*)b, mask);
  return check_launch("ipcb_contact_hessian");
}

template <class S>
int launch_hessian_sorted(int kind, const ipcb_soup* soup, const ipcb_contacts* L, int n, int offset,
                          const int* offset_dev, double kappa, int* rows, int* cols, void* vals, void* b,
                          unsigned short* mask, void* ws, cudaStream_t st) {
  int threads = n >= 0 ? n : L->capacity;
  if (threads == 0) return IPCB_OK;
  int* counts = (int*)ws;
  int* cursor = counts + 4;
  const Sorted<S> W = sorted_ws<S>(ws, L->capacity);
  cudaMemsetAsync(ws, 0, 8 * sizeof(int), st);
  const S* x = (const S*)soup->x;
  const S* xcs = (const S*)soup->xcs;
  dim3 g256(div_up(threads, 256)), g128(div_up(threads, 128));
  if (kind == 0) {
    k_classify<S, 0><<<g256, 256, 0, st>>>(x, xcs, *L, n, W.pre, counts);
    k_class_order<S><<<g256, 256, 0, st>>>(*L, n, counts, cursor, W);
    k_contact_hessian_sorted<S, 0><<<g128, 128, 0, st>>>(x, xcs, *L, n, offset, offset_dev, kappa, W, rows, cols,
                                                         (S*)vals, (S*)b, mask);
  } else {
    k_classify<S, 1><<<g256, 256, 0, st>>>(x, xcs, *L, n, W.pre, counts);
    k_class_order<S><<<g256, 256, 0, st>>>(*L, n, counts, cursor, W);
    k_contact_hessian_sorted<S, 1><<<g128, 128, 0, st>>>(x, xcs, *L, n, offset, offset_dev, kappa, W, rows, cols,
                                                         (S*)vals, (S*)b, mask);
  }
  return check_launch("ipcb_contact_hessian_sorted");
}

template <class S>
int launch_energy(int kind, const ipcb_soup* soup, const ipcb_contacts* L, int n, double kappa, double* e,
                  cudaStream_t st) {
  int threads = n >= 0 ? n : L->capacity;
  if (threads == 0) return IPCB_OK;
  dim3 grid(div_up(threads, 256));
  if (kind == 0)
    k_contact_energy<S, 0><<<grid, 256, 0, st>>>((const S*)soup->x, (const S*)soup->xcs, *L, n, kappa, e);
  else
    k_contact_energy<S, 1><<<grid, 256, 0, st>>>((const S*)soup->x, (const S*)soup->xcs, *L, n, kappa, e);
  return check_launch("ipcb_contact_energy");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_contact_hessian(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset, double kappa,
                         int* rows, int* cols, void* vals, void* b, unsigned short* block_mask, ipcb_stream s) {
  return ipcb_contact_hessian_after(kind, soup, list, n, offset, nullptr, kappa, rows, cols, vals, b, block_mask, s);
}

int ipcb_contact_hessian_after(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset,
                               const int* offset_count, double kappa, int* rows, int* cols, void* vals, void* b,
                               unsigned short* block_mask, ipcb_stream s) {
  if (!soup || !list || !rows || !cols || !vals || !b || (kind != 0 && kind != 1) || offset < 0) return IPCB_E_ARG;
  if (n > list->capacity) return IPCB_E_ARG;
  if (soup->fp64)
    return launch_hessian<double>(kind, soup, list, n, offset, offset_count, kappa, rows, cols, vals, b, block_mask,
                                  (cudaStream_t)s);
  return launch_hessian<float>(kind, soup, list, n, offset, offset_count, kappa, rows, cols, vals, b, block_mask,
                               (cudaStream_t)s);
}

size_t ipcb_contact_hessian_workspace(int capacity) { return sorted_workspace(capacity); }

int ipcb_contact_hessian_sorted(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, int offset,
                                const int* offset_count, double kappa, int* rows, int* cols, void* vals, void* b,
                                unsigned short* block_mask, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!soup || !list || !rows || !cols || !vals || !b || (kind != 0 && kind != 1) || offset < 0) return IPCB_E_ARG;
  if (n > list->capacity || !ws || ws_bytes < sorted_workspace(list->capacity)) return IPCB_E_ARG;
  if (soup->fp64)
    return launch_hessian_sorted<double>(kind, soup, list, n, offset, offset_count, kappa, rows, cols, vals, b,
                                         block_mask, ws, (cudaStream_t)s);
  return launch_hessian_sorted<float>(kind, soup, list, n, offset, offset_count, kappa, rows, cols, vals, b,
                                      block_mask, ws, (cudaStream_t)s);
}

int ipcb_contact_energy(int kind, const ipcb_soup* soup, const ipcb_contacts* list, int n, double kappa,
                        double* energy, ipcb_stream s) {
  if (!soup || !list || !energy || (kind != 0 && kind != 1)) return IPCB_E_ARG;
  if (n > list->capacity) return IPCB_E_ARG;
  if (soup->fp64) return launch_energy<double>(kind, soup, list, n, kappa, energy, (cudaStream_t)s);
  return launch_energy<float>(kind, soup, list, n, kappa, energy, (cudaStream_t)s);
}

}  // extern "C"
