// Discrete collision detection: boxes and the EE / PT candidate queries
// (contact.py:30-52, 199-228, 304-336).
#include <cooperative_groups.h>

#include "common.cuh"
#include "geom.cuh"
#include "lbvh.cuh"

namespace cg = cooperative_groups;

namespace ipcb {
int check_launch(const char* where);

namespace {

template <class S>
__global__ void k_pack(const S* __restrict__ x, int n, float4* __restrict__ x4) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  x4[i] = make_float4((float)x[3 * i], (float)x[3 * i + 1], (float)x[3 * i + 2], 0.f);
}

__global__ void k_edge_aabbs(const float4* __restrict__ x4, const int* __restrict__ edges, int n, float pad,
                             float* __restrict__ lo, float* __restrict__ hi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int2 e = __ldg(reinterpret_cast<const int2*>(edges) + i);
  f3 a = load4(x4, e.x), b = load4(x4, e.y);
  lo[3 * i] = fminf(a.x, b.x) - pad;
  lo[3 * i + 1] = fminf(a.y, b.y) - pad;
  lo[3 * i + 2] = fminf(a.z, b.z) - pad;
  hi[3 * i] = fmaxf(a.x, b.x) + pad;
  hi[3 * i + 1] = fmaxf(a.y, b.y) + pad;
  hi[3 * i + 2] = fmaxf(a.z, b.z) + pad;
}

__global__ void k_tri_aabbs(const float4* __restrict__ x4, const int* __restrict__ tris, int n, float pad,
                            float* __restrict__ lo, float* __restrict__ hi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  f3 a = load4(x4, __ldg(tris + 3 * i)), b = load4(x4, __ldg(tris + 3 * i + 1)), c = load4(x4, __ldg(tris + 3 * i + 2));
  lo[3 * i] = fminf(fminf(a.x, b.x), c.x) - pad;
  lo[3 * i + 1] = fminf(fminf(a.y, b.y), c.y) - pad;
  lo[3 * i + 2] = fminf(fminf(a.z, b.z), c.z) - pad;
  hi[3 * i] = fmaxf(fmaxf(a.x, b.x), c.x) + pad;
  hi[3 * i + 1] = fmaxf(fmaxf(a.y, b.y), c.y) + pad;
  hi[3 * i + 2] = fmaxf(fmaxf(a.z, b.z), c.z) + pad;
}

constexpr int kQueue = 32;  // per-thread queue of filtered leaf hits

template <class S>
IPCB_D void write_record(const ipcb_contacts& c, int slot, int a1, int a2, int b1, int b2, int e0, int e1, S l0) {
  if (slot < c.capacity) {
    reinterpret_cast<int4*>(c.a1a2b1b2)[slot] = make_int4(a1, a2, b1, b2);
    reinterpret_cast<int2*>(c.e0e1)[slot] = make_int2(e0, e1);
    static_cast<S*>(c.l0)[slot] = l0;
    static_cast<S*>(c.alpha)[slot] = S(1e-6);
    static_cast<S*>(c.lam)[slot] = S(0);
  }
}

// Append from inside divergent code (rare path: a full queue).
template <class S>
IPCB_D void append_divergent(const ipcb_contacts& c, int a1, int a2, int b1, int b2, int e0, int e1, S l0) {
  cg::coalesced_group g = cg::coalesced_threads();
  int base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(c.cnt, (int)g.size());
  write_record<S>(c, g.shfl(base, 0) + (int)g.thread_rank(), a1, a2, b1, b2, e0, e1, l0);
}

// Append from converged code: one ballot and one atomicAdd per warp.
IPCB_D int warp_reserve(int* cnt, bool accept) {
  const unsigned lane = threadIdx.x & 31;
  unsigned m = __ballot_sync(0xffffffffu, accept);
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(cnt, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  return base + __popc(m & ((1u << lane) - 1u));
}

IPCB_D int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// One thread per edge, visiting edges in the BVH leaf (Morton) order so a
// warp's queries walk neighbouring subtrees.  Traversal only applies the cheap
// filters and queues the surviving leaves; the exact closest-point test and
// the append run afterwards with the warp converged.
template <class S>
__global__ void __launch_bounds__(128) k_dcd_ee(const float4* __restrict__ x4, const int* __restrict__ edges,
                                                const int* __restrict__ body, const float4* __restrict__ nodes,
                                                const int* __restrict__ order, int n, float thickness, float qpad,
                                                int exclude, ipcb_contacts out, int* status) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < n;
  int i = active ? __ldg(order + t) : 0;
  int2 ea = active ? __ldg(reinterpret_cast<const int2*>(edges) + i) : make_int2(0, 0);
  f3 p1 = load4(x4, ea.x), p2 = load4(x4, ea.y);
  int bi = exclude ? __ldg(body + ea.x) : 0;
  const float l0f = xmul(thickness, 2.0f);
  const S l0 = S(thickness) * S(2.0);
  int q[kQueue];
  int nq = 0;
  if (active) {
    f3 qlo = mk3(fminf(p1.x, p2.x) - qpad, fminf(p1.y, p2.y) - qpad, fminf(p1.z, p2.z) - qpad);
    f3 qhi = mk3(fmaxf(p1.x, p2.x) + qpad, fmaxf(p1.y, p2.y) + qpad, fmaxf(p1.z, p2.z) + qpad);
    bool ok = traverse4(nodes, n, qlo, qhi, [&](int j) {
      if (!(i < j)) return;
      int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + j);
      if (ea.x == eb.x || ea.x == eb.y || ea.y == eb.x || ea.y == eb.y) return;
      if (exclude && bi == __ldg(body + eb.x)) return;
      if (nq < kQueue) {
        q[nq++] = j;
      } else {
        CPEE r = closest_point_edge_edge(p1, p2, load4(x4, eb.x), load4(x4, eb.y), 1.0e-6f);
        if (r.d < l0f) append_divergent<S>(out, ea.x, ea.y, eb.x, eb.y, i, j, l0);
      }
    });
    if (!ok) atomicOr(status, IPCB_STATUS_STACK);
  }
  int rounds = warp_max(nq);
  for (int k = 0; k < rounds; ++k) {
    bool has = k < nq;
    int j = has ? q[k] : 0;
    int2 eb = has ? __ldg(reinterpret_cast<const int2*>(edges) + j) : make_int2(0, 0);
    bool accept = false;
    if (has) accept = closest_point_edge_edge(p1, p2, load4(x4, eb.x), load4(x4, eb.y), 1.0e-6f).d < l0f;
    int slot = warp_reserve(out.cnt, accept);
    if (accept) write_record<S>(out, slot, ea.x, ea.y, eb.x, eb.y, i, j, l0);
  }
}

template <class S>
__global__ void __launch_bounds__(128) k_dcd_pt(const float4* __restrict__ x4, const int* __restrict__ tris,
                                                const int* __restrict__ body, const float4* __restrict__ nodes,
                                                int n_tris, const int* __restrict__ order, int nv, float thickness,
                                                float qpad, int exclude, ipcb_contacts out, int* status) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < nv;
  int i = active ? (order ? __ldg(order + t) : t) : 0;
  f3 p = load4(x4, i);
  int bi = exclude ? __ldg(body + i) : 0;
  const float l0f = xmul(thickness, 2.0f);
  const S l0 = S(thickness) * S(2.0);
  int q[kQueue];
  int nq = 0;
  if (active) {
    f3 qlo = mk3(p.x - qpad, p.y - qpad, p.z - qpad), qhi = mk3(p.x + qpad, p.y + qpad, p.z + qpad);
    bool ok = traverse4(nodes, n_tris, qlo, qhi, [&](int j) {
      int t0 = __ldg(tris + 3 * j), t1 = __ldg(tris + 3 * j + 1), t2 = __ldg(tris + 3 * j + 2);
      if (t0 == i || t1 == i || t2 == i) return;
      if (exclude && bi == __ldg(body + t0)) return;
      if (nq < kQueue) {
        q[nq++] = j;
      } else {
        CPT r = closest_point_triangle(p, load4(x4, t0), load4(x4, t1), load4(x4, t2));
        if (r.d < l0f) append_divergent<S>(out, i, t1, t0, t2, i, j, l0);
      }
    });
    if (!ok) atomicOr(status, IPCB_STATUS_STACK);
  }
  int rounds = warp_max(nq);
  for (int k = 0; k < rounds; ++k) {
    bool has = k < nq;
    int j = has ? q[k] : 0;
    int t0 = has ? __ldg(tris + 3 * j) : 0, t1 = has ? __ldg(tris + 3 * j + 1) : 0,
        t2 = has ? __ldg(tris + 3 * j + 2) : 0;
    bool accept = false;
    if (has) accept = closest_point_triangle(p, load4(x4, t0), load4(x4, t1), load4(x4, t2)).d < l0f;
    int slot = warp_reserve(out.cnt, accept);
    if (accept) write_record<S>(out, slot, i, t1, t0, t2, i, j, l0);  // (p, tri[1], tri[0], tri[2])
  }
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_pack_positions(const ipcb_soup* soup, float* x4, ipcb_stream s) {
  if (!soup || !x4 || soup->n_verts < 0) return IPCB_E_ARG;
  int n = soup->n_verts;
  if (n == 0) return IPCB_OK;
  if (soup->fp64)
    k_pack<double><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const double*)soup->x, n, (float4*)x4);
  else
    k_pack<float><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const float*)soup->x, n, (float4*)x4);
  return check_launch("ipcb_pack_positions");
}

int ipcb_edge_aabbs(const ipcb_soup* soup, const float* x4, float pad, float* lower, float* upper, ipcb_stream s) {
  if (!soup || !x4 || !lower || !upper) return IPCB_E_ARG;
  int n = soup->n_edges;
  if (n == 0) return IPCB_OK;
  k_edge_aabbs<<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, n, pad, lower, upper);
  return check_launch("ipcb_edge_aabbs");
}

int ipcb_triangle_aabbs(const ipcb_soup* soup, const float* x4, float pad, float* lower, float* upper,
                        ipcb_stream s) {
  if (!soup || !x4 || !lower || !upper) return IPCB_E_ARG;
  int n = soup->n_tris;
  if (n == 0) return IPCB_OK;
  k_tri_aabbs<<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, n, pad, lower, upper);
  return check_launch("ipcb_triangle_aabbs");
}

int ipcb_dcd_ee(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness, float query_pad,
                int exclude_same_body, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup || !x4 || !bvh || !out || !status || bvh->n != soup->n_edges) return IPCB_E_ARG;
  int n = soup->n_edges;
  if (n == 0) return IPCB_OK;
  dim3 grid(div_up(n, 128));
  if (soup->fp64)
    k_dcd_ee<double><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, soup->body,
                                                        (const float4*)bvh->wide, bvh->sorted, n, thickness,
                                                        query_pad, exclude_same_body, *out, status);
  else
    k_dcd_ee<float><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, soup->body,
                                                       (const float4*)bvh->wide, bvh->sorted, n, thickness,
                                                       query_pad, exclude_same_body, *out, status);
  return check_launch("ipcb_dcd_ee");
}

int ipcb_dcd_pt(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness, float query_pad,
                int exclude_same_body, const int* query_order, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup || !x4 || !bvh || !out || !status || bvh->n != soup->n_tris) return IPCB_E_ARG;
  int nv = soup->n_verts;
  if (nv == 0 || soup->n_tris == 0) return IPCB_OK;
  dim3 grid(div_up(nv, 128));
  if (soup->fp64)
    k_dcd_pt<double><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, soup->body,
                                                        (const float4*)bvh->wide, soup->n_tris, query_order, nv,
                                                        thickness, query_pad, exclude_same_body, *out, status);
  else
    k_dcd_pt<float><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, soup->body,
                                                       (const float4*)bvh->wide, soup->n_tris, query_order, nv,
                                                       thickness, query_pad, exclude_same_body, *out, status);
  return check_launch("ipcb_dcd_pt");
}

}  // extern "C"
