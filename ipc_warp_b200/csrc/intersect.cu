// Intersection check of a surface state: every surface edge that crosses a
// surface triangle (not sharing a vertex with it) is an intersection.  The
// IPC invariant is that an accepted step never produces one; the trajectory
// tests run this after every step.
//
// One thread per edge queries the triangle hierarchy (refit to the current
// positions) with the edge's box padded by a relative 1e-6 (covers the
// float rounding of the hierarchy's boxes), and tests each hit with
// orientation signs in double: the endpoints p, q lie strictly on opposite
// sides of the triangle's plane and the line pq passes strictly inside the
// three edges.  Contacts at exactly zero volume (touching, coplanar) are not
// counted.  Every double operation is a correctly rounded intrinsic, so the
// signs are the ones a plain IEEE evaluation in the same order gives (the CPU
// oracle evaluates the same expressions).
#include "common.cuh"
#include "lbvh.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

IPCB_D double orient(const d3& a, const d3& b, const d3& c, const d3& d) {
  const d3 u = esub(b, a), v = esub(c, a), w = esub(d, a);
  // det[u v w] = u . (v x w), in that order
  return edot(u, ecross(v, w));
}

IPCB_D bool segment_crosses_triangle(const d3& p, const d3& q, const d3& a, const d3& b, const d3& c) {
  const double o1 = orient(a, b, c, p), o2 = orient(a, b, c, q);
  if (!((o1 > 0.0 && o2 < 0.0) || (o1 < 0.0 && o2 > 0.0))) return false;
  const double s1 = orient(p, q, a, b), s2 = orient(p, q, b, c), s3 = orient(p, q, c, a);
  return (s1 > 0.0 && s2 > 0.0 && s3 > 0.0) || (s1 < 0.0 && s2 < 0.0 && s3 < 0.0);
}

template <class S>
__global__ void __launch_bounds__(128) k_edge_triangle_crossings(const S* __restrict__ x, const int* __restrict__ edges,
                                                                 int n_edges, const int* __restrict__ tris,
                                                                 const float4* __restrict__ wide, int n_tris,
                                                                 int* __restrict__ count, int2* __restrict__ pairs,
                                                                 int capacity, int* __restrict__ status) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n_edges) return;
  const int2 ev = __ldg(reinterpret_cast<const int2*>(edges) + e);
  const d3 p = to_d(load3(x, ev.x)), q = to_d(load3(x, ev.y));
  f3 lo, hi;
  const double lx = fmin(p.x, q.x), ly = fmin(p.y, q.y), lz = fmin(p.z, q.z);
  const double hx = fmax(p.x, q.x), hy = fmax(p.y, q.y), hz = fmax(p.z, q.z);
  lo = mk3(__double2float_rd(lx - 1e-6 * (1.0 + fabs(lx))), __double2float_rd(ly - 1e-6 * (1.0 + fabs(ly))),
           __double2float_rd(lz - 1e-6 * (1.0 + fabs(lz))));
  hi = mk3(__double2float_ru(hx + 1e-6 * (1.0 + fabs(hx))), __double2float_ru(hy + 1e-6 * (1.0 + fabs(hy))),
           __double2float_ru(hz + 1e-6 * (1.0 + fabs(hz))));
  const bool ok = traverse4(wide, n_tris, lo, hi, [&](int t) {
    const int t0 = __ldg(tris + 3 * t), t1 = __ldg(tris + 3 * t + 1), t2 = __ldg(tris + 3 * t + 2);
    if (t0 == ev.x || t0 == ev.y || t1 == ev.x || t1 == ev.y || t2 == ev.x || t2 == ev.y) return;
    if (!segment_crosses_triangle(p, q, to_d(load3(x, t0)), to_d(load3(x, t1)), to_d(load3(x, t2)))) return;
    const int k = atomicAdd(count, 1);
    if (k < capacity) pairs[k] = make_int2(e, t);
  });
  if (!ok) atomicOr(status, IPCB_STATUS_STACK);
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_edge_triangle_crossings(const ipcb_soup* soup, const ipcb_lbvh* tri_bvh, int* count, int* pairs,
                                 int capacity, int* status, ipcb_stream s) {
  if (!soup || !tri_bvh || !count || !status || capacity < 0 || (capacity > 0 && !pairs)) return IPCB_E_ARG;
  if (tri_bvh->n != soup->n_tris) return IPCB_E_ARG;
  if (soup->n_edges == 0 || soup->n_tris == 0) return IPCB_OK;
  const dim3 grid(div_up(soup->n_edges, 128));
  cudaStream_t st = (cudaStream_t)s;
  if (soup->fp64)
    k_edge_triangle_crossings<double><<<grid, 128, 0, st>>>((const double*)soup->x, soup->edges, soup->n_edges,
                                                            soup->triangles, (const float4*)tri_bvh->wide,
                                                            soup->n_tris, count, (int2*)pairs, capacity, status);
  else
    k_edge_triangle_crossings<float><<<grid, 128, 0, st>>>((const float*)soup->x, soup->edges, soup->n_edges,
                                                           soup->triangles, (const float4*)tri_bvh->wide,
                                                           soup->n_tris, count, (int2*)pairs, capacity, status);
  return check_launch("ipcb_edge_triangle_crossings");
}

}  // extern "C"
