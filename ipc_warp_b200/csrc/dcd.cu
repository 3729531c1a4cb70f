// Discrete collision detection: boxes and the EE / PT candidate queries
// (contact.py:30-52, 199-228, 304-336).
#include <cooperative_groups.h>

#include "bodies.cuh"
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
// 64-thread blocks, 14 per SM (at most 73 registers; 80 unbounded): more
// warps in flight over the dependent node loads (screw and nut 0.568 ->
// 0.539 ms; 64 registers spill and were slower)
template <class S>
__global__ void __launch_bounds__(64, 14) k_dcd_ee(const float4* __restrict__ x4, const int* __restrict__ edges,
                                                const int* __restrict__ body, const float4* __restrict__ nodes,
                                                const int* __restrict__ order, int n, int first, int count,
                                                float thickness, float qpad, int exclude, ipcb_contacts out,
                                                int* status) {
  // queries: the edges of Morton rank first .. first + count - 1
  int t = first + blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < first + count;
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
    // the hierarchy is over the queries themselves: thread t is the edge of
    // Morton rank t, so only leaves of higher rank are visited and each pair
    // is met once; it is then stated as the reference's (lower id, higher id)
    bool ok = traverse4_after(nodes, n, t, qlo, qhi, [&](int j, int) {
      int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + j);
      if (ea.x == eb.x || ea.x == eb.y || ea.y == eb.x || ea.y == eb.y) return;
      if (exclude && bi == __ldg(body + eb.x)) return;
      if (nq < kQueue) {
        q[nq++] = j;
      } else if (i < j) {
        CPEE r = closest_point_edge_edge(p1, p2, load4(x4, eb.x), load4(x4, eb.y), 1.0e-6f);
        if (r.d < l0f) append_divergent<S>(out, ea.x, ea.y, eb.x, eb.y, i, j, l0);
      } else {
        CPEE r = closest_point_edge_edge(load4(x4, eb.x), load4(x4, eb.y), p1, p2, 1.0e-6f);
        if (r.d < l0f) append_divergent<S>(out, eb.x, eb.y, ea.x, ea.y, j, i, l0);
      }
    });
    if (!ok) atomicOr(status, IPCB_STATUS_STACK);
  }
  int rounds = warp_max(nq);
  for (int k = 0; k < rounds; ++k) {
    bool has = k < nq;
    int j = has ? q[k] : 0;
    int2 eb = has ? __ldg(reinterpret_cast<const int2*>(edges) + j) : make_int2(0, 0);
    // (lower id, higher id): the reference's orientation and argument order
    const bool fwd = i < j;
    const int lo_id = fwd ? i : j, hi_id = fwd ? j : i;
    const int2 e_lo = fwd ? ea : eb, e_hi = fwd ? eb : ea;
    bool accept = false;
    if (has)
      accept = closest_point_edge_edge(load4(x4, e_lo.x), load4(x4, e_lo.y), load4(x4, e_hi.x), load4(x4, e_hi.y),
                                       1.0e-6f).d < l0f;
    int slot = warp_reserve(out.cnt, accept);
    if (accept) write_record<S>(out, slot, e_lo.x, e_lo.y, e_hi.x, e_hi.y, lo_id, hi_id, l0);
  }
}

template <class S>
__global__ void __launch_bounds__(64, 14) k_dcd_pt(const float4* __restrict__ x4, const int* __restrict__ tris,
                                                const int* __restrict__ body, const float4* __restrict__ nodes,
                                                int n_tris, const int* __restrict__ order, int first, int count,
                                                float thickness, float qpad, int exclude, ipcb_contacts out,
                                                int* status) {
  // queries: the vertices first .. first + count - 1 of the visiting order
  int t = first + blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < first + count;
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

// ---------------------------------------------------------------- fixed bodies
// world boxes of the bodies, frames, and the padded pair cull (a < b)
template <class S>
__global__ void k_body_frames(int nb, const S* __restrict__ q, const float* __restrict__ llo,
                              const float* __restrict__ lhi, double* __restrict__ frames,
                              double* __restrict__ wbox, int* __restrict__ status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double p[3], A[9], I[9], wl[3], wh[3];
  bodies::load_affine(q, b, p, A);
  const double det = bodies::det3(A);
  if (!(fabs(det) >= 1e-8)) {
    atomicOr(status, IPCB_STATUS_SINGULAR);
    for (int k = 0; k < 9; ++k) I[k] = (k % 4) == 0 ? 1.0 : 0.0;
  } else {
    bodies::inverse3(A, det, I);
  }
  double fro = 0.0;
  for (int k = 0; k < 9; ++k) {
    frames[13 * b + k] = I[k];
    fro += I[k] * I[k];
  }
  for (int k = 0; k < 3; ++k) frames[13 * b + 9 + k] = p[k];
  frames[13 * b + 12] = sqrt(fro);
  bodies::world_box(p, A, llo + 3 * b, lhi + 3 * b, wl, wh);
  for (int k = 0; k < 3; ++k) {
    wbox[6 * b + k] = wl[k];
    wbox[6 * b + 3 + k] = wh[k];
  }
}

__global__ void k_body_pair_cull(int nb, const double* __restrict__ wbox, double pad, int2* __restrict__ pairs,
                                 int capacity, int* __restrict__ count) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int a = (int)(t / nb), b = (int)(t % nb);
  bool hit = false;
  if (a < nb && a < b) {
    hit = true;
    for (int k = 0; k < 3; ++k)
      hit = hit && wbox[6 * a + k] - pad <= wbox[6 * b + 3 + k] && wbox[6 * b + k] - pad <= wbox[6 * a + 3 + k];
  }
  const int slot = warp_reserve(count, hit);
  if (hit && slot < capacity) pairs[slot] = make_int2(a, b);
}

// one thread per (body pair, source edge of pair.x): the edge mapped into
// pair.y's frame, padded by |A^-1|_F 2 thickness, against pair.y's hierarchy
template <class S>
__global__ void __launch_bounds__(128) k_fixed_dcd_ee(const float4* __restrict__ x4, const int* __restrict__ edges,
                                                      ipcb_bodies B, const int2* __restrict__ pairs, int n_pairs,
                                                      float thickness, ipcb_contacts out, int* status) {
  const int chunks = (B.max_edges + 127) / 128;
  const int pair = blockIdx.x / chunks;
  const int k = (blockIdx.x % chunks) * blockDim.x + threadIdx.x;
  const int2 pr = pairs[pair];
  const int sb = pr.x, tb = pr.y;
  const int s0 = __ldg(B.edge_off + sb), sn = __ldg(B.edge_off + sb + 1) - s0;
  const bool active = k < sn;
  const int i = active ? __ldg(B.edge_ids + s0 + k) : 0;
  const int2 ea = active ? __ldg(reinterpret_cast<const int2*>(edges) + i) : make_int2(0, 0);
  const f3 p1 = load4(x4, ea.x), p2 = load4(x4, ea.y);
  const float l0f = xmul(thickness, 2.0f);
  const S l0 = S(thickness) * S(2.0);
  const int t0 = __ldg(B.edge_off + tb), tn = __ldg(B.edge_off + tb + 1) - t0;
  int q[kQueue];
  int nq = 0;
  if (active && tn > 0) {
    const bodies::Frame f = bodies::load_frame(B.frames, tb);
    double a[3], c[3], lo[3], hi[3], pad[3];
    bodies::to_local(f, p1.x, p1.y, p1.z, a);
    bodies::to_local(f, p2.x, p2.y, p2.z, c);
    for (int r = 0; r < 3; ++r) {
      lo[r] = fmin(a[r], c[r]);
      hi[r] = fmax(a[r], c[r]);
      pad[r] = f.fro * 2.0 * (double)thickness + 1e-6 * (1.0 + fmax(fabs(lo[r]), fabs(hi[r])));
    }
    f3 qlo, qhi;
    bodies::float_box(lo, hi, pad, qlo, qhi);
    const float4* wide = reinterpret_cast<const float4*>(B.edge_wide[tb]);
    bool ok = traverse4(wide, tn, qlo, qhi, [&](int j) {
      const int e2 = __ldg(B.edge_ids + t0 + j);
      if (nq < kQueue) {
        q[nq++] = e2;
      } else {
        const int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + e2);
        CPEE r = closest_point_edge_edge(p1, p2, load4(x4, eb.x), load4(x4, eb.y), 1.0e-6f);
        if (r.d < l0f) append_divergent<S>(out, ea.x, ea.y, eb.x, eb.y, i, e2, l0);
      }
    });
    if (!ok) atomicOr(status, IPCB_STATUS_STACK);
  }
  const int rounds = warp_max(nq);
  for (int r = 0; r < rounds; ++r) {
    const bool has = r < nq;
    const int e2 = has ? q[r] : 0;
    const int2 eb = has ? __ldg(reinterpret_cast<const int2*>(edges) + e2) : make_int2(0, 0);
    bool accept = false;
    if (has) accept = closest_point_edge_edge(p1, p2, load4(x4, eb.x), load4(x4, eb.y), 1.0e-6f).d < l0f;
    const int slot = warp_reserve(out.cnt, accept);
    if (accept) write_record<S>(out, slot, ea.x, ea.y, eb.x, eb.y, i, e2, l0);
  }
}

// one thread per (body pair, direction, source vertex)
template <class S>
__global__ void __launch_bounds__(128) k_fixed_dcd_pt(const float4* __restrict__ x4, const int* __restrict__ tris,
                                                      ipcb_bodies B, const int2* __restrict__ pairs, int n_pairs,
                                                      float thickness, ipcb_contacts out, int* status) {
  const int chunks = (B.max_verts + 127) / 128;
  const int pair = blockIdx.x / chunks, dir = blockIdx.y;
  const int k = (blockIdx.x % chunks) * blockDim.x + threadIdx.x;
  const int2 pr = pairs[pair];
  const int sb = dir ? pr.y : pr.x, tb = dir ? pr.x : pr.y;
  const int s0 = __ldg(B.vert_off + sb), sn = __ldg(B.vert_off + sb + 1) - s0;
  const bool active = k < sn;
  const int i = active ? __ldg(B.vert_ids + s0 + k) : 0;
  const f3 p = load4(x4, i);
  const float l0f = xmul(thickness, 2.0f);
  const S l0 = S(thickness) * S(2.0);
  const int t0 = __ldg(B.tri_off + tb), tn = __ldg(B.tri_off + tb + 1) - t0;
  int q[kQueue];
  int nq = 0;
  if (active && tn > 0) {
    const bodies::Frame f = bodies::load_frame(B.frames, tb);
    double a[3], pad[3];
    bodies::to_local(f, p.x, p.y, p.z, a);
    for (int r = 0; r < 3; ++r) pad[r] = f.fro * 2.0 * (double)thickness + 1e-6 * (1.0 + fabs(a[r]));
    f3 qlo, qhi;
    bodies::float_box(a, a, pad, qlo, qhi);
    const float4* wide = reinterpret_cast<const float4*>(B.tri_wide[tb]);
    bool ok = traverse4(wide, tn, qlo, qhi, [&](int j) {
      const int tr = __ldg(B.tri_ids + t0 + j);
      if (nq < kQueue) {
        q[nq++] = tr;
      } else {
        const int u0 = __ldg(tris + 3 * tr), u1 = __ldg(tris + 3 * tr + 1), u2 = __ldg(tris + 3 * tr + 2);
        CPT r = closest_point_triangle(p, load4(x4, u0), load4(x4, u1), load4(x4, u2));
        if (r.d < l0f) append_divergent<S>(out, i, u1, u0, u2, i, tr, l0);
      }
    });
    if (!ok) atomicOr(status, IPCB_STATUS_STACK);
  }
  const int rounds = warp_max(nq);
  for (int r = 0; r < rounds; ++r) {
    const bool has = r < nq;
    const int tr = has ? q[r] : 0;
    const int u0 = has ? __ldg(tris + 3 * tr) : 0, u1 = has ? __ldg(tris + 3 * tr + 1) : 0,
              u2 = has ? __ldg(tris + 3 * tr + 2) : 0;
    bool accept = false;
    if (has) accept = closest_point_triangle(p, load4(x4, u0), load4(x4, u1), load4(x4, u2)).d < l0f;
    const int slot = warp_reserve(out.cnt, accept);
    if (accept) write_record<S>(out, slot, i, u1, u0, u2, i, tr, l0);
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

int ipcb_dcd_ee_range(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness,
                      float query_pad, int exclude_same_body, int first, int count, ipcb_contacts* out, int* status,
                      ipcb_stream s) {
  if (!soup || !x4 || !bvh || !out || !status || bvh->n != soup->n_edges) return IPCB_E_ARG;
  int n = soup->n_edges;
  if (first < 0 || count < 0 || first > n || count > n - first) return IPCB_E_ARG;
  if (count == 0) return IPCB_OK;
  // 64-thread blocks: queries end at different depths, and a small block
  // frees its slot sooner (measured a few percent faster than 128)
  dim3 grid(div_up(count, 64));
  if (soup->fp64)
    k_dcd_ee<double><<<grid, 64, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, soup->body,
                                                        (const float4*)bvh->wide, bvh->sorted, n, first, count,
                                                        thickness, query_pad, exclude_same_body, *out, status);
  else
    k_dcd_ee<float><<<grid, 64, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, soup->body,
                                                       (const float4*)bvh->wide, bvh->sorted, n, first, count,
                                                       thickness, query_pad, exclude_same_body, *out, status);
  return check_launch("ipcb_dcd_ee");
}

int ipcb_dcd_ee(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness, float query_pad,
                int exclude_same_body, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup) return IPCB_E_ARG;
  return ipcb_dcd_ee_range(soup, x4, bvh, thickness, query_pad, exclude_same_body, 0, soup->n_edges, out, status, s);
}

int ipcb_dcd_pt_range(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness,
                      float query_pad, int exclude_same_body, const int* query_order, int first, int count,
                      ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup || !x4 || !bvh || !out || !status || bvh->n != soup->n_tris) return IPCB_E_ARG;
  int nv = soup->n_verts;
  if (first < 0 || count < 0 || first > nv || count > nv - first) return IPCB_E_ARG;
  if (count == 0 || soup->n_tris == 0) return IPCB_OK;
  dim3 grid(div_up(count, 64));
  if (soup->fp64)
    k_dcd_pt<double><<<grid, 64, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, soup->body,
                                                        (const float4*)bvh->wide, soup->n_tris, query_order, first,
                                                        count, thickness, query_pad, exclude_same_body, *out, status);
  else
    k_dcd_pt<float><<<grid, 64, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, soup->body,
                                                       (const float4*)bvh->wide, soup->n_tris, query_order, first,
                                                       count, thickness, query_pad, exclude_same_body, *out, status);
  return check_launch("ipcb_dcd_pt");
}

int ipcb_dcd_pt(const ipcb_soup* soup, const float* x4, const ipcb_lbvh* bvh, float thickness, float query_pad,
                int exclude_same_body, const int* query_order, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup) return IPCB_E_ARG;
  return ipcb_dcd_pt_range(soup, x4, bvh, thickness, query_pad, exclude_same_body, query_order, 0, soup->n_verts,
                           out, status, s);
}


static bool bodies_ok(const ipcb_bodies* B) {
  return B && B->n_bodies > 0 && B->local_lower && B->local_upper && B->edge_off && B->edge_ids && B->tri_off &&
         B->tri_ids && B->vert_off && B->vert_ids && B->edge_wide && B->tri_wide && B->frames && B->motion;
}

int ipcb_body_pairs(const ipcb_bodies* B, int fp64, const void* q, double padding, int* pairs, int capacity,
                    int* count, int* status, ipcb_stream s) {
  if (!bodies_ok(B) || !q || !pairs || capacity < 0 || !count || !status) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int nb = B->n_bodies;
  double* wbox = B->frames + 13 * (size_t)nb;  // world boxes: 6 doubles per body after the frames
  if (fp64)
    k_body_frames<double><<<div_up(nb, 128), 128, 0, st>>>(nb, (const double*)q, B->local_lower, B->local_upper,
                                                            B->frames, wbox, status);
  else
    k_body_frames<float><<<div_up(nb, 128), 128, 0, st>>>(nb, (const float*)q, B->local_lower, B->local_upper,
                                                           B->frames, wbox, status);
  k_body_pair_cull<<<div_up((long long)nb * nb, 256), 256, 0, st>>>(nb, wbox, padding, (int2*)pairs, capacity, count);
  return check_launch("ipcb_body_pairs");
}

int ipcb_fixed_dcd_ee(const ipcb_soup* soup, const float* x4, const ipcb_bodies* B, const int* pairs, int n_pairs,
                      float thickness, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup || !x4 || !bodies_ok(B) || !pairs || n_pairs < 0 || !out || !status) return IPCB_E_ARG;
  if (n_pairs == 0 || B->max_edges == 0) return IPCB_OK;
  dim3 grid(div_up(B->max_edges, 128) * n_pairs);
  if (soup->fp64)
    k_fixed_dcd_ee<double><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, *B,
                                                              (const int2*)pairs, n_pairs, thickness, *out, status);
  else
    k_fixed_dcd_ee<float><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->edges, *B,
                                                             (const int2*)pairs, n_pairs, thickness, *out, status);
  return check_launch("ipcb_fixed_dcd_ee");
}

int ipcb_fixed_dcd_pt(const ipcb_soup* soup, const float* x4, const ipcb_bodies* B, const int* pairs, int n_pairs,
                      float thickness, ipcb_contacts* out, int* status, ipcb_stream s) {
  if (!soup || !x4 || !bodies_ok(B) || !pairs || n_pairs < 0 || !out || !status) return IPCB_E_ARG;
  if (n_pairs == 0 || B->max_verts == 0) return IPCB_OK;
  dim3 grid(div_up(B->max_verts, 128) * n_pairs, 2);
  if (soup->fp64)
    k_fixed_dcd_pt<double><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, *B,
                                                              (const int2*)pairs, n_pairs, thickness, *out, status);
  else
    k_fixed_dcd_pt<float><<<grid, 128, 0, (cudaStream_t)s>>>((const float4*)x4, soup->triangles, *B,
                                                             (const int2*)pairs, n_pairs, thickness, *out, status);
  return check_launch("ipcb_fixed_dcd_pt");
}

}  // extern "C"
