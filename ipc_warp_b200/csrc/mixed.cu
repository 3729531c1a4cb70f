// Mixed FEM + affine-body Newton systems (deformable tets and affine bodies in
// one solve, e.g. affine wrecking balls striking a wall of FEM cubes).
//
// Unknowns: one vec3 array q of n_fem + 4 n_bodies entries -- the FEM vertex
// positions, then per affine body p, a0, a1, a2 (x = p + A r, r the vertex's
// body-local rest position; the layout of affine_body_dynamics.py:42-48).
// The contact soup lists the FEM vertices first (vertex v < n_fem is unknown
// v) and then the affine bodies' vertices (vertex v >= n_fem belongs to
// body[v - n_fem]).  The Jacobian of a vertex is I (FEM), [I, r0 I, r1 I,
// r2 I] (free body) or empty (fixed body), so the contact part of the
// Newton matrix is J^T H J: the 3x3 vertex block (u, v) of a contact record
// becomes n_u n_v unknown blocks w_u,a w_v,c H_uv (n = 1, 4 or 0), written
// compactly after a count and a scan, and the vertex contact force reduces
// the same way into the gradient.  A pin holds a body-local point of an
// affine body at a world point with a quadratic penalty (a pendulum rod).
#include "common.cuh"
#include "scan.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

template <class S>
struct Mixed {
  int n_fem, n_verts, n_bodies;
  const int* body;
  const int* fixed;
  const S* rest;
};

template <class S>
Mixed<S> mview(const ipcb_mixed* m) {
  return Mixed<S>{m->n_fem, m->n_verts, m->n_bodies, m->body, m->fixed, (const S*)m->rest};
}

// unknowns of vertex v: count (0, 1 or 4), first unknown, weights (1, r)
template <class S>
IPCB_D int vertex_dofs(const Mixed<S>& M, int v, int& first, S w[4]) {
  if (v < M.n_fem) {
    first = v;
    w[0] = S(1);
    return 1;
  }
  const int b = __ldg(M.body + (v - M.n_fem));
  if (__ldg(M.fixed + b) != 0) return 0;
  first = M.n_fem + 4 * b;
  w[0] = S(1);
  w[1] = __ldg(M.rest + 3 * v);
  w[2] = __ldg(M.rest + 3 * v + 1);
  w[3] = __ldg(M.rest + 3 * v + 2);
  return 4;
}

template <class S>
__global__ void k_mixed_map(Mixed<S> M, const S* __restrict__ q, S* __restrict__ x) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  if (v >= M.n_verts) return;
  v3<S> out;
  if (v < M.n_fem) {
    out = load3(q, v);
  } else {
    const int o = M.n_fem + 4 * __ldg(M.body + (v - M.n_fem));
    const v3<S> r = load3(M.rest, v);
    out = load3(q, o) + load3(q, o + 1) * r.x + load3(q, o + 2) * r.y + load3(q, o + 3) * r.z;
  }
  x[3 * v] = out.x;
  x[3 * v + 1] = out.y;
  x[3 * v + 2] = out.z;
}

// g[unknowns of v] += scale J_v^T f_v.  FEM unknowns belong to one vertex
// each (plain add); a warp whose affine vertices share one body sums in
// registers and adds once.
template <class S>
__global__ void k_mixed_reduce_force(Mixed<S> M, const S* __restrict__ f, S scale, S* __restrict__ g) {
  const int v = blockIdx.x * blockDim.x + threadIdx.x;
  const bool in = v < M.n_verts;
  if (in && v < M.n_fem) {
    const v3<S> fv = load3(f, v);
    g[3 * v] += scale * fv.x;
    g[3 * v + 1] += scale * fv.y;
    g[3 * v + 2] += scale * fv.z;
  }
  // warp-uniform from here: lanes with no affine vertex take part with b = -1
  int b = -1;
  S c[12];
#pragma unroll
  for (int k = 0; k < 12; ++k) c[k] = S(0);
  if (in && v >= M.n_fem) {
    b = __ldg(M.body + (v - M.n_fem));
    if (__ldg(M.fixed + b) != 0) b = -1;
  }
  if (b >= 0) {
    const v3<S> fv = load3(f, v) * scale, r = load3(M.rest, v);
    const S w[4] = {S(1), r.x, r.y, r.z};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      c[3 * k] = w[k] * fv.x;
      c[3 * k + 1] = w[k] * fv.y;
      c[3 * k + 2] = w[k] * fv.z;
    }
  }
  int lead = b;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) lead = max(lead, __shfl_xor_sync(0xffffffffu, lead, o));
  if (lead < 0) return;
  if (__all_sync(0xffffffffu, b == lead || b < 0)) {
#pragma unroll
    for (int k = 0; k < 12; ++k)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], o);
    if ((threadIdx.x & 31) == 0) {
      S* d = g + 3 * ((size_t)M.n_fem + 4 * (size_t)lead);
#pragma unroll
      for (int k = 0; k < 12; ++k) atomicAdd(d + k, c[k]);
    }
  } else if (b >= 0) {
    S* d = g + 3 * ((size_t)M.n_fem + 4 * (size_t)b);
#pragma unroll
    for (int k = 0; k < 12; ++k) atomicAdd(d + k, c[k]);
  }
}

template <class S>
IPCB_D bool block_live(int s, const S* __restrict__ vals, const unsigned short* __restrict__ mask) {
  if (mask) return (__ldg(mask + (s >> 4)) >> (s & 15)) & 1u;
  bool nz = false;
#pragma unroll
  for (int k = 0; k < 9; ++k) nz |= vals[9LL * s + k] != S(0);
  return nz;
}

template <class S>
__global__ void k_mixed_count(Mixed<S> M, int n_src, const int* __restrict__ rows, const int* __restrict__ cols,
                              const S* __restrict__ vals, const unsigned short* __restrict__ mask,
                              int* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_src) return;
  int c = 0;
  if (block_live(s, vals, mask)) {
    int f;
    S w[4];
    c = vertex_dofs(M, __ldg(rows + s), f, w) * vertex_dofs(M, __ldg(cols + s), f, w);
  }
  counts[s] = c;
}

template <class S>
__global__ void k_mixed_fill(Mixed<S> M, int n_src, const int* __restrict__ rows, const int* __restrict__ cols,
                             const S* __restrict__ vals, const int* __restrict__ start, S scale, int capacity,
                             int* __restrict__ drows, int* __restrict__ dcols, S* __restrict__ dvals) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_src) return;
  const int o = __ldg(start + s);
  if (__ldg(start + s + 1) == o) return;  // a dropped block
  int fu, fv;
  S wu[4], wv[4];
  const int nu = vertex_dofs(M, __ldg(rows + s), fu, wu);
  const int nv = vertex_dofs(M, __ldg(cols + s), fv, wv);
  if (nu == 0 || nv == 0) return;
  S h[9];
#pragma unroll
  for (int k = 0; k < 9; ++k) h[k] = scale * vals[9LL * s + k];
  int k = o;
  for (int a = 0; a < nu; ++a)
    for (int c = 0; c < nv; ++c, ++k) {
      if (k >= capacity) return;
      const S w = wu[a] * wv[c];
      drows[k] = fu + a;
      dcols[k] = fv + c;
#pragma unroll
      for (int q = 0; q < 9; ++q) dvals[9LL * k + q] = w * h[q];
    }
}

__global__ void k_mixed_total(const int* __restrict__ total, int capacity, int* __restrict__ n_out,
                              int* __restrict__ status) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    *n_out = *total;
    if (*total > capacity) atomicOr(status, IPCB_STATUS_PATTERN);
  }
}

// one thread per (body, i, j) of the pinned bodies: the block h2 k w_i w_j I,
// the gradient h2 k w_i (x_pin - target) (j == 0) and the energy
// 0.5 h2 k |x_pin - target|^2 (i == j == 0), w = (1, pin_rest)
template <class S>
__global__ void k_mixed_pins(Mixed<S> M, const S* __restrict__ q, const S* __restrict__ pin_rest,
                             const S* __restrict__ pin_target, const S* __restrict__ pin_k, S h2,
                             int* __restrict__ rows, int* __restrict__ cols, S* __restrict__ vals,
                             S* __restrict__ g, double* __restrict__ energy) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 16 * M.n_bodies) return;
  const int b = t >> 4, i = (t >> 2) & 3, j = t & 3;
  const S k = __ldg(pin_k + b);
  const bool live = k != S(0) && __ldg(M.fixed + b) == 0;
  const v3<S> r = load3(pin_rest, b);
  const S w[4] = {S(1), r.x, r.y, r.z};
  const int o = M.n_fem + 4 * b;
  if (rows) {
    rows[t] = o + i;
    cols[t] = o + j;
    const S d = live ? h2 * k * w[i] * w[j] : S(0);
    S* dst = vals + 9LL * t;
#pragma unroll
    for (int q = 0; q < 9; ++q) dst[q] = (q == 0 || q == 4 || q == 8) ? d : S(0);
  }
  if (!live || j != 0 || (!g && !energy)) return;
  const v3<S> e = load3(q, o) + load3(q, o + 1) * r.x + load3(q, o + 2) * r.y + load3(q, o + 3) * r.z -
                  load3(pin_target, b);
  if (g) {
    const S s = h2 * k * w[i];
    g[3 * (o + i)] += s * e.x;
    g[3 * (o + i) + 1] += s * e.y;
    g[3 * (o + i) + 2] += s * e.z;
  }
  if (energy && i == 0) atomicAdd(energy, 0.5 * (double)h2 * (double)k * (double)dot(e, e));
}

inline bool mixed_ok(const ipcb_mixed* m) {
  return m && m->n_fem >= 0 && m->n_verts >= m->n_fem && m->n_bodies >= 0 &&
         (m->n_verts == m->n_fem || (m->body && m->fixed && m->rest));
}

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_mixed_map(const ipcb_mixed* m, const void* q, void* x, ipcb_stream s) {
  if (!mixed_ok(m) || !q || !x) return IPCB_E_ARG;
  if (m->n_verts == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(m->n_verts, 256);
  if (m->fp64) k_mixed_map<double><<<g, 256, 0, st>>>(mview<double>(m), (const double*)q, (double*)x);
  else k_mixed_map<float><<<g, 256, 0, st>>>(mview<float>(m), (const float*)q, (float*)x);
  return check_launch("ipcb_mixed_map");
}

int ipcb_mixed_reduce_force(const ipcb_mixed* m, const void* vertex_force, double scale, void* gradient,
                            ipcb_stream s) {
  if (!mixed_ok(m) || !vertex_force || !gradient) return IPCB_E_ARG;
  if (m->n_verts == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(m->n_verts, 256);
  if (m->fp64)
    k_mixed_reduce_force<double><<<g, 256, 0, st>>>(mview<double>(m), (const double*)vertex_force, scale,
                                                    (double*)gradient);
  else
    k_mixed_reduce_force<float><<<g, 256, 0, st>>>(mview<float>(m), (const float*)vertex_force, (float)scale,
                                                   (float*)gradient);
  return check_launch("ipcb_mixed_reduce_force");
}

size_t ipcb_mixed_hessian_workspace(int n_src) {
  const int n = n_src > 0 ? n_src : 1;
  return al((size_t)(n + 1) * 4) + 256 + scan::scratch_bytes(n + 1);
}

int ipcb_mixed_reduce_hessian(const ipcb_mixed* m, int n_src, const int* rows, const int* cols, const void* vals,
                              const unsigned short* block_mask, double scale, int capacity, int* drows, int* dcols,
                              void* dvals, int* n_out, int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!mixed_ok(m) || n_src < 0 || capacity < 0 || !n_out || !status) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (n_src == 0) {
    cudaMemsetAsync(n_out, 0, sizeof(int), st);
    return check_launch("ipcb_mixed_reduce_hessian");
  }
  if (!rows || !cols || !vals || !ws || ws_bytes < ipcb_mixed_hessian_workspace(n_src)) return IPCB_E_ARG;
  if (capacity > 0 && (!drows || !dcols || !dvals)) return IPCB_E_ARG;
  int* start = (int*)ws;
  int* total = (int*)((char*)ws + al((size_t)(n_src + 1) * 4));
  void* scratch = (char*)total + 256;
  const int g = div_up(n_src, 256);
  if (m->fp64)
    k_mixed_count<double><<<g, 256, 0, st>>>(mview<double>(m), n_src, rows, cols, (const double*)vals, block_mask,
                                             start);
  else
    k_mixed_count<float><<<g, 256, 0, st>>>(mview<float>(m), n_src, rows, cols, (const float*)vals, block_mask,
                                            start);
  cudaMemsetAsync(start + n_src, 0, sizeof(int), st);
  scan::exclusive<int>(start, n_src + 1, scratch, total, st);
  // start[n_src] = the total, so every source's range is [start[s], start[s + 1])
  if (m->fp64)
    k_mixed_fill<double><<<g, 256, 0, st>>>(mview<double>(m), n_src, rows, cols, (const double*)vals, start, scale,
                                            capacity, drows, dcols, (double*)dvals);
  else
    k_mixed_fill<float><<<g, 256, 0, st>>>(mview<float>(m), n_src, rows, cols, (const float*)vals, start,
                                           (float)scale, capacity, drows, dcols, (float*)dvals);
  k_mixed_total<<<1, 32, 0, st>>>(total, capacity, n_out, status);
  return check_launch("ipcb_mixed_reduce_hessian");
}

int ipcb_mixed_pins(const ipcb_mixed* m, const void* q, const void* pin_rest, const void* pin_target,
                    const void* pin_k, double h2, int* rows, int* cols, void* vals, void* gradient, double* energy,
                    ipcb_stream s) {
  if (!mixed_ok(m) || !q || !pin_rest || !pin_target || !pin_k) return IPCB_E_ARG;
  if ((rows || cols || vals) && !(rows && cols && vals)) return IPCB_E_ARG;
  if (m->n_bodies == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(16 * m->n_bodies, 128);
  if (m->fp64)
    k_mixed_pins<double><<<g, 128, 0, st>>>(mview<double>(m), (const double*)q, (const double*)pin_rest,
                                            (const double*)pin_target, (const double*)pin_k, h2, rows, cols,
                                            (double*)vals, (double*)gradient, energy);
  else
    k_mixed_pins<float><<<g, 128, 0, st>>>(mview<float>(m), (const float*)q, (const float*)pin_rest,
                                           (const float*)pin_target, (const float*)pin_k, (float)h2, rows, cols,
                                           (float*)vals, (float*)gradient, energy);
  return check_launch("ipcb_mixed_pins");
}

}  // extern "C"
