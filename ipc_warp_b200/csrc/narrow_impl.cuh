// Narrow-phase device code shared by the per-list kernels (narrow.cu) and
// the batched work-queue kernel (terms.cu).  See narrow.cu for the method.
#pragma once
#include "common.cuh"
#include "geom.cuh"

namespace ipcb {
namespace {

constexpr int kMaxH = 6;  // grad + up to 5 eigenvectors

// ------------------------------------------------------------------ barrier
struct Barrier {
  double b, db, d2b;
};
IPCB_D Barrier barrier(double x, double xh, double kappa) {
  Barrier r{0.0, 0.0, 0.0};
  if (!(x < xh)) return r;
  double dx = x - xh, lg = log(x / xh);
  r.b = -kappa * dx * dx * lg;
  r.db = kappa * (-2.0 * dx * lg - dx * dx / x);
  r.d2b = kappa * (-2.0 * lg - 4.0 * dx / x + dx * dx / (x * x));
  return r;
}

// ------------------------------------------------------------------ Jacobi
template <class T, int N>
IPCB_D void jacobi(T (&a)[N][N], T (&v)[N][N]) {
#pragma unroll
  for (int i = 0; i < N; ++i)
#pragma unroll
    for (int j = 0; j < N; ++j) v[i][j] = (i == j) ? T(1) : T(0);
  const T tiny = sizeof(T) == 4 ? T(1e-14) : T(1e-30);
  for (int sweep = 0; sweep < 12; ++sweep) {
    T off = 0, dg = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
      dg += a[i][i] * a[i][i];
#pragma unroll
      for (int j = i + 1; j < N; ++j) off += a[i][j] * a[i][j];
    }
    if (off <= tiny * dg) break;
    // cyclic sweep of symmetric rotations: each (p, q) rotation updates the
    // two pivots in closed form, zeroes a_pq, and rotates the other entries
    // of rows/columns p and q once (a is kept symmetric)
#pragma unroll
    for (int p = 0; p < N - 1; ++p)
#pragma unroll
      for (int q = p + 1; q < N; ++q) {
        const T apq = a[p][q];
        if (apq != T(0)) {
          const T theta = (a[q][q] - a[p][p]) / (T(2) * apq);
          const T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
          const T c = T(1) / sqrt(t * t + T(1)), s = t * c;
          a[p][p] -= t * apq;
          a[q][q] += t * apq;
          a[p][q] = a[q][p] = T(0);
#pragma unroll
          for (int k = 0; k < N; ++k) {
            if (k == p || k == q) continue;
            const T akp = a[k][p], akq = a[k][q];
            a[k][p] = a[p][k] = c * akp - s * akq;
            a[k][q] = a[q][k] = s * akp + c * akq;
          }
#pragma unroll
          for (int k = 0; k < N; ++k) {
            const T vkp = v[k][p], vkq = v[k][q];
            v[k][p] = c * vkp - s * vkq;
            v[k][q] = s * vkp + c * vkq;
          }
        }
      }
  }
}

// --------------------------------------------------------------- features
struct Feature {
  int np;         // number of distance parameters: 0 PP, 1 PE, 2 PT/EE
  double c[4];    // r = sum_k c_k x_k over the 4 record slots
  double D[2][4]; // dc/dtau_j
  d3 E[2];        // dr/dtau_j
  d3 n;           // unit normal of the parameter span (np >= 1)
  double rho;     // signed distance along n
  d3 r;           // closest-point difference
};

IPCB_D d3 dnorm(d3 a) { return a * (1.0 / sqrt(dot(a, a))); }

// register-resident selection of x[s] for a runtime slot s
IPCB_D d3 pick(const d3* x, int s) { return s == 0 ? x[0] : (s == 1 ? x[1] : (s == 2 ? x[2] : x[3])); }

IPCB_D void feature_pp(Feature& f, const d3* x, int sa, int sb) {
  f.np = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) f.c[k] = k == sa ? 1.0 : (k == sb ? -1.0 : 0.0);
  f.r = pick(x, sa) - pick(x, sb);
}

IPCB_D void feature_pe(Feature& f, const d3* x, int sp, int s0, int s1) {
  f.np = 1;
  d3 p = pick(x, sp), e0 = pick(x, s0), e1 = pick(x, s1), e = e1 - e0;
  double t = dot(p - e0, e) / dot(e, e);
  d3 r = p - e0 - e * t;
  double rl = sqrt(dot(r, r));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    f.c[k] = k == sp ? 1.0 : (k == s0 ? -(1.0 - t) : (k == s1 ? -t : 0.0));
    f.D[0][k] = k == s0 ? 1.0 : (k == s1 ? -1.0 : 0.0);
    f.D[1][k] = 0.0;
  }
  f.E[0] = e0 - e1;
  f.rho = rl;
  f.n = r * (1.0 / rl);
  f.r = r;
}

IPCB_D void feature_pt(Feature& f, const d3* x) {
  f.np = 2;
  d3 e1 = x[2] - x[1], e2 = x[3] - x[1], w = x[0] - x[1];
  double g11 = dot(e1, e1), g12 = dot(e1, e2), g22 = dot(e2, e2);
  double b1 = dot(e1, w), b2 = dot(e2, w), det = g11 * g22 - g12 * g12;
  double be = (g22 * b1 - g12 * b2) / det, ga = (g11 * b2 - g12 * b1) / det;
  f.n = dnorm(cross(e1, e2));
  f.rho = dot(w, f.n);
  f.r = f.n * f.rho;
  f.c[0] = 1.0; f.c[1] = -1.0 + be + ga; f.c[2] = -be; f.c[3] = -ga;
  f.D[0][0] = 0; f.D[0][1] = 1; f.D[0][2] = -1; f.D[0][3] = 0;
  f.D[1][0] = 0; f.D[1][1] = 1; f.D[1][2] = 0; f.D[1][3] = -1;
  f.E[0] = e1 * -1.0;
  f.E[1] = e2 * -1.0;
}

IPCB_D void feature_ee(Feature& f, const d3* x) {
  f.np = 2;
  d3 ea = x[1] - x[0], eb = x[3] - x[2], w = x[0] - x[2];
  double g11 = dot(ea, ea), g12 = -dot(ea, eb), g22 = dot(eb, eb);
  double r1 = -dot(ea, w), r2 = dot(eb, w), det = g11 * g22 - g12 * g12;
  double s = (g22 * r1 - g12 * r2) / det, t = (g11 * r2 - g12 * r1) / det;
  f.n = dnorm(cross(ea, eb));
  f.rho = dot(w, f.n);
  f.r = f.n * f.rho;
  f.c[0] = 1.0 - s; f.c[1] = s; f.c[2] = -(1.0 - t); f.c[3] = -t;
  f.D[0][0] = -1; f.D[0][1] = 1; f.D[0][2] = 0; f.D[0][3] = 0;
  f.D[1][0] = 0; f.D[1][1] = 0; f.D[1][2] = 1; f.D[1][3] = -1;
  f.E[0] = ea;
  f.E[1] = eb * -1.0;
}

// Negative spectral part of hess(d^2) as sum_e lam_e u_e u_e^T; fills h[1..]
// and w[1..] (w = scale * lam).  Returns the number of vectors written.
template <class T, int NP, int MH>
IPCB_D int nsd_subspace(const Feature& f, double scale, T (&h)[MH][12], T (&w)[MH]) {
  static_assert(MH >= 2 * NP + 2, "room for the gradient and every eigenvector");
  constexpr int NZ = 1 + NP, NS = 2 * NP + 1;
  double cn = sqrt(f.c[0] * f.c[0] + f.c[1] * f.c[1] + f.c[2] * f.c[2] + f.c[3] * f.c[3]);
  double ch[4], fv[NP][4];
#pragma unroll
  for (int k = 0; k < 4; ++k) ch[k] = f.c[k] / cn;
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    double v[4];
    double pc = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) pc += f.D[j][k] * ch[k];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = f.D[j][k] - pc * ch[k];
#pragma unroll
    for (int q = 0; q < j; ++q) {
      double pf = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) pf += v[k] * fv[q][k];
#pragma unroll
      for (int k = 0; k < 4; ++k) v[k] -= pf * fv[q][k];
    }
    double vn = rsqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3]);
#pragma unroll
    for (int k = 0; k < 4; ++k) fv[j][k] = v[k] * vn;
  }
  double Gi[NP][NP];
  if (NP == 1) {
    Gi[0][0] = 1.0 / dot(f.E[0], f.E[0]);
  } else {
    double g00 = dot(f.E[0], f.E[0]), g01 = dot(f.E[0], f.E[NP - 1]), g11 = dot(f.E[NP - 1], f.E[NP - 1]);
    double idet = 1.0 / (g00 * g11 - g01 * g01);
    Gi[0][0] = g11 * idet;
    Gi[NP - 1][NP - 1] = g00 * idet;
    Gi[0][NP - 1] = -g01 * idet;
    Gi[NP - 1][0] = -g01 * idet;
  }
  d3 th[NP];
  th[0] = dnorm(f.E[0]);
  if (NP == 2) th[NP - 1] = cross(f.n, th[0]);
  double Dm[NP][NZ], Tm[NP][NP];
#pragma unroll
  for (int j = 0; j < NP; ++j) {
    double s0 = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) s0 += f.D[j][k] * ch[k];
    Dm[j][0] = s0;
#pragma unroll
    for (int a = 0; a < NP; ++a) {
      double sa = 0;
#pragma unroll
      for (int k = 0; k < 4; ++k) sa += f.D[j][k] * fv[a][k];
      Dm[j][1 + a] = sa;
    }
    d3 ed = f.E[0] * Gi[j][0];
#pragma unroll
    for (int k = 1; k < NP; ++k) ed = ed + f.E[k] * Gi[j][k];
#pragma unroll
    for (int i = 0; i < NP; ++i) Tm[j][i] = dot(th[i], ed);
  }
  T M[NS][NS], V[NS][NS];
  const double r2 = -2.0 * f.rho * f.rho, rc = -2.0 * f.rho * cn;
#pragma unroll
  for (int a = 0; a < NZ; ++a)
#pragma unroll
    for (int b = 0; b < NZ; ++b) {
      double s = 0;
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int j = 0; j < NP; ++j) s += Dm[i][a] * Gi[i][j] * Dm[j][b];
      M[a][b] = T(r2 * s + ((a == 0 && b == 0) ? 2.0 * cn * cn : 0.0));
    }
#pragma unroll
  for (int a = 0; a < NZ; ++a)
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      double s = 0;
#pragma unroll
      for (int j = 0; j < NP; ++j) s += Dm[j][a] * Tm[j][i];
      M[a][NZ + i] = M[NZ + i][a] = T(rc * s);
    }
#pragma unroll
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int j = 0; j < NP; ++j) M[NZ + i][NZ + j] = T(0);
  jacobi<T, NS>(M, V);
  // basis: phi_0 = ch (x) n, phi_{1+a} = f_a (x) n, phi_{NZ+i} = ch (x) th_i
  T nf[3] = {T(f.n.x), T(f.n.y), T(f.n.z)};
  T tf[NP][3];
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    tf[i][0] = T(th[i].x);
    tf[i][1] = T(th[i].y);
    tf[i][2] = T(th[i].z);
  }
  int cnt = 0;
#pragma unroll
  for (int e = 0; e < NS; ++e) {
    T lam = M[e][e];
    // spatial parts: vector on ch (x) s and on f_a (x) n
    T sc[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      T v = V[0][e] * nf[k];
#pragma unroll
      for (int i = 0; i < NP; ++i) v += V[NZ + i][e] * tf[i][k];
      sc[k] = v;
    }
#pragma unroll
    for (int vtx = 0; vtx < 4; ++vtx) {
      T fa = T(0);
#pragma unroll
      for (int a = 0; a < NP; ++a) fa += V[1 + a][e] * T(fv[a][vtx]);
#pragma unroll
      for (int k = 0; k < 3; ++k) h[1 + e][3 * vtx + k] = T(ch[vtx]) * sc[k] + fa * nf[k];
    }
    w[1 + e] = lam < T(0) ? T(scale) * lam : T(0);
    cnt = e + 1;
  }
  return cnt;
}

template <class S>
IPCB_D v3<S> ldx(const S* __restrict__ x, int i) {
  return load3(x, i);
}

struct Rec {
  int4 id;
  bool active;
};

template <class S>
IPCB_D int list_count(const ipcb_contacts& L, int n) {
  if (n >= 0) return n;
  int c = *L.cnt;
  return c < L.capacity ? c : L.capacity;
}

// Feature selection for an EE record (dynamic_contacts.py:49-108).  Uses the
// float32 (s, t) of the segment closest points.
template <class S>
IPCB_D void ee_dispatch(Feature& f, const d3* xd, float ds, float dt, bool near_par) {
  S s = S(ds), t = S(dt);
  const S feps = S(1.0e-6), one = S(1.0), hi = S(1.0) - S(1.0e-6);
  bool sb = s <= feps || s >= hi;
  bool tb = t <= feps || t >= hi;
  if (sb && tb) {
    feature_pp(f, xd, s >= hi ? 1 : 0, t >= hi ? 3 : 2);
    return;
  }
  if (sb) {
    feature_pe(f, xd, s >= hi ? 1 : 0, 2, 3);
    return;
  }
  if (tb) {
    feature_pe(f, xd, t >= hi ? 3 : 2, 0, 1);
    return;
  }
  if (near_par) {
    S ds0 = s, ds1 = xsub(one, s), dt0 = t, dt1 = xsub(one, t);
    S mn = tmin(tmin(ds0, ds1), tmin(dt0, dt1));
    if (mn == ds0) feature_pe(f, xd, 0, 2, 3);
    else if (mn == ds1) feature_pe(f, xd, 1, 2, 3);
    else if (mn == dt0) feature_pe(f, xd, 2, 0, 1);
    else feature_pe(f, xd, 3, 0, 1);
    return;
  }
  feature_ee(f, xd);
}

// dynamic_contacts.py:111-125; t: the closest-point region type of the record
IPCB_D int pt_dispatch(Feature& f, int t, const d3* xd) {
  if (t <= 2) feature_pp(f, xd, 0, t + 1);
  else if (t == 3) feature_pe(f, xd, 0, 1, 2);
  else if (t == 4) feature_pe(f, xd, 0, 1, 3);
  else if (t == 5) feature_pe(f, xd, 0, 2, 3);
  else feature_pt(f, xd);
  return t;
}

template <class S>
IPCB_D S ee_eps_x(const S* __restrict__ xcs, int4 id) {
  v3<S> r0 = load3(xcs, id.x), r1 = load3(xcs, id.y), r2 = load3(xcs, id.z), r3 = load3(xcs, id.w);
  v3<S> ea = esub(r1, r0), eb = esub(r3, r2);
  return xmul(xmul(S(1.0e-3), edot(ea, ea)), edot(eb, eb));
}

// 16-byte stores of n (multiple of 16 bytes) values; dst 16-byte aligned
IPCB_D void store16(float* dst, const float* v, int n) {
#pragma unroll
  for (int k = 0; k < n; k += 4) *reinterpret_cast<float4*>(dst + k) = make_float4(v[k], v[k + 1], v[k + 2], v[k + 3]);
}
IPCB_D void store16(double* dst, const double* v, int n) {
#pragma unroll
  for (int k = 0; k < n; k += 2) *reinterpret_cast<double2*>(dst + k) = make_double2(v[k], v[k + 1]);
}

// inactive record: zero blocks at (0, 0) (the reference's zero-initialised
// triplet arrays)
template <class S>
IPCB_D void write_zero(int* rows, int* cols, S* vals, long long base) {
  int4 z = make_int4(0, 0, 0, 0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    reinterpret_cast<int4*>(rows + base)[k] = z;
    reinterpret_cast<int4*>(cols + base)[k] = z;
  }
  S zv[72];
#pragma unroll
  for (int k = 0; k < 72; ++k) zv[k] = S(0);
  store16(vals + 9 * base, zv, 72);
  store16(vals + 9 * base + 72, zv, 72);
}

// 16 blocks of H = sum_m w_m h_m h_m^T; the record's 144 values are
// contiguous and 16-byte aligned (576 B per record in float), written as two
// halves of 8 blocks with vector stores.
template <class S, class T, int MH>
IPCB_D unsigned write_blocks(const int4 id, int* rows, int* cols, S* vals, long long base, const T (&h)[MH][12],
                             const T (&w)[MH], int nh) {
  unsigned mask = 0;
  const int vid[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
  for (int ii = 0; ii < 4; ++ii) {
    reinterpret_cast<int4*>(rows + base)[ii] = make_int4(vid[ii], vid[ii], vid[ii], vid[ii]);
    reinterpret_cast<int4*>(cols + base)[ii] = make_int4(vid[0], vid[1], vid[2], vid[3]);
  }
  // one block row (4 blocks, 144 B in float) at a time: w_m h_m[3 ii + a] is
  // formed once per row component and the staging buffer stays at 36 values,
  // which keeps the kernel at <= 168 registers (3 CTAs of 128 per SM)
#pragma unroll
  for (int ii = 0; ii < 4; ++ii) {
    S buf[36];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      T wh[MH];
#pragma unroll
      for (int m = 0; m < MH; ++m) wh[m] = m < nh ? w[m] * h[m][3 * ii + a] : T(0);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          T v = T(0);
#pragma unroll
          for (int m = 0; m < MH; ++m)
            if (m < nh) v += wh[m] * h[m][3 * jj + b];  // rows m >= nh of h are not set
          buf[jj * 9 + 3 * a + b] = S(v);
          if (S(v) != S(0)) mask |= 1u << (ii * 4 + jj);
        }
    }
    store16(vals + 9 * base + 36 * ii, buf, 36);
  }
  return mask;
}

template <class S>
IPCB_D void add_force(S* b, int4 id, const double (&fc)[12]) {
  const int vid[4] = {id.x, id.y, id.z, id.w};
#pragma unroll
  for (int k = 0; k < 4; ++k)
#pragma unroll
    for (int c = 0; c < 3; ++c) atomicAdd(b + 3 * vid[k] + c, S(fc[3 * k + c]));
}

// mollifier value and gradient for near-parallel edges
IPCB_D void mollifier(const d3* xd, double eps_x, double& mv, double (&gm)[12]) {
  d3 ea = xd[1] - xd[0], eb = xd[3] - xd[2];
  d3 cr = cross(ea, eb);
  double xc = dot(cr, cr), q = xc / eps_x;
  mv = (2.0 - q) * q;
  double dm = 2.0 * (1.0 - q) / eps_x;
  double ab = dot(ea, eb);
  d3 dxa = ea * (2.0 * dot(eb, eb)) - eb * (2.0 * ab);
  d3 dxb = eb * (2.0 * dot(ea, ea)) - ea * (2.0 * ab);
  gm[0] = -dm * dxa.x; gm[1] = -dm * dxa.y; gm[2] = -dm * dxa.z;
  gm[3] = dm * dxa.x; gm[4] = dm * dxa.y; gm[5] = dm * dxa.z;
  gm[6] = -dm * dxb.x; gm[7] = -dm * dxb.y; gm[8] = -dm * dxb.z;
  gm[9] = dm * dxb.x; gm[10] = dm * dxb.y; gm[11] = dm * dxb.z;
}

// The float32 part of a record (the reference's wp.vec3 casts, F9): the
// closest distance, the segment parameters (EE) or region type (PT), the
// near-parallel test of the EE mollifier, and the record's cost class, for
// giving records that take the same path through the Hessian to the same
// warps: 0 inactive (dist >= l0: zero blocks), 1 no eigen-solve (point-point
// feature, or near-parallel EE edges: mollified gradient term only), 2 the
// 3x3 restriction (point-edge), 3 the 5x5 restriction (edge-edge,
// point-triangle).  Packed in a float4: (dist, s, t, flags) with flags bits
// 0-1 the class, bit 2 near-parallel, bits 3-5 the PT region type.
struct Pre {
  float d, s, t;
  int flags;
  IPCB_D int cls() const { return flags & 3; }
  IPCB_D bool near_par() const { return (flags >> 2) & 1; }
  IPCB_D int type() const { return (flags >> 3) & 7; }
};
IPCB_D float4 pack(const Pre& p) { return make_float4(p.d, p.s, p.t, __int_as_float(p.flags)); }
IPCB_D Pre unpack(float4 v) { return Pre{v.x, v.y, v.z, __float_as_int(v.w)}; }

template <class S, int KIND>
IPCB_D Pre predicate(const S* __restrict__ xcs, int4 id, S l0, const v3<S>* xs) {
  const f3 xf[4] = {to_f(xs[0]), to_f(xs[1]), to_f(xs[2]), to_f(xs[3])};
  Pre p{0.f, 0.f, 0.f, 0};
  if (KIND == 0) {
    const CPEE d = closest_point_edge_edge(xf[0], xf[1], xf[2], xf[3], 1.0e-6f);
    p.d = d.d;
    p.s = d.s;
    p.t = d.t;
    if (!(S(d.d) < l0)) return p;
    const S eps_x = ee_eps_x(xcs, id);
    const v3<S> ea = esub(xs[1], xs[0]), eb = esub(xs[3], xs[2]);
    const v3<S> cr = ecross(ea, eb);
    const bool near_par = eps_x > S(0) && edot(cr, cr) < eps_x;
    const S s = S(d.s), t = S(d.t), feps = S(1.0e-6), hi = S(1.0) - S(1.0e-6);
    const bool sb = s <= feps || s >= hi, tb = t <= feps || t >= hi;
    const int cls = near_par ? 1 : (sb && tb ? 1 : (sb || tb ? 2 : 3));
    p.flags = cls | (near_par ? 4 : 0);
  } else {
    const CPT cp = closest_point_triangle(xf[0], xf[1], xf[2], xf[3]);
    p.d = cp.d;
    p.flags = cp.type << 3;
    if (!(S(cp.d) < l0)) return p;
    p.flags |= cp.type <= 2 ? 1 : (cp.type <= 5 ? 2 : 3);
  }
  return p;
}

template <class S, int KIND>
IPCB_D int record_class(const S* __restrict__ x, const S* __restrict__ xcs, const ipcb_contacts& L, int i) {
  const int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
  const S l0 = static_cast<const S*>(L.l0)[i];
  const v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
  return predicate<S, KIND>(xcs, id, l0, xs).cls();
}

// One record of contact_hessian_ee / _pt from its float32 part p: 16 blocks
// at (offset + i)*16, force into bforce, block mask.  T: arithmetic type of
// the eigen-solve and of H (float for S=float).
// Rank-one terms of one active record: H = sum_m w_m h_m h_m^T (the
// gradient, plus up to 3 (point-edge) or 5 (edge-edge, point-triangle)
// negative eigenvectors) and the force fc.  Returns the number of terms.
template <class S, int KIND>
IPCB_D int hessian_terms(const S* __restrict__ x, const S* __restrict__ xcs, int4 id, S l0, double kappa,
                         const Pre& p, S (&h)[kMaxH][12], S (&w)[kMaxH], double (&fc)[12]) {
  typedef S T;
  v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
  d3 xd[4] = {to_d(xs[0]), to_d(xs[1]), to_d(xs[2]), to_d(xs[3])};
  const float dist = p.d;
  Feature f;
  const bool near_par = KIND == 0 && p.near_par();
  if (KIND == 0) ee_dispatch<S>(f, xd, p.s, p.t, near_par);
  else pt_dispatch(f, p.type(), xd);
  double d2 = (double)dist * (double)dist, d02 = (double)l0 * (double)l0;
  Barrier br = barrier(d2, d02, kappa);
#pragma unroll
  for (int m = 0; m < kMaxH; ++m) w[m] = T(0);
  double g[12];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    g[3 * k] = 2.0 * f.c[k] * f.r.x;
    g[3 * k + 1] = 2.0 * f.c[k] * f.r.y;
    g[3 * k + 2] = 2.0 * f.c[k] * f.r.z;
  }
#pragma unroll
  for (int k = 0; k < 12; ++k) h[0][k] = T(g[k]);
  int nh = 1;
  if (near_par) {
    double mv, gm[12];
    mollifier(xd, (double)ee_eps_x(xcs, id), mv, gm);
    w[0] = T(mv * br.d2b);
#pragma unroll
    for (int k = 0; k < 12; ++k) fc[k] = -(mv * br.db * g[k] + br.b * gm[k]);
  } else {
    w[0] = T(br.d2b);
    if (f.np == 1) nh = 1 + nsd_subspace<T, 1, kMaxH>(f, br.db, h, w);
    else if (f.np == 2) nh = 1 + nsd_subspace<T, 2, kMaxH>(f, br.db, h, w);
#pragma unroll
    for (int k = 0; k < 12; ++k) fc[k] = -br.db * g[k];
  }
  return nh;
}

// record i of the list (vertex ids id, l0); its outputs go to slot offset + i
template <class S, int KIND>
IPCB_D void hessian_from(const S* __restrict__ x, const S* __restrict__ xcs, int4 id, S l0, int i, int offset,
                         double kappa, const Pre& p, int* __restrict__ rows, int* __restrict__ cols,
                         S* __restrict__ vals, S* __restrict__ bforce, unsigned short* __restrict__ block_mask) {
  long long base = (long long)(offset + i) * 16;
  if (p.cls() == 0) {
    write_zero<S>(rows, cols, vals, base);
    if (block_mask) block_mask[offset + i] = 0;
    return;
  }
  S h[kMaxH][12], w[kMaxH];
  double fc[12];
  const int nh = hessian_terms<S, KIND>(x, xcs, id, l0, kappa, p, h, w, fc);
  unsigned mask = write_blocks<S, S, kMaxH>(id, rows, cols, vals, base, h, w, nh);
  if (block_mask) block_mask[offset + i] = (unsigned short)mask;
  add_force<S>(bforce, id, fc);
}

// The same, written by the 32 lanes of a warp together (every lane calls it;
// a lane without a record passes active = false): each lane forms one block
// row of its record at a time into the warp's shared-memory stage, then the
// warp stores the 32 block rows -- each 36 contiguous values -- as runs of
// 16-byte vectors, instead of every lane storing 16 bytes to 32 different
// records per instruction.  stage: 32 * 36 values, 16-byte aligned.
template <class S, int KIND>
IPCB_D void hessian_from_warp(const S* __restrict__ x, const S* __restrict__ xcs, int4 id, S l0, int i, int offset,
                              double kappa, const Pre& p, bool active, int* __restrict__ rows,
                              int* __restrict__ cols, S* __restrict__ vals, S* __restrict__ bforce,
                              unsigned short* __restrict__ block_mask, S* __restrict__ stage) {
  constexpr int kVec = 36 * (int)sizeof(S) / 16;  // 16-byte vectors per block row
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const bool live = active && p.cls() != 0;
  S h[kMaxH][12], w[kMaxH];
  double fc[12];
  int nh = 0;
  if (live) {
    nh = hessian_terms<S, KIND>(x, xcs, id, l0, kappa, p, h, w, fc);
    add_force<S>(bforce, id, fc);  // before the blocks: fc is not live while they are formed
  }
  const long long base = (long long)(offset + i) * 16;
  const int4 rid = live ? id : make_int4(0, 0, 0, 0);
  if (active) {
    const int vid[4] = {rid.x, rid.y, rid.z, rid.w};
#pragma unroll
    for (int ii = 0; ii < 4; ++ii) {
      reinterpret_cast<int4*>(rows + base)[ii] = make_int4(vid[ii], vid[ii], vid[ii], vid[ii]);
      reinterpret_cast<int4*>(cols + base)[ii] = make_int4(vid[0], vid[1], vid[2], vid[3]);
    }
  }
  unsigned mask = 0;
#pragma unroll
  for (int ii = 0; ii < 4; ++ii) {
    S buf[36];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      S wh[kMaxH];
#pragma unroll
      for (int m = 0; m < kMaxH; ++m) wh[m] = m < nh ? w[m] * h[m][3 * ii + a] : S(0);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int b = 0; b < 3; ++b) {
          S v = S(0);
#pragma unroll
          for (int m = 0; m < kMaxH; ++m)
            if (m < nh) v += wh[m] * h[m][3 * jj + b];
          buf[jj * 9 + 3 * a + b] = v;
          if (v != S(0)) mask |= 1u << (ii * 4 + jj);
        }
    }
    const float4* st4 = reinterpret_cast<const float4*>(stage);
    store16(stage + 36 * lane, buf, 36);  // 16-byte aligned: 36 values are 144 (288) bytes
    __syncwarp(full);
    // vector u of the warp's 32 * kVec belongs to lane u / kVec's block row
#pragma unroll
    for (int r = 0; r < kVec; ++r) {
      const int u = 32 * r + lane, owner = u / kVec, piece = u - owner * kVec;
      const long long ob = __shfl_sync(full, base, owner);
      const bool on = __shfl_sync(full, active, owner);
      if (on) reinterpret_cast<float4*>(vals + 9 * ob + 36 * ii)[piece] = st4[u];
    }
    __syncwarp(full);
  }
  if (active && block_mask) block_mask[offset + i] = (unsigned short)mask;
}

// ---- class-sorted path: the records of the whole list are put in cost-class
// order (most expensive first) before the Hessian kernel, so nearly every
// warp runs one path.  The ordering pass also copies each record's float32
// part, vertex ids and l0 to its sorted position, so the Hessian kernel reads
// its inputs coalesced and only the positions are gathered.  Workspace:
// [class counts int[4] | cursors int[4] | pad to 256 B | float4 pre[cap] |
// int order[cap] | float4 sorted pre[cap] | int4 sorted ids[cap] | S sorted
// l0[cap]], each array 256-byte aligned.
template <class S, int KIND>
__global__ void __launch_bounds__(256) k_classify(const S* __restrict__ x, const S* __restrict__ xcs, ipcb_contacts L,
                                                  int n, float4* __restrict__ pre, int* __restrict__ counts) {
  __shared__ int sc[4];
  const int cnt = list_count<S>(L, n);
  if ((int)(blockIdx.x * blockDim.x) >= cnt) return;  // the whole block
  if (threadIdx.x < 4) sc[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cnt) {
    const int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
    const S l0 = static_cast<const S*>(L.l0)[i];
    const v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
    const Pre p = predicate<S, KIND>(xcs, id, l0, xs);
    pre[i] = pack(p);
    atomicAdd(&sc[p.cls()], 1);
  }
  __syncthreads();
  if (threadIdx.x < 4 && sc[threadIdx.x]) atomicAdd(counts + threadIdx.x, sc[threadIdx.x]);
}

template <class S>
struct Sorted {
  float4* pre;
  int* order;
  float4* spre;
  int4* sids;
  S* sl0;
};

// host side: the device addresses of the workspace's arrays
template <class S>
inline Sorted<S> sorted_ws(void* ws, int capacity) {
  const size_t c = (size_t)(capacity < 1 ? 1 : capacity);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  char* p = (char*)ws + 256;
  Sorted<S> r;
  r.pre = (float4*)p;
  p += al(c * 16);
  r.order = (int*)p;
  p += al(c * 4);
  r.spre = (float4*)p;
  p += al(c * 16);
  r.sids = (int4*)p;
  p += al(c * 16);
  r.sl0 = (S*)p;
  return r;
}

template <class S>
__global__ void __launch_bounds__(256) k_class_order(ipcb_contacts L, int n, const int* __restrict__ counts,
                                                     int* __restrict__ cursor, Sorted<S> W) {
  __shared__ int sc[4], sbase[4];
  const int cnt = list_count<S>(L, n);
  if ((int)(blockIdx.x * blockDim.x) >= cnt) return;
  if (threadIdx.x < 4) sc[threadIdx.x] = 0;
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  int cls = -1, local = 0;
  float4 pr = make_float4(0.f, 0.f, 0.f, 0.f);
  if (i < cnt) {
    pr = W.pre[i];
    cls = __float_as_int(pr.w) & 3;
    local = atomicAdd(&sc[cls], 1);
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    // classes in the order 3, 2, 1, 0: the costliest records start first
    const int k = threadIdx.x;
    int start = 0;
    for (int c = 3; c > k; --c) start += counts[c];
    sbase[k] = sc[k] ? start + atomicAdd(cursor + k, sc[k]) : 0;
  }
  __syncthreads();
  if (cls >= 0) {
    const int pos = sbase[cls] + local;
    W.order[pos] = i;
    W.spre[pos] = pr;
    W.sids[pos] = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
    W.sl0[pos] = static_cast<const S*>(L.l0)[i];
  }
}

inline size_t sorted_workspace(int capacity) {
  const size_t c = (size_t)(capacity < 1 ? 1 : capacity);
  auto al = [](size_t b) { return (b + 255) / 256 * 256; };
  return 256 + al(c * 16) + al(c * 4) + al(c * 16) + al(c * 16) + al(c * 8);
}

// One record of contact_hessian_ee / _pt: the float32 part, then the rest.
template <class S, int KIND>
IPCB_D void contact_hessian_item(const S* __restrict__ x, const S* __restrict__ xcs, const ipcb_contacts& L, int i,
                                 int offset, double kappa, int* __restrict__ rows, int* __restrict__ cols,
                                 S* __restrict__ vals, S* __restrict__ bforce,
                                 unsigned short* __restrict__ block_mask) {
  const int4 id = __ldg(reinterpret_cast<const int4*>(L.a1a2b1b2) + i);
  const S l0 = static_cast<const S*>(L.l0)[i];
  const v3<S> xs[4] = {ldx(x, id.x), ldx(x, id.y), ldx(x, id.z), ldx(x, id.w)};
  const Pre p = predicate<S, KIND>(xcs, id, l0, xs);
  hessian_from<S, KIND>(x, xcs, id, l0, i, offset, kappa, p, rows, cols, vals, bforce, block_mask);
}

}  // namespace
}  // namespace ipcb
