// Continuous collision detection: swept boxes, coplanarity-cubic time of
// impact (ccd/ccd.py:166-427, ccd/cubic_roots.py:7-193), all root arithmetic
// in double.  This file is compiled with -fmad=false: every operation rounds
// on its own, in source order, so the TOI is reproducible bit for bit by a
// plain IEEE evaluation.
#include <cooperative_groups.h>

#include "bodies.cuh"
#include "common.cuh"
#include "lbvh.cuh"

namespace cg = cooperative_groups;

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr int kFindIters = 200;  // bound on the bracketed Newton/bisection loop
constexpr double kXError = 1e-10;  // cubic_roots.py:4

struct Q4 {
  double c[4];
};
struct D3v {
  double v[3];
};

IPCB_D double evaluate(const Q4& p, double x) { return p.c[0] + x * (p.c[1] + x * (p.c[2] + x * p.c[3])); }
IPCB_D double multi_sign(double a, double b) { return b < 0.0 ? -a : a; }
IPCB_D bool diff_sign(double y0, double yr) { return y0 * yr < 0.0; }
IPCB_D double dmin(double a, double b) { return a < b ? a : b; }
IPCB_D double dmax(double a, double b) { return a > b ? a : b; }

IPCB_D D3v deflate(const Q4& p, double root) {
  D3v d;
  d.v[2] = p.c[3];
  d.v[1] = p.c[2] + root * d.v[2];
  d.v[0] = p.c[1] + root * d.v[1];
  return d;
}

IPCB_D double find_closed(const Q4& p, const Q4& dp, double x0, double x1, double y0, double y1, int& status) {
  (void)y1;
  double xr = (x0 + x1) / 2.0;
  double yr = evaluate(p, xr);
  double xb0 = x0, xb1 = x1;
  if (x1 - x0 <= kXError * 2.0) return xr;
  for (int it = 0;; ++it) {
    if (it >= kFindIters) {
      status |= IPCB_STATUS_ROOT_ITERS;
      break;
    }
    if (diff_sign(y0, yr)) xb1 = xr;
    else xb0 = xr;
    double dy = evaluate(dp, xr);
    double dx = yr / dy;
    double xn = xr - dx;
    if (xn > xb0 && xn < xb1) {
      double step = fabs(xr - xn);
      xr = xn;
      if (step > kXError) yr = evaluate(p, xr);
      else break;
    } else {
      xr = (xb0 + xb1) / 2.0;
      yr = evaluate(p, xr);
      if (xb0 == xr || xb1 == xr || xb1 - xb0 <= 2.0 * kXError) break;
    }
  }
  return xr;
}

IPCB_D int quadratic_roots(const D3v& q, double x0, double x1, double* roots) {
  double c = q.v[0], b = q.v[1], a = q.v[2];
  double delta = b * b - 4.0 * a * c;
  int ret = 0;
  roots[0] = roots[1] = 0.0;
  if (delta > 0.0) {
    double d = sqrt(delta);
    double qq = -(b + multi_sign(d, b)) * 0.5;
    double rv0 = qq / a, rv1 = c / qq;
    double xa = dmin(rv0, rv1), xb = dmax(rv0, rv1);
    if (xa >= x0 && xa <= x1) roots[ret++] = xa;
    if (xb >= x0 && xb <= x1) roots[ret++] = xb;
  } else if (delta < 0.0) {
    ret = 0;
  } else {
    double r0 = -0.5 * b / a;
    roots[0] = r0;
    if (r0 >= x0 && r0 <= x1) ret = 1;
  }
  return ret;
}

// cubic_roots.py:96-193: real roots in [x0, x1], ascending.
IPCB_D int cubic_roots(const Q4& p, double x0, double x1, double* roots, int& status) {
  roots[0] = roots[1] = roots[2] = 0.0;
  double y0 = evaluate(p, x0), y1 = evaluate(p, x1);
  double a = p.c[3] * 3.0, b_2 = p.c[2], c = p.c[1];
  Q4 dp{{c, 2.0 * b_2, a, 0.0}};
  double delta_4 = b_2 * b_2 - a * c;
  double q2[2];
  if (delta_4 > 0.0) {
    double d_2 = sqrt(delta_4);
    double q = -(b_2 + multi_sign(d_2, b_2));
    double rv0 = q / a, rv1 = c / q;
    double xa = dmin(rv0, rv1), xb = dmax(rv0, rv1);
    if (diff_sign(y0, y1)) {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) {
        roots[0] = find_closed(p, dp, x0, x1, y0, y1, status);
        return 1;
      }
    } else {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) return 0;
    }
    if (xa > x0) {
      double ya = evaluate(p, xa);
      if (diff_sign(y0, ya)) {
        roots[0] = find_closed(p, dp, x0, xa, y0, ya, status);
        if (diff_sign(ya, y1) || (xb < x1 && diff_sign(ya, evaluate(p, xb)))) {
          int r = quadratic_roots(deflate(p, roots[0]), xa, x1, q2);
          roots[1] = q2[0];
          roots[2] = q2[1];
          return r + 1;
        }
        return 1;
      }
      if (xb < x1) {
        double yb = evaluate(p, xb);
        if (diff_sign(ya, yb)) {
          roots[0] = find_closed(p, dp, xa, xb, ya, yb, status);
          if (diff_sign(yb, y1)) {
            int r = quadratic_roots(deflate(p, roots[0]), xb, x1, q2);
            roots[1] = q2[0];
            roots[2] = q2[1];
            return r + 1;
          }
          return 1;
        }
        if (diff_sign(yb, y1)) {
          roots[0] = find_closed(p, dp, xb, x1, yb, y1, status);
          return 1;
        }
      } else if (diff_sign(ya, y1)) {
        roots[0] = find_closed(p, dp, xa, x1, ya, y1, status);
        return 1;
      }
    } else {
      double yb = evaluate(p, xb);
      if (diff_sign(y0, yb)) {
        roots[0] = find_closed(p, dp, x0, xb, y0, yb, status);
        if (diff_sign(yb, y1)) {
          int r = quadratic_roots(deflate(p, roots[0]), xb, x1, q2);
          roots[1] = q2[0];
          roots[2] = q2[1];
          return r + 1;
        }
        return 1;
      }
      if (diff_sign(yb, y1)) {
        roots[0] = find_closed(p, dp, xb, x1, yb, y1, status);
        return 1;
      }
    }
    return 0;
  }
  if (diff_sign(y0, y1)) {
    roots[0] = find_closed(p, dp, x0, x1, y0, y1, status);
    return 1;
  }
  return 0;
}

// ccd.py:293-300: coefficients of prod_k (b_k + t a_k), ascending powers
IPCB_D Q4 cubic_binomial(double a0, double a1, double a2, double b0, double b1, double b2) {
  Q4 r;
  r.c[0] = b0 * b1 * b2;
  r.c[1] = a0 * b1 * b2 + b0 * b1 * a2 + b0 * a1 * b2;
  r.c[2] = a0 * a1 * b2 + a0 * b1 * a2 + b0 * a1 * a2;
  r.c[3] = a0 * a1 * a2;
  return r;
}

// det(B + t A) for 3x3 matrices given by columns (ccd.py:252-290)
IPCB_D Q4 det_polynomial(const d3* A, const d3* B) {
  // M[r][c] = col_c[r]
  auto m = [](const d3* C, int r, int c) -> double { return r == 0 ? C[c].x : (r == 1 ? C[c].y : C[c].z); };
  Q4 pos{{0, 0, 0, 0}}, neg{{0, 0, 0, 0}};
  const int P[3][3][2] = {{{0, 0}, {1, 1}, {2, 2}}, {{0, 1}, {1, 2}, {2, 0}}, {{0, 2}, {1, 0}, {2, 1}}};
  const int N[3][3][2] = {{{0, 0}, {1, 2}, {2, 1}}, {{0, 1}, {1, 0}, {2, 2}}, {{0, 2}, {1, 1}, {2, 0}}};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Q4 t = cubic_binomial(m(A, P[k][0][0], P[k][0][1]), m(A, P[k][1][0], P[k][1][1]), m(A, P[k][2][0], P[k][2][1]),
                          m(B, P[k][0][0], P[k][0][1]), m(B, P[k][1][0], P[k][1][1]), m(B, P[k][2][0], P[k][2][1]));
#pragma unroll
    for (int q = 0; q < 4; ++q) pos.c[q] = pos.c[q] + t.c[q];
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    Q4 t = cubic_binomial(m(A, N[k][0][0], N[k][0][1]), m(A, N[k][1][0], N[k][1][1]), m(A, N[k][2][0], N[k][2][1]),
                          m(B, N[k][0][0], N[k][0][1]), m(B, N[k][1][0], N[k][1][1]), m(B, N[k][2][0], N[k][2][1]));
#pragma unroll
    for (int q = 0; q < 4; ++q) neg.c[q] = neg.c[q] + t.c[q];
  }
  Q4 r;
#pragma unroll
  for (int q = 0; q < 4; ++q) r.c[q] = pos.c[q] - neg.c[q];
  return r;
}

// ccd.py:226-249: roots in [0,1] of det[p1-p0 ...] coplanarity polynomial
IPCB_D int coplanar_roots(const d3* p0, const d3* p1, double* roots, int& status) {
  const int cols[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  Q4 acc{{0, 0, 0, 0}};
#pragma unroll
  for (int m = 0; m < 4; ++m) {
    d3 A[3], B[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      B[c] = p0[cols[m][c]];
      A[c] = p1[cols[m][c]] - p0[cols[m][c]];
    }
    Q4 d = det_polynomial(A, B);
    double sg = (m & 1) ? -1.0 : 1.0;
    if (m == 0) acc = d;
    else
#pragma unroll
      for (int q = 0; q < 4; ++q) acc.c[q] = sg > 0 ? acc.c[q] + d.c[q] : acc.c[q] - d.c[q];
  }
  return cubic_roots(acc, 0.0, 1.0, roots, status);
}

IPCB_D d3 lerp(d3 a, d3 b, double t) { return a * (1.0 - t) + b * t; }

// Least-squares coordinates of the coplanar configuration (ipctkwp
// beta_gamma_pt/ee, restated): PT solves x0 - x1 = beta e1 + gamma e2,
// EE solves x2 - x0 = beta ea + gamma eb.
IPCB_D void solve2(double a11, double a12, double a22, double b1, double b2, double& be, double& ga) {
  double det = a11 * a22 - a12 * a12;
  be = (b1 * a22 - a12 * b2) / det;
  ga = (a11 * b2 - a12 * b1) / det;
}

IPCB_D bool verify_pt(const d3* x) {
  d3 e1 = x[2] - x[1], e2 = x[3] - x[1], w = x[0] - x[1];
  double be, ga;
  solve2(dot(e1, e1), dot(e1, e2), dot(e2, e2), dot(e1, w), dot(e2, w), be, ga);
  const double tol = 1e-8;
  return be >= -tol && ga >= -tol && be + ga <= 1.0 + tol;
}

IPCB_D bool verify_ee(const d3* x) {
  d3 ea = x[1] - x[0], eb = x[3] - x[2], w = x[2] - x[0];
  double be, ga;
  solve2(dot(ea, ea), dot(ea, eb), dot(eb, eb), dot(ea, w), dot(eb, w), be, ga);
  const double tol = 1e-8;
  return be >= -tol && be <= 1.0 + tol && -ga >= -tol && -ga <= 1.0 + tol;
}

// ccd.py:304-357
template <int KIND>
IPCB_D double collision_time(const d3* p0, const d3* p1, int& status) {
  double roots[3];
  int nr = coplanar_roots(p0, p1, roots, status);
  double root = 1.0;
  bool ok = false;
  for (int i = 0; i < nr; ++i) {
    root = roots[i];
    d3 xt[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) xt[k] = lerp(p0[k], p1[k], root);
    ok = KIND == 0 ? verify_ee(xt) : verify_pt(xt);
    if (ok) break;
  }
  return ok ? root : 1.0;
}

template <class S>
IPCB_D d3 ld(const S* __restrict__ x, int i) {
  return mk3((double)__ldg(x + 3 * i), (double)__ldg(x + 3 * i + 1), (double)__ldg(x + 3 * i + 2));
}

IPCB_D void store_toi(float* toi, double t) { atomic_min_nonneg(toi, __double2float_rz(t)); }
IPCB_D void store_toi(double* toi, double t) { atomic_min_nonneg(toi, t); }

// Optional output of new_intersections (contact.py:587-670): every pair whose
// time of impact is < 1 is appended as a record (append_ccd, contact.py:186-197:
// a1a2b1b2, e0e1 = (query primitive, hit primitive), l0 = 2 thickness,
// alpha = toi, lam = 0); records beyond the capacity are only counted.
struct Sink {
  ipcb_contacts L;
  double l0;
  int on;
};

template <class S>
IPCB_D void sink_append(const Sink& k, int4 ids, int e0, int e1, double t) {
  if (!k.on) return;
  const int idx = atomicAdd(k.L.cnt, 1);
  if (idx >= k.L.capacity) return;
  reinterpret_cast<int4*>(k.L.a1a2b1b2)[idx] = ids;
  reinterpret_cast<int2*>(k.L.e0e1)[idx] = make_int2(e0, e1);
  static_cast<S*>(k.L.l0)[idx] = S(k.l0);
  static_cast<S*>(k.L.alpha)[idx] = sizeof(S) == 4 ? S(__double2float_rz(t)) : S(t);
  static_cast<S*>(k.L.lam)[idx] = S(0);
}

template <class S>
__global__ void k_add_dx(const S* __restrict__ x, const S* __restrict__ dx, S* __restrict__ x1, int n3) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3) x1[i] = x[i] - dx[i];
}

template <class S, int NV>
__global__ void k_swept(const S* __restrict__ x0, const S* __restrict__ x1, const int* __restrict__ prims, int n,
                        double pad, float* __restrict__ lo, float* __restrict__ hi) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    int k = __ldg(prims + NV * i + v);
    d3 a = ld(x0, k), b = ld(x1, k);
    mn[0] = dmin(mn[0], dmin(a.x, b.x)); mx[0] = dmax(mx[0], dmax(a.x, b.x));
    mn[1] = dmin(mn[1], dmin(a.y, b.y)); mx[1] = dmax(mx[1], dmax(a.y, b.y));
    mn[2] = dmin(mn[2], dmin(a.z, b.z)); mx[2] = dmax(mx[2], dmax(a.z, b.z));
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    lo[3 * i + k] = __double2float_rd(mn[k] - pad);
    hi[3 * i + k] = __double2float_ru(mx[k] + pad);
  }
}

// Candidate pairs are staged in a list so the cubic solves run one pair per
// thread (balanced) instead of inside divergent traversal loops.  Workspace:
// [count int32 | overflow int32 | pad to 256 B | int2 pairs[capacity]].  When
// a pair finds the list full the overflow flag is raised and an inline pass
// solves every pair of the query during traversal, so the result never
// depends on the capacity.
struct CandList {
  int* count;
  int* overflow;  // set by a collect pass that dropped pairs (the inline pass then redoes the query)
  int2* pairs;
  int capacity;
};


// ---- exact skip of pairs that cannot reach contact within the step ----
// The primitives move linearly, so their distance obeys
//   d(t) >= d(0) - t * (max_a |dx_a - m| + max_b |dx_b - m|)
// for any common translation m (the vertex-mean here).  A verified root needs
// the primitives to touch up to the barycentric tolerance of the root check
// (1e-8 in parameter units), so a pair with d(0) - motion above a margin of
// 1e-6 (1 + extent) returns 1 from the cubic path; skipping it does not change
// the TOI.
IPCB_D double seg_seg_dist(d3 p1, d3 q1, d3 p2, d3 q2) {
  d3 d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  double s = 0, t = 0;
  if (a <= 1e-30 && e <= 1e-30) {
  } else if (a <= 1e-30) {
    t = fmin(fmax(f / e, 0.0), 1.0);
  } else {
    double c = dot(d1, r);
    if (e <= 1e-30) {
      s = fmin(fmax(-c / a, 0.0), 1.0);
    } else {
      double b = dot(d1, d2), den = a * e - b * b;
      s = den > 0 ? fmin(fmax((b * f - c * e) / den, 0.0), 1.0) : 0.0;
      t = (b * s + f) / e;
      if (t < 0) {
        t = 0;
        s = fmin(fmax(-c / a, 0.0), 1.0);
      } else if (t > 1) {
        t = 1;
        s = fmin(fmax((b - c) / a, 0.0), 1.0);
      }
    }
  }
  d3 w = (p1 + d1 * s) - (p2 + d2 * t);
  return sqrt(dot(w, w));
}

IPCB_D double pt_dist(d3 p, d3 a, d3 b, d3 c) {
  d3 ab = b - a, ac = c - a, ap = p - a;
  double d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return sqrt(dot(ap, ap));
  d3 bp = p - b;
  double d3v = dot(ab, bp), d4 = dot(ac, bp);
  if (d3v >= 0 && d4 <= d3v) return sqrt(dot(bp, bp));
  double vc = d1 * d4 - d3v * d2;
  if (vc <= 0 && d1 >= 0 && d3v <= 0) {
    d3 w = p - (a + ab * (d1 / (d1 - d3v)));
    return sqrt(dot(w, w));
  }
  d3 cp = p - c;
  double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return sqrt(dot(cp, cp));
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) {
    d3 w = p - (a + ac * (d2 / (d2 - d6)));
    return sqrt(dot(w, w));
  }
  double va = d3v * d6 - d5 * d4;
  if (va <= 0 && (d4 - d3v) >= 0 && (d5 - d6) >= 0) {
    d3 w = p - (b + (c - b) * ((d4 - d3v) / ((d4 - d3v) + (d5 - d6))));
    return sqrt(dot(w, w));
  }
  double den = va + vb + vc;
  if (!(fabs(den) > 0)) {  // degenerate triangle: distance to its edges
    return fmin(seg_seg_dist(p, p, a, b), fmin(seg_seg_dist(p, p, a, c), seg_seg_dist(p, p, b, c)));
  }
  d3 w = p - (a + ab * (vb / den) + ac * (vc / den));
  return sqrt(dot(w, w));
}

// KIND 0: (a0, a1 | b0, b1); KIND 1: (p | t0, t1, t2).  Lower bound on the
// time at which the pair can touch: (d(0) - margin) / (relative motion bound),
// 0 when it already touches, infinity when it does not move.  A verified root
// at t needs d(t) within the margin, so no root lies below the bound.
template <int KIND>
IPCB_D double touch_time_bound(const d3* p0, const d3* p1) {
  d3 dx[4];
  d3 m = mk3(0.0, 0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    dx[k] = p1[k] - p0[k];
    m = m + dx[k];
  }
  m = m * 0.25;
  double ma = 0, mb = 0, ext = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d3 u = dx[k] - m;
    double l = sqrt(dot(u, u));
    if ((KIND == 0 && k < 2) || (KIND == 1 && k < 1)) ma = fmax(ma, l);
    else mb = fmax(mb, l);
    ext = fmax(ext, fmax(fabs(p0[k].x), fmax(fabs(p0[k].y), fabs(p0[k].z))));
    ext = fmax(ext, fmax(fabs(p1[k].x), fmax(fabs(p1[k].y), fabs(p1[k].z))));
  }
  const double d0 = KIND == 0 ? seg_seg_dist(p0[0], p0[1], p0[2], p0[3]) : pt_dist(p0[0], p0[1], p0[2], p0[3]);
  const double gap = d0 - 1e-6 * (1.0 + ext);
  if (!(gap > 0.0)) return 0.0;
  const double v = ma + mb;
  return v > 0.0 ? gap / v : INFINITY;
}

template <int KIND>
IPCB_D bool cannot_touch(const d3* p0, const d3* p1) {
  d3 dx[4];
  d3 m = mk3(0.0, 0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    dx[k] = p1[k] - p0[k];
    m = m + dx[k];
  }
  m = m * 0.25;
  double ma = 0, mb = 0, ext = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    d3 u = dx[k] - m;
    double l = sqrt(dot(u, u));
    if ((KIND == 0 && k < 2) || (KIND == 1 && k < 1)) ma = fmax(ma, l);
    else mb = fmax(mb, l);
    ext = fmax(ext, fmax(fabs(p0[k].x), fmax(fabs(p0[k].y), fabs(p0[k].z))));
    ext = fmax(ext, fmax(fabs(p1[k].x), fmax(fabs(p1[k].y), fabs(p1[k].z))));
  }
  double d0 = KIND == 0 ? seg_seg_dist(p0[0], p0[1], p0[2], p0[3]) : pt_dist(p0[0], p0[1], p0[2], p0[3]);
  return d0 - (ma + mb) > 1e-6 * (1.0 + ext);
}

template <class S>
IPCB_D double ee_pair_time(const S* __restrict__ x0, const S* __restrict__ x1, int2 ea, int2 eb, int& st) {
  d3 p0[4] = {ld(x0, ea.x), ld(x0, ea.y), ld(x0, eb.x), ld(x0, eb.y)};
  d3 p1[4] = {ld(x1, ea.x), ld(x1, ea.y), ld(x1, eb.x), ld(x1, eb.y)};
  if (cannot_touch<0>(p0, p1)) return 1.0;
  return collision_time<0>(p0, p1, st);
}

template <class S>
IPCB_D double pt_pair_time(const S* __restrict__ x0, const S* __restrict__ x1, int v, int3 t, int& st) {
  d3 p0[4] = {ld(x0, v), ld(x0, t.x), ld(x0, t.y), ld(x0, t.z)};
  d3 p1[4] = {ld(x1, v), ld(x1, t.x), ld(x1, t.y), ld(x1, t.z)};
  if (cannot_touch<1>(p0, p1)) return 1.0;
  return collision_time<1>(p0, p1, st);
}

constexpr int kQueue = 32;  // per-thread queue of filtered leaf hits

IPCB_D int warp_max(int v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// converged push: one ballot and one atomicAdd per warp; returns false for a
// lane whose pair did not fit (the caller solves it in place)
IPCB_D bool push_converged(const CandList& L, bool has, int a, int b) {
  const unsigned lane = threadIdx.x & 31;
  unsigned m = __ballot_sync(0xffffffffu, has);
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(L.count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  int slot = base + __popc(m & ((1u << lane) - 1u));
  if (has && slot < L.capacity) {
    L.pairs[slot] = make_int2(a, b);
    return true;
  }
  return !has;
}

// Traversal applies the cheap filters and queues leaves; the warp then pushes
// the queued pairs converged (divergent pushes would serialise on the count).
// FAST: stage pairs only (a lane whose queue is full pushes on its own); a
// pair that does not fit in the list raises cand.overflow instead of being
// solved here, which keeps the cubic solver out of this kernel (56 instead of
// 255 registers).  !FAST (run only when *gate is set, with a zero-capacity
// list): every pair solved in place.
template <class S, bool FAST>
__global__ void __launch_bounds__(128) k_ee_collect(const S* __restrict__ x0, const S* __restrict__ x1,
                                                    const int* __restrict__ edges, const int* __restrict__ body,
                                                    const float4* __restrict__ nodes, const int* __restrict__ order,
                                                    int n, int first, int count, const float* __restrict__ lo,
                                                    const float* __restrict__ hi, int exclude, CandList cand, S* toi,
                                                    int* status, Sink sink, const int* gate) {
  if (gate && *gate == 0) return;
  bool dropped = false;
  // queries: the edges of Morton rank first .. first + count - 1
  int t = first + blockIdx.x * blockDim.x + threadIdx.x;
  bool active = t < first + count;
  int i = active ? __ldg(order + t) : 0;
  int2 ea = __ldg(reinterpret_cast<const int2*>(edges) + i);
  int bi = exclude ? __ldg(body + ea.x) : 0;
  int st = 0;
  int q[kQueue];
  int nq = 0;
  if (active) {
    f3 qlo = mk3(__ldg(lo + 3 * i), __ldg(lo + 3 * i + 1), __ldg(lo + 3 * i + 2));
    f3 qhi = mk3(__ldg(hi + 3 * i), __ldg(hi + 3 * i + 1), __ldg(hi + 3 * i + 2));
    // thread t queries the edge of Morton rank t in its own hierarchy: only
    // leaves of higher rank are visited, so each pair is met once; it is then
    // taken as the reference's (lower id, higher id) pair
    bool ok = traverse4_after(nodes, n, t, qlo, qhi, [&](int j, int) {
      int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + j);
      if (ea.x == eb.x || ea.x == eb.y || ea.y == eb.x || ea.y == eb.y) return;
      if (exclude && bi == __ldg(body + eb.x)) return;
      if (nq < kQueue) {
        q[nq++] = j;
      } else if (FAST) {  // lane queue full: stage this pair directly
        const int slot = atomicAdd(cand.count, 1);
        if (slot < cand.capacity) cand.pairs[slot] = make_int2(min(i, j), max(i, j));
        else dropped = true;
      } else {
        const bool fwd = i < j;
        const int2 e_lo = fwd ? ea : eb, e_hi = fwd ? eb : ea;
        double tt = ee_pair_time(x0, x1, e_lo, e_hi, st);
        if (tt < 1.0) {
          store_toi(toi, tt);
          sink_append<S>(sink, make_int4(e_lo.x, e_lo.y, e_hi.x, e_hi.y), min(i, j), max(i, j), tt);
        }
      }
    });
    if (!ok) st |= IPCB_STATUS_STACK;
  }
  int rounds = warp_max(nq);
  for (int k = 0; k < rounds; ++k) {
    bool has = k < nq;
    int j = has ? q[k] : 0;
    if (!push_converged(cand, has, min(i, j), max(i, j))) {
      if (FAST) {
        dropped = true;
        continue;
      }
      int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + j);
      const bool fwd = i < j;
      const int2 e_lo = fwd ? ea : eb, e_hi = fwd ? eb : ea;
      double tt = ee_pair_time(x0, x1, e_lo, e_hi, st);
      if (tt < 1.0) {
        store_toi(toi, tt);
        sink_append<S>(sink, make_int4(e_lo.x, e_lo.y, e_hi.x, e_hi.y), min(i, j), max(i, j), tt);
      }
    }
  }
  if (dropped) *cand.overflow = 1;
  if (st) atomicOr(status, st);
}

template <class S, bool FAST>
__global__ void __launch_bounds__(128) k_pt_collect(const S* __restrict__ x0, const S* __restrict__ x1,
                                                    const int* __restrict__ tris, const int* __restrict__ body,
                                                    const float4* __restrict__ nodes, int n_tris, int first, int count,
                                                    double pad, int exclude, CandList cand, S* toi, int* status,
                                                    Sink sink, const int* gate) {
  if (gate && *gate == 0) return;
  bool dropped = false;
  // queries: the vertices first .. first + count - 1
  int i0 = first + blockIdx.x * blockDim.x + threadIdx.x;
  bool active = i0 < first + count;
  int i = active ? i0 : 0;
  d3 a = ld(x0, i), b = ld(x1, i);
  int bi = exclude ? __ldg(body + i) : 0;
  int st = 0;
  int q[kQueue];
  int nq = 0;
  if (active) {
    f3 qlo = mk3(__double2float_rd(dmin(a.x, b.x) - pad), __double2float_rd(dmin(a.y, b.y) - pad),
                 __double2float_rd(dmin(a.z, b.z) - pad));
    f3 qhi = mk3(__double2float_ru(dmax(a.x, b.x) + pad), __double2float_ru(dmax(a.y, b.y) + pad),
                 __double2float_ru(dmax(a.z, b.z) + pad));
    bool ok = traverse4(nodes, n_tris, qlo, qhi, [&](int j) {
      int3 tj = make_int3(__ldg(tris + 3 * j), __ldg(tris + 3 * j + 1), __ldg(tris + 3 * j + 2));
      if (i == tj.x || i == tj.y || i == tj.z) return;
      if (exclude && bi == __ldg(body + tj.x)) return;
      if (nq < kQueue) {
        q[nq++] = j;
      } else if (FAST) {  // lane queue full: stage this pair directly
        const int slot = atomicAdd(cand.count, 1);
        if (slot < cand.capacity) cand.pairs[slot] = make_int2(i, j);
        else dropped = true;
      } else {
        double tt = pt_pair_time(x0, x1, i, tj, st);
        if (tt < 1.0) {
          store_toi(toi, tt);
          sink_append<S>(sink, make_int4(i, tj.x, tj.y, tj.z), i, j, tt);
        }
      }
    });
    if (!ok) st |= IPCB_STATUS_STACK;
  }
  int rounds = warp_max(nq);
  for (int k = 0; k < rounds; ++k) {
    bool has = k < nq;
    int j = has ? q[k] : 0;
    if (!push_converged(cand, has, i, j)) {
      if (FAST) {
        dropped = true;
        continue;
      }
      int3 tj = make_int3(__ldg(tris + 3 * j), __ldg(tris + 3 * j + 1), __ldg(tris + 3 * j + 2));
      double tt = pt_pair_time(x0, x1, i, tj, st);
      if (tt < 1.0) {
        store_toi(toi, tt);
        sink_append<S>(sink, make_int4(i, tj.x, tj.y, tj.z), i, j, tt);
      }
    }
  }
  if (dropped) *cand.overflow = 1;
  if (st) atomicOr(status, st);
}

// one thread per staged candidate; kind 0 EE (edge, edge), 1 PT (vertex, triangle)
// One thread per staged pair, grid-stride.  Without a sink only the minimum
// matters: a pair whose touch-time bound is at or above the TOI stored so far
// (re-read from L2 for every pair; it only decreases) cannot lower it, so its
// cubic is not solved -- the result is the same minimum, bit for bit.  With
// a sink every pair that can touch within the step is solved.
IPCB_D double current_toi(float* toi) { return (double)__ldcg(toi); }
IPCB_D double current_toi(double* toi) { return __ldcg(toi); }

template <class S, int KIND>
__global__ void __launch_bounds__(128) k_cand_toi(const S* __restrict__ x0, const S* __restrict__ x1,
                                                  const int* __restrict__ prims, CandList cand, S* toi,
                                                  int* status, Sink sink, const int* skip_if) {
  if (skip_if && *skip_if) return;  // the inline pass redoes every pair
  const int n = min(*cand.count, cand.capacity);
  int st = 0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const int2 pr = cand.pairs[k];
    int4 ids;
    if (KIND == 0) {
      const int2 ea = __ldg(reinterpret_cast<const int2*>(prims) + pr.x);
      const int2 eb = __ldg(reinterpret_cast<const int2*>(prims) + pr.y);
      ids = make_int4(ea.x, ea.y, eb.x, eb.y);
    } else {
      ids = make_int4(pr.x, __ldg(prims + 3 * pr.y), __ldg(prims + 3 * pr.y + 1), __ldg(prims + 3 * pr.y + 2));
    }
    d3 p0[4] = {ld(x0, ids.x), ld(x0, ids.y), ld(x0, ids.z), ld(x0, ids.w)};
    d3 p1[4] = {ld(x1, ids.x), ld(x1, ids.y), ld(x1, ids.z), ld(x1, ids.w)};
    const double lb = touch_time_bound<KIND>(p0, p1);
    if (lb > 1.0) continue;  // cannot touch within the step
    if (!sink.on && lb >= current_toi(toi)) continue;  // cannot lower the minimum
    const double tt = collision_time<KIND>(p0, p1, st);
    if (tt < 1.0) {
      store_toi(toi, tt);
      sink_append<S>(sink, ids, pr.x, pr.y, tt);
    }
  }
  if (st) atomicOr(status, st);
}

// ---- ordered candidate solve (no record sink): the staged pairs' touch-time
// bounds are computed first by a light kernel and the pairs bucketed by them
// (32 buckets over [0, 1]; a pair that cannot touch within the step is
// dropped); the solve then takes the pairs in bucket order, so the pairs that
// can touch earliest set the TOI first, and a pair whose bound is at or above
// the TOI stored so far is skipped (it cannot lower the minimum: the result is
// the same minimum, bit for bit); a warp that meets a bucket starting at or
// above the stored TOI stops.  Divergence between pruned and solved pairs and
// the cubic solver's registers stay out of the bound pass.
constexpr int kBuckets = 32;
struct CandOrder {
  int* bcount;   // pairs per bucket
  int* bcursor;  // fill cursors
  int* work;     // next position of the ordered solve
  float* tlb;    // per staged pair: touch-time bound rounded down, or 2 (cannot touch)
  int* order;    // staged pair indices in bucket order
};

IPCB_D int bucket_of(float tl) { return min(kBuckets - 1, (int)(tl * (float)kBuckets)); }

// 3 blocks per SM (at most 85 registers; 88 unbounded): the pass waits on
// gathers of the pair's positions, and the extra warps hide them (screw and
// nut edge-edge query 1.21 -> 1.14 ms)
template <class S, int KIND>
__global__ void __launch_bounds__(256, 3) k_cand_bound(const S* __restrict__ x0, const S* __restrict__ x1,
                                                    const int* __restrict__ prims, CandList cand, CandOrder o,
                                                    const int* skip_if) {
  __shared__ int sb[kBuckets];
  if (skip_if && *skip_if) return;  // the inline pass redoes every pair
  const int n = min(*cand.count, cand.capacity);
  if ((int)(blockIdx.x * blockDim.x) >= n) return;
  if (threadIdx.x < kBuckets) sb[threadIdx.x] = 0;
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    const int2 pr = cand.pairs[k];
    int4 ids;
    if (KIND == 0) {
      const int2 ea = __ldg(reinterpret_cast<const int2*>(prims) + pr.x);
      const int2 eb = __ldg(reinterpret_cast<const int2*>(prims) + pr.y);
      ids = make_int4(ea.x, ea.y, eb.x, eb.y);
    } else {
      ids = make_int4(pr.x, __ldg(prims + 3 * pr.y), __ldg(prims + 3 * pr.y + 1), __ldg(prims + 3 * pr.y + 2));
    }
    d3 p0[4] = {ld(x0, ids.x), ld(x0, ids.y), ld(x0, ids.z), ld(x0, ids.w)};
    d3 p1[4] = {ld(x1, ids.x), ld(x1, ids.y), ld(x1, ids.z), ld(x1, ids.w)};
    const double lb = touch_time_bound<KIND>(p0, p1);
    float tl = 2.0f;
    if (lb <= 1.0) {
      tl = __double2float_rd(lb);  // not above the bound
      atomicAdd(&sb[bucket_of(tl)], 1);
    }
    o.tlb[k] = tl;
  }
  __syncthreads();
  if (threadIdx.x < kBuckets && sb[threadIdx.x]) atomicAdd(o.bcount + threadIdx.x, sb[threadIdx.x]);
}

__global__ void __launch_bounds__(256) k_cand_bucket(CandList cand, CandOrder o, const int* skip_if) {
  __shared__ int sb[kBuckets], sbase[kBuckets];
  if (skip_if && *skip_if) return;
  const int n = min(*cand.count, cand.capacity);
  if ((int)(blockIdx.x * blockDim.x) >= n) return;
  if (threadIdx.x < kBuckets) sb[threadIdx.x] = 0;
  __syncthreads();
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  int b = -1, local = 0;
  if (k < n) {
    const float tl = o.tlb[k];
    if (tl <= 1.0f) {
      b = bucket_of(tl);
      local = atomicAdd(&sb[b], 1);
    }
  }
  __syncthreads();
  if (threadIdx.x < kBuckets) {
    const int q = threadIdx.x;
    int start = 0;
    for (int c = 0; c < q; ++c) start += o.bcount[c];
    sbase[q] = sb[q] ? start + atomicAdd(o.bcursor + q, sb[q]) : 0;
  }
  __syncthreads();
  if (b >= 0) o.order[sbase[b] + local] = k;
}

template <class S, int KIND>
__global__ void __launch_bounds__(128) k_cand_solve(const S* __restrict__ x0, const S* __restrict__ x1,
                                                    const int* __restrict__ prims, CandList cand, CandOrder o, S* toi,
                                                    int* status, const int* skip_if) {
  if (skip_if && *skip_if) return;
  int total = 0;
#pragma unroll 1
  for (int q = 0; q < kBuckets; ++q) total += o.bcount[q];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int st = 0;
  for (;;) {
    int base = 0;
    if (lane == 0) base = atomicAdd(o.work, 32);
    base = __shfl_sync(full, base, 0);
    if (base >= total) break;
    const int item = base + lane;
    const int k = item < total ? __ldg(o.order + item) : -1;
    const float tl = k >= 0 ? __ldg(o.tlb + k) : 2.0f;
    const double cur = current_toi(toi);
    // the chunk's first pair starts its bucket range: every later pair lies
    // in this bucket or a later one, so none can lower a TOI at or below it
    const float first = __shfl_sync(full, tl, 0);
    if ((double)bucket_of(first) / kBuckets >= cur) break;
    if (k < 0 || (double)tl >= cur) continue;
    const int2 pr = cand.pairs[k];
    int4 ids;
    if (KIND == 0) {
      const int2 ea = __ldg(reinterpret_cast<const int2*>(prims) + pr.x);
      const int2 eb = __ldg(reinterpret_cast<const int2*>(prims) + pr.y);
      ids = make_int4(ea.x, ea.y, eb.x, eb.y);
    } else {
      ids = make_int4(pr.x, __ldg(prims + 3 * pr.y), __ldg(prims + 3 * pr.y + 1), __ldg(prims + 3 * pr.y + 2));
    }
    d3 p0[4] = {ld(x0, ids.x), ld(x0, ids.y), ld(x0, ids.z), ld(x0, ids.w)};
    d3 p1[4] = {ld(x1, ids.x), ld(x1, ids.y), ld(x1, ids.z), ld(x1, ids.w)};
    const double tt = collision_time<KIND>(p0, p1, st);
    if (tt < 1.0) store_toi(toi, tt);
  }
  if (st) atomicOr(status, st);
}

// ---------------------------------------------------------------- fixed bodies
// frames at q, swept world boxes of the bodies over the step q -> q - dq, the
// singular test at both ends, and the target-frame motion extent
// (_target_motion_extent, fixed_bvh_contacts.py:121-141):
//   d = A0^-1 (A1 - A0), c = A0^-1 (p1 - p0), m = |d mid + c| + |d| ext
template <class S>
__global__ void k_body_frames_swept(int nb, const S* __restrict__ q, const S* __restrict__ dq,
                                    const float* __restrict__ llo, const float* __restrict__ lhi,
                                    double* __restrict__ frames, double* __restrict__ motion,
                                    int* __restrict__ status) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= nb) return;
  double p0[3], A0[9], p1[3], A1[9], I[9], w0l[3], w0h[3], w1l[3], w1h[3];
  bodies::load_affine(q, b, p0, A0);
  for (int k = 0; k < 3; ++k) p1[k] = p0[k] - (double)dq[12 * b + k];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) A1[3 * r + c] = A0[3 * r + c] - (double)dq[12 * b + 3 + 3 * c + r];
  const double d0 = bodies::det3(A0), d1 = bodies::det3(A1);
  if (!(fmin(fabs(d0), fabs(d1)) >= 1e-8)) {
    atomicOr(status, IPCB_STATUS_SINGULAR);
    for (int k = 0; k < 9; ++k) I[k] = (k % 4) == 0 ? 1.0 : 0.0;
  } else {
    bodies::inverse3(A0, d0, I);
  }
  double fro = 0.0;
  for (int k = 0; k < 9; ++k) {
    frames[13 * b + k] = I[k];
    fro += I[k] * I[k];
  }
  for (int k = 0; k < 3; ++k) frames[13 * b + 9 + k] = p0[k];
  frames[13 * b + 12] = sqrt(fro);
  const float* lo = llo + 3 * b;
  const float* hi = lhi + 3 * b;
  bodies::world_box(p0, A0, lo, hi, w0l, w0h);
  bodies::world_box(p1, A1, lo, hi, w1l, w1h);
  double* wbox = frames + 13 * (size_t)nb + 6 * b;
  for (int k = 0; k < 3; ++k) {
    wbox[k] = fmin(w0l[k], w1l[k]);
    wbox[3 + k] = fmax(w0h[k], w1h[k]);
  }
  double D[9], cvec[3];
  for (int r = 0; r < 3; ++r) {
    for (int c = 0; c < 3; ++c) {
      double acc = 0.0;
      for (int k = 0; k < 3; ++k) acc += I[3 * r + k] * (A1[3 * k + c] - A0[3 * k + c]);
      D[3 * r + c] = acc;
    }
    cvec[r] = I[3 * r] * (p1[0] - p0[0]) + I[3 * r + 1] * (p1[1] - p0[1]) + I[3 * r + 2] * (p1[2] - p0[2]);
  }
  for (int r = 0; r < 3; ++r) {
    double dc = cvec[r], e = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double mid = 0.5 * ((double)lo[k] + (double)hi[k]), ext = 0.5 * ((double)hi[k] - (double)lo[k]);
      dc += D[3 * r + k] * mid;
      e += fabs(D[3 * r + k]) * ext;
    }
    motion[3 * b + r] = fabs(dc) + e;
  }
}

__global__ void k_swept_pair_cull(int nb, const double* __restrict__ wbox, double pad, int2* __restrict__ pairs,
                                  int capacity, int* __restrict__ count) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int a = (int)(t / nb), b = (int)(t % nb);
  bool hit = false;
  if (a < nb && a < b) {
    hit = true;
    for (int k = 0; k < 3; ++k)
      hit = hit && wbox[6 * a + k] - pad <= wbox[6 * b + 3 + k] && wbox[6 * b + k] - pad <= wbox[6 * a + 3 + k];
  }
  const unsigned lane = threadIdx.x & 31;
  const unsigned m = __ballot_sync(0xffffffffu, hit);
  int base = 0;
  if (lane == 0 && m) base = atomicAdd(count, __popc(m));
  base = __shfl_sync(0xffffffffu, base, 0);
  const int slot = base + __popc(m & ((1u << lane) - 1u));
  if (hit && slot < capacity) pairs[slot] = make_int2(a, b);
}

// swept local box of world points (x0 and x1 of each) in the target frame,
// inflated by the frame's motion extent and |A^-1|_F pad
template <class S, int NP>
IPCB_D void swept_local_box(const bodies::Frame& f, const double* __restrict__ motion, int tb, const S* __restrict__ x0,
                            const S* __restrict__ x1, const int (&v)[NP], double pad, f3& qlo, f3& qhi) {
  double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300}, pd[3], a[3];
  for (int k = 0; k < NP; ++k) {
    const d3 p = ld(x0, v[k]), r = ld(x1, v[k]);
    bodies::to_local(f, p.x, p.y, p.z, a);
    for (int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], a[c]);
      hi[c] = fmax(hi[c], a[c]);
    }
    bodies::to_local(f, r.x, r.y, r.z, a);
    for (int c = 0; c < 3; ++c) {
      lo[c] = fmin(lo[c], a[c]);
      hi[c] = fmax(hi[c], a[c]);
    }
  }
  for (int c = 0; c < 3; ++c)
    pd[c] = motion[3 * tb + c] + f.fro * pad + 1e-6 * (1.0 + fmax(fabs(lo[c]), fabs(hi[c])));
  bodies::float_box(lo, hi, pd, qlo, qhi);
}

template <class S>
__global__ void __launch_bounds__(128) k_fixed_ee_collect(const S* __restrict__ x0, const S* __restrict__ x1,
                                                          const int* __restrict__ edges, ipcb_bodies B,
                                                          const int* __restrict__ fixed, const int2* __restrict__ pairs,
                                                          double pad, CandList cand, S* toi, int* status) {
  const int chunks = (B.max_edges + 127) / 128;
  const int pair = blockIdx.x / chunks;
  const int k = (blockIdx.x % chunks) * blockDim.x + threadIdx.x;
  int2 pr = pairs[pair];
  if (fixed && fixed[pr.x] != 0 && fixed[pr.y] == 0) pr = make_int2(pr.y, pr.x);  // query from the moving body
  const int sb = pr.x, tb = pr.y;
  const int s0 = __ldg(B.edge_off + sb), sn = __ldg(B.edge_off + sb + 1) - s0;
  const bool active = k < sn;
  const int i = active ? __ldg(B.edge_ids + s0 + k) : 0;
  const int2 ea = __ldg(reinterpret_cast<const int2*>(edges) + i);
  const int t0 = __ldg(B.edge_off + tb), tn = __ldg(B.edge_off + tb + 1) - t0;
  int st = 0;
  int q[kQueue];
  int nq = 0;
  if (active && tn > 0) {
    const bodies::Frame f = bodies::load_frame(B.frames, tb);
    const int v[2] = {ea.x, ea.y};
    f3 qlo, qhi;
    swept_local_box<S, 2>(f, B.motion, tb, x0, x1, v, pad, qlo, qhi);
    const float4* wide = reinterpret_cast<const float4*>(B.edge_wide[tb]);
    bool ok = traverse4(wide, tn, qlo, qhi, [&](int j) {
      const int e2 = __ldg(B.edge_ids + t0 + j);
      if (nq < kQueue) {
        q[nq++] = e2;
      } else {
        const int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + e2);
        double tt = ee_pair_time(x0, x1, ea, eb, st);
        if (tt < 1.0) store_toi(toi, tt);
      }
    });
    if (!ok) st |= IPCB_STATUS_STACK;
  }
  const int rounds = warp_max(nq);
  for (int r = 0; r < rounds; ++r) {
    const bool has = r < nq;
    const int e2 = has ? q[r] : 0;
    if (!push_converged(cand, has, i, e2)) {
      const int2 eb = __ldg(reinterpret_cast<const int2*>(edges) + e2);
      double tt = ee_pair_time(x0, x1, ea, eb, st);
      if (tt < 1.0) store_toi(toi, tt);
    }
  }
  if (st) atomicOr(status, st);
}

template <class S>
__global__ void __launch_bounds__(128) k_fixed_pt_collect(const S* __restrict__ x0, const S* __restrict__ x1,
                                                          const int* __restrict__ tris, ipcb_bodies B,
                                                          const int2* __restrict__ pairs, double pad, CandList cand,
                                                          S* toi, int* status) {
  const int chunks = (B.max_verts + 127) / 128;
  const int pair = blockIdx.x / chunks, dir = blockIdx.y;
  const int k = (blockIdx.x % chunks) * blockDim.x + threadIdx.x;
  const int2 pr = pairs[pair];
  const int sb = dir ? pr.y : pr.x, tb = dir ? pr.x : pr.y;
  const int s0 = __ldg(B.vert_off + sb), sn = __ldg(B.vert_off + sb + 1) - s0;
  const bool active = k < sn;
  const int i = active ? __ldg(B.vert_ids + s0 + k) : 0;
  const int t0 = __ldg(B.tri_off + tb), tn = __ldg(B.tri_off + tb + 1) - t0;
  int st = 0;
  int q[kQueue];
  int nq = 0;
  if (active && tn > 0) {
    const bodies::Frame f = bodies::load_frame(B.frames, tb);
    const int v[1] = {i};
    f3 qlo, qhi;
    swept_local_box<S, 1>(f, B.motion, tb, x0, x1, v, pad, qlo, qhi);
    const float4* wide = reinterpret_cast<const float4*>(B.tri_wide[tb]);
    bool ok = traverse4(wide, tn, qlo, qhi, [&](int j) {
      const int tr = __ldg(B.tri_ids + t0 + j);
      if (nq < kQueue) {
        q[nq++] = tr;
      } else {
        const int3 tj = make_int3(__ldg(tris + 3 * tr), __ldg(tris + 3 * tr + 1), __ldg(tris + 3 * tr + 2));
        double tt = pt_pair_time(x0, x1, i, tj, st);
        if (tt < 1.0) store_toi(toi, tt);
      }
    });
    if (!ok) st |= IPCB_STATUS_STACK;
  }
  const int rounds = warp_max(nq);
  for (int r = 0; r < rounds; ++r) {
    const bool has = r < nq;
    const int tr = has ? q[r] : 0;
    if (!push_converged(cand, has, i, tr)) {
      const int3 tj = make_int3(__ldg(tris + 3 * tr), __ldg(tris + 3 * tr + 1), __ldg(tris + 3 * tr + 2));
      double tt = pt_pair_time(x0, x1, i, tj, st);
      if (tt < 1.0) store_toi(toi, tt);
    }
  }
  if (st) atomicOr(status, st);
}

// Candidate workspace: a 512-byte header (count, overflow flag, bucket counts
// and cursors, work counter), then per staged pair its int2, its touch-time
// bound (float) and the bucket order (int): 16 bytes a pair.
constexpr size_t kCandHeader = 512;
constexpr size_t kCandPerPair = sizeof(int2) + sizeof(float) + sizeof(int);

inline CandList cand_list(void* ws, size_t ws_bytes) {
  CandList c;
  c.count = (int*)ws;
  c.overflow = (int*)ws + 1;
  c.pairs = (int2*)((char*)ws + kCandHeader);
  size_t cap = ws_bytes > kCandHeader ? (ws_bytes - kCandHeader) / kCandPerPair : 0;
  c.capacity = cap > 0x7fffffff ? 0x7fffffff : (int)cap;
  return c;
}

inline CandOrder cand_order(void* ws, const CandList& c) {
  CandOrder o;
  int* h = (int*)ws;
  o.bcount = h + 2;
  o.bcursor = h + 2 + kBuckets;
  o.work = h + 2 + 2 * kBuckets;
  o.tlb = (float*)(c.pairs + c.capacity);
  o.order = (int*)(o.tlb + c.capacity);
  return o;
}

template <class S, int KIND>
void solve_candidates(const S* x0, const S* x1, const int* prims, void* ws, const CandList& c, S* toi, int* status,
                      const Sink& sink, cudaStream_t st) {
  if (!c.capacity) return;
  if (sink.on) {  // every pair that collides is a record: solve them all
    const dim3 gc(min(div_up(c.capacity, 128), 2048));
    k_cand_toi<S, KIND><<<gc, 128, 0, st>>>(x0, x1, prims, c, toi, status, sink, c.overflow);
    return;
  }
  const CandOrder o = cand_order(ws, c);
  cudaMemsetAsync(o.bcount, 0, (2 * kBuckets + 1) * sizeof(int), st);
  const dim3 g256(div_up(c.capacity, 256));
  k_cand_bound<S, KIND><<<g256, 256, 0, st>>>(x0, x1, prims, c, o, c.overflow);
  k_cand_bucket<<<g256, 256, 0, st>>>(c, o, c.overflow);
  k_cand_solve<S, KIND><<<148 * 3, 128, 0, st>>>(x0, x1, prims, c, o, toi, status, c.overflow);
}


__global__ void k_pair_time(int kind, int n, const double* __restrict__ a, const double* __restrict__ b,
                            double* __restrict__ t, int* status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  d3 p0[4], p1[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    p0[k] = mk3(a[12 * i + 3 * k], a[12 * i + 3 * k + 1], a[12 * i + 3 * k + 2]);
    p1[k] = mk3(b[12 * i + 3 * k], b[12 * i + 3 * k + 1], b[12 * i + 3 * k + 2]);
  }
  int st = 0;
  t[i] = kind == 0 ? collision_time<0>(p0, p1, st) : collision_time<1>(p0, p1, st);
  if (st) atomicOr(status, st);
}

__global__ void k_cubic(int n, const double* __restrict__ coef, double x0, double x1, double* __restrict__ roots,
                        int* __restrict__ nr, int* status) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  Q4 p{{coef[4 * i], coef[4 * i + 1], coef[4 * i + 2], coef[4 * i + 3]}};
  int st = 0;
  double r[3];
  nr[i] = cubic_roots(p, x0, x1, r, st);
  roots[3 * i] = r[0];
  roots[3 * i + 1] = r[1];
  roots[3 * i + 2] = r[2];
  if (st) atomicOr(status, st);
}

// The CCD query of one kind: a staging-only collect pass, the per-candidate
// TOI pass, and (only when the first pass dropped pairs) an inline pass that
// solves every pair of the query in place.
template <class S>
void run_ee(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, const float* lower, const float* upper,
            int exclude, CandList c, void* toi, int* status, Sink sink, cudaStream_t st, int first, int count) {
  const int n = soup->n_edges;
  const dim3 g(div_up(count, 64));  // 64-thread blocks, as the discrete queries
  cudaMemsetAsync(c.count, 0, 2 * sizeof(int), st);
  k_ee_collect<S, true><<<g, 64, 0, st>>>((const S*)soup->x, (const S*)x1, soup->edges, soup->body,
                                           (const float4*)bvh->wide, bvh->sorted, n, first, count, lower, upper,
                                           exclude, c, (S*)toi, status, sink, nullptr);
  solve_candidates<S, 0>((const S*)soup->x, (const S*)x1, soup->edges, c.count, c, (S*)toi, status, sink, st);
  CandList none = c;
  none.capacity = 0;
  k_ee_collect<S, false><<<g, 64, 0, st>>>((const S*)soup->x, (const S*)x1, soup->edges, soup->body,
                                            (const float4*)bvh->wide, bvh->sorted, n, first, count, lower, upper,
                                            exclude, none, (S*)toi, status, sink, c.overflow);
}

template <class S>
void run_pt(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, double pad, int exclude, CandList c,
            void* toi, int* status, Sink sink, cudaStream_t st, int first, int count) {
  const dim3 g(div_up(count, 64));
  cudaMemsetAsync(c.count, 0, 2 * sizeof(int), st);
  k_pt_collect<S, true><<<g, 64, 0, st>>>((const S*)soup->x, (const S*)x1, soup->triangles, soup->body,
                                           (const float4*)bvh->wide, soup->n_tris, first, count, pad, exclude, c,
                                           (S*)toi, status, sink, nullptr);
  solve_candidates<S, 1>((const S*)soup->x, (const S*)x1, soup->triangles, c.count, c, (S*)toi, status, sink, st);
  CandList none = c;
  none.capacity = 0;
  k_pt_collect<S, false><<<g, 64, 0, st>>>((const S*)soup->x, (const S*)x1, soup->triangles, soup->body,
                                            (const float4*)bvh->wide, soup->n_tris, first, count, pad, exclude, none,
                                            (S*)toi, status, sink, c.overflow);
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_add_dx(const ipcb_soup* soup, const void* dx, void* x1, ipcb_stream s) {
  if (!soup || !dx || !x1) return IPCB_E_ARG;
  int n3 = 3 * soup->n_verts;
  if (n3 == 0) return IPCB_OK;
  if (soup->fp64)
    k_add_dx<double><<<div_up(n3, 256), 256, 0, (cudaStream_t)s>>>((const double*)soup->x, (const double*)dx,
                                                                   (double*)x1, n3);
  else
    k_add_dx<float><<<div_up(n3, 256), 256, 0, (cudaStream_t)s>>>((const float*)soup->x, (const float*)dx,
                                                                  (float*)x1, n3);
  return check_launch("ipcb_add_dx");
}

int ipcb_swept_edge_aabbs(const ipcb_soup* soup, const void* x1, double pad, float* lower, float* upper,
                          ipcb_stream s) {
  if (!soup || !x1 || !lower || !upper) return IPCB_E_ARG;
  int n = soup->n_edges;
  if (n == 0) return IPCB_OK;
  if (soup->fp64)
    k_swept<double, 2><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const double*)soup->x, (const double*)x1,
                                                                    soup->edges, n, pad, lower, upper);
  else
    k_swept<float, 2><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const float*)soup->x, (const float*)x1,
                                                                   soup->edges, n, pad, lower, upper);
  return check_launch("ipcb_swept_edge_aabbs");
}

int ipcb_swept_triangle_aabbs(const ipcb_soup* soup, const void* x1, double pad, float* lower, float* upper,
                              ipcb_stream s) {
  if (!soup || !x1 || !lower || !upper) return IPCB_E_ARG;
  int n = soup->n_tris;
  if (n == 0) return IPCB_OK;
  if (soup->fp64)
    k_swept<double, 3><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const double*)soup->x, (const double*)x1,
                                                                    soup->triangles, n, pad, lower, upper);
  else
    k_swept<float, 3><<<div_up(n, 256), 256, 0, (cudaStream_t)s>>>((const float*)soup->x, (const float*)x1,
                                                                   soup->triangles, n, pad, lower, upper);
  return check_launch("ipcb_swept_triangle_aabbs");
}

size_t ipcb_toi_workspace(int capacity) { return kCandHeader + (size_t)(capacity > 0 ? capacity : 0) * kCandPerPair; }

int ipcb_edge_edge_toi_range(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, const float* lower,
                             const float* upper, int exclude_same_body, int first, int count, void* toi, int* status,
                             void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!soup || !x1 || !bvh || !lower || !upper || !toi || !status || !ws || ws_bytes < kCandHeader ||
      bvh->n != soup->n_edges)
    return IPCB_E_ARG;
  const int n = soup->n_edges;
  if (first < 0 || count < 0 || first > n || count > n - first) return IPCB_E_ARG;
  if (count == 0) return IPCB_OK;
  const CandList c = cand_list(ws, ws_bytes);
  if (soup->fp64)
    run_ee<double>(soup, x1, bvh, lower, upper, exclude_same_body, c, toi, status, Sink{}, (cudaStream_t)s, first,
                   count);
  else
    run_ee<float>(soup, x1, bvh, lower, upper, exclude_same_body, c, toi, status, Sink{}, (cudaStream_t)s, first,
                  count);
  return check_launch("ipcb_edge_edge_toi");
}

int ipcb_edge_edge_toi(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, const float* lower,
                       const float* upper, int exclude_same_body, void* toi, int* status, void* ws, size_t ws_bytes,
                       ipcb_stream s) {
  if (!soup) return IPCB_E_ARG;
  return ipcb_edge_edge_toi_range(soup, x1, bvh, lower, upper, exclude_same_body, 0, soup->n_edges, toi, status, ws,
                                  ws_bytes, s);
}

int ipcb_point_triangle_toi_range(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, double pad,
                                  int exclude_same_body, int first, int count, void* toi, int* status, void* ws,
                                  size_t ws_bytes, ipcb_stream s) {
  if (!soup || !x1 || !bvh || !toi || !status || !ws || ws_bytes < kCandHeader || bvh->n != soup->n_tris)
    return IPCB_E_ARG;
  const int nv = soup->n_verts;
  if (first < 0 || count < 0 || first > nv || count > nv - first) return IPCB_E_ARG;
  if (count == 0 || soup->n_tris == 0) return IPCB_OK;
  const CandList c = cand_list(ws, ws_bytes);
  if (soup->fp64)
    run_pt<double>(soup, x1, bvh, pad, exclude_same_body, c, toi, status, Sink{}, (cudaStream_t)s, first, count);
  else
    run_pt<float>(soup, x1, bvh, pad, exclude_same_body, c, toi, status, Sink{}, (cudaStream_t)s, first, count);
  return check_launch("ipcb_point_triangle_toi");
}

int ipcb_point_triangle_toi(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, double pad,
                            int exclude_same_body, void* toi, int* status, void* ws, size_t ws_bytes,
                            ipcb_stream s) {
  if (!soup) return IPCB_E_ARG;
  return ipcb_point_triangle_toi_range(soup, x1, bvh, pad, exclude_same_body, 0, soup->n_verts, toi, status, ws,
                                       ws_bytes, s);
}

int ipcb_edge_edge_intersections(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, const float* lower,
                                 const float* upper, int exclude_same_body, double thickness, void* toi,
                                 const ipcb_contacts* out, int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!soup || !x1 || !bvh || !lower || !upper || !toi || !out || !out->cnt || !status || !ws || ws_bytes < kCandHeader ||
      bvh->n != soup->n_edges)
    return IPCB_E_ARG;
  if (out->capacity > 0 && (!out->a1a2b1b2 || !out->e0e1 || !out->l0 || !out->alpha || !out->lam)) return IPCB_E_ARG;
  if (soup->n_edges == 0) return IPCB_OK;
  const CandList c = cand_list(ws, ws_bytes);
  const Sink sink{*out, thickness * 2.0, 1};
  const int n = soup->n_edges;
  if (soup->fp64)
    run_ee<double>(soup, x1, bvh, lower, upper, exclude_same_body, c, toi, status, sink, (cudaStream_t)s, 0, n);
  else
    run_ee<float>(soup, x1, bvh, lower, upper, exclude_same_body, c, toi, status, sink, (cudaStream_t)s, 0, n);
  return check_launch("ipcb_edge_edge_intersections");
}

int ipcb_point_triangle_intersections(const ipcb_soup* soup, const void* x1, const ipcb_lbvh* bvh, double pad,
                                      int exclude_same_body, double thickness, void* toi, const ipcb_contacts* out,
                                      int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!soup || !x1 || !bvh || !toi || !out || !out->cnt || !status || !ws || ws_bytes < kCandHeader ||
      bvh->n != soup->n_tris)
    return IPCB_E_ARG;
  if (out->capacity > 0 && (!out->a1a2b1b2 || !out->e0e1 || !out->l0 || !out->alpha || !out->lam)) return IPCB_E_ARG;
  if (soup->n_verts == 0 || soup->n_tris == 0) return IPCB_OK;
  const CandList c = cand_list(ws, ws_bytes);
  const Sink sink{*out, thickness * 2.0, 1};
  const int nv = soup->n_verts;
  if (soup->fp64)
    run_pt<double>(soup, x1, bvh, pad, exclude_same_body, c, toi, status, sink, (cudaStream_t)s, 0, nv);
  else
    run_pt<float>(soup, x1, bvh, pad, exclude_same_body, c, toi, status, sink, (cudaStream_t)s, 0, nv);
  return check_launch("ipcb_point_triangle_intersections");
}

int ipcb_collision_time(int kind, int n, const double* p_t0, const double* p_t1, double* t, int* status,
                        ipcb_stream s) {
  if (n < 0 || (kind != 0 && kind != 1)) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  if (!p_t0 || !p_t1 || !t || !status) return IPCB_E_ARG;
  k_pair_time<<<div_up(n, 128), 128, 0, (cudaStream_t)s>>>(kind, n, p_t0, p_t1, t, status);
  return check_launch("ipcb_collision_time");
}

int ipcb_cubic_roots(int n, const double* coef, double x0, double x1, double* roots, int* n_roots, int* status,
                     ipcb_stream s) {
  if (n < 0) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  if (!coef || !roots || !n_roots || !status) return IPCB_E_ARG;
  k_cubic<<<div_up(n, 128), 128, 0, (cudaStream_t)s>>>(n, coef, x0, x1, roots, n_roots, status);
  return check_launch("ipcb_cubic_roots");
}


static bool bodies_ok(const ipcb_bodies* B) {
  return B && B->n_bodies > 0 && B->local_lower && B->local_upper && B->edge_off && B->edge_ids && B->tri_off &&
         B->tri_ids && B->vert_off && B->vert_ids && B->edge_wide && B->tri_wide && B->frames && B->motion;
}

int ipcb_body_pairs_swept(const ipcb_bodies* B, int fp64, const void* q, const void* dq, double padding, int* pairs,
                          int capacity, int* count, int* status, ipcb_stream s) {
  if (!bodies_ok(B) || !q || !dq || !pairs || capacity < 0 || !count || !status) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int nb = B->n_bodies;
  if (fp64)
    k_body_frames_swept<double><<<div_up(nb, 128), 128, 0, st>>>(nb, (const double*)q, (const double*)dq,
                                                                  B->local_lower, B->local_upper, B->frames,
                                                                  B->motion, status);
  else
    k_body_frames_swept<float><<<div_up(nb, 128), 128, 0, st>>>(nb, (const float*)q, (const float*)dq,
                                                                 B->local_lower, B->local_upper, B->frames,
                                                                 B->motion, status);
  k_swept_pair_cull<<<div_up((long long)nb * nb, 256), 256, 0, st>>>(nb, B->frames + 13 * (size_t)nb, padding,
                                                                     (int2*)pairs, capacity, count);
  return check_launch("ipcb_body_pairs_swept");
}

int ipcb_fixed_edge_edge_toi(const ipcb_soup* soup, const void* x1, const ipcb_bodies* B, const int* fixed,
                             const int* pairs, int n_pairs, double pad, void* toi, int* status, void* ws,
                             size_t ws_bytes, ipcb_stream s) {
  if (!soup || !x1 || !bodies_ok(B) || !pairs || n_pairs < 0 || !toi || !status || !ws || ws_bytes < kCandHeader)
    return IPCB_E_ARG;
  if (n_pairs == 0 || B->max_edges == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  CandList c = cand_list(ws, ws_bytes);
  cudaMemsetAsync(c.count, 0, sizeof(int), st);
  dim3 grid(div_up(B->max_edges, 128) * n_pairs);
  const int gc = min(div_up(c.capacity > 0 ? c.capacity : 1, 128), 2048);
  if (soup->fp64) {
    k_fixed_ee_collect<double><<<grid, 128, 0, st>>>((const double*)soup->x, (const double*)x1, soup->edges, *B,
                                                     fixed, (const int2*)pairs, pad, c, (double*)toi, status);
    if (c.capacity)
      k_cand_toi<double, 0><<<gc, 128, 0, st>>>((const double*)soup->x, (const double*)x1, soup->edges, c,
                                              (double*)toi, status, Sink{}, nullptr);
  } else {
    k_fixed_ee_collect<float><<<grid, 128, 0, st>>>((const float*)soup->x, (const float*)x1, soup->edges, *B, fixed,
                                                    (const int2*)pairs, pad, c, (float*)toi, status);
    if (c.capacity)
      k_cand_toi<float, 0><<<gc, 128, 0, st>>>((const float*)soup->x, (const float*)x1, soup->edges, c, (float*)toi,
                                             status, Sink{}, nullptr);
  }
  return check_launch("ipcb_fixed_edge_edge_toi");
}

int ipcb_fixed_point_triangle_toi(const ipcb_soup* soup, const void* x1, const ipcb_bodies* B, const int* pairs,
                                  int n_pairs, double pad, void* toi, int* status, void* ws, size_t ws_bytes,
                                  ipcb_stream s) {
  if (!soup || !x1 || !bodies_ok(B) || !pairs || n_pairs < 0 || !toi || !status || !ws || ws_bytes < kCandHeader)
    return IPCB_E_ARG;
  if (n_pairs == 0 || B->max_verts == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  CandList c = cand_list(ws, ws_bytes);
  cudaMemsetAsync(c.count, 0, sizeof(int), st);
  dim3 grid(div_up(B->max_verts, 128) * n_pairs, 2);
  const int gc = min(div_up(c.capacity > 0 ? c.capacity : 1, 128), 2048);
  if (soup->fp64) {
    k_fixed_pt_collect<double><<<grid, 128, 0, st>>>((const double*)soup->x, (const double*)x1, soup->triangles, *B,
                                                     (const int2*)pairs, pad, c, (double*)toi, status);
    if (c.capacity)
      k_cand_toi<double, 1><<<gc, 128, 0, st>>>((const double*)soup->x, (const double*)x1, soup->triangles, c,
                                              (double*)toi, status, Sink{}, nullptr);
  } else {
    k_fixed_pt_collect<float><<<grid, 128, 0, st>>>((const float*)soup->x, (const float*)x1, soup->triangles, *B,
                                                    (const int2*)pairs, pad, c, (float*)toi, status);
    if (c.capacity)
      k_cand_toi<float, 1><<<gc, 128, 0, st>>>((const float*)soup->x, (const float*)x1, soup->triangles, c,
                                             (float*)toi, status, Sink{}, nullptr);
  }
  return check_launch("ipcb_fixed_point_triangle_toi");
}

}  // extern "C"
