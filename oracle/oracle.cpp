// CPU oracle for the ipc_warp contact pipeline.  TEST INFRASTRUCTURE ONLY:
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it as
// the checker.  The product (ipc_warp_b200) never links or calls it.
//
// Restates, in plain C++17 (g++ -O3 -fopenmp -ffp-contract=off):
//   * closest_point_triangle             contact.py:230-302  (float32, exact op order)
//   * segment-segment closest points     Warp builtin wp.closest_point_edge_edge used at
//                                        contact.py:101,226 -- not in the reference tree;
//                                        restated from Ericson, Real-Time Collision
//                                        Detection (2005) 5.1.9.  Parity unpinned.
//   * EE / PT candidate acceptance       contact.py:199-228, 304-336 (filters, F10 order)
//   * feature dispatch + Hessian compose dynamic_contacts.py:49-125, 152-246, 375-398
//   * IPC barrier / EE mollifier         ipctkwp (empty submodule): restated from
//                                        Li et al. 2020 (IPC) eqs. for b(d^2) and the
//                                        EE mollifier.  Parity unpinned.
//   * NSD part of the squared-distance   ipctkwp x_to_grad_nsd_hess_*: restated as the
//     Hessian                            exact negative spectral part.  Mode 0 computes
//                                        it independently (hyper-dual second derivatives
//                                        of the explicit distance formula + 12x12
//                                        Jacobi); mode 1 uses the analytic low-rank
//                                        subspace form (the one the CUDA kernels use).
//   * cubic CCD                          ccd/ccd.py:212-357, ccd/cubic_roots.py:7-193
//                                        (beta_gamma_* restated: ipctkwp is empty)
// Candidate sets are pinned against outputs of the reference's own Python
// functions run under a Warp stand-in (tests/golden/make_golden.py).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>
#include <omp.h>

namespace {

template <class T>
struct V3 {
  T x, y, z;
};
template <class T> inline V3<T> mk(T x, T y, T z) { return V3<T>{x, y, z}; }
template <class T> inline V3<T> operator+(V3<T> a, V3<T> b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> inline V3<T> operator-(V3<T> a, V3<T> b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> inline V3<T> operator*(V3<T> a, T s) { return mk(a.x * s, a.y * s, a.z * s); }
template <class T> inline V3<T> operator*(T s, V3<T> a) { return mk(s * a.x, s * a.y, s * a.z); }
template <class T> inline T dot(V3<T> a, V3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> inline V3<T> cross(V3<T> a, V3<T> b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class T> inline T length(V3<T> a) { return std::sqrt(dot(a, a)); }
template <class T> inline T tmin(T a, T b) { return a < b ? a : b; }
template <class T> inline T tmax(T a, T b) { return a > b ? a : b; }
template <class T> inline T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }

template <class T> inline V3<T> load3(const T* p, int i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
template <class T> inline V3<float> f32(V3<T> a) { return mk((float)a.x, (float)a.y, (float)a.z); }
template <class T> inline V3<double> f64(V3<T> a) { return mk((double)a.x, (double)a.y, (double)a.z); }

// ---------------------------------------------------------------- predicates
// contact.py:230-302.  Returns (u, v, dist) and the Voronoi type 0..6.
struct CPT {
  float u, v, d;
  int type;
};
CPT closest_point_triangle(V3<float> p, V3<float> a, V3<float> b, V3<float> c) {
  CPT r{0.f, 0.f, 0.f, -1};
  V3<float> ab = b - a, ac = c - a, ap = p - a;
  float d1 = dot(ab, ap), d2 = dot(ac, ap);
  if (d1 <= 0.f && d2 <= 0.f) { r = {1.f, 0.f, length(p - a), 0}; }
  V3<float> bp = p - b;
  float d3 = dot(ab, bp), d4 = dot(ac, bp);
  if (d3 >= 0.f && d4 <= d3 && r.type == -1) { r = {0.f, 1.f, length(p - b), 1}; }
  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f && r.type == -1) {
    float v = d1 / (d1 - d3);
    V3<float> pt = a + v * ab;
    r = {1.f - v, v, length(p - pt), 3};
  }
  V3<float> cp = p - c;
  float d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.f && d5 <= d6 && r.type == -1) { r = {0.f, 0.f, length(p - c), 2}; }
  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f && r.type == -1) {
    float w = d2 / (d2 - d6);
    V3<float> pt = a + w * ac;
    r = {1.f - w, 0.f, length(p - pt), 4};
  }
  float va = d3 * d6 - d5 * d4;
  if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f && r.type == -1) {
    float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    V3<float> pt = b + w * (c - b);
    r = {0.f, 1.f - w, length(p - pt), 5};
  }
  if (r.type == -1) {
    float denom = 1.f / (va + vb + vc);
    float v = vb * denom, w = vc * denom;
    float u = 1.f - v - w;
    V3<float> pt = a + ab * v + ac * w;
    r = {u, v, length(p - pt), 6};
  }
  return r;
}

// Ericson RTCD 5.1.9, segment p1q1 vs p2q2; returns (s, t, dist).
struct CPEE {
  float s, t, d;
};
CPEE closest_point_edge_edge(V3<float> p1, V3<float> q1, V3<float> p2, V3<float> q2, float eps) {
  V3<float> d1 = q1 - p1, d2 = q2 - p2, r = p1 - p2;
  float a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  float s = 0.f, t = 0.f;
  if (a <= eps && e <= eps) {
    s = 0.f;
    t = 0.f;
  } else if (a <= eps) {
    s = 0.f;
    t = clampv(f / e, 0.f, 1.f);
  } else {
    float c = dot(d1, r);
    if (e <= eps) {
      t = 0.f;
      s = clampv(-c / a, 0.f, 1.f);
    } else {
      float b = dot(d1, d2);
      float denom = a * e - b * b;
      if (denom != 0.f) s = clampv((b * f - c * e) / denom, 0.f, 1.f);
      else s = 0.f;
      t = (b * s + f) / e;
      if (t < 0.f) {
        t = 0.f;
        s = clampv(-c / a, 0.f, 1.f);
      } else if (t > 1.f) {
        t = 1.f;
        s = clampv((b - c) / a, 0.f, 1.f);
      }
    }
  }
  V3<float> c1 = p1 + d1 * s, c2 = p2 + d2 * t;
  return CPEE{s, t, length(c1 - c2)};
}

// ------------------------------------------------------------ barrier (IPC)
// b(x) = -kappa (x - xh)^2 ln(x / xh) for 0 < x < xh, x = d^2, xh = dhat^2.
struct Barrier {
  double b, db, d2b;
};
Barrier barrier(double x, double xh, double kappa) {
  Barrier r{0.0, 0.0, 0.0};
  if (x >= xh) return r;
  double dx = x - xh, lg = std::log(x / xh);
  r.b = -kappa * dx * dx * lg;
  r.db = kappa * (-2.0 * dx * lg - dx * dx / x);
  r.d2b = kappa * (-2.0 * lg - 4.0 * dx / x + dx * dx / (x * x));
  return r;
}

// ------------------------------------------------------- symmetric eigen
// Cyclic Jacobi; a is n x n row-major symmetric, destroyed.  w: eigenvalues,
// v: eigenvectors in columns.
void jacobi_eig(double* a, int n, double* w, double* v) {
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) v[i * n + j] = (i == j) ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += a[i * n + j] * a[i * n + j];
        if (i != j) off += a[i * n + j] * a[i * n + j];
      }
    if (off <= 1e-32 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        double apq = a[p * n + q];
        if (apq == 0.0) continue;
        double app = a[p * n + p], aqq = a[q * n + q];
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          double vkp = v[k * n + p], vkq = v[k * n + q];
          v[k * n + p] = c * vkp - s * vkq;
          v[k * n + q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
}

// --------------------------------------------- hyper-dual (2nd-order) jets
struct Jet {
  double v;
  double g[12];
  double h[12][12];
};
inline Jet jconst(double c) {
  Jet r;
  std::memset(&r, 0, sizeof(r));
  r.v = c;
  return r;
}
inline Jet jvar(double c, int i) {
  Jet r = jconst(c);
  r.g[i] = 1.0;
  return r;
}
inline Jet operator+(const Jet& a, const Jet& b) {
  Jet r;
  r.v = a.v + b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] + b.g[i];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) r.h[i][j] = a.h[i][j] + b.h[i][j];
  return r;
}
inline Jet operator-(const Jet& a, const Jet& b) {
  Jet r;
  r.v = a.v - b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] - b.g[i];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j) r.h[i][j] = a.h[i][j] - b.h[i][j];
  return r;
}
inline Jet operator*(const Jet& a, const Jet& b) {
  Jet r;
  r.v = a.v * b.v;
  for (int i = 0; i < 12; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j)
      r.h[i][j] = a.h[i][j] * b.v + a.g[i] * b.g[j] + a.g[j] * b.g[i] + a.v * b.h[i][j];
  return r;
}
inline Jet recip(const Jet& a) {
  Jet r;
  double iv = 1.0 / a.v;
  r.v = iv;
  for (int i = 0; i < 12; ++i) r.g[i] = -a.g[i] * iv * iv;
  for (int i = 0; i < 12; ++i)
    for (int j = 0; j < 12; ++j)
      r.h[i][j] = 2.0 * a.g[i] * a.g[j] * iv * iv * iv - a.h[i][j] * iv * iv;
  return r;
}
struct JV {
  Jet x, y, z;
};
inline JV jv(const double* p, int slot) {
  return JV{jvar(p[0], 3 * slot), jvar(p[1], 3 * slot + 1), jvar(p[2], 3 * slot + 2)};
}
inline JV operator-(const JV& a, const JV& b) { return JV{a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Jet jdot(const JV& a, const JV& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline JV jcross(const JV& a, const JV& b) {
  return JV{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// Squared distance of the active feature, as an explicit function of up to 4
// points (slots 0..3 of the 12 jet variables).
//   kind 0 PP: |a-b|^2;  1 PE: |(p-e0)x(e1-e0)|^2/|e1-e0|^2;
//   2 PT-plane: ((p-t0).n)^2/|n|^2;  3 EE-line: ((a0-b0).n)^2/|n|^2
Jet feature_d2_jet(int kind, const double* P /*4x3*/) {
  JV v0 = jv(P + 0, 0), v1 = jv(P + 3, 1), v2 = jv(P + 6, 2), v3 = jv(P + 9, 3);
  if (kind == 0) {
    JV d = v0 - v1;
    return jdot(d, d);
  }
  if (kind == 1) {
    JV e = v2 - v1, u = v0 - v1;
    JV c = jcross(u, e);
    return jdot(c, c) * recip(jdot(e, e));
  }
  if (kind == 2) {
    JV n = jcross(v2 - v1, v3 - v1);
    Jet s = jdot(v0 - v1, n);
    return s * s * recip(jdot(n, n));
  }
  JV n = jcross(v1 - v0, v3 - v2);
  Jet s = jdot(v0 - v2, n);
  return s * s * recip(jdot(n, n));
}

// Gradient (12) and NSD part (12x12) of the squared distance of a feature on
// `nv` local points, embedded at `slots` of the 4 contact vertices.
struct FeatureDH {
  double g[12];
  double h[144];
};

void embed(const double* gl, const double* hl, int nv, const int* slots, FeatureDH& out) {
  std::memset(&out, 0, sizeof(out));
  for (int a = 0; a < nv; ++a)
    for (int k = 0; k < 3; ++k) out.g[3 * slots[a] + k] = gl[3 * a + k];
  int m = 3 * nv;
  for (int a = 0; a < nv; ++a)
    for (int b = 0; b < nv; ++b)
      for (int k = 0; k < 3; ++k)
        for (int l = 0; l < 3; ++l)
          out.h[(3 * slots[a] + k) * 12 + 3 * slots[b] + l] = hl[(3 * a + k) * m + 3 * b + l];
}

// Mode 0: jets + full Jacobi.
void feature_dh_jet(int kind, const V3<double>* pts, int nv, const int* slots, FeatureDH& out) {
  double P[12] = {0};
  for (int a = 0; a < nv; ++a) {
    P[3 * a] = pts[a].x;
    P[3 * a + 1] = pts[a].y;
    P[3 * a + 2] = pts[a].z;
  }
  Jet f = feature_d2_jet(kind, P);
  int m = 3 * nv;
  double gl[12], hl[144], a[144], w[12], v[144];
  for (int i = 0; i < m; ++i) gl[i] = f.g[i];
  for (int i = 0; i < m; ++i)
    for (int j = 0; j < m; ++j) a[i * m + j] = 0.5 * (f.h[i][j] + f.h[j][i]);
  std::memset(hl, 0, sizeof(hl));
  if (kind != 0) {
    jacobi_eig(a, m, w, v);
    for (int e = 0; e < m; ++e) {
      if (!(w[e] < 0.0)) continue;
      for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) hl[i * m + j] += w[e] * v[i * m + e] * v[j * m + e];
    }
  }
  embed(gl, hl, nv, slots, out);
}

// Mode 1: analytic low-rank subspace.  d^2 = min_tau |sum_k c_k(tau) x_k|^2 with
// c affine in tau; Hessian = 2(cc^T)(x)(I-P) - 2 sum_j[(c d_j^T)(x)(E~_j r^T) + T]
//                            - 2 (D G^-1 D^T)(x)(r r^T)
// restricted to span{c^ (x) frame, f_a (x) n^}.
static inline V3<double> nrm(V3<double> a) { return a * (1.0 / length(a)); }

void feature_dh_subspace(int kind, const V3<double>* pts, int nv, const int* slots, FeatureDH& out) {
  double gl[12] = {0}, hl[144] = {0};
  int m = 3 * nv;
  if (kind == 0) {
    V3<double> d = pts[0] - pts[1];
    gl[0] = 2 * d.x; gl[1] = 2 * d.y; gl[2] = 2 * d.z;
    gl[3] = -2 * d.x; gl[4] = -2 * d.y; gl[5] = -2 * d.z;
    embed(gl, hl, nv, slots, out);
    return;
  }
  // c: weights, D: param derivatives of c, E: param edge vectors, n: unit normal
  double c[4] = {0}, D[2][4] = {{0}}, rho;
  V3<double> E[2], nh;
  int np;
  if (kind == 1) {  // p, e0, e1
    V3<double> p = pts[0], e0 = pts[1], e1 = pts[2];
    V3<double> e = e1 - e0;
    double t = dot(p - e0, e) / dot(e, e);
    V3<double> r = p - e0 - e * t;
    rho = length(r);
    nh = r * (1.0 / rho);
    c[0] = 1; c[1] = -(1 - t); c[2] = -t;
    D[0][1] = 1; D[0][2] = -1;
    E[0] = e0 - e1;
    np = 1;
  } else if (kind == 2) {  // p, t0, t1, t2
    V3<double> p = pts[0], t0 = pts[1], t1 = pts[2], t2 = pts[3];
    V3<double> e1 = t1 - t0, e2 = t2 - t0, w = p - t0;
    double g11 = dot(e1, e1), g12 = dot(e1, e2), g22 = dot(e2, e2);
    double b1 = dot(e1, w), b2 = dot(e2, w), det = g11 * g22 - g12 * g12;
    double be = (g22 * b1 - g12 * b2) / det, ga = (g11 * b2 - g12 * b1) / det;
    nh = nrm(cross(e1, e2));
    rho = dot(w, nh);
    c[0] = 1; c[1] = -1 + be + ga; c[2] = -be; c[3] = -ga;
    D[0][1] = 1; D[0][2] = -1;
    D[1][1] = 1; D[1][3] = -1;
    E[0] = t0 - t1; E[1] = t0 - t2;
    np = 2;
  } else {  // a0, a1, b0, b1
    V3<double> a0 = pts[0], a1 = pts[1], b0 = pts[2], b1 = pts[3];
    V3<double> ea = a1 - a0, eb = b1 - b0, w = a0 - b0;
    double g11 = dot(ea, ea), g12 = -dot(ea, eb), g22 = dot(eb, eb);
    double r1 = -dot(ea, w), r2 = dot(eb, w), det = g11 * g22 - g12 * g12;
    double s = (g22 * r1 - g12 * r2) / det, t = (g11 * r2 - g12 * r1) / det;
    nh = nrm(cross(ea, eb));
    rho = dot(w, nh);
    c[0] = 1 - s; c[1] = s; c[2] = -(1 - t); c[3] = -t;
    D[0][0] = -1; D[0][1] = 1;
    D[1][2] = 1; D[1][3] = -1;
    E[0] = ea; E[1] = eb * -1.0;
    np = 2;
  }
  // gradient: 2 c_k r, r = rho n^
  V3<double> r = nh * rho;
  for (int k = 0; k < nv; ++k) {
    gl[3 * k] = 2 * c[k] * r.x;
    gl[3 * k + 1] = 2 * c[k] * r.y;
    gl[3 * k + 2] = 2 * c[k] * r.z;
  }
  // 4D orthonormal basis: ch, f1 (, f2)
  double cn = 0;
  for (int k = 0; k < 4; ++k) cn += c[k] * c[k];
  cn = std::sqrt(cn);
  double ch[4], f[2][4];
  for (int k = 0; k < 4; ++k) ch[k] = c[k] / cn;
  for (int j = 0; j < np; ++j) {
    double v[4];
    for (int k = 0; k < 4; ++k) v[k] = D[j][k];
    double pc = 0;
    for (int k = 0; k < 4; ++k) pc += v[k] * ch[k];
    for (int k = 0; k < 4; ++k) v[k] -= pc * ch[k];
    for (int q = 0; q < j; ++q) {
      double pf = 0;
      for (int k = 0; k < 4; ++k) pf += v[k] * f[q][k];
      for (int k = 0; k < 4; ++k) v[k] -= pf * f[q][k];
    }
    double vn = 0;
    for (int k = 0; k < 4; ++k) vn += v[k] * v[k];
    vn = std::sqrt(vn);
    for (int k = 0; k < 4; ++k) f[j][k] = v[k] / vn;
  }
  // Gram of E and its inverse
  double G[2][2], Gi[2][2];
  if (np == 1) {
    G[0][0] = dot(E[0], E[0]);
    Gi[0][0] = 1.0 / G[0][0];
  } else {
    G[0][0] = dot(E[0], E[0]); G[0][1] = dot(E[0], E[1]); G[1][1] = dot(E[1], E[1]);
    G[1][0] = G[0][1];
    double det = G[0][0] * G[1][1] - G[0][1] * G[0][1];
    Gi[0][0] = G[1][1] / det; Gi[1][1] = G[0][0] / det;
    Gi[0][1] = Gi[1][0] = -G[0][1] / det;
  }
  // spatial in-span frame t1 (, t2)
  V3<double> th[2];
  th[0] = nrm(E[0]);
  if (np == 2) th[1] = cross(nh, th[0]);
  // dual vectors
  V3<double> Ed[2];
  for (int j = 0; j < np; ++j) {
    Ed[j] = mk(0.0, 0.0, 0.0);
    for (int k = 0; k < np; ++k) Ed[j] = Ed[j] + E[k] * Gi[j][k];
  }
  int nz = 1 + np, nw = np, ns = nz + nw;
  double Dm[2][3] = {{0}}, Tm[2][2] = {{0}};
  for (int j = 0; j < np; ++j) {
    double s0 = 0;
    for (int k = 0; k < 4; ++k) s0 += D[j][k] * ch[k];
    Dm[j][0] = s0;
    for (int a = 0; a < np; ++a) {
      double sa = 0;
      for (int k = 0; k < 4; ++k) sa += D[j][k] * f[a][k];
      Dm[j][1 + a] = sa;
    }
    for (int i = 0; i < np; ++i) Tm[j][i] = dot(th[i], Ed[j]);
  }
  double M[25] = {0};
  for (int a = 0; a < nz; ++a)
    for (int b = 0; b < nz; ++b) {
      double s = 0;
      for (int i = 0; i < np; ++i)
        for (int j = 0; j < np; ++j) s += Dm[i][a] * Gi[i][j] * Dm[j][b];
      M[a * ns + b] = -2.0 * rho * rho * s + ((a == 0 && b == 0) ? 2.0 * cn * cn : 0.0);
    }
  for (int a = 0; a < nz; ++a)
    for (int i = 0; i < nw; ++i) {
      double s = 0;
      for (int j = 0; j < np; ++j) s += Dm[j][a] * Tm[j][i];
      M[a * ns + nz + i] = M[(nz + i) * ns + a] = -2.0 * rho * cn * s;
    }
  double w[5], V[25];
  jacobi_eig(M, ns, w, V);
  // basis vectors (12): phi_a for z then w
  double phi[5][12] = {{0}};
  auto setkron = [&](double* dst, const double* a4, V3<double> s) {
    for (int k = 0; k < 4; ++k) {
      dst[3 * k] = a4[k] * s.x;
      dst[3 * k + 1] = a4[k] * s.y;
      dst[3 * k + 2] = a4[k] * s.z;
    }
  };
  setkron(phi[0], ch, nh);
  for (int a = 0; a < np; ++a) setkron(phi[1 + a], f[a], nh);
  for (int i = 0; i < np; ++i) setkron(phi[nz + i], ch, th[i]);
  for (int e = 0; e < ns; ++e) {
    if (!(w[e] < 0.0)) continue;
    double u[12] = {0};
    for (int b = 0; b < ns; ++b)
      for (int i = 0; i < 12; ++i) u[i] += V[b * ns + e] * phi[b][i];
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) hl[i * m + j] += w[e] * u[i] * u[j];
  }
  embed(gl, hl, nv, slots, out);
}

typedef void (*FeatureFn)(int, const V3<double>*, int, const int*, FeatureDH&);

// ------------------------------------------------------------ narrow phase
// Per-pair output of the restated contact kernels (dynamic_contacts.py:152-246):
// force (12, = -gradient of the barrier energy), Hessian (12x12), energy.
template <class S>
struct NarrowOut {
  double* force;   // n x 12
  double* hess;    // n x 144
  double* energy;  // n
  int* active;     // n  (1 if dist < l0), feature code in bits 8..
};

// dynamic_contacts.py:49-108 with the F9 float32 closest-point cast.
template <class S>
void ee_feature(const V3<S> x[4], S parallel_eps, int& kind, int& nv, V3<double> pts[4], int slots[4], bool& near_par) {
  CPEE dab = closest_point_edge_edge(f32(x[0]), f32(x[1]), f32(x[2]), f32(x[3]), 1.0e-6f);
  S s = (S)dab.s, t = (S)dab.t;
  S feps = (S)1.0e-6;
  S one = (S)1.0;
  bool sb = s <= feps || s >= one - feps;
  bool tb = t <= feps || t >= one - feps;
  near_par = false;
  if (sb && tb) {
    int oa = 0, ob = 2;
    if (s >= one - feps) oa = 1;
    if (t >= one - feps) ob = 3;
    kind = 0; nv = 2;
    pts[0] = f64(x[oa]); pts[1] = f64(x[ob]);
    slots[0] = oa; slots[1] = ob;
    return;
  }
  if (sb) {
    int oa = (s >= one - feps) ? 1 : 0;
    kind = 1; nv = 3;
    pts[0] = f64(x[oa]); pts[1] = f64(x[2]); pts[2] = f64(x[3]);
    slots[0] = oa; slots[1] = 2; slots[2] = 3;
    return;
  }
  if (tb) {
    int ob = (t >= one - feps) ? 3 : 2;
    kind = 1; nv = 3;
    pts[0] = f64(x[ob]); pts[1] = f64(x[0]); pts[2] = f64(x[1]);
    slots[0] = ob; slots[1] = 0; slots[2] = 1;
    return;
  }
  V3<S> ea = x[1] - x[0], eb = x[3] - x[2];
  V3<S> cr = cross(ea, eb);
  if (parallel_eps > (S)0 && dot(cr, cr) < parallel_eps) {
    S ds0 = s, ds1 = one - s, dt0 = t, dt1 = one - t;
    S mn = tmin(tmin(ds0, ds1), tmin(dt0, dt1));
    int p, q0, q1;
    if (mn == ds0) { p = 0; q0 = 2; q1 = 3; }
    else if (mn == ds1) { p = 1; q0 = 2; q1 = 3; }
    else if (mn == dt0) { p = 2; q0 = 0; q1 = 1; }
    else { p = 3; q0 = 0; q1 = 1; }
    kind = 1; nv = 3;
    pts[0] = f64(x[p]); pts[1] = f64(x[q0]); pts[2] = f64(x[q1]);
    slots[0] = p; slots[1] = q0; slots[2] = q1;
    return;
  }
  kind = 3; nv = 4;
  for (int k = 0; k < 4; ++k) { pts[k] = f64(x[k]); slots[k] = k; }
}

// dynamic_contacts.py:111-125
template <class S>
void pt_feature(const V3<S> x[4], int& kind, int& nv, V3<double> pts[4], int slots[4]) {
  CPT cp = closest_point_triangle(f32(x[0]), f32(x[1]), f32(x[2]), f32(x[3]));
  int t = cp.type;
  if (t <= 2) {
    int o = t + 1;
    kind = 0; nv = 2;
    pts[0] = f64(x[0]); pts[1] = f64(x[o]);
    slots[0] = 0; slots[1] = o;
    return;
  }
  if (t <= 5) {
    int a = (t == 5) ? 2 : 1, b = (t == 3) ? 2 : 3;
    kind = 1; nv = 3;
    pts[0] = f64(x[0]); pts[1] = f64(x[a]); pts[2] = f64(x[b]);
    slots[0] = 0; slots[1] = a; slots[2] = b;
    return;
  }
  kind = 2; nv = 4;
  for (int k = 0; k < 4; ++k) { pts[k] = f64(x[k]); slots[k] = k; }
}

// EE mollifier (IPC): eps_x = 1e-3 |ea_rest|^2 |eb_rest|^2,
// m(x) = (2 - x/eps_x) x/eps_x for x < eps_x else 1, x = |ea x eb|^2.
template <class S>
S ee_eps_x(const V3<S> r[4]) {
  V3<S> ea = r[1] - r[0], eb = r[3] - r[2];
  return (S)1.0e-3 * dot(ea, ea) * dot(eb, eb);
}

template <class S>
void narrow_ee(int n, const int* idx, const S* l0, const S* x, const S* xcs, double kappa, FeatureFn fn, NarrowOut<S> o) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const int* id = idx + 4 * i;
    V3<S> xs[4], rs[4];
    for (int k = 0; k < 4; ++k) { xs[k] = load3(x, id[k]); rs[k] = load3(xcs, id[k]); }
    double* F = o.force + 12 * i;
    double* H = o.hess + 144 * i;
    std::memset(F, 0, 12 * sizeof(double));
    std::memset(H, 0, 144 * sizeof(double));
    o.energy[i] = 0.0;
    o.active[i] = 0;
    CPEE dab = closest_point_edge_edge(f32(xs[0]), f32(xs[1]), f32(xs[2]), f32(xs[3]), 1.0e-6f);
    S dist = (S)dab.d;
    if (!(dist < l0[i])) continue;
    S eps_x = ee_eps_x(rs);
    V3<S> ea = xs[1] - xs[0], eb = xs[3] - xs[2];
    V3<S> cr = cross(ea, eb);
    S crn = dot(cr, cr);
    bool near_par = eps_x > (S)0 && crn < eps_x;
    int kind, nv, slots[4];
    V3<double> pts[4];
    bool np_unused;
    ee_feature(xs, eps_x, kind, nv, pts, slots, np_unused);
    FeatureDH fd;
    fn(kind, pts, nv, slots, fd);
    double d2 = (double)dab.d * (double)dab.d;
    double d02 = (double)l0[i] * (double)l0[i];
    Barrier br = barrier(d2, d02, kappa);
    // mollifier value and gradient (only differs from 1 when near parallel)
    double mv = 1.0, gm[12] = {0};
    if (near_par) {
      V3<double> ead = f64(xs[1]) - f64(xs[0]), ebd = f64(xs[3]) - f64(xs[2]);
      double xc = dot(cross(ead, ebd), cross(ead, ebd)), ex = (double)eps_x;
      double q = xc / ex;
      mv = (2.0 - q) * q;
      double dm = 2.0 * (1.0 - q) / ex;
      V3<double> dxa = ead * (2.0 * dot(ebd, ebd)) - ebd * (2.0 * dot(ead, ebd));
      V3<double> dxb = ebd * (2.0 * dot(ead, ead)) - ead * (2.0 * dot(ead, ebd));
      double gx[12] = {-dxa.x, -dxa.y, -dxa.z, dxa.x, dxa.y, dxa.z, -dxb.x, -dxb.y, -dxb.z, dxb.x, dxb.y, dxb.z};
      for (int k = 0; k < 12; ++k) gm[k] = dm * gx[k];
    }
    if (near_par) {
      for (int a = 0; a < 12; ++a)
        for (int b = 0; b < 12; ++b) H[a * 12 + b] = mv * br.d2b * fd.g[a] * fd.g[b];
    } else {
      for (int a = 0; a < 12; ++a)
        for (int b = 0; b < 12; ++b) H[a * 12 + b] = br.d2b * fd.g[a] * fd.g[b] + br.db * fd.h[a * 12 + b];
    }
    for (int k = 0; k < 12; ++k) F[k] = -(mv * br.db * fd.g[k] + br.b * gm[k]);
    o.energy[i] = mv * br.b;
    o.active[i] = 1 | (kind << 8) | (near_par ? 1 << 12 : 0);
  }
}

template <class S>
void narrow_pt(int n, const int* idx, const S* l0, const S* x, double kappa, FeatureFn fn, NarrowOut<S> o) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    const int* id = idx + 4 * i;
    V3<S> xs[4];
    for (int k = 0; k < 4; ++k) xs[k] = load3(x, id[k]);
    double* F = o.force + 12 * i;
    double* H = o.hess + 144 * i;
    std::memset(F, 0, 12 * sizeof(double));
    std::memset(H, 0, 144 * sizeof(double));
    o.energy[i] = 0.0;
    o.active[i] = 0;
    CPT cp = closest_point_triangle(f32(xs[0]), f32(xs[1]), f32(xs[2]), f32(xs[3]));
    S dist = (S)cp.d;
    if (!(dist < l0[i])) continue;
    int kind, nv, slots[4];
    V3<double> pts[4];
    pt_feature(xs, kind, nv, pts, slots);
    FeatureDH fd;
    fn(kind, pts, nv, slots, fd);
    double d2 = (double)cp.d * (double)cp.d;
    double d02 = (double)l0[i] * (double)l0[i];
    Barrier br = barrier(d2, d02, kappa);
    for (int a = 0; a < 12; ++a)
      for (int b = 0; b < 12; ++b) H[a * 12 + b] = br.d2b * fd.g[a] * fd.g[b] + br.db * fd.h[a * 12 + b];
    for (int k = 0; k < 12; ++k) F[k] = -br.db * fd.g[k];
    o.energy[i] = br.b;
    o.active[i] = 1 | (kind << 8);
  }
}

// ------------------------------------------------------------ broad phase
struct Box {
  float lo[3], hi[3];
};
inline bool overlap(const Box& a, const Box& b) {
  return a.lo[0] <= b.hi[0] && b.lo[0] <= a.hi[0] && a.lo[1] <= b.hi[1] && b.lo[1] <= a.hi[1] &&
         a.lo[2] <= b.hi[2] && b.lo[2] <= a.hi[2];
}

// Uniform-grid pruning: calls fn(i, j) once for every query i and target j
// whose boxes overlap.  Targets are binned into every cell of a uniform grid
// (cell edge = twice the mean target extent) that their box touches; a query
// visits the cells its box touches and reports a pair only from the cell that
// holds the lower corner of the two boxes' intersection, so each pair is
// reported once.  Exactness of the candidate set comes from the predicate;
// the pruning only has to be conservative.
template <class Fn>
void sweep(const std::vector<Box>& q, const std::vector<Box>& t, Fn&& fn) {
  const int nt = (int)t.size(), nq = (int)q.size();
  if (nt == 0 || nq == 0) return;
  float lo[3] = {3.4e38f, 3.4e38f, 3.4e38f}, hi[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  double ext = 0.0;
  for (int j = 0; j < nt; ++j)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], t[j].lo[k]);
      hi[k] = std::max(hi[k], t[j].hi[k]);
      ext += (double)t[j].hi[k] - (double)t[j].lo[k];
    }
  double h = std::max(2.0 * ext / (3.0 * nt), 1e-30);
  long long dims[3];
  for (;;) {  // at most ~64M cells
    long long tot = 1;
    for (int k = 0; k < 3; ++k) {
      dims[k] = std::max(1LL, (long long)std::ceil(((double)hi[k] - lo[k]) / h) + 1);
      tot *= dims[k];
    }
    if (tot <= (1LL << 26)) break;
    h *= 1.5;
  }
  auto cell = [&](float v, int k) -> long long {
    double c = std::floor(((double)v - lo[k]) / h);
    return (long long)std::min(std::max(c, 0.0), (double)(dims[k] - 1));
  };
  auto key = [&](long long a, long long b, long long c) { return (a * dims[1] + b) * dims[2] + c; };
  std::vector<std::pair<long long, int>> bins;
  bins.reserve((size_t)nt * 2);
  for (int j = 0; j < nt; ++j) {
    long long a0 = cell(t[j].lo[0], 0), a1 = cell(t[j].hi[0], 0), b0 = cell(t[j].lo[1], 1),
              b1 = cell(t[j].hi[1], 1), c0 = cell(t[j].lo[2], 2), c1 = cell(t[j].hi[2], 2);
    for (long long a = a0; a <= a1; ++a)
      for (long long b = b0; b <= b1; ++b)
        for (long long c = c0; c <= c1; ++c) bins.push_back({key(a, b, c), j});
  }
  std::sort(bins.begin(), bins.end());
  std::vector<long long> keys(bins.size());
  for (size_t i = 0; i < bins.size(); ++i) keys[i] = bins[i].first;
#pragma omp parallel for schedule(dynamic, 256)
  for (int i = 0; i < nq; ++i) {
    const Box& Q = q[i];
    long long a0 = cell(Q.lo[0], 0), a1 = cell(Q.hi[0], 0), b0 = cell(Q.lo[1], 1), b1 = cell(Q.hi[1], 1),
              c0 = cell(Q.lo[2], 2), c1 = cell(Q.hi[2], 2);
    for (long long a = a0; a <= a1; ++a)
      for (long long b = b0; b <= b1; ++b)
        for (long long c = c0; c <= c1; ++c) {
          long long k = key(a, b, c);
          size_t p = (size_t)(std::lower_bound(keys.begin(), keys.end(), k) - keys.begin());
          for (; p < keys.size() && keys[p] == k; ++p) {
            int j = bins[p].second;
            const Box& T = t[j];
            if (!overlap(Q, T)) continue;
            // report from the cell of the intersection's lower corner only
            if (cell(std::max(Q.lo[0], T.lo[0]), 0) != a || cell(std::max(Q.lo[1], T.lo[1]), 1) != b ||
                cell(std::max(Q.lo[2], T.lo[2]), 2) != c)
              continue;
            fn(i, j);
          }
        }
  }
}


// ------------------------------------------------------------------- CCD
// ccd/cubic_roots.py:7-193 and ccd/ccd.py:212-357, in double.
struct P4 {
  double c[4];
};
inline double evaluate(const P4& p, double x) { return p.c[0] + x * (p.c[1] + x * (p.c[2] + x * p.c[3])); }
inline double multi_sign(double a, double b) { return b < 0.0 ? -a : a; }
inline bool diff_sign(double y0, double yr) { return y0 * yr < 0.0; }
const double kXError = 1e-10;
const int kFindIters = 200;

double find_closed(const P4& p, const P4& dp, double x0, double x1, double y0, double y1, int& st) {
  (void)y1;
  double xr = (x0 + x1) / 2.0, yr = evaluate(p, xr), xb0 = x0, xb1 = x1;
  if (x1 - x0 <= kXError * 2.0) return xr;
  for (int it = 0;; ++it) {
    if (it >= kFindIters) { st |= 2; break; }
    if (diff_sign(y0, yr)) xb1 = xr; else xb0 = xr;
    double dy = evaluate(dp, xr);
    double dx = yr / dy;
    double xn = xr - dx;
    if (xn > xb0 && xn < xb1) {
      double step = std::fabs(xr - xn);
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

int quadratic_roots(const double* q, double x0, double x1, double* roots) {
  double c = q[0], b = q[1], a = q[2];
  double delta = b * b - 4.0 * a * c;
  int ret = 0;
  roots[0] = roots[1] = 0.0;
  if (delta > 0.0) {
    double d = std::sqrt(delta);
    double qq = -(b + multi_sign(d, b)) * 0.5;
    double rv0 = qq / a, rv1 = c / qq;
    double xa = tmin(rv0, rv1), xb = tmax(rv0, rv1);
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

void deflate(const P4& p, double root, double* d) {
  d[2] = p.c[3];
  d[1] = p.c[2] + root * d[2];
  d[0] = p.c[1] + root * d[1];
}

int cubic_roots(const P4& p, double x0, double x1, double* roots, int& st) {
  roots[0] = roots[1] = roots[2] = 0.0;
  double y0 = evaluate(p, x0), y1 = evaluate(p, x1);
  double a = p.c[3] * 3.0, b_2 = p.c[2], c = p.c[1];
  P4 dp{{c, 2.0 * b_2, a, 0.0}};
  double delta_4 = b_2 * b_2 - a * c;
  double q2[2], dfl[3];
  auto with_quad = [&](double lo) {
    deflate(p, roots[0], dfl);
    int r = quadratic_roots(dfl, lo, x1, q2);
    roots[1] = q2[0];
    roots[2] = q2[1];
    return r + 1;
  };
  if (delta_4 > 0.0) {
    double d_2 = std::sqrt(delta_4);
    double q = -(b_2 + multi_sign(d_2, b_2));
    double rv0 = q / a, rv1 = c / q;
    double xa = tmin(rv0, rv1), xb = tmax(rv0, rv1);
    if (diff_sign(y0, y1)) {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) { roots[0] = find_closed(p, dp, x0, x1, y0, y1, st); return 1; }
    } else {
      if (xa >= x1 || xb <= x0 || (xa <= x0 && xb >= x1)) return 0;
    }
    if (xa > x0) {
      double ya = evaluate(p, xa);
      if (diff_sign(y0, ya)) {
        roots[0] = find_closed(p, dp, x0, xa, y0, ya, st);
        if (diff_sign(ya, y1) || (xb < x1 && diff_sign(ya, evaluate(p, xb)))) return with_quad(xa);
        return 1;
      }
      if (xb < x1) {
        double yb = evaluate(p, xb);
        if (diff_sign(ya, yb)) {
          roots[0] = find_closed(p, dp, xa, xb, ya, yb, st);
          if (diff_sign(yb, y1)) return with_quad(xb);
          return 1;
        }
        if (diff_sign(yb, y1)) { roots[0] = find_closed(p, dp, xb, x1, yb, y1, st); return 1; }
      } else if (diff_sign(ya, y1)) {
        roots[0] = find_closed(p, dp, xa, x1, ya, y1, st);
        return 1;
      }
    } else {
      double yb = evaluate(p, xb);
      if (diff_sign(y0, yb)) {
        roots[0] = find_closed(p, dp, x0, xb, y0, yb, st);
        if (diff_sign(yb, y1)) return with_quad(xb);
        return 1;
      }
      if (diff_sign(yb, y1)) { roots[0] = find_closed(p, dp, xb, x1, yb, y1, st); return 1; }
    }
    return 0;
  }
  if (diff_sign(y0, y1)) { roots[0] = find_closed(p, dp, x0, x1, y0, y1, st); return 1; }
  return 0;
}

P4 cubic_binomial(const double* a, const double* b) {
  P4 r;
  r.c[0] = b[0] * b[1] * b[2];
  r.c[1] = a[0] * b[1] * b[2] + b[0] * b[1] * a[2] + b[0] * a[1] * b[2];
  r.c[2] = a[0] * a[1] * b[2] + a[0] * b[1] * a[2] + b[0] * a[1] * a[2];
  r.c[3] = a[0] * a[1] * a[2];
  return r;
}

// det(B + tA), matrices as 3x3 row-major built from columns
P4 det_polynomial(const double A[3][3], const double B[3][3]) {
  static const int Pi[3][3][2] = {{{0, 0}, {1, 1}, {2, 2}}, {{0, 1}, {1, 2}, {2, 0}}, {{0, 2}, {1, 0}, {2, 1}}};
  static const int Ni[3][3][2] = {{{0, 0}, {1, 2}, {2, 1}}, {{0, 1}, {1, 0}, {2, 2}}, {{0, 2}, {1, 1}, {2, 0}}};
  P4 pos{{0, 0, 0, 0}}, neg{{0, 0, 0, 0}};
  for (int k = 0; k < 3; ++k) {
    double a[3], b[3];
    for (int m = 0; m < 3; ++m) { a[m] = A[Pi[k][m][0]][Pi[k][m][1]]; b[m] = B[Pi[k][m][0]][Pi[k][m][1]]; }
    P4 t = cubic_binomial(a, b);
    for (int q = 0; q < 4; ++q) pos.c[q] = pos.c[q] + t.c[q];
  }
  for (int k = 0; k < 3; ++k) {
    double a[3], b[3];
    for (int m = 0; m < 3; ++m) { a[m] = A[Ni[k][m][0]][Ni[k][m][1]]; b[m] = B[Ni[k][m][0]][Ni[k][m][1]]; }
    P4 t = cubic_binomial(a, b);
    for (int q = 0; q < 4; ++q) neg.c[q] = neg.c[q] + t.c[q];
  }
  P4 r;
  for (int q = 0; q < 4; ++q) r.c[q] = pos.c[q] - neg.c[q];
  return r;
}

int coplanar_roots(const V3<double>* p0, const V3<double>* p1, double* roots, int& st) {
  static const int cols[4][3] = {{1, 2, 3}, {0, 2, 3}, {0, 1, 3}, {0, 1, 2}};
  P4 acc{{0, 0, 0, 0}};
  for (int m = 0; m < 4; ++m) {
    double A[3][3], B[3][3];
    for (int c = 0; c < 3; ++c) {
      V3<double> b = p0[cols[m][c]], e = p1[cols[m][c]];
      B[0][c] = b.x; B[1][c] = b.y; B[2][c] = b.z;
      A[0][c] = e.x - b.x; A[1][c] = e.y - b.y; A[2][c] = e.z - b.z;
    }
    P4 d = det_polynomial(A, B);
    if (m == 0) acc = d;
    else for (int q = 0; q < 4; ++q) acc.c[q] = (m & 1) ? acc.c[q] - d.c[q] : acc.c[q] + d.c[q];
  }
  return cubic_roots(acc, 0.0, 1.0, roots, st);
}

inline V3<double> lerpd(V3<double> a, V3<double> b, double t) { return a * (1.0 - t) + b * t; }
void solve2(double a11, double a12, double a22, double b1, double b2, double& be, double& ga) {
  double det = a11 * a22 - a12 * a12;
  be = (b1 * a22 - a12 * b2) / det;
  ga = (a11 * b2 - a12 * b1) / det;
}
bool verify_pt(const V3<double>* x) {
  V3<double> e1 = x[2] - x[1], e2 = x[3] - x[1], w = x[0] - x[1];
  double be, ga;
  solve2(dot(e1, e1), dot(e1, e2), dot(e2, e2), dot(e1, w), dot(e2, w), be, ga);
  const double tol = 1e-8;
  return be >= -tol && ga >= -tol && be + ga <= 1.0 + tol;
}
bool verify_ee(const V3<double>* x) {
  V3<double> ea = x[1] - x[0], eb = x[3] - x[2], w = x[2] - x[0];
  double be, ga;
  solve2(dot(ea, ea), dot(ea, eb), dot(eb, eb), dot(ea, w), dot(eb, w), be, ga);
  const double tol = 1e-8;
  return be >= -tol && be <= 1.0 + tol && -ga >= -tol && -ga <= 1.0 + tol;
}
double collision_time(int kind_ee, const V3<double>* p0, const V3<double>* p1, int& st) {
  double roots[3];
  int nr = coplanar_roots(p0, p1, roots, st);
  double root = 1.0;
  bool ok = false;
  for (int i = 0; i < nr; ++i) {
    root = roots[i];
    V3<double> xt[4];
    for (int k = 0; k < 4; ++k) xt[k] = lerpd(p0[k], p1[k], root);
    ok = kind_ee ? verify_ee(xt) : verify_pt(xt);
    if (ok) break;
  }
  return ok ? root : 1.0;
}

// swept boxes rounded outward to float with pad (at least as wide as the product's)
template <class S>
Box swept_box(const S* x0, const S* x1, const int* ids, int nv, double pad) {
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int v = 0; v < nv; ++v) {
    V3<double> a = f64(load3(x0, ids[v])), b = f64(load3(x1, ids[v]));
    double av[3] = {a.x, a.y, a.z}, bv[3] = {b.x, b.y, b.z};
    for (int k = 0; k < 3; ++k) { mn[k] = tmin(mn[k], tmin(av[k], bv[k])); mx[k] = tmax(mx[k], tmax(av[k], bv[k])); }
  }
  Box bx;
  for (int k = 0; k < 3; ++k) {
    bx.lo[k] = std::nextafter((float)(mn[k] - pad), -INFINITY);
    bx.hi[k] = std::nextafter((float)(mx[k] + pad), INFINITY);
  }
  return bx;
}

template <class S>
double scene_toi(int nv, const S* x0, const S* x1, int ne, const int* edges, int nt, const int* tris, const int* body,
                 int exclude, int& st_out) {
  const double pad = 1e-7;
  std::vector<Box> eb(ne), tb(nt), vb(nv);
  for (int i = 0; i < ne; ++i) eb[i] = swept_box(x0, x1, edges + 2 * i, 2, pad);
  for (int j = 0; j < nt; ++j) tb[j] = swept_box(x0, x1, tris + 3 * j, 3, pad);
  for (int i = 0; i < nv; ++i) vb[i] = swept_box(x0, x1, &i, 1, pad);
  int nth = omp_get_max_threads();
  std::vector<double> best(nth, 1.0);
  std::vector<int> stv(nth, 0);
  sweep(eb, eb, [&](int i, int j) {
    if (!(i < j)) return;
    int a0 = edges[2 * i], a1 = edges[2 * i + 1], b0 = edges[2 * j], b1 = edges[2 * j + 1];
    if (a0 == b0 || a0 == b1 || a1 == b0 || a1 == b1) return;
    if (exclude && body[a0] == body[b0]) return;
    V3<double> p0[4] = {f64(load3(x0, a0)), f64(load3(x0, a1)), f64(load3(x0, b0)), f64(load3(x0, b1))};
    V3<double> p1[4] = {f64(load3(x1, a0)), f64(load3(x1, a1)), f64(load3(x1, b0)), f64(load3(x1, b1))};
    int tid = omp_get_thread_num();
    double t = collision_time(1, p0, p1, stv[tid]);
    if (t < best[tid]) best[tid] = t;
  });
  sweep(vb, tb, [&](int i, int j) {
    int t0 = tris[3 * j], t1 = tris[3 * j + 1], t2 = tris[3 * j + 2];
    if (i == t0 || i == t1 || i == t2) return;
    if (exclude && body[i] == body[t0]) return;
    V3<double> p0[4] = {f64(load3(x0, i)), f64(load3(x0, t0)), f64(load3(x0, t1)), f64(load3(x0, t2))};
    V3<double> p1[4] = {f64(load3(x1, i)), f64(load3(x1, t0)), f64(load3(x1, t1)), f64(load3(x1, t2))};
    int tid = omp_get_thread_num();
    double t = collision_time(0, p0, p1, stv[tid]);
    if (t < best[tid]) best[tid] = t;
  });
  double b = 1.0;
  st_out = 0;
  for (int k = 0; k < nth; ++k) { b = tmin(b, best[k]); st_out |= stv[k]; }
  return b;
}


// ------------------------------------------------------------------- FEM
// fem/fem.py:22-34, 139-203; fem/snh.py, neo_hookean.py, stvk.py (double)
struct M3d {
  double a[3][3];
};
M3d mz() { M3d m; std::memset(&m, 0, sizeof(m)); return m; }
M3d mm(const M3d& x, const M3d& y) {
  M3d r = mz();
  for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) for (int k = 0; k < 3; ++k) r.a[i][j] += x.a[i][k] * y.a[k][j];
  return r;
}
M3d mt(const M3d& x) { M3d r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[j][i]; return r; }
M3d lin(double a, const M3d& x, double b, const M3d& y) {
  M3d r; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) r.a[i][j] = a * x.a[i][j] + b * y.a[i][j]; return r;
}
double dd(const M3d& x, const M3d& y) { double s = 0; for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s += x.a[i][j] * y.a[i][j]; return s; }
double det(const M3d& m) {
  return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) - m.a[0][1] * (m.a[1][0] * m.a[2][2] - m.a[1][2] * m.a[2][0]) +
         m.a[0][2] * (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]);
}
M3d inv(const M3d& m) {
  double id = 1.0 / det(m);
  M3d r;
  r.a[0][0] = (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) * id; r.a[0][1] = (m.a[0][2] * m.a[2][1] - m.a[0][1] * m.a[2][2]) * id;
  r.a[0][2] = (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]) * id; r.a[1][0] = (m.a[1][2] * m.a[2][0] - m.a[1][0] * m.a[2][2]) * id;
  r.a[1][1] = (m.a[0][0] * m.a[2][2] - m.a[0][2] * m.a[2][0]) * id; r.a[1][2] = (m.a[0][2] * m.a[1][0] - m.a[0][0] * m.a[1][2]) * id;
  r.a[2][0] = (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]) * id; r.a[2][1] = (m.a[0][1] * m.a[2][0] - m.a[0][0] * m.a[2][1]) * id;
  r.a[2][2] = (m.a[0][0] * m.a[1][1] - m.a[0][1] * m.a[1][0]) * id;
  return r;
}
V3<double> colm(const M3d& m, int j) { return mk(m.a[0][j], m.a[1][j], m.a[2][j]); }
M3d cols3(V3<double> c0, V3<double> c1, V3<double> c2) {
  M3d r;
  double v[3][3] = {{c0.x, c1.x, c2.x}, {c0.y, c1.y, c2.y}, {c0.z, c1.z, c2.z}};
  std::memcpy(r.a, v, sizeof(v));
  return r;
}
M3d cof(const M3d& F) {
  V3<double> f0 = colm(F, 0), f1 = colm(F, 1), f2 = colm(F, 2);
  return cols3(cross(f1, f2), cross(f2, f0), cross(f0, f1));
}
M3d green(const M3d& F) {
  M3d E = mm(mt(F), F);
  for (int i = 0; i < 3; ++i) E.a[i][i] -= 1.0;
  return lin(0.5, E, 0.0, E);
}
double fem_psi(int mat, const M3d& F, double mu, double lam) {
  if (mat == 0) {
    double smu = 4.0 / 3.0 * mu, slam = lam + 5.0 / 6.0 * mu, alpha = 1.0 + 0.75 * smu / slam;
    double Ic = dd(F, F), Ja = det(F) - alpha;
    return 0.5 * (slam * Ja * Ja + smu * (Ic - 3.0) - smu * std::log(Ic + 1.0));
  }
  if (mat == 1) {
    double lJ = std::log(det(F));
    return mu * 0.5 * (dd(F, F) - 3.0) - mu * lJ + lam * 0.5 * lJ * lJ;
  }
  M3d E = green(F);
  double tr = E.a[0][0] + E.a[1][1] + E.a[2][2];
  return mu * dd(E, E) + lam * 0.5 * tr * tr;
}
M3d fem_pk1(int mat, const M3d& F, double mu, double lam) {
  if (mat == 0) {
    double smu = 4.0 / 3.0 * mu, slam = lam + 5.0 / 6.0 * mu, alpha = 1.0 + 0.75 * smu / slam;
    double Ic = dd(F, F);
    return lin(smu * (1.0 - 1.0 / (Ic + 1.0)), F, slam * (det(F) - alpha), cof(F));
  }
  if (mat == 1) {
    M3d FiT = mt(inv(F));
    return lin(mu, lin(1.0, F, -1.0, FiT), lam * std::log(det(F)), FiT);
  }
  M3d E = green(F);
  double tr = E.a[0][0] + E.a[1][1] + E.a[2][2];
  M3d S = lin(2.0 * mu, E, 0.0, E);
  for (int i = 0; i < 3; ++i) S.a[i][i] += lam * tr;
  return mm(F, S);
}
M3d fem_tangent(int mat, const M3d& F, const M3d& dF, double mu, double lam) {
  if (mat == 0) {
    double smu = 4.0 / 3.0 * mu, slam = lam + 5.0 / 6.0 * mu, alpha = 1.0 + 0.75 * smu / slam;
    M3d C = cof(F);
    double Ic1 = dd(F, F) + 1.0, dIc = 2.0 * dd(F, dF);
    V3<double> f0 = colm(F, 0), f1 = colm(F, 1), f2 = colm(F, 2), d0 = colm(dF, 0), d1 = colm(dF, 1), d2 = colm(dF, 2);
    M3d dC = cols3(cross(d1, f2) + cross(f1, d2), cross(d2, f0) + cross(f2, d0), cross(d0, f1) + cross(f0, d1));
    M3d r = lin(smu * (1.0 - 1.0 / Ic1), dF, smu * dIc / (Ic1 * Ic1), F);
    r = lin(1.0, r, slam * dd(C, dF), C);
    return lin(1.0, r, slam * (det(F) - alpha), dC);
  }
  if (mat == 1) {
    M3d Fi = inv(F), FiT = mt(Fi), B = mm(Fi, dF);
    double lJ = std::log(det(F)), trB = B.a[0][0] + B.a[1][1] + B.a[2][2];
    return lin(1.0, lin(mu, dF, mu - lam * lJ, mm(mm(FiT, mt(dF)), FiT)), lam * trB, FiT);
  }
  M3d E = green(F), dE = mm(mt(dF), F);
  dE = lin(0.5, dE, 0.5, mt(dE));
  double trE = E.a[0][0] + E.a[1][1] + E.a[2][2], trdE = dE.a[0][0] + dE.a[1][1] + dE.a[2][2];
  M3d S = lin(2.0 * mu, E, 0.0, E), dS = lin(2.0 * mu, dE, 0.0, dE);
  for (int i = 0; i < 3; ++i) { S.a[i][i] += lam * trE; dS.a[i][i] += lam * trdE; }
  return lin(1.0, mm(dF, S), 1.0, mm(F, dS));
}
}  // namespace

// ===================================================================== C ABI
extern "C" {

int ora_version() { return 1; }

void ora_closest_point_triangle(int n, const float* p, const float* a, const float* b, const float* c,
                                float* out_uvd, int* out_type) {
  for (int i = 0; i < n; ++i) {
    CPT r = closest_point_triangle(load3(p, i), load3(a, i), load3(b, i), load3(c, i));
    out_uvd[3 * i] = r.u;
    out_uvd[3 * i + 1] = r.v;
    out_uvd[3 * i + 2] = r.d;
    out_type[i] = r.type;
  }
}

void ora_closest_point_edge_edge(int n, const float* p1, const float* q1, const float* p2, const float* q2,
                                 float eps, float* out_std) {
  for (int i = 0; i < n; ++i) {
    CPEE r = closest_point_edge_edge(load3(p1, i), load3(q1, i), load3(p2, i), load3(q2, i), eps);
    out_std[3 * i] = r.s;
    out_std[3 * i + 1] = r.t;
    out_std[3 * i + 2] = r.d;
  }
}

// Candidate records are 6 ints: a1 a2 b1 b2 e0 e1 (contact.py:171-183).
// Returns the number of candidates; writes at most `cap`.
int ora_dcd_ee(int nv, const float* x, int ne, const int* edges, const int* body, float th, int exclude,
               int* out, int cap) {
  (void)nv;
  std::vector<Box> boxes(ne);
  float pad = 2.0f * th * 1.0001f + 1e-6f;
  for (int i = 0; i < ne; ++i) {
    V3<float> p = load3(x, edges[2 * i]), q = load3(x, edges[2 * i + 1]);
    boxes[i] = Box{{tmin(p.x, q.x) - pad, tmin(p.y, q.y) - pad, tmin(p.z, q.z) - pad},
                   {tmax(p.x, q.x) + pad, tmax(p.y, q.y) + pad, tmax(p.z, q.z) + pad}};
  }
  int nth = omp_get_max_threads();
  std::vector<std::vector<int>> loc(nth);
  float l0 = th * 2.0f;
  sweep(boxes, boxes, [&](int i, int j) {
    if (!(i < j)) return;
    int a1 = edges[2 * i], a2 = edges[2 * i + 1], b1 = edges[2 * j], b2 = edges[2 * j + 1];
    if (a1 == b1 || a1 == b2 || a2 == b1 || a2 == b2) return;
    if (exclude && body[a1] == body[b1]) return;
    CPEE r = closest_point_edge_edge(load3(x, a1), load3(x, a2), load3(x, b1), load3(x, b2), 1.0e-6f);
    if (r.d < l0) {
      auto& v = loc[omp_get_thread_num()];
      v.insert(v.end(), {a1, a2, b1, b2, i, j});
    }
  });
  int cnt = 0;
  for (auto& v : loc)
    for (size_t k = 0; k < v.size(); k += 6, ++cnt)
      if (cnt < cap) std::memcpy(out + 6 * (size_t)cnt, v.data() + k, 6 * sizeof(int));
  return cnt;
}

int ora_dcd_pt(int nv, const float* x, int nt, const int* tris, const int* body, float th, int exclude, int* out,
               int cap) {
  std::vector<Box> tb(nt), vb(nv);
  float eps = 1e-6f;
  for (int j = 0; j < nt; ++j) {
    V3<float> a = load3(x, tris[3 * j]), b = load3(x, tris[3 * j + 1]), c = load3(x, tris[3 * j + 2]);
    tb[j] = Box{{tmin(tmin(a.x, b.x), c.x) - eps, tmin(tmin(a.y, b.y), c.y) - eps, tmin(tmin(a.z, b.z), c.z) - eps},
                {tmax(tmax(a.x, b.x), c.x) + eps, tmax(tmax(a.y, b.y), c.y) + eps, tmax(tmax(a.z, b.z), c.z) + eps}};
  }
  float pad = 2.0f * th * 1.0001f + 1e-6f;
  for (int i = 0; i < nv; ++i) {
    V3<float> p = load3(x, i);
    vb[i] = Box{{p.x - pad, p.y - pad, p.z - pad}, {p.x + pad, p.y + pad, p.z + pad}};
  }
  int nth = omp_get_max_threads();
  std::vector<std::vector<int>> loc(nth);
  float l0 = th * 2.0f;
  sweep(vb, tb, [&](int i, int j) {
    int t1 = tris[3 * j], t2 = tris[3 * j + 1], t3 = tris[3 * j + 2];
    if (t1 == i || t2 == i || t3 == i) return;
    if (exclude && body[i] == body[t1]) return;
    CPT r = closest_point_triangle(load3(x, i), load3(x, t1), load3(x, t2), load3(x, t3));
    if (r.d < l0) {
      auto& v = loc[omp_get_thread_num()];
      v.insert(v.end(), {i, t2, t1, t3, i, j});  // F10 order: (p, tri[1], tri[0], tri[2])
    }
  });
  int cnt = 0;
  for (auto& v : loc)
    for (size_t k = 0; k < v.size(); k += 6, ++cnt)
      if (cnt < cap) std::memcpy(out + 6 * (size_t)cnt, v.data() + k, 6 * sizeof(int));
  return cnt;
}

// Narrow phase.  fp64: S = double else float.  mode 0 = jets+Jacobi, 1 = subspace.
void ora_narrow(int kind_ee, int fp64, int mode, int n, const int* idx, const void* l0, const void* x,
                const void* xcs, double kappa, double* force, double* hess, double* energy, int* active) {
  FeatureFn fn = mode == 0 ? feature_dh_jet : feature_dh_subspace;
  if (fp64) {
    NarrowOut<double> o{force, hess, energy, active};
    if (kind_ee) narrow_ee<double>(n, idx, (const double*)l0, (const double*)x, (const double*)xcs, kappa, fn, o);
    else narrow_pt<double>(n, idx, (const double*)l0, (const double*)x, kappa, fn, o);
  } else {
    NarrowOut<float> o{force, hess, energy, active};
    if (kind_ee) narrow_ee<float>(n, idx, (const float*)l0, (const float*)x, (const float*)xcs, kappa, fn, o);
    else narrow_pt<float>(n, idx, (const float*)l0, (const float*)x, kappa, fn, o);
  }
}

// Gradient + NSD of a single explicit feature (kind 0..3) on 4 double points,
// for direct tests of the two Hessian routes.
void ora_feature_dh(int kind, int mode, const double* pts12, double* g12, double* h144) {
  int nv = kind == 0 ? 2 : (kind == 1 ? 3 : 4);
  V3<double> p[4];
  int slots[4] = {0, 1, 2, 3};
  for (int k = 0; k < 4; ++k) p[k] = mk(pts12[3 * k], pts12[3 * k + 1], pts12[3 * k + 2]);
  FeatureDH fd;
  (mode == 0 ? feature_dh_jet : feature_dh_subspace)(kind, p, nv, slots, fd);
  std::memcpy(g12, fd.g, sizeof(fd.g));
  std::memcpy(h144, fd.h, sizeof(fd.h));
}

void ora_barrier(int n, const double* x, const double* xh, double kappa, double* out3) {
  for (int i = 0; i < n; ++i) {
    Barrier b = barrier(x[i], xh[i], kappa);
    out3[3 * i] = b.b;
    out3[3 * i + 1] = b.db;
    out3[3 * i + 2] = b.d2b;
  }
}


int ora_cubic_roots(int n, const double* coef, double x0, double x1, double* roots, int* nroots) {
  int st = 0;
  for (int i = 0; i < n; ++i) {
    P4 p{{coef[4 * i], coef[4 * i + 1], coef[4 * i + 2], coef[4 * i + 3]}};
    nroots[i] = cubic_roots(p, x0, x1, roots + 3 * i, st);
  }
  return st;
}

int ora_collision_time(int kind_ee, int n, const double* a, const double* b, double* t) {
  int st = 0;
  for (int i = 0; i < n; ++i) {
    V3<double> p0[4], p1[4];
    for (int k = 0; k < 4; ++k) {
      p0[k] = mk(a[12 * i + 3 * k], a[12 * i + 3 * k + 1], a[12 * i + 3 * k + 2]);
      p1[k] = mk(b[12 * i + 3 * k], b[12 * i + 3 * k + 1], b[12 * i + 3 * k + 2]);
    }
    t[i] = collision_time(kind_ee, p0, p1, st);
  }
  return st;
}

// Minimum TOI over all EE and PT pairs whose swept boxes overlap (ccd.py:360-427).
double ora_scene_toi(int fp64, int nv, const void* x0, const void* x1, int ne, const int* edges, int nt, const int* tris,
                     const int* body, int exclude, int* status) {
  int st = 0;
  double t = fp64 ? scene_toi<double>(nv, (const double*)x0, (const double*)x1, ne, edges, nt, tris, body, exclude, st)
                  : scene_toi<float>(nv, (const float*)x0, (const float*)x1, ne, edges, nt, tris, body, exclude, st);
  if (status) *status = st;
  return t;
}


// Elastic forces (V x 3, added), 16 blocks per tet (n x 16 x 9) and energy
// sum W psi for positions x and rest positions xcs (both double).
double ora_tet(int mat, int nv, const double* x, const double* xcs, int nt, const int* tets, double mu, double lam,
               double* force, double* blocks) {
  (void)nv;
  double energy = 0.0;
  for (int e = 0; e < nt; ++e) {
    const int* t = tets + 4 * e;
    M3d Dm = cols3(load3(xcs, t[0]) - load3(xcs, t[3]), load3(xcs, t[1]) - load3(xcs, t[3]), load3(xcs, t[2]) - load3(xcs, t[3]));
    M3d B = inv(Dm);
    double w = std::fabs(det(Dm)) / 6.0;
    M3d F = mm(cols3(load3(x, t[0]) - load3(x, t[3]), load3(x, t[1]) - load3(x, t[3]), load3(x, t[2]) - load3(x, t[3])), B);
    energy += w * fem_psi(mat, F, mu, lam);
    M3d H = lin(-w, mm(fem_pk1(mat, F, mu, lam), mt(B)), 0.0, F);
    for (int i = 0; i < 4; ++i)
      for (int l = 0; l < 3; ++l)
        force[3 * t[i] + l] += i < 3 ? H.a[l][i] : -(H.a[l][0] + H.a[l][1] + H.a[l][2]);
    for (int j = 0; j < 4; ++j)
      for (int k = 0; k < 3; ++k) {
        M3d dDs = mz();
        if (j < 3) dDs.a[k][j] = -1.0;
        else dDs.a[k][0] = dDs.a[k][1] = dDs.a[k][2] = 1.0;
        M3d dH = lin(-w, mm(fem_tangent(mat, F, mm(dDs, B), mu, lam), mt(B)), 0.0, F);
        for (int i = 0; i < 4; ++i)
          for (int l = 0; l < 3; ++l)
            blocks[((size_t)e * 16 + i * 4 + j) * 9 + 3 * l + k] = i < 3 ? dH.a[l][i] : -(dH.a[l][0] + dH.a[l][1] + dH.a[l][2]);
      }
  }
  return energy;
}

// Contact-block BSR assembly (dynamic_contacts.py:281-297: triplets
// i*16 + ii*4 + jj of each record -> bsr_from_triplets): record p's 12x12
// Hessian hess[p] gives 16 blocks keyed (idx[p][ii], idx[p][jj]); all-zero
// blocks are dropped (warp's prune_numerical_zeros); equal keys are summed in
// record order.  offsets[nv + 1]; cols/vals sized by the caller (cap blocks).
// Returns nnz (when > cap nothing past cap is written).
int ora_contact_bsr(int nv, int n, const int* idx, const double* hess, int* offsets, int* cols, double* vals,
                    int cap) {
  std::vector<int> cnt(nv + 1, 0);
  auto block_nz = [&](long p, int ii, int jj) {
    const double* H = hess + (size_t)p * 144;
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b)
        if (H[(3 * ii + a) * 12 + 3 * jj + b] != 0.0) return true;
    return false;
  };
  for (long p = 0; p < n; ++p)
    for (int ii = 0; ii < 4; ++ii)
      for (int jj = 0; jj < 4; ++jj)
        if (block_nz(p, ii, jj)) cnt[idx[4 * p + ii] + 1]++;
  for (int r = 0; r < nv; ++r) cnt[r + 1] += cnt[r];
  std::vector<int> slot(cnt.begin(), cnt.end() - 1);
  std::vector<int> ids(cnt[nv]);
  for (long p = 0; p < n; ++p)
    for (int ii = 0; ii < 4; ++ii)
      for (int jj = 0; jj < 4; ++jj)
        if (block_nz(p, ii, jj)) ids[slot[idx[4 * p + ii]]++] = (int)(p * 16 + ii * 4 + jj);
  auto col_of = [&](int id) { return idx[4 * (id / 16) + (id % 4)]; };
  std::vector<int> distinct(nv + 1, 0);
#pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < nv; ++r) {
    int* b = ids.data() + cnt[r];
    int* e = ids.data() + cnt[r + 1];
    std::sort(b, e, [&](int x, int y) { return col_of(x) != col_of(y) ? col_of(x) < col_of(y) : x < y; });
    int d = 0;
    for (int* q = b; q < e; ++q)
      if (q == b || col_of(*q) != col_of(*(q - 1))) ++d;
    distinct[r + 1] = d;
  }
  for (int r = 0; r < nv; ++r) distinct[r + 1] += distinct[r];
  for (int r = 0; r <= nv; ++r) offsets[r] = distinct[r];
  const int nnz = distinct[nv];
  if (nnz > cap) return nnz;
#pragma omp parallel for schedule(dynamic, 64)
  for (int r = 0; r < nv; ++r) {
    int o = distinct[r] - 1;
    for (int q = cnt[r]; q < cnt[r + 1]; ++q) {
      const int id = ids[q];
      const long p = id / 16;
      const int ii = (id / 4) % 4, jj = id % 4;
      if (q == cnt[r] || col_of(id) != col_of(ids[q - 1])) {
        ++o;
        cols[o] = col_of(id);
        for (int k = 0; k < 9; ++k) vals[(size_t)o * 9 + k] = 0.0;
      }
      const double* H = hess + (size_t)p * 144;
      for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) vals[(size_t)o * 9 + 3 * a + b] += H[(3 * ii + a) * 12 + 3 * jj + b];
    }
  }
  return nnz;
}

// Intersection check (the reference's trajectories must stay intersection
// free): every (edge, triangle) pair without a shared vertex whose segment
// strictly crosses the triangle, by orientation signs in double (plain IEEE
// operations in a fixed order; the product evaluates the same expressions).
// The sorted-grid pruning over tight boxes is conservative, so the count is
// that of all E x T pairs.  Returns the count; the first cap pairs go to out.
static double ora_orient(const double* a, const double* b, const double* c, const double* d) {
  double u[3], v[3], w[3];
  for (int k = 0; k < 3; ++k) {
    u[k] = b[k] - a[k];
    v[k] = c[k] - a[k];
    w[k] = d[k] - a[k];
  }
  const double cx = v[1] * w[2] - v[2] * w[1], cy = v[2] * w[0] - v[0] * w[2], cz = v[0] * w[1] - v[1] * w[0];
  return (u[0] * cx + u[1] * cy) + u[2] * cz;
}

int ora_edge_triangle_crossings(int nv, const double* x, int ne, const int* edges, int nt, const int* tris, int* out,
                                int cap) {
  (void)nv;
  std::vector<Box> eb(ne), tb(nt);
  for (int e = 0; e < ne; ++e)
    for (int k = 0; k < 3; ++k) {
      const double a = x[3 * edges[2 * e] + k], b = x[3 * edges[2 * e + 1] + k];
      eb[e].lo[k] = std::nextafter((float)std::min(a, b), -3.4e38f);
      eb[e].hi[k] = std::nextafter((float)std::max(a, b), 3.4e38f);
    }
  for (int t = 0; t < nt; ++t)
    for (int k = 0; k < 3; ++k) {
      double mn = 1e300, mx = -1e300;
      for (int v = 0; v < 3; ++v) {
        mn = std::min(mn, x[3 * tris[3 * t + v] + k]);
        mx = std::max(mx, x[3 * tris[3 * t + v] + k]);
      }
      tb[t].lo[k] = std::nextafter((float)mn, -3.4e38f);
      tb[t].hi[k] = std::nextafter((float)mx, 3.4e38f);
    }
  std::vector<std::pair<int, int>> found;
  std::mutex mu;
  sweep(eb, tb, [&](int e, int t) {
    const int p = edges[2 * e], q = edges[2 * e + 1];
    const int a = tris[3 * t], b = tris[3 * t + 1], c = tris[3 * t + 2];
    if (a == p || a == q || b == p || b == q || c == p || c == q) return;
    const double *P = x + 3 * p, *Q = x + 3 * q, *A = x + 3 * a, *B = x + 3 * b, *C = x + 3 * c;
    const double o1 = ora_orient(A, B, C, P), o2 = ora_orient(A, B, C, Q);
    if (!((o1 > 0.0 && o2 < 0.0) || (o1 < 0.0 && o2 > 0.0))) return;
    const double s1 = ora_orient(P, Q, A, B), s2 = ora_orient(P, Q, B, C), s3 = ora_orient(P, Q, C, A);
    if (!((s1 > 0.0 && s2 > 0.0 && s3 > 0.0) || (s1 < 0.0 && s2 < 0.0 && s3 < 0.0))) return;
    std::lock_guard<std::mutex> lock(mu);
    found.push_back({e, t});
  });
  std::sort(found.begin(), found.end());
  for (int k = 0; k < (int)found.size() && k < cap; ++k) {
    out[2 * k] = found[k].first;
    out[2 * k + 1] = found[k].second;
  }
  return (int)found.size();
}

}  // extern "C"
