// Tet FEM device code shared by fem.cu and the batched work-queue kernel
// (terms.cu).  See fem.cu for the method.
#pragma once
#include "common.cuh"

namespace ipcb {
namespace {

template <class T>
struct M3 {
  T a[3][3];
};

template <class T> IPCB_HD M3<T> mzero() {
  M3<T> m;
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) m.a[i][j] = T(0);
  return m;
}
template <class T> IPCB_HD M3<T> mmul(const M3<T>& x, const M3<T>& y) {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][0] * y.a[0][j] + x.a[i][1] * y.a[1][j] + x.a[i][2] * y.a[2][j];
  return r;
}
template <class T> IPCB_HD M3<T> mmulT(const M3<T>& x, const M3<T>& y) {  // x y^T
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[i][0] * y.a[j][0] + x.a[i][1] * y.a[j][1] + x.a[i][2] * y.a[j][2];
  return r;
}
template <class T> IPCB_HD M3<T> mT(const M3<T>& x) {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.a[i][j] = x.a[j][i];
  return r;
}
template <class T> IPCB_HD T ddot(const M3<T>& x, const M3<T>& y) {
  T s = T(0);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) s += x.a[i][j] * y.a[i][j];
  return s;
}
template <class T> IPCB_HD T det3(const M3<T>& m) {
  return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) -
         m.a[0][1] * (m.a[1][0] * m.a[2][2] - m.a[1][2] * m.a[2][0]) +
         m.a[0][2] * (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]);
}
template <class T> IPCB_HD M3<T> inv3(const M3<T>& m) {
  T d = det3(m), id = T(1) / d;
  M3<T> r;
  r.a[0][0] = (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) * id;
  r.a[0][1] = (m.a[0][2] * m.a[2][1] - m.a[0][1] * m.a[2][2]) * id;
  r.a[0][2] = (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]) * id;
  r.a[1][0] = (m.a[1][2] * m.a[2][0] - m.a[1][0] * m.a[2][2]) * id;
  r.a[1][1] = (m.a[0][0] * m.a[2][2] - m.a[0][2] * m.a[2][0]) * id;
  r.a[1][2] = (m.a[0][2] * m.a[1][0] - m.a[0][0] * m.a[1][2]) * id;
  r.a[2][0] = (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]) * id;
  r.a[2][1] = (m.a[0][1] * m.a[2][0] - m.a[0][0] * m.a[2][1]) * id;
  r.a[2][2] = (m.a[0][0] * m.a[1][1] - m.a[0][1] * m.a[1][0]) * id;
  return r;
}
template <class T> IPCB_HD M3<T> axpby(T a, const M3<T>& x, T b, const M3<T>& y) {
  M3<T> r;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) r.a[i][j] = a * x.a[i][j] + b * y.a[i][j];
  return r;
}
template <class T> IPCB_HD v3<T> colv(const M3<T>& m, int j) { return mk3(m.a[0][j], m.a[1][j], m.a[2][j]); }
template <class T> IPCB_HD M3<T> from_cols(v3<T> c0, v3<T> c1, v3<T> c2) {
  M3<T> r;
  r.a[0][0] = c0.x; r.a[1][0] = c0.y; r.a[2][0] = c0.z;
  r.a[0][1] = c1.x; r.a[1][1] = c1.y; r.a[2][1] = c1.z;
  r.a[0][2] = c2.x; r.a[1][2] = c2.y; r.a[2][2] = c2.z;
  return r;
}

enum { MAT_SNH = 0, MAT_NH = 1, MAT_STVK = 2 };

// cofactor dJ/dF: columns f1 x f2, f2 x f0, f0 x f1 (snh.py:30-37)
template <class T> IPCB_HD M3<T> cofactor(const M3<T>& F) {
  v3<T> f0 = colv(F, 0), f1 = colv(F, 1), f2 = colv(F, 2);
  return from_cols(cross(f1, f2), cross(f2, f0), cross(f0, f1));
}

// snh.py:6-13 reparametrisation
template <class T> IPCB_HD void snh_params(T mu, T lam, T& smu, T& slam, T& alpha) {
  smu = T(4.0 / 3.0) * mu;
  slam = lam + T(5.0 / 6.0) * mu;
  alpha = T(1) + T(0.75) * smu / slam;
}

template <class T> IPCB_HD T psi(int mat, const M3<T>& F, T mu, T lam) {
  if (mat == MAT_SNH) {
    T smu, slam, alpha;
    snh_params(mu, lam, smu, slam, alpha);
    T Ic = ddot(F, F), Ja = det3(F) - alpha;
    return T(0.5) * (slam * Ja * Ja + smu * (Ic - T(3)) - smu * log(Ic + T(1)));
  }
  if (mat == MAT_NH) {
    T I1 = ddot(F, F), lJ = log(det3(F));
    return mu * T(0.5) * (I1 - T(3)) - mu * lJ + lam * T(0.5) * lJ * lJ;
  }
  M3<T> E = mmul(mT(F), F);
  E.a[0][0] -= T(1); E.a[1][1] -= T(1); E.a[2][2] -= T(1);
  E = axpby(T(0.5), E, T(0), E);
  T tr = E.a[0][0] + E.a[1][1] + E.a[2][2];
  return mu * ddot(E, E) + lam * T(0.5) * tr * tr;
}

template <class T> IPCB_HD M3<T> pk1(int mat, const M3<T>& F, T mu, T lam) {
  if (mat == MAT_SNH) {
    T smu, slam, alpha;
    snh_params(mu, lam, smu, slam, alpha);
    T Ic = ddot(F, F);
    return axpby(smu * (T(1) - T(1) / (Ic + T(1))), F, slam * (det3(F) - alpha), cofactor(F));
  }
  if (mat == MAT_NH) {
    M3<T> FiT = mT(inv3(F));
    T lJ = log(det3(F));
    return axpby(mu, axpby(T(1), F, T(-1), FiT), lam * lJ, FiT);
  }
  M3<T> E = mmul(mT(F), F);
  E.a[0][0] -= T(1); E.a[1][1] -= T(1); E.a[2][2] -= T(1);
  E = axpby(T(0.5), E, T(0), E);
  T tr = E.a[0][0] + E.a[1][1] + E.a[2][2];
  M3<T> S = axpby(T(2) * mu, E, T(0), E);
  S.a[0][0] += lam * tr; S.a[1][1] += lam * tr; S.a[2][2] += lam * tr;
  return mmul(F, S);
}

// directional derivative dP(F; dF)
template <class T> IPCB_HD M3<T> tangent(int mat, const M3<T>& F, const M3<T>& dF, T mu, T lam) {
  if (mat == MAT_SNH) {
    T smu, slam, alpha;
    snh_params(mu, lam, smu, slam, alpha);
    M3<T> cof = cofactor(F);
    T Ic = ddot(F, F), Ic1 = Ic + T(1), dIc = T(2) * ddot(F, dF);
    T dist = smu * (T(1) - T(1) / Ic1), ddist = smu * dIc / (Ic1 * Ic1);
    T dJ = ddot(cof, dF), vol = slam * (det3(F) - alpha);
    v3<T> f0 = colv(F, 0), f1 = colv(F, 1), f2 = colv(F, 2);
    v3<T> d0 = colv(dF, 0), d1 = colv(dF, 1), d2 = colv(dF, 2);
    M3<T> dcof = from_cols(cross(d1, f2) + cross(f1, d2), cross(d2, f0) + cross(f2, d0), cross(d0, f1) + cross(f0, d1));
    M3<T> r = axpby(dist, dF, ddist, F);
    r = axpby(T(1), r, slam * dJ, cof);
    return axpby(T(1), r, vol, dcof);
  }
  if (mat == MAT_NH) {
    M3<T> Fi = inv3(F), FiT = mT(Fi);
    M3<T> B = mmul(Fi, dF);
    T lJ = log(det3(F)), trB = B.a[0][0] + B.a[1][1] + B.a[2][2];
    M3<T> m1 = mmul(mmul(FiT, mT(dF)), FiT);
    return axpby(T(1), axpby(mu, dF, mu - lam * lJ, m1), lam * trB, FiT);
  }
  M3<T> E = mmul(mT(F), F);
  E.a[0][0] -= T(1); E.a[1][1] -= T(1); E.a[2][2] -= T(1);
  E = axpby(T(0.5), E, T(0), E);
  T trE = E.a[0][0] + E.a[1][1] + E.a[2][2];
  M3<T> dE = mmul(mT(dF), F);
  dE = axpby(T(0.5), dE, T(0.5), mT(dE));
  T trdE = dE.a[0][0] + dE.a[1][1] + dE.a[2][2];
  M3<T> S = axpby(T(2) * mu, E, T(0), E);
  S.a[0][0] += lam * trE; S.a[1][1] += lam * trE; S.a[2][2] += lam * trE;
  M3<T> dS = axpby(T(2) * mu, dE, T(0), dE);
  dS.a[0][0] += lam * trdE; dS.a[1][1] += lam * trdE; dS.a[2][2] += lam * trdE;
  return axpby(T(1), mmul(dF, S), T(1), mmul(F, dS));
}

template <class S>
IPCB_D M3<S> load_bm(const S* __restrict__ Bm, int e) {
  M3<S> B;
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) B.a[i][j] = Bm[9 * e + 3 * i + j];
  return B;
}

// The 16 blocks of one tet of tet_kernel_sparse, handed to put(q, l, k, v)
// with q = i*4 + j the block slot, and the nodal forces into b.
template <class S, class Put>
IPCB_D void tet_hessian_blocks(int mat, const S* __restrict__ x, const int4* __restrict__ tets, int e,
                               const S* __restrict__ Bm, const S* __restrict__ W, S mu, S lam, S* __restrict__ b,
                               Put&& put) {
  int4 t = tets[e];
  const int vid[4] = {t.x, t.y, t.z, t.w};
  v3<S> p0 = load3(x, t.x), p1 = load3(x, t.y), p2 = load3(x, t.z), p3 = load3(x, t.w);
  M3<S> B = load_bm(Bm, e);
  S w = W[e];
  M3<S> F = mmul(from_cols(p0 - p3, p1 - p3, p2 - p3), B);
  M3<S> H = axpby(-w, mmulT(pk1(mat, F, mu, lam), B), S(0), F);  // -W P Bm^T; forces are its columns
  v3<S> f[4] = {colv(H, 0), colv(H, 1), colv(H, 2), mk3(S(0), S(0), S(0))};
  f[3] = mk3(-(f[0].x + f[1].x + f[2].x), -(f[0].y + f[1].y + f[2].y), -(f[0].z + f[1].z + f[2].z));
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    atomicAdd(b + 3 * vid[i], f[i].x);
    atomicAdd(b + 3 * vid[i] + 1, f[i].y);
    atomicAdd(b + 3 * vid[i] + 2, f[i].z);
  }
  for (int j = 0; j < 4; ++j) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      M3<S> dDs = mzero<S>();
      if (j < 3) dDs.a[k][j] = S(-1);
      else dDs.a[k][0] = dDs.a[k][1] = dDs.a[k][2] = S(1);
      M3<S> dF = mmul(dDs, B);
      M3<S> dH = axpby(-w, mmulT(tangent(mat, F, dF, mu, lam), B), S(0), dF);
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int l = 0; l < 3; ++l) put(i * 4 + j, l, k, dH.a[l][i]);
#pragma unroll
      for (int l = 0; l < 3; ++l) put(12 + j, l, k, -(dH.a[l][0] + dH.a[l][1] + dH.a[l][2]));
    }
  }
}

// One tet: 16 blocks at e*16 + i*4 + j (rows/cols skipped when null: a fixed
// pattern knows them), nodal forces into b.
template <class S>
IPCB_D void tet_hessian_item(int mat, const S* __restrict__ x, const int4* __restrict__ tets, int e,
                             const S* __restrict__ Bm, const S* __restrict__ W, S mu, S lam, int* __restrict__ rows,
                             int* __restrict__ cols, S* __restrict__ vals, S* __restrict__ b) {
  const long long base = 16LL * e;
  if (rows) {
    const int4 t = tets[e];
    const int vid[4] = {t.x, t.y, t.z, t.w};
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      rows[base + q] = vid[q >> 2];
      cols[base + q] = vid[q & 3];
    }
  }
  S* out = vals + 9 * base;
  tet_hessian_blocks<S>(mat, x, tets, e, Bm, W, mu, lam, b,
                        [&](int q, int l, int k, S v) { out[9 * q + 3 * l + k] = v; });
}

// Shared-memory stride of one tet's 144 values (odd: conflict-free lanes).
constexpr int kTetStage = 145;

// The 32 lanes of a warp build tets e0 .. e0+31 (those < n) into the warp's
// stage sm[32 * kTetStage], then write the tets' contiguous 144-value records
// (and rows/cols) with coalesced stores.  Called by all 32 lanes.
template <class S>
IPCB_D void tet_hessian_warp(int mat, const S* __restrict__ x, const int4* __restrict__ tets, int e0, int n,
                             const S* __restrict__ Bm, const S* __restrict__ W, S mu, S lam, int* __restrict__ rows,
                             int* __restrict__ cols, S* __restrict__ vals, S* __restrict__ b, S* sm) {
  const int lane = threadIdx.x & 31;
  const int e = e0 + lane;
  if (e < n) {
    S* mine = sm + lane * kTetStage;
    tet_hessian_blocks<S>(mat, x, tets, e, Bm, W, mu, lam, b,
                          [&](int q, int l, int k, S v) { mine[9 * q + 3 * l + k] = v; });
  }
  __syncwarp();
  const int cnt = n - e0 < 32 ? n - e0 : 32;
  S* dst = vals + 144LL * e0;
  for (int idx = lane; idx < cnt * 144; idx += 32) {
    const int te = idx / 144;
    dst[idx] = sm[te * kTetStage + (idx - te * 144)];
  }
  if (rows) {
    for (int idx = lane; idx < cnt * 16; idx += 32) {
      const int4 t = tets[e0 + (idx >> 4)];
      const int vid[4] = {t.x, t.y, t.z, t.w};
      rows[16LL * e0 + idx] = vid[(idx >> 2) & 3];
      cols[16LL * e0 + idx] = vid[idx & 3];
    }
  }
  __syncwarp();
}

}  // namespace
}  // namespace ipcb
