// Affine-body terms shared by the ABD kernels (abd.cu) and the batched
// per-iteration launch (terms.cu): the device view of an ipcb_abd, and the
// per-body inertia + orthogonality block and gradient
// (affine_body_dynamics.py:88-141).
#pragma once
#include "common.cuh"

namespace ipcb {
namespace {

template <class S>
struct Abd {
  int nb;
  S* q;
  S* q0;
  S* qt;
  S* qdot;
  S* dx;
  const S* mass;
  const S* volume;
  const S* stiffness;
  const int* fixed;
};

template <class S>
IPCB_HD Abd<S> view(const ipcb_abd* a) {
  return Abd<S>{a->n_bodies, (S*)a->q, (S*)a->q0, (S*)a->q_tilde, (S*)a->qdot, (S*)a->dx,
                (const S*)a->mass, (const S*)a->volume, (const S*)a->stiffness, a->fixed};
}

template <class S> IPCB_D v3<S> ld(const S* p, int i) { return mk3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
template <class S> IPCB_D void st3(S* p, int i, v3<S> v) {
  p[3 * i] = v.x;
  p[3 * i + 1] = v.y;
  p[3 * i + 2] = v.z;
}

// --------------------------------------------------------- body system
// Block (i, j) of body b: M_ij I, plus for i, j >= 1 the orthogonality
// Hessian 4 kappa V h^2 [(a_i.a_i - 1) I + 2 a_i a_i^T + sum_{k != i} a_k a_k^T]
// (i == j) or 4 kappa V h^2 [(a_i.a_j) I + a_j a_i^T]; fixed bodies get I / 0.
template <class S>
IPCB_D void body_block(const Abd<S>& A, int b, int i, int j, S h2, S out[9]) {
  for (int k = 0; k < 9; ++k) out[k] = S(0);
  if (A.fixed[b] != 0) {
    if (i == j) out[0] = out[4] = out[8] = S(1);
    return;
  }
  const S m = A.mass[16 * b + 4 * i + j];
  out[0] = out[4] = out[8] = m;
  if (i > 0 && j > 0) {
    const S* Q = A.q + 12 * (size_t)b;
    const v3<S> ai = ld(Q, i), aj = ld(Q, j);
    const S sc = S(4) * A.stiffness[b] * A.volume[b] * h2;
    const S av[3] = {ai.x, ai.y, ai.z}, bv[3] = {aj.x, aj.y, aj.z};
    if (i == j) {
      const S s = dot(ai, ai) - S(1);
      S acc[9];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) acc[3 * r + c] = (r == c ? s : S(0)) + S(2) * av[r] * av[c];
      for (int k = 1; k < 4; ++k) {
        if (k == i) continue;
        const v3<S> ak = ld(Q, k);
        const S kv[3] = {ak.x, ak.y, ak.z};
        for (int r = 0; r < 3; ++r)
          for (int c = 0; c < 3; ++c) acc[3 * r + c] += kv[r] * kv[c];
      }
      for (int k = 0; k < 9; ++k) out[k] += sc * acc[k];
    } else {
      const S d = dot(ai, aj);
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) out[3 * r + c] += sc * ((r == c ? d : S(0)) + bv[r] * av[c]);
    }
  }
}

template <class S>
IPCB_D v3<S> body_gradient(const Abd<S>& A, int b, int i, S h2) {
  if (A.fixed[b] != 0) return mk3(S(0), S(0), S(0));
  const S* Q = A.q + 12 * (size_t)b;
  const S* T = A.qt + 12 * (size_t)b;
  v3<S> g = mk3(S(0), S(0), S(0));
  for (int k = 0; k < 4; ++k) g = g + (ld(Q, k) - ld(T, k)) * A.mass[16 * b + 4 * i + k];
  if (i > 0) {
    const v3<S> ai = ld(Q, i);
    v3<S> og = ai * (dot(ai, ai) - S(1));
    for (int k = 1; k < 4; ++k)
      if (k != i) {
        const v3<S> ak = ld(Q, k);
        og = og + ak * dot(ai, ak);
      }
    g = g + og * (S(4) * A.stiffness[b] * A.volume[b] * h2);
  }
  return g;
}

}  // namespace
}  // namespace ipcb
