// Affine-body frames for the body-local (fixed) hierarchies
// (fixed_bvh_contacts.py:32-175): per body the inverse of A, p and
// |A^-1|_F in double, world boxes of the rest bounds, and the motion extent
// of the body's frame over a step.
#pragma once
#include "common.cuh"

namespace ipcb {
namespace bodies {

struct Frame {
  double inv[9];  // row-major A^-1
  double p[3];
  double fro;     // |A^-1|_F
};

template <class S>
IPCB_D void load_affine(const S* __restrict__ q, int b, double (&p)[3], double (&A)[9]) {
  // q: p, then the columns A[:,0], A[:,1], A[:,2]; A row-major here
  for (int k = 0; k < 3; ++k) p[k] = (double)q[12 * b + k];
  for (int c = 0; c < 3; ++c)
    for (int r = 0; r < 3; ++r) A[3 * r + c] = (double)q[12 * b + 3 + 3 * c + r];
}

IPCB_D double det3(const double (&A)[9]) {
  return A[0] * (A[4] * A[8] - A[5] * A[7]) - A[1] * (A[3] * A[8] - A[5] * A[6]) + A[2] * (A[3] * A[7] - A[4] * A[6]);
}

IPCB_D void inverse3(const double (&A)[9], double det, double (&I)[9]) {
  const double id = 1.0 / det;
  I[0] = (A[4] * A[8] - A[5] * A[7]) * id;
  I[1] = (A[2] * A[7] - A[1] * A[8]) * id;
  I[2] = (A[1] * A[5] - A[2] * A[4]) * id;
  I[3] = (A[5] * A[6] - A[3] * A[8]) * id;
  I[4] = (A[0] * A[8] - A[2] * A[6]) * id;
  I[5] = (A[2] * A[3] - A[0] * A[5]) * id;
  I[6] = (A[3] * A[7] - A[4] * A[6]) * id;
  I[7] = (A[1] * A[6] - A[0] * A[7]) * id;
  I[8] = (A[0] * A[4] - A[1] * A[3]) * id;
}

// world box of the rest box [lo, hi] under x = p + A r
IPCB_D void world_box(const double (&p)[3], const double (&A)[9], const float* lo, const float* hi, double (&wl)[3],
                      double (&wh)[3]) {
  for (int r = 0; r < 3; ++r) {
    double c = p[r], e = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double mid = 0.5 * ((double)lo[k] + (double)hi[k]), ext = 0.5 * ((double)hi[k] - (double)lo[k]);
      c += A[3 * r + k] * mid;
      e += fabs(A[3 * r + k]) * ext;
    }
    wl[r] = c - e;
    wh[r] = c + e;
  }
}

IPCB_D Frame load_frame(const double* __restrict__ frames, int b) {
  Frame f;
  const double* s = frames + 13 * b;
  for (int k = 0; k < 9; ++k) f.inv[k] = s[k];
  for (int k = 0; k < 3; ++k) f.p[k] = s[9 + k];
  f.fro = s[12];
  return f;
}

// x_local = A^-1 (x - p)
IPCB_D void to_local(const Frame& f, double x, double y, double z, double (&o)[3]) {
  const double dx = x - f.p[0], dy = y - f.p[1], dz = z - f.p[2];
  for (int r = 0; r < 3; ++r) o[r] = f.inv[3 * r] * dx + f.inv[3 * r + 1] * dy + f.inv[3 * r + 2] * dz;
}

// outward-rounded float box of [lo - pad_k, hi + pad_k]
IPCB_D void float_box(const double (&lo)[3], const double (&hi)[3], const double (&pad)[3], f3& flo, f3& fhi) {
  flo = mk3(__double2float_rd(lo[0] - pad[0]), __double2float_rd(lo[1] - pad[1]), __double2float_rd(lo[2] - pad[2]));
  fhi = mk3(__double2float_ru(hi[0] + pad[0]), __double2float_ru(hi[1] + pad[1]), __double2float_ru(hi[2] + pad[2]));
}

}  // namespace bodies
}  // namespace ipcb
