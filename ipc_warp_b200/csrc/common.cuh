// Shared device helpers for the ipc_warp_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/ipcb.h"

#define IPCB_HD __host__ __device__ __forceinline__
#define IPCB_D __device__ __forceinline__

namespace ipcb {

// ------------------------------------------------------------------ exact ops
// Correctly rounded single operations that the compiler may not contract into
// FMAs.  Every predicate whose outcome decides a candidate, a gate or a feature
// branch is written with these so the float32 results are bit-identical to a
// plain IEEE evaluation in the same order.
IPCB_D float xadd(float a, float b) { return __fadd_rn(a, b); }
IPCB_D float xsub(float a, float b) { return __fsub_rn(a, b); }
IPCB_D float xmul(float a, float b) { return __fmul_rn(a, b); }
IPCB_D float xdiv(float a, float b) { return __fdiv_rn(a, b); }
IPCB_D float xsqrt(float a) { return __fsqrt_rn(a); }
IPCB_D double xadd(double a, double b) { return __dadd_rn(a, b); }
IPCB_D double xsub(double a, double b) { return __dsub_rn(a, b); }
IPCB_D double xmul(double a, double b) { return __dmul_rn(a, b); }
IPCB_D double xdiv(double a, double b) { return __ddiv_rn(a, b); }
IPCB_D double xsqrt(double a) { return __dsqrt_rn(a); }

template <class T>
struct v3 {
  T x, y, z;
};
typedef v3<float> f3;
typedef v3<double> d3;

template <class T> IPCB_HD v3<T> mk3(T x, T y, T z) { return v3<T>{x, y, z}; }

// exact-op vector helpers (evaluation order: ((x*x + y*y) + z*z))
template <class T> IPCB_D v3<T> esub(v3<T> a, v3<T> b) { return mk3(xsub(a.x, b.x), xsub(a.y, b.y), xsub(a.z, b.z)); }
template <class T> IPCB_D v3<T> eadd(v3<T> a, v3<T> b) { return mk3(xadd(a.x, b.x), xadd(a.y, b.y), xadd(a.z, b.z)); }
template <class T> IPCB_D v3<T> escale(v3<T> a, T s) { return mk3(xmul(a.x, s), xmul(a.y, s), xmul(a.z, s)); }
template <class T> IPCB_D T edot(v3<T> a, v3<T> b) { return xadd(xadd(xmul(a.x, b.x), xmul(a.y, b.y)), xmul(a.z, b.z)); }
template <class T> IPCB_D v3<T> ecross(v3<T> a, v3<T> b) {
  return mk3(xsub(xmul(a.y, b.z), xmul(a.z, b.y)), xsub(xmul(a.z, b.x), xmul(a.x, b.z)),
             xsub(xmul(a.x, b.y), xmul(a.y, b.x)));
}
template <class T> IPCB_D T elength(v3<T> a) { return xsqrt(edot(a, a)); }

// plain (contractible) vector helpers for non-predicate arithmetic
template <class T> IPCB_HD v3<T> operator+(v3<T> a, v3<T> b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
template <class T> IPCB_HD v3<T> operator-(v3<T> a, v3<T> b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
template <class T> IPCB_HD v3<T> operator*(v3<T> a, T s) { return mk3(a.x * s, a.y * s, a.z * s); }
template <class T> IPCB_HD T dot(v3<T> a, v3<T> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T> IPCB_HD v3<T> cross(v3<T> a, v3<T> b) {
  return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}

template <class T> IPCB_HD T tmin(T a, T b) { return a < b ? a : b; }
template <class T> IPCB_HD T tmax(T a, T b) { return a > b ? a : b; }
template <class T> IPCB_HD T clampv(T x, T lo, T hi) { return x < lo ? lo : (x > hi ? hi : x); }

IPCB_D d3 to_d(f3 a) { return mk3((double)a.x, (double)a.y, (double)a.z); }
IPCB_D d3 to_d(d3 a) { return a; }
IPCB_D f3 to_f(d3 a) { return mk3((float)a.x, (float)a.y, (float)a.z); }
IPCB_D f3 to_f(f3 a) { return a; }

// positions: AoS scalar[3*V]
template <class S> IPCB_D v3<S> load3(const S* __restrict__ p, int i) {
  return mk3(__ldg(p + 3 * i), __ldg(p + 3 * i + 1), __ldg(p + 3 * i + 2));
}
IPCB_D f3 load4(const float4* __restrict__ p, int i) {
  float4 v = __ldg(p + i);
  return mk3(v.x, v.y, v.z);
}

// ----------------------------------------------------------- float atomics
// Non-negative floats order like their bit patterns.
IPCB_D void atomic_min_nonneg(float* a, float v) { atomicMin((int*)a, __float_as_int(v)); }
IPCB_D void atomic_min_nonneg(double* a, double v) {
  atomicMin((unsigned long long*)a, (unsigned long long)__double_as_longlong(v));
}

// order-preserving float <-> uint for min/max reductions of signed floats
IPCB_D unsigned f2ord(float f) {
  unsigned u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
IPCB_D float ord2f(unsigned u) { return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u); }

inline int div_up(long long a, long long b) { return (int)((a + b - 1) / b); }

}  // namespace ipcb
