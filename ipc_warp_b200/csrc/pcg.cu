// Device-resident preconditioned conjugate gradients on the 3x3-block Newton
// system (include/ipcb.h): the scalars (rz, pAp, |r|^2, ...) live in device
// memory, every kernel of an iteration reads them there, and a finished solve
// turns the remaining launches into no-ops, so the host launches k iterations
// at a time (or replays them as a CUDA graph) and reads one flag per batch.
//
// Per iteration: q = A p fused with p.q (warp per block row over the row's
// contiguous values); x += alpha p, r -= alpha q with |r|^2, fused with the
// block-Jacobi z = D^-1 r and r.z (or, for the FSAI factor, followed by its
// two sweeps); p = z + beta p, whose last block to finish rotates the
// scalars and tests |r| <= tol |b|: three launches per iteration with block
// Jacobi, four with the learned factor.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <type_traits>

#include "common.cuh"

namespace ipcb {
int check_launch(const char* where);
void set_error_msg(const char* msg);
}  // namespace ipcb

namespace {

using bf16 = __nv_bfloat16;
constexpr int kBlock = 256;

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double s[kBlock / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) s[w] = v;
  __syncthreads();
  double t = 0.0;
  if (w == 0) {
    t = lane < (int)(blockDim.x >> 5) ? s[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

// two block sums at once (valid in thread 0)
__device__ __forceinline__ void block_sum2(double& a, double& b) {
  __shared__ double s[2][kBlock / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    s[0][w] = a;
    s[1][w] = b;
  }
  __syncthreads();
  if (w == 0) {
    double x = lane < (int)(blockDim.x >> 5) ? s[0][lane] : 0.0;
    double y = lane < (int)(blockDim.x >> 5) ? s[1][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(0xffffffffu, x, o);
      y += __shfl_down_sync(0xffffffffu, y, o);
    }
    a = x;
    b = y;
  }
}

template <class T> __device__ __forceinline__ T ldv(const T* p) { return __ldg(p); }
__device__ __forceinline__ float ldv(const bf16* p) { return __bfloat162float(*p); }

// Block-row products with 8 lanes per row (4 rows in flight per warp): lane
// `sub` takes blocks b + sub, b + sub + 8, ... of the row, reads the whole 3x3
// block (consecutive lanes read consecutive blocks, so a row's values stream
// contiguously), gathers x of the block's column and accumulates 3 outputs;
// the 8 lanes then reduce.  xs scales x per scalar (NULL: none);
// transpose_at: block index used transposed.
constexpr int kLanes = 8;

template <class T> __device__ __forceinline__ void ld9(const T* __restrict__ v, float (&a)[9]) {
#pragma unroll
  for (int q = 0; q < 9; ++q) a[q] = (float)__ldg(v + q);
}
__device__ __forceinline__ void ld9(const double* __restrict__ v, double (&a)[9]) {
#pragma unroll
  for (int q = 0; q < 9; ++q) a[q] = __ldg(v + q);
}
__device__ __forceinline__ void ld9(const bf16* __restrict__ v, float (&a)[9]) {
#pragma unroll
  for (int q = 0; q < 9; ++q) a[q] = __bfloat162float(v[q]);
}

template <class T, class V, int L = kLanes>
__device__ __forceinline__ void row_mv(const int* __restrict__ cols, const V* __restrict__ vals, int b, int e,
                                       const T* __restrict__ x, const float* __restrict__ xs, int transpose_at,
                                       T& o0, T& o1, T& o2) {
  const int sub = threadIdx.x & (L - 1);
  using A = typename std::conditional<std::is_same<V, double>::value, double, float>::type;
  T a0 = 0, a1 = 0, a2 = 0;
#pragma unroll 2
  for (int k = b + sub; k < e; k += L) {
    const int c = __ldg(cols + k);
    A m[9];
    ld9(vals + 9LL * k, m);
    T x0 = x[3 * c], x1 = x[3 * c + 1], x2 = x[3 * c + 2];
    if (xs) {
      x0 *= (T)__ldg(xs + 3 * c);
      x1 *= (T)__ldg(xs + 3 * c + 1);
      x2 *= (T)__ldg(xs + 3 * c + 2);
    }
    if (k == transpose_at) {
      a0 += (T)m[0] * x0 + (T)m[3] * x1 + (T)m[6] * x2;
      a1 += (T)m[1] * x0 + (T)m[4] * x1 + (T)m[7] * x2;
      a2 += (T)m[2] * x0 + (T)m[5] * x1 + (T)m[8] * x2;
    } else {
      a0 += (T)m[0] * x0 + (T)m[1] * x1 + (T)m[2] * x2;
      a1 += (T)m[3] * x0 + (T)m[4] * x1 + (T)m[5] * x2;
      a2 += (T)m[6] * x0 + (T)m[7] * x1 + (T)m[8] * x2;
    }
  }
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
  }
  o0 = a0;
  o1 = a1;
  o2 = a2;
}

// q = A p ; state.pAp += p.q  (grid-stride row groups: one atomic per block)
template <class T>
__global__ void __launch_bounds__(kBlock) k_spmv_dot(int n, const int* __restrict__ off, const int* __restrict__ cols,
                                                     const T* __restrict__ vals, const T* __restrict__ p,
                                                     T* __restrict__ q, ipcb_pcg_state* st) {
  if (st->done) return;
  const int sub = threadIdx.x & (kLanes - 1);
  const int groups = (gridDim.x * blockDim.x) / kLanes;
  double part = 0.0;
  // every lane of a warp runs the same number of trips (shuffles need all 32)
  const int trips = (n + groups - 1) / groups;
  int row = (blockIdx.x * blockDim.x + threadIdx.x) / kLanes;
  for (int t = 0; t < trips; ++t, row += groups) {
    const bool ok = row < n;
    T o0, o1, o2;
    row_mv<T, T>(cols, vals, ok ? off[row] : 0, ok ? off[row + 1] : 0, p, nullptr, -1, o0, o1, o2);
    if (ok && sub == 0) {
      q[3 * row] = o0;
      q[3 * row + 1] = o1;
      q[3 * row + 2] = o2;
      part += (double)p[3 * row] * o0 + (double)p[3 * row + 1] * o1 + (double)p[3 * row + 2] * o2;
    }
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->pAp, part);
}

// x += alpha p ; r -= alpha q ; state.rr += r.r
template <class T>
__global__ void __launch_bounds__(kBlock) k_update_xr(int m, T* __restrict__ x, T* __restrict__ r,
                                                      const T* __restrict__ p, const T* __restrict__ q,
                                                      ipcb_pcg_state* st) {
  if (st->done) return;
  const double alpha = st->pAp > 0.0 ? st->rz / st->pAp : 0.0;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x) {
    x[i] += (T)alpha * p[i];
    const T ri = r[i] - (T)alpha * q[i];
    r[i] = ri;
    part += (double)ri * ri;
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->rr, part);
}

// x += alpha p ; r -= alpha q ; z = D^-1 r (block Jacobi), per block row ;
// state.rr += r.r ; state.rz_new += r.z
template <class T>
__global__ void __launch_bounds__(kBlock) k_update_xr_jacobi(int n, T* __restrict__ x, T* __restrict__ r,
                                                             const T* __restrict__ p, const T* __restrict__ q,
                                                             const T* __restrict__ dinv, T* __restrict__ z,
                                                             ipcb_pcg_state* st) {
  if (st->done) return;
  const double alpha = st->pAp > 0.0 ? st->rz / st->pAp : 0.0;
  double prr = 0.0, prz = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    T rv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int k = 3 * i + c;
      x[k] += (T)alpha * p[k];
      rv[c] = r[k] - (T)alpha * q[k];
      r[k] = rv[c];
      prr += (double)rv[c] * rv[c];
    }
    const T* d = dinv + 9LL * i;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T zc = d[3 * c] * rv[0] + d[3 * c + 1] * rv[1] + d[3 * c + 2] * rv[2];
      z[3 * i + c] = zc;
      prz += (double)rv[c] * zc;
    }
  }
  block_sum2(prr, prz);
  if (threadIdx.x == 0) {
    atomicAdd(&st->rr, prr);
    atomicAdd(&st->rz_new, prz);
  }
}

// Item layout of the grouped update: items i < n_point are the 3x3 block
// rows; from the next multiple of 32 on, 16 lanes per group (lanes 0..11 its
// rows, 12..15 idle), so a warp holds two whole groups.
__host__ __device__ inline int group_base(int n_point) { return (n_point + 31) & ~31; }
__host__ __device__ inline long long group_items(int n_point, int n_groups) {
  return group_base(n_point) + 16LL * ((n_groups + 1) & ~1);
}

// The same for a system with row groups (one affine body each): a group's
// 16-lane half-warp updates its 12 rows of x and r, exchanges the new
// residuals by shuffles, and lane c takes row c of the 12x12 inverse block.
template <class T>
__global__ void __launch_bounds__(kBlock) k_update_xr_groups(int n_point, int n_groups, T* __restrict__ x,
                                                             T* __restrict__ r, const T* __restrict__ p,
                                                             const T* __restrict__ q, const T* __restrict__ dinv,
                                                             const T* __restrict__ dinv_group, T* __restrict__ z,
                                                             ipcb_pcg_state* st) {
  if (st->done) return;
  const double alpha = st->pAp > 0.0 ? st->rz / st->pAp : 0.0;
  const int base = group_base(n_point);
  const long long total = group_items(n_point, n_groups);
  double prr = 0.0, prz = 0.0;
  // total and the stride are multiples of 32: a warp runs the loop as a whole
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    if (i < n_point) {
      T rv[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const long long k = 3 * i + c;
        x[k] += (T)alpha * p[k];
        rv[c] = r[k] - (T)alpha * q[k];
        r[k] = rv[c];
        prr += (double)rv[c] * rv[c];
      }
      const T* d = dinv + 9 * i;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T zc = d[3 * c] * rv[0] + d[3 * c + 1] * rv[1] + d[3 * c + 2] * rv[2];
        z[3 * i + c] = zc;
        prz += (double)rv[c] * zc;
      }
    } else if (i >= base) {  // whole warps only (base is a multiple of 32)
      const long long j = i - base;
      const int g = (int)(j >> 4), c = (int)(j & 15);
      const bool on = g < n_groups && c < 12;
      const long long o = 3LL * n_point + 12LL * g + c;
      T rv = T(0);
      if (on) {
        x[o] += (T)alpha * p[o];
        rv = r[o] - (T)alpha * q[o];
        r[o] = rv;
        prr += (double)rv * rv;
      }
      const T* d = dinv_group + 144LL * g + 12 * c;
      T zc = T(0);
#pragma unroll
      for (int k = 0; k < 12; ++k) {
        const T rk = __shfl_sync(0xffffffffu, rv, k, 16);
        if (on) zc += d[k] * rk;
      }
      if (on) {
        z[o] = zc;
        prz += (double)rv * zc;
      }
    }
  }
  block_sum2(prr, prz);
  if (threadIdx.x == 0) {
    atomicAdd(&st->rr, prr);
    atomicAdd(&st->rz_new, prz);
  }
}

// z = (group) block-Jacobi r ; state.rz_new += r.z (the start of a solve)
template <class T>
__global__ void __launch_bounds__(kBlock) k_jacobi_groups(int n_point, int n_groups, const T* __restrict__ dinv,
                                                          const T* __restrict__ dinv_group, const T* __restrict__ r,
                                                          T* __restrict__ z, ipcb_pcg_state* st) {
  if (st->done) return;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_point + n_groups; i += gridDim.x * blockDim.x) {
    const bool grp = i >= n_point;
    const int w = grp ? 12 : 3;
    const long long o = grp ? 3LL * n_point + 12LL * (i - n_point) : 3LL * i;
    const T* d = grp ? dinv_group + 144LL * (i - n_point) : dinv + 9LL * i;
    for (int c = 0; c < w; ++c) {
      T zc = T(0);
      for (int k = 0; k < w; ++k) zc += d[w * c + k] * r[o + k];
      z[o + c] = zc;
      part += (double)r[o + c] * zc;
    }
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->rz_new, part);
}

// one warp per group: gather the 16 3x3 blocks of rows / columns
// n_point + 4 g .. + 3 from the BSR into the warp's shared [12 | I] matrix,
// then Gauss-Jordan in double with partial pivoting (the first largest pivot,
// as a sequential scan picks), one row swap, scaling and elimination step per
// column with the lanes over the entries
constexpr int kInvWarps = 4;

template <class T>
__global__ void __launch_bounds__(32 * kInvWarps) k_group_inverse(int n_point, int n_groups,
                                                                 const int* __restrict__ off,
                                                                 const int* __restrict__ cols,
                                                                 const T* __restrict__ vals, T* __restrict__ out,
                                                                 int* __restrict__ status) {
  __shared__ double sa[kInvWarps][12][24];
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = blockIdx.x * kInvWarps + w;
  if (g >= n_groups) return;  // the whole warp
  double(&a)[12][24] = sa[w];
  for (int e = lane; e < 12 * 24; e += 32) {
    const int i = e / 24, j = e - 24 * i;
    a[i][j] = (j == 12 + i) ? 1.0 : 0.0;
  }
  __syncwarp(full);
  const int r0 = n_point + 4 * g;
  for (int bi = 0; bi < 4; ++bi) {
    const int row = r0 + bi;
    for (int k = off[row] + lane; k < off[row + 1]; k += 32) {  // a row's columns are distinct
      const int c = cols[k] - r0;
      if (c < 0 || c >= 4) continue;
      for (int u = 0; u < 3; ++u)
        for (int v = 0; v < 3; ++v) a[3 * bi + u][3 * c + v] += (double)vals[9LL * k + 3 * u + v];
    }
  }
  __syncwarp(full);
  bool ok = true;
  for (int c = 0; c < 12; ++c) {
    // pivot: the largest |a[i][c]| over i >= c, the smallest such i
    double v = lane >= c && lane < 12 ? fabs(a[lane][c]) : -1.0;
    int piv = lane;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ov = __shfl_xor_sync(full, v, o);
      const int op = __shfl_xor_sync(full, piv, o);
      if (ov > v || (ov == v && op < piv)) {
        v = ov;
        piv = op;
      }
    }
    if (!(v > 0.0)) {
      ok = false;
      break;
    }
    if (piv != c && lane < 24) {
      const double t = a[c][lane];
      a[c][lane] = a[piv][lane];
      a[piv][lane] = t;
    }
    __syncwarp(full);
    const double inv = 1.0 / a[c][c];
    __syncwarp(full);
    if (lane < 24) a[c][lane] *= inv;
    __syncwarp(full);
    double f[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) f[i] = a[i][c];
    __syncwarp(full);
    if (lane < 24) {
#pragma unroll
      for (int i = 0; i < 12; ++i)
        if (i != c && f[i] != 0.0) a[i][lane] -= f[i] * a[c][lane];
    }
    __syncwarp(full);
  }
  T* d = out + 144LL * g;
  if (!ok && lane == 0) atomicOr(status, IPCB_STATUS_PATTERN);
  for (int e = lane; e < 144; e += 32) {
    const int i = e / 12, j = e - 12 * i;
    d[e] = ok ? (T)a[i][12 + j] : (T)(i == j ? 1.0 : 0.0);
  }
}

// z = D^-1 r (block Jacobi) ; state.rz_new += r.z
template <class T>
__global__ void __launch_bounds__(kBlock) k_jacobi(int n, const T* __restrict__ dinv, const T* __restrict__ r,
                                                   T* __restrict__ z, ipcb_pcg_state* st) {
  if (st->done) return;
  double part = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const T* d = dinv + 9LL * i;
    const T r0 = r[3 * i], r1 = r[3 * i + 1], r2 = r[3 * i + 2];
    const T z0 = d[0] * r0 + d[1] * r1 + d[2] * r2;
    const T z1 = d[3] * r0 + d[4] * r1 + d[5] * r2;
    const T z2 = d[6] * r0 + d[7] * r1 + d[8] * r2;
    z[3 * i] = z0;
    z[3 * i + 1] = z1;
    z[3 * i + 2] = z2;
    part += (double)r0 * z0 + (double)r1 * z1 + (double)r2 * z2;
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->rz_new, part);
}

// lanes per row of the factor sweeps: each reads half a row of the pattern
// (measured on the wound rod bundle: 61.7 us an iteration with 4, 63.3 with
// 8, 70.0 with 2)
constexpr int kFsaiLanes = 4;

// t = G_lower (S r)
template <class T>
__global__ void __launch_bounds__(kBlock) k_fsai_lower(int n, const int* __restrict__ off, const int* __restrict__ diag,
                                                       const int* __restrict__ cols, const bf16* __restrict__ g,
                                                       const float* __restrict__ scale, const T* __restrict__ r,
                                                       T* __restrict__ t, ipcb_pcg_state* st) {
  if (st->done) return;
  const int sub = threadIdx.x & (kFsaiLanes - 1);
  const int groups = (gridDim.x * blockDim.x) / kFsaiLanes;
  const int trips = (n + groups - 1) / groups;
  int row = (blockIdx.x * blockDim.x + threadIdx.x) / kFsaiLanes;
  for (int it = 0; it < trips; ++it, row += groups) {
    const bool ok = row < n;
    T o0, o1, o2;
    row_mv<T, bf16, kFsaiLanes>(cols, g, ok ? off[row] : 0, ok ? diag[row] + 1 : 0, r, scale, -1, o0, o1, o2);
    if (ok && sub == 0) {
      t[3 * row] = o0;
      t[3 * row + 1] = o1;
      t[3 * row + 2] = o2;
    }
  }
}

// z = S G_upper t (upper slots hold the transposed lower blocks; the diagonal
// block is read transposed) ; state.rz_new += r.z
template <class T>
__global__ void __launch_bounds__(kBlock) k_fsai_upper(int n, const int* __restrict__ off, const int* __restrict__ diag,
                                                       const int* __restrict__ cols, const bf16* __restrict__ g,
                                                       const float* __restrict__ scale, const T* __restrict__ t,
                                                       const T* __restrict__ r, T* __restrict__ z,
                                                       ipcb_pcg_state* st) {
  if (st->done) return;
  const int sub = threadIdx.x & (kFsaiLanes - 1);
  const int groups = (gridDim.x * blockDim.x) / kFsaiLanes;
  const int trips = (n + groups - 1) / groups;
  double part = 0.0;
  int row = (blockIdx.x * blockDim.x + threadIdx.x) / kFsaiLanes;
  for (int it = 0; it < trips; ++it, row += groups) {
    const bool ok = row < n;
    T o0, o1, o2;
    const int d = ok ? diag[row] : 0;
    row_mv<T, bf16, kFsaiLanes>(cols, g, d, ok ? off[row + 1] : 0, t, nullptr, d, o0, o1, o2);
    if (ok && sub == 0) {
      const T z0 = o0 * (T)scale[3 * row], z1 = o1 * (T)scale[3 * row + 1], z2 = o2 * (T)scale[3 * row + 2];
      z[3 * row] = z0;
      z[3 * row + 1] = z1;
      z[3 * row + 2] = z2;
      part += (double)r[3 * row] * z0 + (double)r[3 * row + 1] * z1 + (double)r[3 * row + 2] * z2;
    }
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->rz_new, part);
}

// the end of an iteration (start: of the setup): rotate the scalars and
// test convergence, breakdown and the iteration bound
__device__ __forceinline__ void finish_state(ipcb_pcg_state* st, int start) {
  if (!start) {
    st->it += 1;
    if (st->rr <= st->tol2 * st->bb) st->done = 1;
    st->last_rr = st->rr;
    if (st->it >= st->maxiter) st->done = 1;
    if (!(st->pAp > 0.0)) {  // breakdown: the operator is not positive definite along p
      st->status |= 1;
      st->done = 1;
    }
  } else if (!(st->bb > 0.0)) {
    st->done = 1;
  }
  st->rz = st->rz_new;
  st->rz_new = 0.0;
  st->pAp = 0.0;
  st->rr = 0.0;
}

// p = z + beta p (beta = rz_new / rz; start: p = z); the last block to finish
// (every block has read rz / rz_new by then) runs finish_state
template <class T>
__global__ void __launch_bounds__(kBlock) k_update_p_finish(int m, const T* __restrict__ z, T* __restrict__ p,
                                                            ipcb_pcg_state* st, int start) {
  if (st->done) return;
  const double beta = start ? 0.0 : (st->rz != 0.0 ? st->rz_new / st->rz : 0.0);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m; i += gridDim.x * blockDim.x)
    p[i] = z[i] + (T)beta * (start ? (T)0 : p[i]);
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const int k = atomicAdd(&st->arrived, 1);
    if (k == (int)gridDim.x - 1) {
      __threadfence();
      st->arrived = 0;
      finish_state(st, start);
    }
  }
}

// x = 0, r = b, bb = b.b
template <class T>
__global__ void __launch_bounds__(kBlock) k_start(int m, const T* __restrict__ b, T* __restrict__ x, T* __restrict__ r,
                                                  ipcb_pcg_state* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (i < m) {
    const T bi = b[i];
    x[i] = 0;
    r[i] = bi;
    part = (double)bi * bi;
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->bb, part);
}

// the start from a guess: x = x0 was copied and q = A x0 computed; r = b - q
template <class T>
__global__ void __launch_bounds__(kBlock) k_start_guess(int m, const T* __restrict__ b, const T* __restrict__ q,
                                                        T* __restrict__ r, ipcb_pcg_state* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (i < m) {
    const T bi = b[i];
    r[i] = bi - q[i];
    part = (double)bi * bi;
  }
  part = block_sum(part);
  if (threadIdx.x == 0) atomicAdd(&st->bb, part);
}

__global__ void k_state_init(ipcb_pcg_state* st, double tol, int maxiter) {
  st->rz = st->rz_new = st->pAp = st->rr = st->bb = st->last_rr = 0.0;
  st->tol2 = tol * tol;
  st->it = 0;
  st->done = 0;
  st->maxiter = maxiter;
  st->status = 0;
  st->arrived = 0;
}

// inverse of the diagonal blocks
template <class T>
__global__ void k_block_jacobi(int n, const int* __restrict__ diag_of, const int* __restrict__ off,
                               const int* __restrict__ cols, const T* __restrict__ vals, T* __restrict__ dinv,
                               int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int d = -1;
  if (diag_of) d = diag_of[i];
  else
    for (int k = off[i]; k < off[i + 1]; ++k)
      if (cols[k] == i) { d = k; break; }
  double a[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  if (d >= 0)
    for (int q = 0; q < 9; ++q) a[q] = (double)vals[9LL * d + q];
  const double c0 = a[4] * a[8] - a[5] * a[7], c1 = a[5] * a[6] - a[3] * a[8], c2 = a[3] * a[7] - a[4] * a[6];
  double det = a[0] * c0 + a[1] * c1 + a[2] * c2;
  if (!(fabs(det) > 0.0)) {
    atomicOr(status, IPCB_STATUS_PATTERN);
    for (int q = 0; q < 9; ++q) dinv[9LL * i + q] = (q % 4 == 0) ? T(1) : T(0);
    return;
  }
  const double id = 1.0 / det;
  const double inv[9] = {c0 * id, (a[2] * a[7] - a[1] * a[8]) * id, (a[1] * a[5] - a[2] * a[4]) * id,
                         c1 * id, (a[0] * a[8] - a[2] * a[6]) * id, (a[2] * a[3] - a[0] * a[5]) * id,
                         c2 * id, (a[1] * a[6] - a[0] * a[7]) * id, (a[0] * a[4] - a[1] * a[3]) * id};
  for (int q = 0; q < 9; ++q) dinv[9LL * i + q] = (T)inv[q];
}

// bf16 factor for the apply: lower and diagonal slots G[e], upper slots the
// transpose of the lower block at rev[e]
__global__ void k_fsai_mirror(int nnz, const int* __restrict__ rows, const int* __restrict__ cols,
                              const int* __restrict__ rev, const float* __restrict__ G, bf16* __restrict__ g) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const bool upper = cols[e] > rows[e];
  const float* s = G + 9LL * (upper ? rev[e] : e);
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) g[9LL * e + 3 * r + c] = __float2bfloat16_rn(upper ? s[3 * c + r] : s[3 * r + c]);
}

inline int gridn(long long n, int b = kBlock) { return (int)((n + b - 1) / b); }

// row-group kernels loop over rows: a fixed grid of 8 blocks per SM
int warp_grid(int n) {
  static int sms = 0;
  if (!sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (sms <= 0) sms = 148;
  }
  const int need = gridn((long long)kLanes * n);
  return need < 8 * sms ? need : 8 * sms;
}

// element-wise kernels with a dot product: at most 4 blocks per SM, so that
// the per-block atomics on the scalar stay few
int flat_grid(long long m) {
  const int need = gridn(m);
  const int cap = 4 * (warp_grid(1 << 30) / 8);
  return need < cap ? need : cap;
}

template <class T>
int precond(const ipcb_pcg* P, cudaStream_t s) {
  const int n = P->n;
  if (P->precond == 0 && P->n_groups > 0)
    k_jacobi_groups<T><<<flat_grid(P->n_point + P->n_groups), kBlock, 0, s>>>(
        P->n_point, P->n_groups, (const T*)P->dinv, (const T*)P->dinv_group, (const T*)P->r, (T*)P->z, P->state);
  else if (P->precond == 0)
    k_jacobi<T><<<flat_grid(n), kBlock, 0, s>>>(n, (const T*)P->dinv, (const T*)P->r, (T*)P->z, P->state);
  else {
    k_fsai_lower<T><<<warp_grid(n), kBlock, 0, s>>>(n, P->g_offsets, P->diag, P->g_columns, (const bf16*)P->g,
                                                   P->scale, (const T*)P->r, (T*)P->t, P->state);
    k_fsai_upper<T><<<warp_grid(n), kBlock, 0, s>>>(n, P->g_offsets, P->diag, P->g_columns, (const bf16*)P->g,
                                                   P->scale, (const T*)P->t, (const T*)P->r, (T*)P->z, P->state);
  }
  return 0;
}

template <class T>
int start(const ipcb_pcg* P, double tol, int maxiter, cudaStream_t s) {
  const int m = 3 * P->n;
  k_state_init<<<1, 1, 0, s>>>(P->state, tol, maxiter);
  if (P->x0) {
    // the product's p.q lands in pAp, which the setup's finish_state clears
    cudaMemcpyAsync(P->x, P->x0, (size_t)m * sizeof(T), cudaMemcpyDeviceToDevice, s);
    k_spmv_dot<T><<<warp_grid(P->n), kBlock, 0, s>>>(P->n, P->offsets, P->columns, (const T*)P->values,
                                                        (const T*)P->x, (T*)P->q, P->state);
    k_start_guess<T><<<gridn(m), kBlock, 0, s>>>(m, (const T*)P->b, (const T*)P->q, (T*)P->r, P->state);
  } else {
    k_start<T><<<gridn(m), kBlock, 0, s>>>(m, (const T*)P->b, (T*)P->x, (T*)P->r, P->state);
  }
  precond<T>(P, s);
  k_update_p_finish<T><<<flat_grid(m), kBlock, 0, s>>>(m, (const T*)P->z, (T*)P->p, P->state, 1);
  return 0;
}

template <class T>
int iterate(const ipcb_pcg* P, int k, cudaStream_t s) {
  const int n = P->n, m = 3 * n;
  for (int it = 0; it < k; ++it) {
    k_spmv_dot<T><<<warp_grid(n), kBlock, 0, s>>>(n, P->offsets, P->columns, (const T*)P->values, (const T*)P->p,
                                                     (T*)P->q, P->state);
    if (P->precond == 0 && P->n_groups > 0) {
      k_update_xr_groups<T><<<flat_grid(group_items(P->n_point, P->n_groups)), kBlock, 0, s>>>(
          P->n_point, P->n_groups, (T*)P->x, (T*)P->r, (const T*)P->p, (const T*)P->q, (const T*)P->dinv,
          (const T*)P->dinv_group, (T*)P->z, P->state);
    } else if (P->precond == 0) {
      k_update_xr_jacobi<T><<<flat_grid(n), kBlock, 0, s>>>(n, (T*)P->x, (T*)P->r, (const T*)P->p, (const T*)P->q,
                                                            (const T*)P->dinv, (T*)P->z, P->state);
    } else {
      k_update_xr<T><<<flat_grid(m), kBlock, 0, s>>>(m, (T*)P->x, (T*)P->r, (const T*)P->p, (const T*)P->q,
                                                     P->state);
      precond<T>(P, s);
    }
    k_update_p_finish<T><<<flat_grid(m), kBlock, 0, s>>>(m, (const T*)P->z, (T*)P->p, P->state, 0);
  }
  return 0;
}

bool pcg_ok(const ipcb_pcg* P) {
  if (!P || P->n <= 0 || !P->offsets || !P->columns || !P->values || !P->x || !P->r || !P->z || !P->p || !P->q ||
      !P->b || !P->state)
    return false;
  if (P->n_groups < 0 || P->n_point < 0 || P->n_point > (1 << 30)) return false;
  if (P->precond == 0 && P->n_groups > 0)
    return P->dinv && P->dinv_group && P->n == P->n_point + 4 * P->n_groups;
  if (P->precond == 0) return P->dinv != nullptr;
  if (P->precond == 1) return P->g_offsets && P->g_columns && P->diag && P->g && P->scale && P->t;
  return false;
}

}  // namespace

extern "C" {

int ipcb_pcg_start(const ipcb_pcg* P, double tol, int maxiter, ipcb_stream s) {
  if (!pcg_ok(P) || maxiter < 0 || !(tol >= 0.0)) {
    ipcb::set_error_msg("pcg_start: bad arguments");
    return IPCB_E_ARG;
  }
  if (P->fp64) start<double>(P, tol, maxiter, (cudaStream_t)s);
  else start<float>(P, tol, maxiter, (cudaStream_t)s);
  return ipcb::check_launch("ipcb_pcg_start");
}

int ipcb_pcg_iterate(const ipcb_pcg* P, int k, ipcb_stream s) {
  if (!pcg_ok(P) || k < 0) {
    ipcb::set_error_msg("pcg_iterate: bad arguments");
    return IPCB_E_ARG;
  }
  if (P->fp64) iterate<double>(P, k, (cudaStream_t)s);
  else iterate<float>(P, k, (cudaStream_t)s);
  return ipcb::check_launch("ipcb_pcg_iterate");
}

int ipcb_block_jacobi(int n, const int* offsets, const int* columns, const int* diag, const void* values, int fp64,
                      void* dinv, int* status, ipcb_stream s) {
  if (n < 0 || !offsets || !columns || !values || !dinv || !status) {
    ipcb::set_error_msg("block_jacobi: bad arguments");
    return IPCB_E_ARG;
  }
  if (n == 0) return 0;
  if (fp64)
    k_block_jacobi<double><<<gridn(n), kBlock, 0, (cudaStream_t)s>>>(n, diag, offsets, columns, (const double*)values,
                                                                     (double*)dinv, status);
  else
    k_block_jacobi<float><<<gridn(n), kBlock, 0, (cudaStream_t)s>>>(n, diag, offsets, columns, (const float*)values,
                                                                    (float*)dinv, status);
  return ipcb::check_launch("ipcb_block_jacobi");
}

int ipcb_group_jacobi(int n_point, int n_groups, const int* offsets, const int* columns, const void* values,
                      int fp64, void* dinv_group, int* status, ipcb_stream s) {
  if (n_point < 0 || n_groups < 0 || (n_groups && (!offsets || !columns || !values || !dinv_group || !status)))
    return IPCB_E_ARG;
  if (n_groups == 0) return IPCB_OK;
  const int g = gridn(n_groups, kInvWarps);
  if (fp64)
    k_group_inverse<double><<<g, 32 * kInvWarps, 0, (cudaStream_t)s>>>(n_point, n_groups, offsets, columns,
                                                                       (const double*)values, (double*)dinv_group,
                                                                       status);
  else
    k_group_inverse<float><<<g, 32 * kInvWarps, 0, (cudaStream_t)s>>>(n_point, n_groups, offsets, columns,
                                                                      (const float*)values, (float*)dinv_group,
                                                                      status);
  return ipcb::check_launch("ipcb_group_jacobi");
}

int ipcb_fsai_mirror(const ipcb_graph* g, const float* G, void* gh, ipcb_stream s) {
  if (!g || g->nnz <= 0 || !g->rows || !g->columns || !g->rev || !G || !gh) {
    ipcb::set_error_msg("fsai_mirror: bad arguments");
    return IPCB_E_ARG;
  }
  k_fsai_mirror<<<gridn(g->nnz), kBlock, 0, (cudaStream_t)s>>>(g->nnz, g->rows, g->columns, g->rev, G, (bf16*)gh);
  return ipcb::check_launch("ipcb_fsai_mirror");
}

}  // extern "C"
