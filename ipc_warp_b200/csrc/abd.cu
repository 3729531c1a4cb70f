// Affine body dynamics terms (affine_body_dynamics.py:42-217): the vertex map,
// predictor and velocity update, the per-body 4x4 system of inertia plus
// orthogonality potential, the body energies, and the reduction of the vertex
// contact force and Hessian onto the 12 affine DOFs of each body.
//
// q layout: scalar[12 nb], per body p, a0, a1, a2 (x = p + A r with the
// columns a_k of A).  Mass: the scalar moments M[16 nb] (the reference stores
// M_ij * I as mat33; only the scalar is ever non-zero off the identity).
//
// The reference reduces a contact Hessian by fanning every vertex block out
// into 16 body-space triplets and sorting all of them (256 per contact
// record).  Here the reduced matrix is assembled directly: its block pattern
// comes from the set of touching body pairs (a bitmap over body pairs, one
// scan), and one group of 16 lanes per contact record folds the record's 16
// vertex blocks into its <= 4 body-pair blocks (lane = (a, c) of the 4x4 body
// block), keeping running sums across a contiguous range of records of the
// same body pair and flushing them with one atomic add per value when the
// pair changes.  The 16x fan-out triplet kernel is kept for the generic path.
#include "abd_impl.cuh"
#include "scan.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

// ------------------------------------------------------------ vertex map
template <class S>
__global__ void k_affine_map(int n, const S* __restrict__ q, const S* __restrict__ rest, const int* __restrict__ body,
                             S* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = __ldg(body + i);
  const v3<S> r = load3(rest, i);
  const S* Q = q + 12 * (size_t)b;
  v3<S> x = ld(Q, 0) + ld(Q, 1) * r.x + ld(Q, 2) * r.y + ld(Q, 3) * r.z;
  st3(out, i, x);
}

template <class S>
__global__ void k_step_from(int n, const S* __restrict__ q_start, const S* __restrict__ dq, S alpha,
                            S* __restrict__ q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) q[i] = q_start[i] - alpha * dq[i];
}

// ------------------------------------------------------ predictor / update
template <class S>
__global__ void k_prepare_tilde(Abd<S> A, S h, S gx, S gy, S gz, const S* __restrict__ omega,
                                const int* __restrict__ enabled) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= A.nb) return;
  const int o = 4 * b;
  v3<S> p = ld(A.q0, o) + ld(A.qdot, o) * h + mk3(gx, gy, gz) * (h * h);
  st3(A.qt, o, p);
  const bool motor = enabled && enabled[b] != 0;
  const v3<S> w = motor ? ld(omega, b) : mk3(S(0), S(0), S(0));
  for (int j = 1; j < 4; ++j) {
    const v3<S> a0 = ld(A.q0, o + j);
    const v3<S> v = motor ? cross(w, a0) : ld(A.qdot, o + j);
    st3(A.qt, o + j, a0 + v * h);
  }
}

template <class S>
__global__ void k_update_velocity(Abd<S> A, S h) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 12 * A.nb) return;
  const S q = A.q[i];
  A.qdot[i] = (q - A.q0[i]) / h;
  A.q0[i] = q;
}

// rank of body c in the sorted neighbour list of body r (-1 if absent)
IPCB_D int find_body(const int* __restrict__ body_off, const int* __restrict__ body_cols, int r, int c) {
  int lo = __ldg(body_off + r), hi = __ldg(body_off + r + 1) - 1;
  const int base = lo;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int v = __ldg(body_cols + mid);
    if (v == c) return mid - base;
    if (v < c) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// one thread per (body, i, j): reference triplets (pattern == null) or a
// store into the assembled block (b*4+i, b*4+j)
template <class S>
__global__ void k_body_system(Abd<S> A, S h2, int* __restrict__ rows, int* __restrict__ cols, S* __restrict__ vals,
                              const int* __restrict__ body_off, const int* __restrict__ body_cols,
                              const int* __restrict__ offsets, int capacity, S* __restrict__ gradient,
                              int* status) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 16 * A.nb) return;
  const int b = t >> 4, i = (t >> 2) & 3, j = t & 3;
  S blk[9];
  body_block(A, b, i, j, h2, blk);
  S* dst;
  if (body_off) {
    const int rank = find_body(body_off, body_cols, b, b);
    if (rank < 0) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      return;
    }
    const long long pos = (long long)__ldg(offsets + 4 * b + i) + 4 * rank + j;
    if (pos >= capacity) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      return;
    }
    dst = vals + 9 * pos;
  } else {
    rows[t] = 4 * b + i;
    cols[t] = 4 * b + j;
    dst = vals + 9 * (size_t)t;
  }
  for (int k = 0; k < 9; ++k) dst[k] = blk[k];
  if (j == 0) st3(gradient, 4 * b + i, body_gradient(A, b, i, h2));
}

// ------------------------------------------------------------- energies
template <class S>
__global__ void k_body_energy(Abd<S> A, S h2, double* __restrict__ out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0, oe = 0.0;
  if (b < A.nb && A.fixed[b] == 0) {
    const S* Q = A.q + 12 * (size_t)b;
    const S* T = A.qt + 12 * (size_t)b;
    v3<S> d[4];
    for (int k = 0; k < 4; ++k) d[k] = ld(Q, k) - ld(T, k);
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) e += (double)(S(0.5) * dot(d[i], d[j]) * A.mass[16 * b + 4 * i + j]);
    double o = 0.0;
    for (int i = 1; i < 4; ++i) {
      const v3<S> ai = ld(Q, i);
      const S s = dot(ai, ai) - S(1);
      o += (double)(s * s);
      for (int j = i + 1; j < 4; ++j) {
        const S c = dot(ai, ld(Q, j));
        o += (double)(S(2) * c * c);
      }
    }
    oe = (double)(A.stiffness[b] * A.volume[b] * h2) * o;
  }
  for (int o = 16; o > 0; o >>= 1) {
    e += __shfl_xor_sync(0xffffffffu, e, o);
    oe += __shfl_xor_sync(0xffffffffu, oe, o);
  }
  if ((threadIdx.x & 31) == 0 && (e != 0.0 || oe != 0.0)) {
    atomicAdd(out, e);
    atomicAdd(out + 1, oe);
  }
}

// ------------------------------------------------------ force reduction
// reduced[b] += [f, r0 f, r1 f, r2 f]; gradient (optional) -= h2 * the same.
// A warp whose vertices share one body sums in registers first.
template <class S>
__global__ void k_reduce_force(int n, const S* __restrict__ f, const S* __restrict__ rest,
                               const int* __restrict__ body, const int* __restrict__ fixed, S* __restrict__ reduced,
                               S* __restrict__ gradient, S minus_h2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool active = i < n;
  int b = active ? __ldg(body + i) : -1;
  if (b >= 0 && fixed[b] != 0) b = -1;
  S c[12];
  if (b >= 0) {
    const v3<S> fv = load3(f, i), r = load3(rest, i);
    const S w[4] = {S(1), r.x, r.y, r.z};
    for (int k = 0; k < 4; ++k) {
      c[3 * k] = w[k] * fv.x;
      c[3 * k + 1] = w[k] * fv.y;
      c[3 * k + 2] = w[k] * fv.z;
    }
  } else {
    for (int k = 0; k < 12; ++k) c[k] = S(0);
  }
  int lead = b;
  for (int o = 16; o > 0; o >>= 1) lead = max(lead, __shfl_xor_sync(0xffffffffu, lead, o));
  const bool uniform = __all_sync(0xffffffffu, b == lead || b < 0);
  if (uniform) {
    if (lead < 0) return;
    for (int k = 0; k < 12; ++k)
      for (int o = 16; o > 0; o >>= 1) c[k] += __shfl_xor_sync(0xffffffffu, c[k], o);
    if ((threadIdx.x & 31) == 0) {
      for (int k = 0; k < 12; ++k) {
        atomicAdd(reduced + 12 * (size_t)lead + k, c[k]);
        if (gradient) atomicAdd(gradient + 12 * (size_t)lead + k, minus_h2 * c[k]);
      }
    }
  } else if (b >= 0) {
    for (int k = 0; k < 12; ++k) {
      atomicAdd(reduced + 12 * (size_t)b + k, c[k]);
      if (gradient) atomicAdd(gradient + 12 * (size_t)b + k, minus_h2 * c[k]);
    }
  }
}

template <class S>
__global__ void k_axpy(int n, S* __restrict__ y, const S* __restrict__ x, S a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}

// ------------------------------------- reference-layout Hessian reduction
template <class S>
__global__ void k_reduce_hessian_triplets(int n_src, const int* __restrict__ srows, const int* __restrict__ scols,
                                          const S* __restrict__ svals, const S* __restrict__ rest,
                                          const int* __restrict__ body, const int* __restrict__ fixed, S scale,
                                          int* __restrict__ drows, int* __restrict__ dcols, S* __restrict__ dvals) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 16LL * n_src) return;
  const int s = (int)(t >> 4), a = (int)((t >> 2) & 3), c = (int)(t & 3);
  const int vi = __ldg(srows + s), vj = __ldg(scols + s);
  const int bi = __ldg(body + vi), bj = __ldg(body + vj);
  drows[t] = 4 * bi + a;
  dcols[t] = 4 * bj + c;
  S* d = dvals + 9 * t;
  if (fixed[bi] != 0 || fixed[bj] != 0) {
    for (int k = 0; k < 9; ++k) d[k] = S(0);
    return;
  }
  const S ca = a > 0 ? __ldg(rest + 3 * vi + a - 1) : S(1);
  const S cc = c > 0 ? __ldg(rest + 3 * vj + c - 1) : S(1);
  const S w = scale * ca * cc;
  for (int k = 0; k < 9; ++k) d[k] = w * __ldg(svals + 9 * (size_t)s + k);
}

// ------------------------------------------------ reduced block pattern
// body pair of a contact record: bi = body of its first vertex, bj = the
// body of its first vertex not in bi (bi when all four share it)
IPCB_D bool record_bodies(const int* __restrict__ trows, const int* __restrict__ tcols, const int* __restrict__ body,
                          long long base, int v[4], int& bi, int& bj) {
  v[0] = __ldg(trows + base);
  v[1] = __ldg(tcols + base + 1);
  v[2] = __ldg(tcols + base + 2);
  v[3] = __ldg(tcols + base + 3);
  bi = __ldg(body + v[0]);
  bj = bi;
  bool ok = true;
  for (int k = 1; k < 4; ++k) {
    const int b = __ldg(body + v[k]);
    if (b == bi) continue;
    if (bj == bi) bj = b;
    else if (b != bj) ok = false;
  }
  return ok;
}

__global__ void k_mark_pairs(int n_rec, const int* __restrict__ trows, const int* __restrict__ tcols,
                             const unsigned short* __restrict__ mask, const int* __restrict__ body,
                             const int* __restrict__ fixed, int nb, int words, unsigned* __restrict__ bits,
                             int* status) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < nb) atomicOr(bits + (size_t)r * words + (r >> 5), 1u << (r & 31));
  if (r >= n_rec) return;
  if (mask && mask[r] == 0) return;
  int v[4], bi, bj;
  if (!record_bodies(trows, tcols, body, 16LL * r, v, bi, bj)) {
    atomicOr(status, IPCB_STATUS_PATTERN);
    return;
  }
  if (bi == bj || fixed[bi] != 0 || fixed[bj] != 0) return;
  atomicOr(bits + (size_t)bi * words + (bj >> 5), 1u << (bj & 31));
  atomicOr(bits + (size_t)bj * words + (bi >> 5), 1u << (bi & 31));
}

// one warp per body row: degree = popcount of its bitmap row
__global__ void k_row_degree(int nb, int words, const unsigned* __restrict__ bits, int* __restrict__ deg) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nb) return;
  int c = 0;
  for (int k = lane; k < words; k += 32) c += __popc(bits[(size_t)w * words + k]);
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) deg[w] = c;
}

// one warp per body row: the set bits in ascending order
__global__ void k_row_fill(int nb, int words, const unsigned* __restrict__ bits, const int* __restrict__ body_off,
                           int* __restrict__ body_cols, int pair_capacity) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (w >= nb) return;
  int pos = body_off[w];
  for (int k0 = 0; k0 < words; k0 += 32) {
    const int k = k0 + lane;
    unsigned m = k < words ? bits[(size_t)w * words + k] : 0u;
    const int cnt = __popc(m);
    const int incl = scan::warp_inclusive(cnt, lane);
    int p = pos + incl - cnt;
    while (m) {
      const int bit = __ffs(m) - 1;
      m &= m - 1;
      if (p < pair_capacity) body_cols[p] = 32 * k + bit;
      ++p;
    }
    pos += __shfl_sync(0xffffffffu, incl, 31);
  }
}

// block rows 4b + a: 4 deg(b) blocks, columns 4c + j for c in the row list
__global__ void k_block_pattern(int nb, const int* __restrict__ body_off, const int* __restrict__ body_cols,
                                int pair_capacity, int* __restrict__ offsets, int* __restrict__ columns,
                                int* __restrict__ nnz, int* status) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r > 4 * nb) return;
  const bool over = body_off[nb] > pair_capacity;
  if (r == 4 * nb) {
    offsets[r] = 16 * body_off[nb];
    if (nnz) *nnz = 16 * body_off[nb];
    if (over) atomicOr(status, IPCB_STATUS_PATTERN);
    return;
  }
  if (over) {
    offsets[r] = 0;
    return;
  }
  const int b = r >> 2, a = r & 3;
  const int o = body_off[b], d = body_off[b + 1] - o;
  const int start = 16 * o + 4 * d * a;
  offsets[r] = start;
  for (int k = 0; k < d; ++k) {
    const int c = body_cols[o + k];
    for (int j = 0; j < 4; ++j) columns[start + 4 * k + j] = 4 * c + j;
  }
}

template <class S>
__global__ void k_zero_values(const int* __restrict__ nnz, int cap, S* __restrict__ vals) {
  const long long n = 9LL * min(*nnz, cap);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    vals[i] = S(0);
}

// ---------------------------------------------- grouped Hessian reduction
constexpr int kGroupLanes = 16;
constexpr int kGroupsPerBlock = 8;  // 128 threads

template <class S>
struct PairSums {
  S v[4][9];  // slots (side_i, side_j) = (0,0), (0,1), (1,0), (1,1)
};

template <class S>
IPCB_D void flush(PairSums<S>& acc, int bi, int bj, int a, int c, const int* __restrict__ fixed,
                  const int* __restrict__ body_off, const int* __restrict__ body_cols, const int* __restrict__ offsets,
                  int capacity, S* __restrict__ vals, int* status) {
  if (bi < 0) return;
  if (bi == bj) {  // all four slots land on the same block
#pragma unroll
    for (int s = 1; s < 4; ++s)
#pragma unroll
      for (int k = 0; k < 9; ++k) acc.v[0][k] += acc.v[s][k];
  }
  const int ns = bi == bj ? 1 : 4;
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    if (s >= ns) break;
    const int r = (s >> 1) ? bj : bi, cb = (s & 1) ? bj : bi;
    if (fixed[r] != 0 || fixed[cb] != 0) continue;
    const int rank = find_body(body_off, body_cols, r, cb);
    if (rank < 0) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      continue;
    }
    const long long pos = (long long)__ldg(offsets + 4 * r + a) + 4 * rank + c;
    if (pos >= capacity) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      continue;
    }
    S* d = vals + 9 * pos;
#pragma unroll
    for (int k = 0; k < 9; ++k)
      if (acc.v[s][k] != S(0)) atomicAdd(d + k, acc.v[s][k]);
  }
}

// records [0, n_ee) are EE (vertices a1 a2 | b1 b2), the rest PT (p | t0 t1
// t2): the side of each vertex is fixed by the kind, so the slots are
// compile-time and the running sums stay in registers
template <int KIND> IPCB_D constexpr int side_of(int k) { return KIND == 0 ? (k >= 2) : (k >= 1); }

template <int KIND, class S>
IPCB_D void accumulate(PairSums<S>& acc, unsigned m, const S (&wa)[4], const S (&wc)[4], const S* __restrict__ h0,
                       S scale) {
#pragma unroll
  for (int ii = 0; ii < 4; ++ii) {
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      if (!((m >> (4 * ii + jj)) & 1u)) continue;
      const S w = scale * wa[ii] * wc[jj];
      const S* h = h0 + 9 * (4 * ii + jj);
      const int s = 2 * side_of<KIND>(ii) + side_of<KIND>(jj);
#pragma unroll
      for (int k = 0; k < 9; ++k) acc.v[s][k] += w * __ldg(h + k);
    }
  }
}

template <class S>
__global__ void __launch_bounds__(kGroupLanes* kGroupsPerBlock)
    k_reduce_hessian_grouped(int n_rec, int n_ee, int per_group, const int* __restrict__ trows,
                             const int* __restrict__ tcols, const S* __restrict__ tvals,
                             const unsigned short* __restrict__ mask, const S* __restrict__ rest,
                             const int* __restrict__ body, const int* __restrict__ fixed, S scale,
                             const int* __restrict__ body_off, const int* __restrict__ body_cols,
                             const int* __restrict__ offsets, int capacity, S* __restrict__ vals, int* status) {
  const int lane = threadIdx.x & (kGroupLanes - 1);
  const int a = lane >> 2, c = lane & 3;
  const long long group = (long long)blockIdx.x * kGroupsPerBlock + (threadIdx.x / kGroupLanes);
  const long long r0 = group * per_group;
  const long long r1 = min((long long)n_rec, r0 + per_group);
  PairSums<S> acc;
#pragma unroll
  for (int s = 0; s < 4; ++s)
#pragma unroll
    for (int k = 0; k < 9; ++k) acc.v[s][k] = S(0);
  int cur_i = -1, cur_j = -1;
  for (long long r = r0; r < r1; ++r) {
    const unsigned m = mask ? (unsigned)__ldg(mask + r) : 0xffffu;
    if (m == 0) continue;
    const long long base = 16 * r;
    const bool ee = r < n_ee;
    int v[4];
    v[0] = __ldg(trows + base);
#pragma unroll
    for (int k = 1; k < 4; ++k) v[k] = __ldg(tcols + base + k);
    int bv[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) bv[k] = __ldg(body + v[k]);
    const int bi = bv[0], bj = ee ? bv[2] : bv[1];
    const bool ok = ee ? (bv[1] == bi && bv[3] == bj) : (bv[2] == bj && bv[3] == bj);
    if (!ok) {
      if (lane == 0) atomicOr(status, IPCB_STATUS_PATTERN);
      continue;
    }
    if (fixed[bi] != 0 && fixed[bj] != 0) continue;
    if (bi != cur_i || bj != cur_j) {
      flush(acc, cur_i, cur_j, a, c, fixed, body_off, body_cols, offsets, capacity, vals, status);
#pragma unroll
      for (int s = 0; s < 4; ++s)
#pragma unroll
        for (int k = 0; k < 9; ++k) acc.v[s][k] = S(0);
      cur_i = bi;
      cur_j = bj;
    }
    S wa[4], wc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      wa[k] = a > 0 ? __ldg(rest + 3 * v[k] + a - 1) : S(1);
      wc[k] = c > 0 ? __ldg(rest + 3 * v[k] + c - 1) : S(1);
    }
    const S* h0 = tvals + 9 * (size_t)base;
    if (ee) accumulate<0>(acc, m, wa, wc, h0, scale);
    else accumulate<1>(acc, m, wa, wc, h0, scale);
  }
  flush(acc, cur_i, cur_j, a, c, fixed, body_off, body_cols, offsets, capacity, vals, status);
}

template <class S>
int launch_reduced(const ipcb_abd* abd, double h2, int n_rec, int n_ee, const int* trows, const int* tcols, const void* tvals,
                   const unsigned short* mask, const void* rest, const int* body, const int* body_off,
                   const int* body_cols, const int* offsets, const int* nnz, int capacity, void* values,
                   void* gradient, void* reduced_force, int n_verts, const void* vertex_force, int* status,
                   cudaStream_t st) {
  Abd<S> A = view<S>(abd);
  k_zero_values<S><<<4 * 148, 256, 0, st>>>(nnz, capacity, (S*)values);
  k_body_system<S><<<div_up(16 * A.nb, 128), 128, 0, st>>>(A, S(h2), nullptr, nullptr, (S*)values, body_off, body_cols,
                                                           offsets, capacity, (S*)gradient, status);
  if (reduced_force) cudaMemsetAsync(reduced_force, 0, sizeof(S) * 12 * (size_t)A.nb, st);
  if (n_verts > 0 && vertex_force && reduced_force)
    k_reduce_force<S><<<div_up(n_verts, 256), 256, 0, st>>>(n_verts, (const S*)vertex_force, (const S*)rest, body,
                                                          A.fixed, (S*)reduced_force, (S*)gradient, S(-h2));
  if (n_rec > 0) {
    // enough groups to fill the machine, at least 4 records per group
    const long long target_groups = 148LL * 16 * kGroupsPerBlock;
    int per = (int)((n_rec + target_groups - 1) / target_groups);
    if (per < 4) per = 4;
    const long long groups = (n_rec + per - 1) / per;
    k_reduce_hessian_grouped<S><<<div_up(groups, kGroupsPerBlock), kGroupLanes * kGroupsPerBlock, 0, st>>>(
        n_rec, n_ee, per, trows, tcols, (const S*)tvals, mask, (const S*)rest, body, A.fixed, S(h2), body_off, body_cols,
        offsets, capacity, (S*)values, status);
  }
  return check_launch("ipcb_abd_assemble");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

static bool abd_ok(const ipcb_abd* a) {
  return a && a->n_bodies > 0 && a->q && a->q0 && a->q_tilde && a->qdot && a->mass && a->volume && a->stiffness &&
         a->fixed;
}

extern "C" {

int ipcb_abd_map(int fp64, int n_verts, const void* q, const void* rest, const int* body, void* out, ipcb_stream s) {
  if (n_verts < 0) return IPCB_E_ARG;
  if (n_verts == 0) return IPCB_OK;
  if (!q || !rest || !body || !out) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (fp64)
    k_affine_map<double><<<div_up(n_verts, 256), 256, 0, st>>>(n_verts, (const double*)q, (const double*)rest, body,
                                                                (double*)out);
  else
    k_affine_map<float><<<div_up(n_verts, 256), 256, 0, st>>>(n_verts, (const float*)q, (const float*)rest, body,
                                                               (float*)out);
  return check_launch("ipcb_abd_map");
}

int ipcb_abd_step_from(int fp64, int n, const void* q_start, const void* dq, double alpha, void* q, ipcb_stream s) {
  if (n < 0 || (n && (!q_start || !dq || !q))) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (fp64)
    k_step_from<double><<<div_up(n, 256), 256, 0, st>>>(n, (const double*)q_start, (const double*)dq, alpha,
                                                         (double*)q);
  else
    k_step_from<float><<<div_up(n, 256), 256, 0, st>>>(n, (const float*)q_start, (const float*)dq, (float)alpha,
                                                        (float*)q);
  return check_launch("ipcb_abd_step_from");
}

int ipcb_abd_prepare_tilde(const ipcb_abd* abd, double h, const double* gravity, const void* motor_omega,
                           const int* motor_enabled, ipcb_stream s) {
  if (!abd_ok(abd) || !gravity) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(abd->n_bodies, 128);
  if (abd->fp64)
    k_prepare_tilde<double><<<g, 128, 0, st>>>(view<double>(abd), h, gravity[0], gravity[1], gravity[2],
                                               (const double*)motor_omega, motor_enabled);
  else
    k_prepare_tilde<float><<<g, 128, 0, st>>>(view<float>(abd), (float)h, (float)gravity[0], (float)gravity[1],
                                              (float)gravity[2], (const float*)motor_omega, motor_enabled);
  return check_launch("ipcb_abd_prepare_tilde");
}

int ipcb_abd_update_velocity(const ipcb_abd* abd, double h, ipcb_stream s) {
  if (!abd_ok(abd)) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(12 * abd->n_bodies, 256);
  if (abd->fp64) k_update_velocity<double><<<g, 256, 0, st>>>(view<double>(abd), h);
  else k_update_velocity<float><<<g, 256, 0, st>>>(view<float>(abd), (float)h);
  return check_launch("ipcb_abd_update_velocity");
}

int ipcb_abd_body_system(const ipcb_abd* abd, double h2, int* rows, int* cols, void* vals, void* gradient,
                         ipcb_stream s) {
  if (!abd_ok(abd) || !rows || !cols || !vals || !gradient) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(16 * abd->n_bodies, 128);
  if (abd->fp64)
    k_body_system<double><<<g, 128, 0, st>>>(view<double>(abd), h2, rows, cols, (double*)vals, nullptr, nullptr,
                                             nullptr, 0, (double*)gradient, nullptr);
  else
    k_body_system<float><<<g, 128, 0, st>>>(view<float>(abd), (float)h2, rows, cols, (float*)vals, nullptr, nullptr,
                                            nullptr, 0, (float*)gradient, nullptr);
  return check_launch("ipcb_abd_body_system");
}

int ipcb_abd_body_energy(const ipcb_abd* abd, double h2, double* energies, ipcb_stream s) {
  if (!abd_ok(abd) || !energies) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(abd->n_bodies, 128);
  if (abd->fp64) k_body_energy<double><<<g, 128, 0, st>>>(view<double>(abd), h2, energies);
  else k_body_energy<float><<<g, 128, 0, st>>>(view<float>(abd), (float)h2, energies);
  return check_launch("ipcb_abd_body_energy");
}

int ipcb_abd_reduce_force(const ipcb_abd* abd, int n_verts, const void* vertex_force, const void* rest,
                          const int* body, void* reduced_force, ipcb_stream s) {
  if (!abd_ok(abd) || n_verts < 0 || !reduced_force) return IPCB_E_ARG;
  if (n_verts == 0) return IPCB_OK;
  if (!vertex_force || !rest || !body) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(n_verts, 256);
  if (abd->fp64)
    k_reduce_force<double><<<g, 256, 0, st>>>(n_verts, (const double*)vertex_force, (const double*)rest, body,
                                              abd->fixed, (double*)reduced_force, nullptr, 0.0);
  else
    k_reduce_force<float><<<g, 256, 0, st>>>(n_verts, (const float*)vertex_force, (const float*)rest, body,
                                             abd->fixed, (float*)reduced_force, nullptr, 0.0f);
  return check_launch("ipcb_abd_reduce_force");
}

int ipcb_abd_add_contact_gradient(int fp64, int n, void* gradient, const void* force, double h2, ipcb_stream s) {
  if (n < 0 || (n && (!gradient || !force))) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  cudaStream_t st = (cudaStream_t)s;
  if (fp64) k_axpy<double><<<div_up(n, 256), 256, 0, st>>>(n, (double*)gradient, (const double*)force, -h2);
  else k_axpy<float><<<div_up(n, 256), 256, 0, st>>>(n, (float*)gradient, (const float*)force, (float)-h2);
  return check_launch("ipcb_abd_add_contact_gradient");
}

int ipcb_abd_reduce_hessian(const ipcb_abd* abd, int n_src, const int* src_rows, const int* src_cols,
                            const void* src_vals, const void* rest, const int* body, double scale, int* dst_rows,
                            int* dst_cols, void* dst_vals, ipcb_stream s) {
  if (!abd_ok(abd) || n_src < 0) return IPCB_E_ARG;
  if (n_src == 0) return IPCB_OK;
  if (!src_rows || !src_cols || !src_vals || !rest || !body || !dst_rows || !dst_cols || !dst_vals) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int g = div_up(16LL * n_src, 256);
  if (abd->fp64)
    k_reduce_hessian_triplets<double><<<g, 256, 0, st>>>(n_src, src_rows, src_cols, (const double*)src_vals,
                                                         (const double*)rest, body, abd->fixed, scale, dst_rows,
                                                         dst_cols, (double*)dst_vals);
  else
    k_reduce_hessian_triplets<float><<<g, 256, 0, st>>>(n_src, src_rows, src_cols, (const float*)src_vals,
                                                        (const float*)rest, body, abd->fixed, (float)scale, dst_rows,
                                                        dst_cols, (float*)dst_vals);
  return check_launch("ipcb_abd_reduce_hessian");
}

size_t ipcb_abd_pattern_workspace(int n_bodies) {
  if (n_bodies <= 0 || n_bodies > IPCB_ABD_MAX_BODIES) return 0;
  const size_t words = (size_t)(n_bodies + 31) / 32;
  const size_t bitmap = ((words * n_bodies * 4) + 255) & ~(size_t)255;
  return bitmap + scan::scratch_bytes(n_bodies + 1);
}

int ipcb_abd_pattern(int n_bodies, const int* fixed, const int* body, int n_records, const int* trows,
                     const int* tcols, const unsigned short* block_mask, int* body_off, int* body_cols,
                     int pair_capacity, int* offsets, int* columns, int* nnz, int* status, void* ws, size_t ws_bytes,
                     ipcb_stream s) {
  if (n_bodies <= 0 || n_bodies > IPCB_ABD_MAX_BODIES || n_records < 0 || pair_capacity < n_bodies || !fixed || !body ||
      !body_off ||
      !body_cols || !offsets || !columns || !nnz || !status || !ws)
    return IPCB_E_ARG;
  if (n_records && (!trows || !tcols)) return IPCB_E_ARG;
  if (ws_bytes < ipcb_abd_pattern_workspace(n_bodies)) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int words = (n_bodies + 31) / 32;
  const size_t words_total = (size_t)words * n_bodies;
  unsigned* bits = (unsigned*)ws;
  void* scratch = (char*)ws + (((words_total * 4) + 255) & ~(size_t)255);
  cudaMemsetAsync(bits, 0, words_total * 4, st);
  const int n_mark = n_records > n_bodies ? n_records : n_bodies;
  k_mark_pairs<<<div_up(n_mark, 256), 256, 0, st>>>(n_records, trows, tcols, block_mask, body, fixed, n_bodies, words,
                                                    bits, status);
  k_row_degree<<<div_up(32LL * n_bodies, 256), 256, 0, st>>>(n_bodies, words, bits, body_off);
  cudaMemsetAsync(body_off + n_bodies, 0, sizeof(int), st);
  scan::exclusive<int>(body_off, n_bodies + 1, scratch, nullptr, st);
  k_row_fill<<<div_up(32LL * n_bodies, 256), 256, 0, st>>>(n_bodies, words, bits, body_off, body_cols,
                                                            pair_capacity);
  k_block_pattern<<<div_up(4 * n_bodies + 1, 256), 256, 0, st>>>(n_bodies, body_off, body_cols, pair_capacity, offsets,
                                                                 columns, nnz, status);
  return check_launch("ipcb_abd_pattern");
}

int ipcb_abd_assemble(const ipcb_abd* abd, double h2, int n_records, int n_ee, const int* trows, const int* tcols,
                      const void* tvals, const unsigned short* block_mask, const void* rest, const int* body,
                      const int* body_off, const int* body_cols, const int* offsets, const int* nnz, int capacity,
                      void* values, void* gradient, int n_verts, const void* vertex_force, void* reduced_force,
                      int* status, ipcb_stream s) {
  if (!abd_ok(abd) || n_records < 0 || n_ee < 0 || n_ee > n_records || n_verts < 0 || !rest || !body || !body_off || !body_cols || !offsets || !nnz ||
      capacity < 16 * abd->n_bodies || !values || !gradient || !status)
    return IPCB_E_ARG;
  if (n_records && (!trows || !tcols || !tvals)) return IPCB_E_ARG;
  if (vertex_force && !reduced_force) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (abd->fp64)
    return launch_reduced<double>(abd, h2, n_records, n_ee, trows, tcols, tvals, block_mask, rest, body, body_off, body_cols,
                                  offsets, nnz, capacity, values, gradient, reduced_force, n_verts, vertex_force,
                                  status, st);
  return launch_reduced<float>(abd, h2, n_records, n_ee, trows, tcols, tvals, block_mask, rest, body, body_off, body_cols,
                               offsets, nnz, capacity, values, gradient, reduced_force, n_verts, vertex_force, status,
                               st);
}

}  // extern "C"
