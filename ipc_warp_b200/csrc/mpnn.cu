// Learned preconditioner: a message-passing net over the 3x3-block graph of
// the Newton matrix predicts the row directions H of an FSAI factor, and an
// exact per-row normalisation turns them into G^ (include/ipcb.h).
//
// Every dense product runs on the tensor cores through one templated kernel,
// k_mlp: a persistent CTA stages 128 rows of its A operand into an SW128
// K-major shared tile (the "stage" functor gathers them: the edge state, node
// state and mean message for an update, ...), one thread issues the UMMAs
// into a TMEM accumulator, and the four warps read their 32 lanes back for a
// fused epilogue (bias, ReLU, residual, segmented message aggregation, head).
// The message map is split by input block, [h_i | h_j | e] W1 = (h W1a)_i +
// (h W1b)_j + e W1c: the two node projections are one node-sized product and
// the edge product stages only the 128-byte edge state.  Weight
// gradients use k_wgrad, which stages X^T and dY^T tiles (rows of the batch
// along K) and keeps the [features x outputs] accumulator in TMEM across all
// the row tiles a CTA visits, plus a bias row from a column of ones.
//
// Storage: node/edge states and messages bf16, accumulation fp32, biases
// fp32, G^ fp32 (the rounding points of oracle/mpnn.py).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "scan.cuh"
#include "umma.cuh"

namespace ipcb {
int check_launch(const char* where);
void set_error_msg(const char* msg);
}  // namespace ipcb

namespace {

using bf16 = __nv_bfloat16;
constexpr int W = IPCB_MPNN_WIDTH;  // 64
constexpr int IN = IPCB_MPNN_IN;    // 16
constexpr int LAYERS = IPCB_MPNN_LAYERS;
constexpr int kThreads = 128;
// k_mlp: warps 0-3 produce (stage tiles, issue the UMMAs), warps 4-7 drain the
// accumulators; hardware barrier ids 1 and 2 synchronise each group
constexpr int kMlpThreads = 256;
constexpr int kProdBarrier = 1, kEpiBarrier = 2;

// ------------------------------------------------------------ parameters
// FP32 master layout (weights in x out row-major, then bias)
constexpr int P_WHIN = 0, P_BHIN = P_WHIN + IN * W;
constexpr int P_WEIN = P_BHIN + W, P_BEIN = P_WEIN + IN * W;
constexpr int P_LAYER0 = P_BEIN + W;
constexpr int P_LAYER = 3 * W * W + W + 2 * W * W + W;  // W1 b1 W2 b2
constexpr int O_W1 = 0, O_B1 = 3 * W * W, O_W2 = O_B1 + W, O_B2 = O_W2 + 2 * W * W;
constexpr int P_WOFF = P_LAYER0 + LAYERS * P_LAYER, P_BOFF = P_WOFF + W * 9;
constexpr int P_COUNT = P_BOFF + 9;

// BF16 operand layout (all offsets in elements, multiples of 8)
constexpr int K_ENC_H = 0;                        // [64 out][64 in]  (in >= 16 zero)
constexpr int K_ENC_E = K_ENC_H + W * 64;         // [64][64]
// message map split by input block: [h_i | h_j | e] W1 = h_i W1a + h_j W1b + e W1c
constexpr int K_W1ABT = K_ENC_E + W * 64;         // LAYERS x [128 out (W1a | W1b)][64 in (h)]
constexpr int K_W1CT = K_W1ABT + LAYERS * 2 * W * W; // LAYERS x [64 out][64 in (e)]
constexpr int K_W2T = K_W1CT + LAYERS * W * W;    // LAYERS x [64 out][128 in]
constexpr int K_HEADT = K_W2T + LAYERS * W * 2 * W; // [16 out][64 in]: rows 0..8 the head
constexpr int K_W1 = K_HEADT + 16 * W;            // LAYERS x [192 in][64 out]
constexpr int K_W2 = K_W1 + LAYERS * 3 * W * W;   // LAYERS x [128 in][64 out]
constexpr int K_HEAD = K_W2 + LAYERS * 2 * W * W; // [64 in][64 cols]: cols 0..8 the head
constexpr int K_COUNT = K_HEAD + W * 64;

__global__ void k_pack(const float* __restrict__ p, bf16* __restrict__ q) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= K_COUNT) return;
  float v = 0.f;
  if (t < K_ENC_E) {  // enc_h^T
    const int o = (t - K_ENC_H) / 64, k = (t - K_ENC_H) % 64;
    v = k < IN ? p[P_WHIN + k * W + o] : 0.f;
  } else if (t < K_W1ABT) {
    const int o = (t - K_ENC_E) / 64, k = (t - K_ENC_E) % 64;
    v = k < IN ? p[P_WEIN + k * W + o] : 0.f;
  } else if (t < K_W1CT) {
    // row o < 64: h_i part (W1 rows 0..63); row 64 + o: h_j part (W1 rows 64..127)
    const int r = t - K_W1ABT, l = r / (2 * W * W), o = (r % (2 * W * W)) / W, k = r % W;
    v = p[P_LAYER0 + l * P_LAYER + O_W1 + ((o / W) * W + k) * W + (o % W)];
  } else if (t < K_W2T) {
    const int r = t - K_W1CT, l = r / (W * W), o = (r % (W * W)) / W, k = r % W;
    v = p[P_LAYER0 + l * P_LAYER + O_W1 + (2 * W + k) * W + o];
  } else if (t < K_HEADT) {
    const int r = t - K_W2T, l = r / (W * 2 * W), o = (r % (W * 2 * W)) / (2 * W), k = r % (2 * W);
    v = p[P_LAYER0 + l * P_LAYER + O_W2 + k * W + o];
  } else if (t < K_W1) {
    const int r = t - K_HEADT, o = r / W, k = r % W;
    if (o < 9) v = p[P_WOFF + k * 9 + o];
  } else if (t < K_W2) {
    const int r = t - K_W1, l = r / (3 * W * W), k = (r % (3 * W * W)) / W, o = r % W;
    v = p[P_LAYER0 + l * P_LAYER + O_W1 + k * W + o];
  } else if (t < K_HEAD) {
    const int r = t - K_W2, l = r / (2 * W * W), k = (r % (2 * W * W)) / W, o = r % W;
    v = p[P_LAYER0 + l * P_LAYER + O_W2 + k * W + o];
  } else {
    const int r = t - K_HEAD, k = r / 64, c = r % 64;
    if (c < 9) v = p[P_WOFF + k * 9 + c];
  }
  q[t] = __float2bfloat16_rn(v);
}

// ------------------------------------------------------------ helpers
__device__ __forceinline__ float bfr(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}
__device__ __forceinline__ uint4 zero4() { return make_uint4(0, 0, 0, 0); }
__device__ __forceinline__ uint4 ld4(const bf16* p) { return *reinterpret_cast<const uint4*>(p); }

__device__ __forceinline__ void unpack8(uint4 u, float (&f)[8]) {
  const __nv_bfloat162* b = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float2 t = __bfloat1622float2(b[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}
__device__ __forceinline__ uint4 pack8(const float* f) {
  uint4 u;
  __nv_bfloat162* b = reinterpret_cast<__nv_bfloat162*>(&u);
#pragma unroll
  for (int i = 0; i < 4; ++i) b[i] = __floats2bfloat162_rn(f[2 * i], f[2 * i + 1]);
  return u;
}

// ------------------------------------------------------------ stages
struct StageDense {  // row-major bf16 rows, columns >= kvalid read as zero
  const bf16* X;
  int ld, kvalid;
  __device__ uint4 group(int row, int c, int g) const {
    const int k = c * 64 + g * 8;
    return k < kvalid ? ld4(X + (size_t)row * ld + k) : zero4();
  }
};

struct StageNode {  // [h | a] of a node (a: mean message, from k_mean_messages)
  const bf16* h;
  const bf16* a;
  __device__ uint4 group(int row, int c, int g) const {
    return ld4((c == 0 ? h : a) + (size_t)row * W + g * 8);
  }
};

struct StageGather {  // X[idx[row]] (64 wide)
  const bf16* X;
  const int* idx;
  __device__ uint4 group(int row, int, int g) const { return ld4(X + (size_t)__ldg(idx + row) * W + g * 8); }
};

// ------------------------------------------------------------ epilogues
// The accumulator tile is moved from TMEM into shared memory (acc: row r at
// r * stride floats), and each epilogue warp then finishes its 32 rows with
// rows32(): lane l works on column group l % 8 (8 columns) of row l / 8 of
// each step of 4 rows, so a row's gathers and stores are contiguous 128- or
// 256-byte accesses, and the 8 steps are unrolled so that their loads are in
// flight together.  Per-row indices are loaded once per warp (lane l: row l)
// and broadcast with shuffles.  tile is the staged A tile (SW128 layout),
// still intact during the epilogue; nvalid rows of the 32 are inside the
// batch.
__device__ __forceinline__ void ld8f(const float* p, float (&f)[8]) {
  const float4 a = reinterpret_cast<const float4*>(p)[0], b = reinterpret_cast<const float4*>(p)[1];
  f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w; f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
}
__device__ __forceinline__ void ld8s(const float* p, float (&f)[8]) {  // shared, any alignment
#pragma unroll
  for (int t = 0; t < 8; ++t) f[t] = p[t];
}

struct EpiBiasRelu {  // out = bf16(relu(v + b)), 64 columns
  const float* b;
  bf16* out;
  __device__ void rows32(int grow0, int nvalid, const float* acc, int stride, const uint8_t*, int, int lane) const {
    const int q = lane >> 3, cg = lane & 7;
    float bb[8];
    ld8f(b + 8 * cg, bb);
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int r = 4 * it + q;
      if (r >= nvalid) continue;
      float v[8];
      ld8s(acc + r * stride + 8 * cg, v);
#pragma unroll
      for (int t = 0; t < 8; ++t) v[t] = fmaxf(v[t] + bb[t], 0.f);
      *reinterpret_cast<uint4*>(out + (size_t)(grow0 + r) * W + 8 * cg) = pack8(v);
    }
  }
};

struct EpiEdge {  // m = relu(v + b1 + P_a[i] + P_b[j]); e_out = e_in + m (e_in: the staged tile)
  const float* b;
  const float* proj;  // [n][128]: columns 0..63 h W1a, 64..127 h W1b
  bf16* e_out;
  bf16* m_out;
  const int* rows;
  const int* cols;
  __device__ void rows32(int grow0, int nvalid, const float* acc, int stride, const uint8_t* tile, int r0,
                         int lane) const {
    const int q = lane >> 3, cg = lane & 7;
    const int my_i = lane < nvalid ? __ldg(rows + grow0 + lane) : 0;
    const int my_j = lane < nvalid ? __ldg(cols + grow0 + lane) : 0;
    float bb[8];
    ld8f(b + 8 * cg, bb);
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int r = 4 * it + q;
      const int i = __shfl_sync(0xffffffffu, my_i, r), j = __shfl_sync(0xffffffffu, my_j, r);
      if (r >= nvalid) continue;
      float pa[8], pb[8], v[8], e[8], m[8];
      ld8f(proj + (size_t)i * 2 * W + 8 * cg, pa);
      ld8f(proj + (size_t)j * 2 * W + W + 8 * cg, pb);
      ld8s(acc + r * stride + 8 * cg, v);
      unpack8(*reinterpret_cast<const uint4*>(tile + umma::sw128_group(r0 + r, 0, cg, 128)), e);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        m[t] = bfr(fmaxf(v[t] + bb[t] + pa[t] + pb[t], 0.f));
        e[t] += m[t];
      }
      *reinterpret_cast<uint4*>(e_out + (size_t)(grow0 + r) * W + 8 * cg) = pack8(e);
      *reinterpret_cast<uint4*>(m_out + (size_t)(grow0 + r) * W + 8 * cg) = pack8(m);
    }
  }
};

struct EpiNode {  // u = relu(v + b2); h_out = h_in + u (h_in: chunk 0 of the staged tile)
  const float* b;
  bf16* h_out;
  bf16* u_out;
  __device__ void rows32(int grow0, int nvalid, const float* acc, int stride, const uint8_t* tile, int r0,
                         int lane) const {
    const int q = lane >> 3, cg = lane & 7;
    float bb[8];
    ld8f(b + 8 * cg, bb);
#pragma unroll
    for (int it = 0; it < 8; ++it) {
      const int r = 4 * it + q;
      if (r >= nvalid) continue;
      float v[8], h[8], u[8];
      ld8s(acc + r * stride + 8 * cg, v);
      unpack8(*reinterpret_cast<const uint4*>(tile + umma::sw128_group(r0 + r, 0, cg, 128)), h);
#pragma unroll
      for (int t = 0; t < 8; ++t) {
        u[t] = bfr(fmaxf(v[t] + bb[t], 0.f));
        h[t] += u[t];
      }
      *reinterpret_cast<uint4*>(h_out + (size_t)(grow0 + r) * W + 8 * cg) = pack8(h);
      if (u_out) *reinterpret_cast<uint4*>(u_out + (size_t)(grow0 + r) * W + 8 * cg) = pack8(u);
    }
  }
};

// rho_i = c / (1 + c), c = sum of |A^_ij|_F over the off-diagonal blocks of
// row i (node feature 10)
__device__ __forceinline__ float coupling(const bf16* __restrict__ x, int i) {
  const float c = __bfloat162float(x[(size_t)i * IN + 10]);
  return c / (1.f + c);
}

// Row directions on a lower block (out: the head output read as a 3x3
// matrix): H_ii = I and H_ij = (rho_i out - I) A^_ij.  A zero head gives
// first-order FSAI; a weakly coupled row stays at first order, where it is
// accurate, whatever the head outputs.  One lane per row.
struct EpiHead {
  const float *b_off, *ahat;
  const bf16* x;
  const int *lower, *rows, *cols;
  float* H;
  __device__ void rows32(int grow0, int nvalid, const float* acc, int stride, const uint8_t*, int, int lane) const {
    if (lane >= nvalid) return;
    const int e = __ldg(lower + grow0 + lane);
    const int i = __ldg(rows + e);
    float* h = H + (size_t)e * 9;
    if (i == __ldg(cols + e)) {
#pragma unroll
      for (int k = 0; k < 9; ++k) h[k] = (k % 4) == 0 ? 1.f : 0.f;
      return;
    }
    const float* a = ahat + (size_t)e * 9;
    const float* v = acc + lane * stride;
    const float rho = coupling(x, i);
    float p[9], am[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      p[k] = rho * (v[k] + __ldg(b_off + k)) - ((k % 4) == 0 ? 1.f : 0.f);
      am[k] = __ldg(a + k);
    }
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) h[3 * r + c] = p[3 * r] * am[c] + p[3 * r + 1] * am[3 + c] + p[3 * r + 2] * am[6 + c];
  }
};

struct EpiF32 {  // plain fp32 rows of width ld (lanes across the columns)
  float* out;
  int ld;
  __device__ void rows32(int grow0, int nvalid, const float* acc, int stride, const uint8_t*, int, int lane) const {
    for (int r = 0; r < nvalid; ++r) {
      float* o = out + (size_t)(grow0 + r) * ld;
      for (int c = lane; c < ld; c += 32) o[c] = acc[r * stride + c];
    }
  }
};

// ------------------------------------------------------------ k_mlp
// Warp-specialised persistent product: D = A B^T + epilogue over 128-row
// tiles of A.  Producer warps (0-3) gather tile k into shared stage k % 2
// (thread t stages row t), then thread 0 issues the UMMAs into TMEM
// accumulator k % 2 and commits to mma_done[k % 2]; epilogue warps (4-7) wait
// for it, read their 32 lanes each (and may read the staged tile) and arrive
// on acc_free[k % 2].  Stage and accumulator k % 2 are reused for tile k + 2
// only after that release, so tile k + 1 is gathered and multiplied while
// tile k is drained.  Every wait is bounded; a wait that
// gives up raises IPCB_STATUS_TIMEOUT and ends the CTA's loop.
template <int N, int C>
constexpr size_t mlp_smem() {
  return 1024 + 2 * (size_t)C * 128 * 128 + (size_t)C * N * 128 + 128 * (size_t)(N + 1) * 4;
}

template <int N, int C, class Stage, class Epi>
__global__ void __launch_bounds__(kMlpThreads) k_mlp(int rows, Stage st, Epi ep, const bf16* __restrict__ Bw,
                                                     int* __restrict__ status) {
  extern __shared__ uint8_t dsmem[];
  __shared__ uint64_t mma_done[2], acc_free[2];
  __shared__ uint32_t tslot;
  // abort flags, each written only by its own group before that group's barrier
  __shared__ int prod_abort, epi_abort;
  // accumulator stride: at least the 32 columns one tcgen05.ld reads
  constexpr int NA = N < 32 ? 32 : N;
  constexpr uint32_t kCols = umma::tmem_cols(2 * NA);
  static_assert(2 * NA <= 512, "two accumulators must fit the 512 TMEM columns");
  constexpr int K = 64 * C;
  constexpr int kStage = C * 128 * 128;
  uint8_t* sA = align1024(dsmem);
  uint8_t* sB = sA + 2 * kStage;
  float* accs = reinterpret_cast<float*>(sB + C * N * 128);  // [128][N + 1]
  constexpr int kStride = N + 1;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int idx = tid; idx < N * C * 8; idx += kMlpThreads) {
    const int r = idx / (C * 8), c = (idx / 8) % C, g = idx % 8;
    *reinterpret_cast<uint4*>(sB + umma::sw128_group(r, c, g, N)) = ld4(Bw + (size_t)r * K + c * 64 + g * 8);
  }
  if (warp == 0) umma::tmem_alloc(&tslot, kCols);
  if (tid == 0) {
    umma::mbar_init(&mma_done[0], 1);
    umma::mbar_init(&mma_done[1], 1);
    umma::mbar_init(&acc_free[0], 128);
    umma::mbar_init(&acc_free[1], 128);
    prod_abort = 0;
    epi_abort = 0;
  }
  umma::fence_async_smem();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  const int ntiles = (rows + 127) / 128;
  const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  int issued = 0;  // tiles whose UMMAs thread 0 committed

  if (warp < 4) {
    for (int k = 0; k < mine; ++k) {
      const int s = k & 1, use = k >> 1;
      // stage s is free once the epilogue of tile k - 2 (which reads it) is done
      if (k >= 2 && !umma::mbar_wait(&acc_free[s], (use - 1) & 1)) prod_abort = 1;
      umma::named_sync(kProdBarrier, 128);
      if (prod_abort) break;  // uniform: read after the group barrier
      // warp w stages rows 32w..32w+31; lanes take consecutive 16-byte groups
      // of a row, so a warp reads contiguous row spans
      const int base = (blockIdx.x + k * gridDim.x) * 128 + 32 * warp;
      uint8_t* a = sA + s * kStage;
      // all of the warp's loads first, then the shared stores
      uint4 buf[C][8];
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int item = it * 32 + lane, row = base + item / 8;
          buf[c][it] = row < rows ? st.group(row, c, item % 8) : zero4();
        }
#pragma unroll
      for (int c = 0; c < C; ++c)
#pragma unroll
        for (int it = 0; it < 8; ++it) {
          const int item = it * 32 + lane;
          *reinterpret_cast<uint4*>(a + umma::sw128_group(32 * warp + item / 8, c, item % 8, 128)) = buf[c][it];
        }
      umma::fence_async_smem();
      umma::named_sync(kProdBarrier, 128);
      if (tid == 0) {
        umma::fence_after();
        umma::issue_tile<N, C>(tmem + s * NA, umma::smem_u32(a), umma::smem_u32(sB), false, &mma_done[s]);
        issued = k + 1;
      }
    }
  } else {
    const int et = tid - 128;
    for (int k = 0; k < mine; ++k) {
      const int s = k & 1, use = k >> 1;
      if (!umma::mbar_wait(&mma_done[s], use & 1)) epi_abort = 1;
      umma::named_sync(kEpiBarrier, 128);
      if (epi_abort) break;  // uniform: read after the group barrier
      umma::fence_after();
      // TMEM -> shared: thread et owns accumulator row et
#pragma unroll
      for (int col = 0; col < N; col += 32) {
        float v[32];
        umma::tmem_ld32(tmem + s * NA + ((uint32_t)(32 * (warp - 4)) << 16) + col, v);
#pragma unroll
        for (int i = 0; i < 32; ++i)
          if (col + i < N) accs[et * kStride + col + i] = v[i];
      }
      umma::fence_before();
      umma::named_sync(kEpiBarrier, 128);
      // each epilogue warp finishes 32 rows
      const int r0 = 32 * (warp - 4);
      const int grow0 = (blockIdx.x + k * gridDim.x) * 128 + r0;
      const int nvalid = rows - grow0 < 32 ? rows - grow0 : 32;
      if (nvalid > 0) ep.rows32(grow0, nvalid, accs + r0 * kStride, kStride, sA + s * kStage, r0, lane);
      umma::named_sync(kEpiBarrier, 128);
      umma::mbar_arrive(&acc_free[s]);
    }
  }
  __syncthreads();
  if (prod_abort || epi_abort) {
    if (tid == 0) {
      atomicOr(status, IPCB_STATUS_TIMEOUT);
      // let UMMAs still in flight finish (bounded) before the TMEM is freed
      for (int k = issued > 2 ? issued - 2 : 0; k < issued; ++k) umma::mbar_wait(&mma_done[k & 1], (k >> 1) & 1);
    }
    __syncthreads();
  }
  umma::fence_after();
  if (warp == 0) umma::tmem_dealloc(tmem, kCols);
}

int g_sms = 0;
int sm_count() {
  if (!g_sms) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sms, cudaDevAttrMultiProcessorCount, dev);
    if (g_sms <= 0) g_sms = 148;
  }
  return g_sms;
}

template <int N, int C, class Stage, class Epi>
int launch_mlp(int rows, const Stage& st, const Epi& ep, const bf16* Bw, int* status, cudaStream_t s,
               const char* what) {
  if (rows <= 0) return 0;
  constexpr size_t smem = mlp_smem<N, C>();
  auto kern = k_mlp<N, C, Stage, Epi>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    ipcb::set_error_msg(what);
    return IPCB_E_CUDA;
  }
  const int by_tmem = (int)(512 / umma::tmem_cols(2 * (N < 32 ? 32 : N)));
  const int by_smem = (int)((227 * 1024) / (smem + 1024));
  const int per_sm = by_tmem < by_smem ? by_tmem : by_smem;
  const int tiles = (rows + 127) / 128;
  const int cap = sm_count() * (per_sm > 0 ? per_sm : 1);
  kern<<<tiles < cap ? tiles : cap, kMlpThreads, smem, s>>>(rows, st, ep, Bw, status);
  return ipcb::check_launch(what);
}

// ------------------------------------------------------------ k_wgrad
// dW[f][o] += sum_r X[r][f] dY[r][o] over all rows, plus the bias gradient in
// row f = kx (a column of ones appended to X).  MT M-tiles of 128 features.
struct EpiGrad {
  float* dW;  // [kx][out]
  float* db;  // [out]
  int kx, out;
  __device__ void add(int f, int col0, const float (&v)[32]) const {
    if (f < kx) {
      for (int i = 0; i < 32 && col0 + i < out; ++i) atomicAdd(dW + (size_t)f * out + col0 + i, v[i]);
    } else if (f == kx) {
      for (int i = 0; i < 32 && col0 + i < out; ++i) atomicAdd(db + col0 + i, v[i]);
    }
  }
};

struct EpiGradHead {  // columns 0..8: the head
  float *dW_off, *db_off;
  __device__ void add(int f, int col0, const float (&v)[32]) const {
    if (col0 != 0 || f > W) return;
    for (int k = 0; k < 9; ++k) {
      if (f < W) atomicAdd(dW_off + f * 9 + k, v[k]);
      else atomicAdd(db_off + k, v[k]);
    }
  }
};

template <int MT, int N>
constexpr size_t wgrad_smem() {
  return 1024 + (size_t)MT * 2 * 128 * 128 + (size_t)2 * N * 128;
}

template <int MT, int N, class Epi>
__global__ void __launch_bounds__(kThreads) k_wgrad(int R, const bf16* __restrict__ X, int ldx, int kx,
                                                    const bf16* __restrict__ dY, int ldy, Epi ep,
                                                    int* __restrict__ status) {
  extern __shared__ uint8_t dsmem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  constexpr uint32_t kCols = umma::tmem_cols(MT * N);
  uint8_t* sA = align1024(dsmem);                // MT x [128 features][128 rows]
  uint8_t* sB = sA + MT * 2 * 128 * 128;         // [N outputs][128 rows]
  const int tid = threadIdx.x, warp = tid >> 5;
  if (warp == 0) umma::tmem_alloc(&tslot, kCols);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  uint32_t phase = 0;
  int ok = 1;
  bool any = false;
  const int ntiles = (R + 127) / 128;
  const bf16 one = __float2bfloat16_rn(1.f), zero = __float2bfloat16_rn(0.f);
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int r = tile * 128 + tid;
    const bool valid = r < R;
    // X^T: element (feature f, k = tid)
    for (int f0 = 0; f0 < MT * 128; f0 += 8) {
      float xv[8];
      if (valid && f0 + 8 <= kx) {
        unpack8(ld4(X + (size_t)r * ldx + f0), xv);
      } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) xv[i] = 0.f;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int f = f0 + i;
        bf16 val = f < kx ? __float2bfloat16_rn(xv[i]) : (f == kx && valid ? one : zero);
        *reinterpret_cast<bf16*>(sA + (f >> 7) * (2 * 128 * 128) + umma::sw128_offset(f & 127, tid, 128)) = val;
      }
    }
    for (int o0 = 0; o0 < N; o0 += 8) {
      float yv[8];
      if (valid) unpack8(ld4(dY + (size_t)r * ldy + o0), yv);
      else {
#pragma unroll
        for (int i = 0; i < 8; ++i) yv[i] = 0.f;
      }
#pragma unroll
      for (int i = 0; i < 8; ++i)
        *reinterpret_cast<bf16*>(sB + umma::sw128_offset(o0 + i, tid, N)) = __float2bfloat16_rn(yv[i]);
    }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after();
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
        umma::issue<N, 2>(tmem + mt * N, umma::smem_u32(sA + mt * 2 * 128 * 128), umma::smem_u32(sB), any);
      umma::commit(&mbar);
    }
    ok = __syncthreads_and(umma::mbar_wait(&mbar, phase) ? 1 : 0);
    phase ^= 1;
    if (!ok) break;
    any = true;
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, IPCB_STATUS_TIMEOUT);
    umma::mbar_wait(&mbar, phase);
  } else if (any) {
    umma::fence_after();
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int col = 0; col < N; col += 32) {
        float v[32];
        umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + mt * N + col, v);
        ep.add(mt * 128 + tid, col, v);
      }
  }
  umma::fence_before();
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kCols);
}

template <int MT, int N, class Epi>
int launch_wgrad(int R, const bf16* X, int ldx, int kx, const bf16* dY, int ldy, const Epi& ep, int* status,
                 cudaStream_t s, const char* what) {
  if (R <= 0) return 0;
  constexpr size_t smem = wgrad_smem<MT, N>();
  auto kern = k_wgrad<MT, N, Epi>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) {
    ipcb::set_error_msg(what);
    return IPCB_E_CUDA;
  }
  const int tiles = (R + 127) / 128;
  // few CTAs: each reduces many tiles in TMEM before its atomics
  const int cap = sm_count();
  kern<<<tiles < cap ? tiles : cap, kThreads, smem, s>>>(R, X, ldx, kx, dY, ldy, ep, status);
  return ipcb::check_launch(what);
}

// ------------------------------------------------------------ graph
__global__ void k_graph_rows(int n, const int* __restrict__ off, const int* __restrict__ col, int* __restrict__ rows,
                             int* __restrict__ rev, int* __restrict__ diag, int* __restrict__ lower_count,
                             int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = off[i], e = off[i + 1];
  int d = -1;
  for (int k = b; k < e; ++k) {
    rows[k] = i;
    const int j = col[k];
    if (j == i) d = k;
    // transposed block (j, i): binary search in row j
    int lo = off[j], hi = off[j + 1] - 1, r = -1;
    while (lo <= hi) {
      const int mid = (lo + hi) >> 1, c = col[mid];
      if (c == i) { r = mid; break; }
      if (c < i) lo = mid + 1; else hi = mid - 1;
    }
    rev[k] = r;
    if (r < 0) atomicOr(status, IPCB_STATUS_PATTERN);
  }
  diag[i] = d;
  if (d < 0) atomicOr(status, IPCB_STATUS_PATTERN);
  lower_count[i] = d < 0 ? 0 : d - b + 1;
}

__global__ void k_graph_lower(int n, const int* __restrict__ off, const int* __restrict__ diag,
                              const int* __restrict__ lower_start, int* __restrict__ lower) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int b = off[i], c = diag[i] < 0 ? 0 : diag[i] - b + 1, s0 = lower_start[i];
  for (int k = 0; k < c; ++k) lower[s0 + k] = b + k;
}

// ------------------------------------------------------------ features
template <class T>
__global__ void k_scale(int n, const int* __restrict__ diag, const T* __restrict__ vals, float* __restrict__ scale,
                        int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int d = diag[i];
  for (int a = 0; a < 3; ++a) {
    double v = d >= 0 ? (double)vals[(size_t)d * 9 + 4 * a] : 0.0;
    if (!(v > 0.0)) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      v = 1.0;
    }
    scale[3 * i + a] = (float)(1.0 / sqrt(v));
  }
}

template <class T>
__global__ void k_edge_features(int nnz, const int* __restrict__ rows, const int* __restrict__ cols,
                                const T* __restrict__ vals, const float* __restrict__ scale, float* __restrict__ ahat,
                                bf16* __restrict__ y) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nnz) return;
  const int i = rows[e], j = cols[e];
  float a[9];
  double fro = 0.0;
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double v = (double)vals[(size_t)e * 9 + 3 * r + c] * (double)scale[3 * i + r] * (double)scale[3 * j + c];
      a[3 * r + c] = (float)v;
      fro += v * v;
    }
  float f[16];
#pragma unroll
  for (int k = 0; k < 9; ++k) {
    ahat[(size_t)e * 9 + k] = a[k];
    f[k] = a[k];
  }
  f[9] = (float)sqrt(fro);
  f[10] = i == j ? 1.f : 0.f;
#pragma unroll
  for (int k = 11; k < 16; ++k) f[k] = 0.f;
  uint4* dst = reinterpret_cast<uint4*>(y + (size_t)e * 16);
  dst[0] = pack8(f);
  dst[1] = pack8(f + 8);
}

__global__ void k_node_features(int n, const int* __restrict__ off, const int* __restrict__ cols,
                                const int* __restrict__ diag, const float* __restrict__ ahat, bf16* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float f[16];
  const int d = diag[i];
#pragma unroll
  for (int k = 0; k < 9; ++k) f[k] = d >= 0 ? ahat[(size_t)d * 9 + k] : 0.f;
  const int b = off[i], e = off[i + 1];
  double rs = 0.0;
  for (int k = b; k < e; ++k) {
    if (cols[k] == i) continue;
    double s = 0.0;
    for (int q = 0; q < 9; ++q) {
      const double v = ahat[(size_t)k * 9 + q];
      s += v * v;
    }
    rs += sqrt(s);
  }
  f[9] = (float)log1p((double)(e - b));
  f[10] = (float)rs;
#pragma unroll
  for (int k = 11; k < 16; ++k) f[k] = 0.f;
  uint4* dst = reinterpret_cast<uint4*>(x + (size_t)i * 16);
  dst[0] = pack8(f);
  dst[1] = pack8(f + 8);
}

// ------------------------------------------------------------ loss
__device__ __forceinline__ int find_col(const int* __restrict__ off, const int* __restrict__ cols, int row, int c) {
  int lo = off[row], hi = off[row + 1] - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1, v = __ldg(cols + mid);
    if (v == c) return mid;
    if (v < c) lo = mid + 1; else hi = mid - 1;
  }
  return -1;
}

__device__ __forceinline__ void mm3_acc(float (&acc)[9], const float* __restrict__ a, const float* __restrict__ b) {
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[3 * r + c] += a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

// T_ij = sum_{k <= i} H_ik A^_kj over the lower blocks (i, j)
__global__ void k_fsai_T(int n_lower, const int* __restrict__ lower, const int* __restrict__ rows,
                         const int* __restrict__ cols, const int* __restrict__ off, const int* __restrict__ diag,
                         const float* __restrict__ ahat, const float* __restrict__ H, float* __restrict__ T) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_lower) return;
  const int e = lower[r], i = rows[e], j = cols[e];
  float t[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int ke = off[i]; ke <= diag[i]; ++ke) {
    const int kj = find_col(off, cols, cols[ke], j);
    if (kj >= 0) mm3_acc(t, H + (size_t)ke * 9, ahat + (size_t)kj * 9);
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) T[(size_t)e * 9 + q] = t[q];
}

// Per row: M_i = sum_j T_ij H_ij^T, Cholesky M_i = C C^T, G^_ij = C^-1 H_ij;
// acc[0] += log det M_i, minv_i = M_i^-1.  A row whose M_i is not positive
// definite keeps G^ = H and raises IPCB_STATUS_PATTERN.
__global__ void k_fsai_rows(int n, const int* __restrict__ off, const int* __restrict__ diag,
                            const float* __restrict__ H, const float* __restrict__ T, float* __restrict__ minv,
                            float* __restrict__ G, double* __restrict__ acc, int* __restrict__ status) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double part = 0.0;
  if (i < n) {
    double M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int e = off[i]; e <= diag[i]; ++e) {
      const float* t = T + (size_t)e * 9;
      const float* h = H + (size_t)e * 9;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          M[3 * r + c] += (double)t[3 * r] * h[3 * c] + (double)t[3 * r + 1] * h[3 * c + 1] +
                          (double)t[3 * r + 2] * h[3 * c + 2];
    }
    // symmetrise, Cholesky
    const double m00 = M[0], m10 = 0.5 * (M[3] + M[1]), m11 = M[4], m20 = 0.5 * (M[6] + M[2]),
                 m21 = 0.5 * (M[7] + M[5]), m22 = M[8];
    bool ok = m00 > 0.0;
    const double c00 = ok ? sqrt(m00) : 1.0;
    const double c10 = m10 / c00, c20 = m20 / c00;
    const double d11 = m11 - c10 * c10;
    ok = ok && d11 > 0.0;
    const double c11 = ok ? sqrt(d11) : 1.0;
    const double c21 = (m21 - c20 * c10) / c11;
    const double d22 = m22 - c20 * c20 - c21 * c21;
    ok = ok && d22 > 0.0;
    const double c22 = ok ? sqrt(d22) : 1.0;
    double L[9];  // C^-1 (lower triangular)
    L[0] = 1.0 / c00; L[1] = 0.0; L[2] = 0.0;
    L[4] = 1.0 / c11; L[3] = -c10 * L[0] / c11; L[5] = 0.0;
    L[8] = 1.0 / c22; L[6] = -(c20 * L[0] + c21 * L[3]) / c22; L[7] = -c21 * L[4] / c22;
    if (!ok) {
      atomicOr(status, IPCB_STATUS_PATTERN);
      for (int q = 0; q < 9; ++q) L[q] = (q % 4) == 0 ? 1.0 : 0.0;
    }
    // M^-1 = L^T L
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        minv[(size_t)i * 9 + 3 * r + c] = (float)(L[r] * L[c] + L[3 + r] * L[3 + c] + L[6 + r] * L[6 + c]);
    part = ok ? 2.0 * log(c00 * c11 * c22) : 0.0;
    for (int e = off[i]; e <= diag[i]; ++e) {
      const float* h = H + (size_t)e * 9;
      float* g = G + (size_t)e * 9;
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          g[3 * r + c] = (float)(L[3 * r] * h[c] + L[3 * r + 1] * h[3 + c] + L[3 * r + 2] * h[6 + c]);
    }
  }
  part = warp_sum(part);
  if ((threadIdx.x & 31) == 0 && part != 0.0) atomicAdd(acc, part);
}

// gradient of weight * (1/N) sum_i log det M_i w.r.t. the head outputs:
// dH_ij = (2/N) M_i^-1 T_ij, d out = rho_i dH A^T, written bf16 in columns
// 0..8 of a 64-wide row (zero for diagonal blocks)
__global__ void k_fsai_dout(int n_lower, int n, const int* __restrict__ lower, const int* __restrict__ rows,
                            const int* __restrict__ cols, const float* __restrict__ ahat, const bf16* __restrict__ x,
                            const float* __restrict__ T, const float* __restrict__ minv, double weight,
                            bf16* __restrict__ dG) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n_lower) return;
  const int e = lower[r], i = rows[e];
  float row[64];
#pragma unroll
  for (int q = 0; q < 64; ++q) row[q] = 0.f;
  if (i != cols[e]) {
    const float* mi = minv + (size_t)i * 9;
    const float* t = T + (size_t)e * 9;
    const float* a = ahat + (size_t)e * 9;
    const float f = (float)(weight * 2.0 / (3.0 * n)) * coupling(x, i);
    float dh[9];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int c = 0; c < 3; ++c) dh[3 * p + c] = mi[3 * p] * t[c] + mi[3 * p + 1] * t[3 + c] + mi[3 * p + 2] * t[6 + c];
#pragma unroll
    for (int p = 0; p < 3; ++p)
#pragma unroll
      for (int c = 0; c < 3; ++c)
        row[3 * p + c] = f * (dh[3 * p] * a[3 * c] + dh[3 * p + 1] * a[3 * c + 1] + dh[3 * p + 2] * a[3 * c + 2]);
  }
  uint4* dst = reinterpret_cast<uint4*>(dG + (size_t)r * 64);
#pragma unroll
  for (int q = 0; q < 8; ++q) dst[q] = pack8(row + 8 * q);
}

// a_i = bf16(sum of the row's messages / deg): a warp per node, lanes = 4 edge
// slots x 8 column groups, so each step reads four contiguous 128-byte rows
__global__ void __launch_bounds__(256) k_mean_messages(int n, const int* __restrict__ off, const bf16* __restrict__ m,
                                                       bf16* __restrict__ a) {
  const int lane = threadIdx.x & 31, slot = lane >> 3, g = lane & 7;
  const int warps = (gridDim.x * blockDim.x) >> 5;
  for (int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int b = __ldg(off + i), e = __ldg(off + i + 1);
    float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll 4
    for (int k = b + slot; k < e; k += 4) {
      float f[8];
      unpack8(ld4(m + (size_t)k * W + g * 8), f);
#pragma unroll
      for (int t = 0; t < 8; ++t) acc[t] += f[t];
    }
#pragma unroll
    for (int t = 0; t < 8; ++t) {
      acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 8);
      acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], 16);
    }
    if (slot == 0) {
      const float deg = (float)(e - b);
#pragma unroll
      for (int t = 0; t < 8; ++t) acc[t] /= deg;
      *reinterpret_cast<uint4*>(a + (size_t)i * W + g * 8) = pack8(acc);
    }
  }
}

// ------------------------------------------------------------ backward helpers
__global__ void k_gather_rows(int R, const bf16* __restrict__ X, const int* __restrict__ idx, bf16* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // one 16-byte group
  if (t >= R * 8) return;
  const int r = t >> 3, g = t & 7;
  reinterpret_cast<uint4*>(out)[t] = ld4(X + (size_t)idx[r] * W + g * 8);
}

__global__ void k_edge_x(int nnz, const bf16* __restrict__ h, const bf16* __restrict__ e, const int* __restrict__ rows,
                         const int* __restrict__ cols, bf16* __restrict__ X) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // 24 groups per edge
  if (t >= nnz * 24) return;
  const int k = t / 24, g = t % 24;
  uint4 v;
  if (g < 8) v = ld4(h + (size_t)rows[k] * W + g * 8);
  else if (g < 16) v = ld4(h + (size_t)cols[k] * W + (g - 8) * 8);
  else v = ld4(e + (size_t)k * W + (g - 16) * 8);
  reinterpret_cast<uint4*>(X)[t] = v;
}

__global__ void k_node_x(int n, const bf16* __restrict__ h, const bf16* __restrict__ a, bf16* __restrict__ X) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;  // 16 groups per node
  if (t >= n * 16) return;
  const int i = t / 16, g = t % 16;
  reinterpret_cast<uint4*>(X)[t] = g < 8 ? ld4(h + (size_t)i * W + g * 8) : ld4(a + (size_t)i * W + (g - 8) * 8);
}

// out = bf16(d * (act > 0)) over rows x 64
__global__ void k_relu_grad(long long count, const float* __restrict__ d, const bf16* __restrict__ act,
                            bf16* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= count) return;
  out[t] = __float2bfloat16_rn(__bfloat162float(act[t]) > 0.f ? d[t] : 0.f);
}

// dm = de + da[row]; out = bf16(dm * (m > 0))
__global__ void k_edge_grad(int nnz, const float* __restrict__ de, const float* __restrict__ da,
                            const int* __restrict__ rows, const bf16* __restrict__ m, bf16* __restrict__ out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnz * W) return;
  const int e = (int)(t / W), c = (int)(t % W);
  const float dm = de[t] + da[(size_t)rows[e] * W + c];
  out[t] = __float2bfloat16_rn(__bfloat162float(m[t]) > 0.f ? dm : 0.f);
}

// dh += dXn[:, :64]; da = dXn[:, 64:] / deg
__global__ void k_node_post(int n, const int* __restrict__ off, const float* __restrict__ dXn, float* __restrict__ dh,
                            float* __restrict__ da) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * W) return;
  const int i = (int)(t / W), c = (int)(t % W);
  const float deg = (float)(off[i + 1] - off[i]);
  dh[t] += dXn[(size_t)i * 2 * W + c];
  da[t] = dXn[(size_t)i * 2 * W + W + c] / deg;
}

// de += dX[:, 128:192]
__global__ void k_edge_post_e(int nnz, const float* __restrict__ dX, float* __restrict__ de) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnz * W) return;
  const int e = (int)(t / W), c = (int)(t % W);
  de[t] += dX[(size_t)e * 3 * W + 2 * W + c];
}

// dh[i] += sum over row i of dX[e][0:64] + dX[rev e][64:128]
__global__ void k_edge_post_h(int n, const int* __restrict__ off, const int* __restrict__ rev,
                              const float* __restrict__ dX, float* __restrict__ dh) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * W) return;
  const int i = (int)(t / W), c = (int)(t % W);
  float s = 0.f;
  for (int e = off[i]; e < off[i + 1]; ++e) s += dX[(size_t)e * 3 * W + c] + dX[(size_t)rev[e] * 3 * W + W + c];
  dh[t] += s;
}

__global__ void k_scatter_rows(int R, const int* __restrict__ idx, const float* __restrict__ src,
                               float* __restrict__ dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)R * W) return;
  const int r = (int)(t / W), c = (int)(t % W);
  dst[(size_t)idx[r] * W + c] = src[t];
}

__global__ void k_adam(int n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// ------------------------------------------------------------ FSAI apply
template <class T>
__global__ void k_fsai_y(int n, const int* __restrict__ off, const int* __restrict__ diag, const int* __restrict__ cols,
                         const float* __restrict__ G, const float* __restrict__ scale, const T* __restrict__ r,
                         T* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  T acc[3] = {0, 0, 0};
  for (int e = off[i]; e <= diag[i]; ++e) {
    const int j = cols[e];
    const float* g = G + (size_t)e * 9;
    const T t0 = r[3 * j] * (T)scale[3 * j], t1 = r[3 * j + 1] * (T)scale[3 * j + 1],
            t2 = r[3 * j + 2] * (T)scale[3 * j + 2];
#pragma unroll
    for (int a = 0; a < 3; ++a) acc[a] += (T)g[3 * a] * t0 + (T)g[3 * a + 1] * t1 + (T)g[3 * a + 2] * t2;
  }
  y[3 * i] = acc[0];
  y[3 * i + 1] = acc[1];
  y[3 * i + 2] = acc[2];
}

template <class T>
__global__ void k_fsai_z(int n, const int* __restrict__ off, const int* __restrict__ diag, const int* __restrict__ cols,
                         const int* __restrict__ rev, const float* __restrict__ G, const float* __restrict__ scale,
                         const T* __restrict__ y, T* __restrict__ z) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  T acc[3] = {0, 0, 0};
  for (int e = diag[j]; e < off[j + 1]; ++e) {
    const int i = cols[e];  // i >= j: block (i, j) of G^ sits at rev[e]
    const float* g = G + (size_t)rev[e] * 9;
    const T y0 = y[3 * i], y1 = y[3 * i + 1], y2 = y[3 * i + 2];
#pragma unroll
    for (int b = 0; b < 3; ++b) acc[b] += (T)g[b] * y0 + (T)g[3 + b] * y1 + (T)g[6 + b] * y2;
  }
  z[3 * j] = acc[0] * (T)scale[3 * j];
  z[3 * j + 1] = acc[1] * (T)scale[3 * j + 1];
  z[3 * j + 2] = acc[2] * (T)scale[3 * j + 2];
}

inline int grid_for(long long n, int b = 256) { return (int)((n + b - 1) / b); }

struct Carve {
  uint8_t* p;
  size_t left;
  template <class T>
  T* take(size_t count) {
    const size_t bytes = (count * sizeof(T) + 255) & ~(size_t)255;
    if (bytes > left) return nullptr;
    T* r = reinterpret_cast<T*>(p);
    p += bytes;
    left -= bytes;
    return r;
  }
};

bool graph_ok(const ipcb_graph* g) {
  return g && g->n > 0 && g->nnz >= g->n && g->offsets && g->columns && g->rows && g->rev && g->diag && g->lower &&
         g->n_lower == (g->nnz + g->n) / 2;
}

}  // namespace

extern "C" {

int ipcb_mpnn_param_count(void) { return P_COUNT; }
int ipcb_mpnn_packed_count(void) { return K_COUNT; }

int ipcb_mpnn_pack(const float* params, void* packed, ipcb_stream s) {
  if (!params || !packed) {
    ipcb::set_error_msg("mpnn_pack: null pointer");
    return IPCB_E_ARG;
  }
  k_pack<<<grid_for(K_COUNT), 256, 0, (cudaStream_t)s>>>(params, (bf16*)packed);
  return ipcb::check_launch("ipcb_mpnn_pack");
}

size_t ipcb_mpnn_graph_workspace(int n) { return 2 * ((size_t)n * 4 + 256) + ipcb::scan::scratch_bytes(n); }

int ipcb_mpnn_graph(ipcb_graph* g, int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!graph_ok(g) || !status || !ws || ws_bytes < ipcb_mpnn_graph_workspace(g->n)) {
    ipcb::set_error_msg("mpnn_graph: bad arguments (n_lower must be (nnz + n) / 2)");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  Carve c{(uint8_t*)ws, ws_bytes};
  int* start = c.take<int>(g->n);
  void* sc = c.take<uint8_t>(ipcb::scan::scratch_bytes(g->n));
  k_graph_rows<<<grid_for(g->n), 256, 0, st>>>(g->n, g->offsets, g->columns, g->rows, g->rev, g->diag, start, status);
  ipcb::scan::exclusive(start, g->n, sc, (int*)nullptr, st);
  k_graph_lower<<<grid_for(g->n), 256, 0, st>>>(g->n, g->offsets, g->diag, start, g->lower);
  return ipcb::check_launch("ipcb_mpnn_graph");
}

int ipcb_mpnn_features(const ipcb_graph* g, int fp64, const void* values, float* scale, float* ahat, void* x,
                       void* y, int* status, ipcb_stream s) {
  if (!graph_ok(g) || !values || !scale || !ahat || !x || !y || !status) {
    ipcb::set_error_msg("mpnn_features: bad arguments");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  if (fp64) {
    k_scale<double><<<grid_for(g->n), 256, 0, st>>>(g->n, g->diag, (const double*)values, scale, status);
    k_edge_features<double><<<grid_for(g->nnz), 256, 0, st>>>(g->nnz, g->rows, g->columns, (const double*)values,
                                                              scale, ahat, (bf16*)y);
  } else {
    k_scale<float><<<grid_for(g->n), 256, 0, st>>>(g->n, g->diag, (const float*)values, scale, status);
    k_edge_features<float><<<grid_for(g->nnz), 256, 0, st>>>(g->nnz, g->rows, g->columns, (const float*)values,
                                                             scale, ahat, (bf16*)y);
  }
  k_node_features<<<grid_for(g->n), 256, 0, st>>>(g->n, g->offsets, g->columns, g->diag, ahat, (bf16*)x);
  return ipcb::check_launch("ipcb_mpnn_features");
}

int ipcb_mpnn_forward(const ipcb_graph* g, const void* packed, const float* params, const float* ahat, const void* x,
                      const void* y, ipcb_mpnn_tape* tape, float* H, int* status, ipcb_stream s) {
  if (!graph_ok(g) || !packed || !params || !ahat || !x || !y || !tape || !tape->h || !tape->e || !tape->m ||
      !tape->a || !tape->proj || !H || !status || (tape->training && !tape->u)) {
    ipcb::set_error_msg("mpnn_forward: bad arguments");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  const bf16* P = (const bf16*)packed;
  const int n = g->n, nnz = g->nnz;
  const bool tr = tape->training != 0;
  bf16* Hs = (bf16*)tape->h;
  bf16* Es = (bf16*)tape->e;
  auto hbuf = [&](int l) { return Hs + (size_t)(tr ? l : (l & 1)) * n * W; };
  auto ebuf = [&](int l) { return Es + (size_t)(tr ? l : (l & 1)) * nnz * W; };
  int rc;
  rc = launch_mlp<64, 1>(n, StageDense{(const bf16*)x, IN, IN}, EpiBiasRelu{params + P_BHIN, hbuf(0)},
                         P + K_ENC_H, status, st, "mpnn node encoder");
  if (rc) return rc;
  rc = launch_mlp<64, 1>(nnz, StageDense{(const bf16*)y, IN, IN}, EpiBiasRelu{params + P_BEIN, ebuf(0)},
                         P + K_ENC_E, status, st, "mpnn edge encoder");
  if (rc) return rc;
  for (int l = 0; l < LAYERS; ++l) {
    const float* pl = params + P_LAYER0 + l * P_LAYER;
    bf16* m = (bf16*)tape->m + (tr ? (size_t)l * nnz * W : 0);  // inference: one buffer
    bf16* a = tr ? (bf16*)tape->a + (size_t)l * n * W : nullptr;
    bf16* u = tr ? (bf16*)tape->u + (size_t)l * n * W : nullptr;
    // per-node projections of both message endpoints, then the edge product
    rc = launch_mlp<128, 1>(n, StageDense{hbuf(l), W, W}, EpiF32{tape->proj, 2 * W}, P + K_W1ABT + l * 2 * W * W,
                            status, st, "mpnn message projection");
    if (rc) return rc;
    rc = launch_mlp<64, 1>(nnz, StageDense{ebuf(l), W, W},
                           EpiEdge{pl + O_B1, tape->proj, ebuf(l + 1), m, g->rows, g->columns},
                           P + K_W1CT + l * W * W, status, st, "mpnn message");
    if (rc) return rc;
    bf16* am = tr ? a : (bf16*)tape->a;
    {
      const int need = (int)(((long long)n * 32 + 255) / 256);
      const int cap = 16 * sm_count();
      k_mean_messages<<<need < cap ? need : cap, 256, 0, st>>>(n, g->offsets, m, am);
    }
    rc = launch_mlp<64, 2>(n, StageNode{hbuf(l), am}, EpiNode{pl + O_B2, hbuf(l + 1), u},
                           P + K_W2T + l * W * 2 * W, status, st, "mpnn update");
    if (rc) return rc;
  }
  return launch_mlp<16, 1>(g->n_lower, StageGather{ebuf(LAYERS), g->lower},
                           EpiHead{params + P_BOFF, ahat, (const bf16*)x, g->lower, g->rows, g->columns, H},
                           P + K_HEADT, status, st, "mpnn head");
}

int ipcb_fsai_normalize(const ipcb_graph* g, const float* ahat, const float* H, float* T, float* minv, float* G,
                        double* acc, int* status, ipcb_stream s) {
  if (!graph_ok(g) || !ahat || !H || !T || !minv || !G || !acc || !status) {
    ipcb::set_error_msg("fsai_normalize: bad arguments");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  k_fsai_T<<<grid_for(g->n_lower), 256, 0, st>>>(g->n_lower, g->lower, g->rows, g->columns, g->offsets, g->diag, ahat,
                                                 H, T);
  k_fsai_rows<<<grid_for(g->n), 256, 0, st>>>(g->n, g->offsets, g->diag, H, T, minv, G, acc, status);
  return ipcb::check_launch("ipcb_fsai_normalize");
}

int ipcb_mpnn_loss_grad(const ipcb_graph* g, const float* ahat, const void* x, const float* T, const float* minv,
                        void* dG, double weight, ipcb_stream s) {
  if (!graph_ok(g) || !ahat || !x || !T || !minv || !dG) {
    ipcb::set_error_msg("mpnn_loss_grad: bad arguments");
    return IPCB_E_ARG;
  }
  k_fsai_dout<<<grid_for(g->n_lower), 256, 0, (cudaStream_t)s>>>(g->n_lower, g->n, g->lower, g->rows, g->columns,
                                                                  ahat, (const bf16*)x, T, minv, weight, (bf16*)dG);
  return ipcb::check_launch("ipcb_mpnn_loss_grad");
}

size_t ipcb_mpnn_backward_workspace(int n, int nnz, int n_lower) {
  const size_t big = (size_t)nnz * 3 * W > (size_t)n * 2 * W ? (size_t)nnz * 3 * W : (size_t)n * 2 * W;
  const size_t rowsmax = (size_t)(nnz > n ? nnz : n);
  size_t b = 0;
  auto add = [&](size_t bytes) { b += (bytes + 255) & ~(size_t)255; };
  add(sizeof(float) * n * W);                 // dh
  add(sizeof(float) * nnz * W);               // de
  add(sizeof(float) * n * W);                 // da
  add(sizeof(float) * (big > (size_t)n_lower * W ? big : (size_t)n_lower * W));  // dX
  add(sizeof(bf16) * (big > (size_t)n_lower * W ? big : (size_t)n_lower * W));   // X
  add(sizeof(bf16) * rowsmax * W);            // dY
  return b + 256;
}

int ipcb_mpnn_backward(const ipcb_graph* g, const void* packed, const float* params, const void* x, const void* y,
                       const ipcb_mpnn_tape* tape, const void* dG, float* grad, int* status, void* ws,
                       size_t ws_bytes, ipcb_stream s) {
  (void)params;
  if (!graph_ok(g) || !packed || !x || !y || !tape || !tape->training || !dG || !grad || !status || !ws ||
      ws_bytes < ipcb_mpnn_backward_workspace(g->n, g->nnz, g->n_lower)) {
    ipcb::set_error_msg("mpnn_backward: bad arguments");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  const bf16* P = (const bf16*)packed;
  const int n = g->n, nnz = g->nnz, L = g->n_lower;
  const size_t big = (size_t)nnz * 3 * W > (size_t)n * 2 * W ? (size_t)nnz * 3 * W : (size_t)n * 2 * W;
  const size_t bigl = big > (size_t)L * W ? big : (size_t)L * W;
  Carve c{(uint8_t*)ws, ws_bytes};
  float* dh = c.take<float>((size_t)n * W);
  float* de = c.take<float>((size_t)nnz * W);
  float* da = c.take<float>((size_t)n * W);
  float* dX = c.take<float>(bigl);
  bf16* X = c.take<bf16>(bigl);
  bf16* dY = c.take<bf16>((size_t)(nnz > n ? nnz : n) * W);
  const bf16* H = (const bf16*)tape->h;
  const bf16* E = (const bf16*)tape->e;
  const bf16* Mt = (const bf16*)tape->m;
  const bf16* At = (const bf16*)tape->a;
  const bf16* Ut = (const bf16*)tape->u;
  const bf16* dGb = (const bf16*)dG;
  int rc;
  // head
  k_gather_rows<<<grid_for((long long)L * 8), 256, 0, st>>>(L, E + (size_t)LAYERS * nnz * W, g->lower, X);
  rc = launch_wgrad<1, 16>(L, X, W, W, dGb, 64, EpiGradHead{grad + P_WOFF, grad + P_BOFF}, status, st,
                           "mpnn head wgrad");
  if (rc) return rc;
  rc = launch_mlp<64, 1>(L, StageDense{dGb, 64, 64}, EpiF32{dX, W}, P + K_HEAD, status, st, "mpnn head dx");
  if (rc) return rc;
  cudaMemsetAsync(de, 0, sizeof(float) * nnz * W, st);
  cudaMemsetAsync(dh, 0, sizeof(float) * n * W, st);
  k_scatter_rows<<<grid_for((long long)L * W), 256, 0, st>>>(L, g->lower, dX, de);
  for (int l = LAYERS - 1; l >= 0; --l) {
    const bf16* h = H + (size_t)l * n * W;
    const bf16* e = E + (size_t)l * nnz * W;
    const bf16* m = Mt + (size_t)l * nnz * W;
    const bf16* a = At + (size_t)l * n * W;
    const bf16* u = Ut + (size_t)l * n * W;
    float* gl = grad + P_LAYER0 + l * P_LAYER;
    // node update: h_out = h + relu([h, a] W2 + b2)
    k_relu_grad<<<grid_for((long long)n * W), 256, 0, st>>>((long long)n * W, dh, u, dY);
    k_node_x<<<grid_for((long long)n * 16), 256, 0, st>>>(n, h, a, X);
    rc = launch_wgrad<2, 64>(n, X, 2 * W, 2 * W, dY, W, EpiGrad{gl + O_W2, gl + O_B2, 2 * W, W}, status, st,
                             "mpnn update wgrad");
    if (rc) return rc;
    rc = launch_mlp<128, 1>(n, StageDense{dY, W, W}, EpiF32{dX, 2 * W}, P + K_W2 + l * 2 * W * W, status, st,
                            "mpnn update dx");
    if (rc) return rc;
    k_node_post<<<grid_for((long long)n * W), 256, 0, st>>>(n, g->offsets, dX, dh, da);
    // message: e_out = e + m, m = relu([h_i, h_j, e] W1 + b1), a = mean m
    k_edge_grad<<<grid_for((long long)nnz * W), 256, 0, st>>>(nnz, de, da, g->rows, m, dY);
    k_edge_x<<<grid_for((long long)nnz * 24), 256, 0, st>>>(nnz, h, e, g->rows, g->columns, X);
    rc = launch_wgrad<2, 64>(nnz, X, 3 * W, 3 * W, dY, W, EpiGrad{gl + O_W1, gl + O_B1, 3 * W, W}, status, st,
                             "mpnn message wgrad");
    if (rc) return rc;
    rc = launch_mlp<192, 1>(nnz, StageDense{dY, W, W}, EpiF32{dX, 3 * W}, P + K_W1 + l * 3 * W * W, status, st,
                            "mpnn message dx");
    if (rc) return rc;
    k_edge_post_e<<<grid_for((long long)nnz * W), 256, 0, st>>>(nnz, dX, de);
    k_edge_post_h<<<grid_for((long long)n * W), 256, 0, st>>>(n, g->offsets, g->rev, dX, dh);
  }
  // encoders
  k_relu_grad<<<grid_for((long long)n * W), 256, 0, st>>>((long long)n * W, dh, H, dY);
  rc = launch_wgrad<1, 64>(n, (const bf16*)x, IN, IN, dY, W, EpiGrad{grad + P_WHIN, grad + P_BHIN, IN, W}, status,
                           st, "mpnn node encoder wgrad");
  if (rc) return rc;
  k_relu_grad<<<grid_for((long long)nnz * W), 256, 0, st>>>((long long)nnz * W, de, E, dY);
  rc = launch_wgrad<1, 64>(nnz, (const bf16*)y, IN, IN, dY, W, EpiGrad{grad + P_WEIN, grad + P_BEIN, IN, W}, status,
                           st, "mpnn edge encoder wgrad");
  if (rc) return rc;
  return ipcb::check_launch("ipcb_mpnn_backward");
}

int ipcb_adam(int n, float* params, const float* grad, float* m, float* v, float lr, float beta1, float beta2,
              float eps, int t, ipcb_stream s) {
  if (n < 0 || !params || !grad || !m || !v || t < 1) {
    ipcb::set_error_msg("adam: bad arguments");
    return IPCB_E_ARG;
  }
  const float c1 = 1.f - powf(beta1, (float)t), c2 = 1.f - powf(beta2, (float)t);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)s>>>(n, params, grad, m, v, lr, beta1, beta2, eps, c1, c2);
  return ipcb::check_launch("ipcb_adam");
}

int ipcb_fsai_apply(const ipcb_graph* g, const float* G, const float* scale, int fp64, const void* r, void* tmp,
                    void* z, ipcb_stream s) {
  if (!graph_ok(g) || !G || !scale || !r || !tmp || !z) {
    ipcb::set_error_msg("fsai_apply: bad arguments");
    return IPCB_E_ARG;
  }
  cudaStream_t st = (cudaStream_t)s;
  if (fp64) {
    k_fsai_y<double><<<grid_for(g->n, 128), 128, 0, st>>>(g->n, g->offsets, g->diag, g->columns, G, scale,
                                                     (const double*)r, (double*)tmp);
    k_fsai_z<double><<<grid_for(g->n, 128), 128, 0, st>>>(g->n, g->offsets, g->diag, g->columns, g->rev, G, scale,
                                                     (const double*)tmp, (double*)z);
  } else {
    k_fsai_y<float><<<grid_for(g->n, 128), 128, 0, st>>>(g->n, g->offsets, g->diag, g->columns, G, scale, (const float*)r,
                                                    (float*)tmp);
    k_fsai_z<float><<<grid_for(g->n, 128), 128, 0, st>>>(g->n, g->offsets, g->diag, g->columns, g->rev, G, scale,
                                                    (const float*)tmp, (float*)z);
  }
  return ipcb::check_launch("ipcb_fsai_apply");
}

}  // extern "C"
