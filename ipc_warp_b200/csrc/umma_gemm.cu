// Dense BF16 GEMM on the tcgen05 engine of umma.cuh: C[M x N] (fp32) =
// A[M x K] * B[N x K]^T with A, B row-major bf16.  It is the unit under test
// for the shared-memory layout, the descriptors and the TMEM epilogue that
// the message-passing kernels (mpnn.cu) are built from, and a plain GEMM for
// callers that need one.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "common.cuh"
#include "ipcb.h"
#include "umma.cuh"

namespace ipcb {
int check_launch(const char* where);
void set_error_msg(const char* msg);
}  // namespace ipcb

namespace {

constexpr int kThreads = 128;

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
  return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

template <int N, int C>
__global__ void __launch_bounds__(kThreads) k_gemm(int M, const __nv_bfloat16* __restrict__ A,
                                                   const __nv_bfloat16* __restrict__ B, float* __restrict__ Cout,
                                                   int* __restrict__ status) {
  extern __shared__ uint8_t dsmem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  constexpr int K = 64 * C;
  constexpr uint32_t kCols = umma::tmem_cols(N);
  uint8_t* sA = align1024(dsmem);
  uint8_t* sB = sA + C * 128 * 128;
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int idx = tid; idx < N * C * 8; idx += kThreads) {
    const int r = idx / (C * 8), c = (idx / 8) % C, g = idx % 8;
    const uint4 v = *reinterpret_cast<const uint4*>(B + (size_t)r * K + c * 64 + g * 8);
    *reinterpret_cast<uint4*>(sB + umma::sw128_group(r, c, g, N)) = v;
  }
  if (warp == 0) umma::tmem_alloc(&tslot, kCols);
  if (tid == 0) umma::mbar_init(&mbar, 1);
  umma::fence_async_smem();
  umma::fence_before();
  __syncthreads();
  umma::fence_after();
  const uint32_t tmem = tslot;
  uint32_t phase = 0;
  int ok = 1;
  const int ntiles = (M + 127) / 128;
  for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row = tile * 128 + tid;
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
      for (int g = 0; g < 8; ++g) {
        uint4 v = make_uint4(0, 0, 0, 0);
        if (row < M) v = *reinterpret_cast<const uint4*>(A + (size_t)row * K + c * 64 + g * 8);
        *reinterpret_cast<uint4*>(sA + umma::sw128_group(tid, c, g, 128)) = v;
      }
    umma::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      umma::fence_after();
      umma::issue_tile<N, C>(tmem, umma::smem_u32(sA), umma::smem_u32(sB), false, &mbar);
    }
    ok = __syncthreads_and(umma::mbar_wait(&mbar, phase) ? 1 : 0);
    phase ^= 1;
    if (!ok) break;
    umma::fence_after();
#pragma unroll
    for (int col = 0; col < N; col += 32) {
      float v[32];
      umma::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + col, v);
      if (row < M) {
        float4* out = reinterpret_cast<float4*>(Cout + (size_t)row * N + col);
        constexpr int kVec = (N < 32 ? N : 32) / 4;  // N = 16 uses half of the 32 loaded columns
#pragma unroll
        for (int i = 0; i < kVec; ++i) out[i] = make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3]);
      }
    }
    umma::fence_before();
    __syncthreads();
  }
  if (!ok) {
    if (tid == 0) atomicOr(status, IPCB_STATUS_TIMEOUT);
    umma::mbar_wait(&mbar, phase);  // bounded: let an MMA still in flight drain
  }
  __syncthreads();
  if (warp == 0) umma::tmem_dealloc(tmem, kCols);
}

template <int N, int C>
int launch(int M, const void* A, const void* B, void* Cout, int* status, cudaStream_t s) {
  const size_t smem = (size_t)C * 128 * 128 + (size_t)C * N * 128 + 1024;
  auto kern = k_gemm<N, C>;
  if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
  {
    ipcb::set_error_msg("umma_gemm: shared memory attribute");
    return IPCB_E_CUDA;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  // keep resident CTAs x TMEM columns within the 512 columns of an SM
  const int per_sm = (int)(512 / umma::tmem_cols(N));
  const int tiles = (M + 127) / 128;
  const int grid = tiles < sms * per_sm ? tiles : sms * per_sm;
  kern<<<grid, kThreads, smem, s>>>(M, (const __nv_bfloat16*)A, (const __nv_bfloat16*)B, (float*)Cout, status);
  return ipcb::check_launch("umma_gemm");
}

}  // namespace

extern "C" int ipcb_umma_gemm_bf16(int M, int N, int K, const void* A, const void* B, void* C, int* status,
                                   ipcb_stream s) {
  if (M < 0 || !A || !B || !C || !status) {
    ipcb::set_error_msg("umma_gemm: bad arguments");
    return IPCB_E_ARG;
  }
  if (M == 0) return 0;
  cudaStream_t st = (cudaStream_t)s;
#define IPCB_GEMM_CASE(NN, CC) \
  if (N == NN && K == 64 * CC) return launch<NN, CC>(M, A, B, C, status, st);
  IPCB_GEMM_CASE(16, 1) IPCB_GEMM_CASE(16, 2) IPCB_GEMM_CASE(16, 3) IPCB_GEMM_CASE(16, 4)
  IPCB_GEMM_CASE(64, 1) IPCB_GEMM_CASE(64, 2) IPCB_GEMM_CASE(64, 3) IPCB_GEMM_CASE(64, 4)
  IPCB_GEMM_CASE(128, 1) IPCB_GEMM_CASE(128, 2) IPCB_GEMM_CASE(128, 3) IPCB_GEMM_CASE(128, 4)
  IPCB_GEMM_CASE(192, 1) IPCB_GEMM_CASE(192, 2) IPCB_GEMM_CASE(192, 3)
  IPCB_GEMM_CASE(256, 1) IPCB_GEMM_CASE(256, 2) IPCB_GEMM_CASE(256, 3) IPCB_GEMM_CASE(256, 4)
#undef IPCB_GEMM_CASE
  ipcb::set_error_msg("umma_gemm: unsupported N/K (N in 16,64,128,192,256; K in 64..256 step 64)");
  return IPCB_E_ARG;
}
