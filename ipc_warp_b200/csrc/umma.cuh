// 5th-generation tensor-core (tcgen05 / UMMA) building blocks for sm_100a:
// BF16 x BF16 -> FP32 products with both operands K-major in shared memory
// (128-byte swizzle) and the accumulator in tensor memory (TMEM).
//
// Operand tile layout in shared memory ("SW128 K-major"): a tile of R rows
// and K = 64 * C columns is stored as C chunks of R x 64 bf16; chunk c starts
// at c * R * 128 bytes (1024-byte aligned), row r of a chunk at r * 128 bytes,
// and the 16-byte group g (elements 8g..8g+7) of a row is stored at group
// position g ^ (r & 7).  A matrix descriptor then has SBO = 1024 bytes (eight
// 128-byte rows), LBO unused (1), layout SWIZZLE_128B and version 1; the K
// steps of 16 elements inside a chunk advance the start address by 32 bytes.
//
// One UMMA computes D[128 x N] (+)= A[128 x 16] * B[N x 16]^T; the
// accumulator row m lives in TMEM lane m, column n in TMEM column base + n.
#pragma once
#include <cstdint>

namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) in an SW128 K-major tile of R rows
__host__ __device__ __forceinline__ uint32_t sw128_offset(int r, int k, int R) {
  const int c = k >> 6, kk = k & 63;
  return (uint32_t)(c * R * 128 + r * 128 + ((((kk >> 3) ^ (r & 7)) & 7) << 4) + ((kk & 7) << 1));
}

// byte offset of the 16-byte group g (elements 8g..8g+7 of the 64-wide chunk
// c) of row r
__host__ __device__ __forceinline__ uint32_t sw128_group(int r, int c, int g, int R) {
  return (uint32_t)(c * R * 128 + r * 128 + (((g ^ (r & 7)) & 7) << 4));
}

__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);  // start address
  d |= (uint64_t)1u << 16;                           // LBO (unused when swizzled K-major)
  d |= (uint64_t)(1024u >> 4) << 32;                 // SBO: 8 rows x 128 B
  d |= (uint64_t)1u << 46;                           // descriptor version (sm_100)
  d |= (uint64_t)2u << 61;                           // SWIZZLE_128B
  return d;
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 D, both K-major, M=128
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int N) {
  return (1u << 4)                       // D format F32
         | (1u << 7)                     // A format BF16
         | (1u << 10)                    // B format BF16
         | ((uint32_t)(N >> 3) << 17)    // N / 8
         | ((uint32_t)(128 >> 4) << 24); // M / 16
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Wait for phase `parity` of the barrier; gives up after `max_polls` polls
// (each poll may suspend the thread for a hardware-defined interval).
// Returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_polls = 1u << 22) {
  const uint32_t a = smem_u32(mbar);
  for (uint32_t i = 0; i < max_polls; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_arrive(uint64_t* mbar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(mbar)) : "memory");
}

// barrier among `count` threads (a multiple of 32) under hardware barrier id
__device__ __forceinline__ void named_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// TMEM allocation by one full warp; the base address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
               : "memory");
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 accumulator columns of this thread's TMEM lane
// (warp w of the CTA reads lanes 32 (w % 4) .. + 31).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
      "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// D[128 x N] (+)= A[128 x 64C] * B[N x 64C]^T from SW128 K-major tiles at
// shared addresses a_base (128 rows) and b_base (N rows).  Issued by one
// thread; the caller commits to an mbarrier afterwards.
template <int N, int C>
__device__ __forceinline__ void issue(uint32_t tmem_d, uint32_t a_base, uint32_t b_base, bool accumulate) {
  constexpr uint32_t idesc = idesc_bf16_f32(N);
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const uint64_t a = desc_sw128(a_base + c * 128 * 128 + s * 32);
      const uint64_t b = desc_sw128(b_base + c * N * 128 + s * 32);
      mma_bf16(tmem_d, a, b, idesc, (accumulate || c > 0 || s > 0) ? 1u : 0u);
    }
}

template <int N, int C>
__device__ __forceinline__ void issue_tile(uint32_t tmem_d, uint32_t a_base, uint32_t b_base, bool accumulate,
                                           uint64_t* mbar) {
  issue<N, C>(tmem_d, a_base, b_base, accumulate);
  commit(mbar);
}

// TMEM columns to allocate for n accumulator columns (a power of two >= 32,
// at most the 512 columns of an SM)
__host__ __device__ constexpr uint32_t tmem_cols(int n) {
  return n <= 32 ? 32 : n <= 64 ? 64 : n <= 128 ? 128 : n <= 256 ? 256 : 512;
}

}  // namespace umma
