// Device-wide exclusive prefix sum of int32/uint32 in three launches:
// block-local scan -> scan of the block totals (one block, looping) -> add.
#pragma once
#include "common.cuh"

namespace ipcb {
namespace scan {

constexpr int kBlock = 1024;

inline int blocks(int n) { return div_up(n > 0 ? n : 1, kBlock); }
// bytes of scratch for n elements (block totals + the total)
inline size_t scratch_bytes(int n) { return (((size_t)blocks(n) + 1) * 4 + 255 + 256) & ~(size_t)255; }

template <class T>
IPCB_D T warp_inclusive(T x, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    T y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  return x;
}

// returns the exclusive prefix of v within the block; *block_total set by every thread
template <class T>
IPCB_D T block_exclusive(T v, T* s_warp, T& block_total) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T x = warp_inclusive(v, lane);
  if (lane == 31) s_warp[w] = x;
  __syncthreads();
  if (w == 0) {
    T y = lane < (int)(blockDim.x >> 5) ? s_warp[lane] : T(0);
    y = warp_inclusive(y, lane);
    s_warp[lane] = y;
  }
  __syncthreads();
  block_total = s_warp[(blockDim.x >> 5) - 1];
  T r = x - v + (w > 0 ? s_warp[w - 1] : T(0));
  __syncthreads();
  return r;
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_local(int n, T* __restrict__ a, T* __restrict__ sums) {
  __shared__ T s[32];
  int t = blockIdx.x * kBlock + threadIdx.x;
  T v = t < n ? a[t] : T(0);
  T tot;
  T e = block_exclusive(v, s, tot);
  if (t < n) a[t] = e;
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

template <class T>
__global__ void __launch_bounds__(kBlock) k_sums(int nb, T* __restrict__ sums, T* __restrict__ total) {
  __shared__ T s[32];
  T carry = T(0);
  for (int base = 0; base < nb; base += kBlock) {
    int t = base + threadIdx.x;
    T v = t < nb ? sums[t] : T(0);
    T tot;
    T e = block_exclusive(v, s, tot);
    if (t < nb) sums[t] = e + carry;
    carry += tot;
  }
  if (threadIdx.x == 0 && total) *total = carry;
}

template <class T>
__global__ void k_add(int n, T* __restrict__ a, const T* __restrict__ sums) {
  int t = blockIdx.x * kBlock + threadIdx.x;
  if (t < n) a[t] += sums[blockIdx.x];
}

// exclusive scan of a[0..n) in place; *total (device, may be null) = sum.
// scratch: scratch_bytes(n) bytes.
template <class T>
inline void exclusive(T* a, int n, void* scratch, T* total, cudaStream_t st) {
  if (n <= 0) return;
  int nb = blocks(n);
  T* sums = (T*)scratch;
  k_local<T><<<nb, kBlock, 0, st>>>(n, a, sums);
  k_sums<T><<<1, kBlock, 0, st>>>(nb, sums, total);
  k_add<T><<<nb, kBlock, 0, st>>>(n, a, sums);
}

}  // namespace scan
}  // namespace ipcb
