// Stable LSD radix sort of (key, value) pairs, 8-bit digits.
//
// One pass = histogram per 2048-key tile -> device-wide exclusive scan of the
// digit-major [256][tiles] table -> stable scatter.  Inside a tile, ranks are
// found 256 keys at a time with __match_any_sync (lanes sharing a digit) and
// a per-warp shared-memory prefix, so equal digits keep input order.
// Workspace: alternate key/value buffers and the [256][tiles] table.
#pragma once
#include "common.cuh"
#include "scan.cuh"

namespace ipcb {
namespace sort {

constexpr int kThreads = 256;
constexpr int kRounds = 8;
constexpr int kTile = kThreads * kRounds;  // 2048 keys per block

inline int tiles(int n) { return div_up(n, kTile); }

template <class K>
inline size_t workspace_bytes(int n) {
  size_t a = ((size_t)n * sizeof(K) + 255) & ~(size_t)255;
  size_t b = ((size_t)n * sizeof(int) + 255) & ~(size_t)255;
  size_t c = ((size_t)256 * tiles(n > 0 ? n : 1) * sizeof(unsigned) + 255) & ~(size_t)255;
  return a + b + c + scan::scratch_bytes(256 * tiles(n > 0 ? n : 1));
}

template <class K>
__global__ void __launch_bounds__(kThreads) k_hist(const K* __restrict__ keys, int n, int shift, int nt,
                                                   unsigned* __restrict__ table) {
  __shared__ unsigned h[256];
  h[threadIdx.x] = 0;
  __syncthreads();
  int base = blockIdx.x * kTile;
#pragma unroll
  for (int r = 0; r < kRounds; ++r) {
    int i = base + r * kThreads + threadIdx.x;
    if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & 255u], 1u);
  }
  __syncthreads();
  table[threadIdx.x * nt + blockIdx.x] = h[threadIdx.x];
}

template <class K, class V>
__global__ void __launch_bounds__(kThreads) k_scatter(const K* __restrict__ kin, const V* __restrict__ vin,
                                                      K* __restrict__ kout, V* __restrict__ vout, int n, int shift,
                                                      int nt, const unsigned* __restrict__ table) {
  __shared__ unsigned s_base[256];
  __shared__ unsigned s_w[kThreads / 32][256];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  s_base[tid] = table[tid * nt + blockIdx.x];
#pragma unroll
  for (int w = 0; w < kThreads / 32; ++w) s_w[w][tid] = 0;
  __syncthreads();
  const unsigned lt = (1u << lane) - 1u;
  int base = blockIdx.x * kTile;
  for (int r = 0; r < kRounds; ++r) {
    int i = base + r * kThreads + tid;
    bool valid = i < n;
    K key = valid ? kin[i] : K(0);
    V val = valid ? vin[i] : V(0);
    unsigned d = valid ? ((unsigned)(key >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    unsigned rank = __popc(peers & lt);
    if (valid && rank == 0) s_w[warp][d] = __popc(peers);
    __syncthreads();
    unsigned run = s_base[tid];
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) {
      unsigned c = s_w[w][tid];
      s_w[w][tid] = run;
      run += c;
    }
    s_base[tid] = run;
    __syncthreads();
    if (valid) {
      unsigned pos = s_w[warp][d] + rank;
      kout[pos] = key;
      vout[pos] = val;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s_w[w][tid] = 0;
    __syncthreads();
  }
}

// Sorts keys/vals in place by bits [0, end_bit).  Returns a cudaError_t.
template <class K>
inline cudaError_t sort_pairs(K* keys, int* vals, int n, int end_bit, void* ws, size_t ws_bytes, cudaStream_t s) {
  if (n <= 1) return cudaSuccess;
  if (ws_bytes < workspace_bytes<K>(n)) return cudaErrorInvalidValue;
  char* p = (char*)ws;
  K* kalt = (K*)p;
  p += ((size_t)n * sizeof(K) + 255) & ~(size_t)255;
  int* valt = (int*)p;
  p += ((size_t)n * sizeof(int) + 255) & ~(size_t)255;
  unsigned* table = (unsigned*)p;
  int nt = tiles(n);
  p += ((size_t)256 * nt * sizeof(unsigned) + 255) & ~(size_t)255;
  void* scan_scratch = p;
  K* kin = keys;
  int* vin = vals;
  K* kout = kalt;
  int* vout = valt;
  int passes = (end_bit + 7) / 8;
  for (int ps = 0; ps < passes; ++ps) {
    int shift = ps * 8;
    k_hist<K><<<nt, kThreads, 0, s>>>(kin, n, shift, nt, table);
    scan::exclusive<unsigned>(table, 256 * nt, scan_scratch, nullptr, s);
    k_scatter<K, int><<<nt, kThreads, 0, s>>>(kin, vin, kout, vout, n, shift, nt, table);
    K* tk = kin; kin = kout; kout = tk;
    int* tv = vin; vin = vout; vout = tv;
  }
  if (kin != keys) {
    cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(K), cudaMemcpyDeviceToDevice, s);
    cudaMemcpyAsync(vals, vin, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, s);
  }
  return cudaGetLastError();
}

}  // namespace sort
}  // namespace ipcb
