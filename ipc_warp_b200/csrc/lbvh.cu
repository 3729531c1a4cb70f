// LBVH build and refit (Karras 2012, "Maximizing parallelism in the
// construction of BVHs, octrees, and k-d trees") and the exported radix sort.
#include <cstdio>
#include <cstring>

#include "common.cuh"
#include "lbvh.cuh"
#include "sort.cuh"

namespace ipcb {

static thread_local char g_err[256] = "";
void set_error(const char* where, cudaError_t e) {
  snprintf(g_err, sizeof(g_err), "%s: %s", where, cudaGetErrorString(e));
}
void set_error_msg(const char* msg) { snprintf(g_err, sizeof(g_err), "%s", msg); }
static int arg_error(const char* msg) {
  set_error_msg(msg);
  return IPCB_E_ARG;
}
const char* last_error() { return g_err; }

int check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(where, e);
    return IPCB_E_CUDA;
  }
  return IPCB_OK;
}

namespace {

// 10-bit spread: b9..b0 -> b9 0 0 b8 0 0 ... b0
IPCB_D unsigned spread10(unsigned v) {
  v = (v * 0x00010001u) & 0xFF0000FFu;
  v = (v * 0x00000101u) & 0x0F00F00Fu;
  v = (v * 0x00000011u) & 0xC30C30C3u;
  v = (v * 0x00000005u) & 0x49249249u;
  return v;
}

__global__ void k_centre_bounds(const float* __restrict__ lo, const float* __restrict__ hi, int n,
                                unsigned* __restrict__ bounds) {
  float mn[3] = {3.4e38f, 3.4e38f, 3.4e38f}, mx[3] = {-3.4e38f, -3.4e38f, -3.4e38f};
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      float c = 0.5f * (lo[3 * i + k] + hi[3 * i + k]);
      mn[k] = fminf(mn[k], c);
      mx[k] = fmaxf(mx[k], c);
    }
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    for (int o = 16; o > 0; o >>= 1) {
      mn[k] = fminf(mn[k], __shfl_xor_sync(0xffffffffu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_xor_sync(0xffffffffu, mx[k], o));
    }
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      atomicMin(bounds + k, f2ord(mn[k]));
      atomicMax(bounds + 3 + k, f2ord(mx[k]));
    }
  }
}

__global__ void k_morton(const float* __restrict__ lo, const float* __restrict__ hi, int n,
                         const unsigned* __restrict__ bounds, unsigned* __restrict__ keys, int* __restrict__ vals) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned code = 0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float bmin = ord2f(bounds[k]), bmax = ord2f(bounds[3 + k]);
    float ext = bmax - bmin;
    float c = 0.5f * (lo[3 * i + k] + hi[3 * i + k]);
    float u = ext > 0.f ? (c - bmin) / ext : 0.5f;
    unsigned q = (unsigned)fminf(fmaxf(u * 1024.f, 0.f), 1023.f);
    code |= spread10(q) << (2 - k);
  }
  keys[i] = code;
  vals[i] = i;
}

// common-prefix length of sorted keys i and j, ties broken by index
IPCB_D int delta(const unsigned* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  unsigned a = k[i], b = k[j];
  if (a == b) return 32 + __clz((unsigned)(i ^ j));
  return __clz(a ^ b);
}

// Bit 31 of a parent entry: the parent's leaf range lies inside one 32-leaf
// block, i.e. inside one warp of the refit.
constexpr unsigned kLocalParent = 0x80000000u;

// One thread per internal node: range, split, child codes and parents (with
// the node's block-local bit).
__global__ void k_karras(const unsigned* __restrict__ keys, const int* __restrict__ sorted, int n,
                         float4* __restrict__ nodes, int* __restrict__ parent, int cap) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = delta(keys, n, i, i - d);
  int lmax = 2;
  while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
  int l = 0;
  for (int t = lmax >> 1; t >= 1; t >>= 1)
    if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
  int j = i + l * d;
  int dnode = delta(keys, n, i, j);
  int s = 0;
  for (int div = 2;; div <<= 1) {
    int t = (l + div - 1) / div;
    if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
    if (t <= 1) break;
  }
  int g = i + s * d + min(d, 0);
  int first = min(i, j), last = max(i, j);
  const unsigned loc = (first >> 5) == (last >> 5) ? kLocalParent : 0u;
  const int up0 = (int)(((unsigned)i << 1) | loc), up1 = (int)(((unsigned)i << 1) | 1u | loc);
  int lcode, rcode;
  if (first == g) {
    lcode = ~sorted[g];
    parent[cap + g] = up0;
  } else {
    lcode = g;
    parent[g] = up0;
  }
  if (last == g + 1) {
    rcode = ~sorted[g + 1];
    parent[cap + g + 1] = up1;
  } else {
    rcode = g + 1;
    parent[g + 1] = up1;
  }
  nodes[4 * i + 0].w = __int_as_float(lcode);
  nodes[4 * i + 2].w = __int_as_float(rcode);
}

// Bottom-up refit: a leaf writes its box into its parent's slot; the second
// child to arrive at a node merges both slots and continues upward.  The .w
// of a slot's hi entry carries the largest leaf rank (position in Morton
// order) below the slot: a node's is its right child's.
//
// The refit also writes the 4-wide view (see traverse4) on the way up: entries
// 2s and 2s + 1 of wide[node] belong to the node's side-s child -- the child's
// own slot and an empty entry when the child is a leaf, the child's two slots
// when it is internal.  The thread that writes its subtree's slot into `node`
// knows both (an internal subtree's two slots are the ones it merged one level
// below), so it writes that half of wide[node] with the slot: no loads and no
// separate gather pass over the nodes.
//
// Two phases.  A node whose leaves lie in one 32-leaf block (kLocalParent in
// the entries pointing to it) has both arrivals in the same warp (lane = leaf
// rank mod 32), and its index -- one end of its range -- is in the block: the
// warp meets there in rounds, each lane delivering its slot to shared memory,
// one __syncwarp, and the side-0 lane of a node with both slots carrying it
// up (no fence, no global atomic).  Above the blocks, the second of the two
// arrivals found by a global atomic counter continues, after a fence.
struct Slot {
  float4 lo, hi;
};

// entries 2 side and 2 side + 1 of the SoA wide node w
IPCB_D void put_wide_half(float4* __restrict__ w, int side, const Slot& a, const Slot& b) {
  float2* h = reinterpret_cast<float2*>(w) + side;
  h[0] = make_float2(a.lo.x, b.lo.x);
  h[2] = make_float2(a.lo.y, b.lo.y);
  h[4] = make_float2(a.lo.z, b.lo.z);
  h[6] = make_float2(a.hi.x, b.hi.x);
  h[8] = make_float2(a.hi.y, b.hi.y);
  h[10] = make_float2(a.hi.z, b.hi.z);
  h[12] = make_float2(a.lo.w, b.lo.w);
  h[14] = make_float2(a.hi.w, b.hi.w);
}

// 64-thread blocks: a warp whose lanes finish early frees its block slot
// without waiting for warps still climbing (1.49M leaves: 211 us against 233
// us with 8-warp blocks)
constexpr int kRefitWarps = 2;

__global__ void __launch_bounds__(32 * kRefitWarps) k_refit(const float* __restrict__ lo, const float* __restrict__ hi,
                                                            int n, const int* __restrict__ sorted,
                                                            const int* __restrict__ parent, int cap,
                                                            float4* __restrict__ nodes, unsigned* __restrict__ flags,
                                                            float4* __restrict__ wide) {
  __shared__ Slot sslot[kRefitWarps][32][2];  // per warp: block-local node x side
  __shared__ unsigned sarr[kRefitWarps][32];  // per warp: sides delivered to each block-local node
  const unsigned full = 0xffffffffu;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const Slot none{make_float4(3.4e38f, 3.4e38f, 3.4e38f, __int_as_float(-1)),
                  make_float4(-3.4e38f, -3.4e38f, -3.4e38f, __int_as_float(-1))};
  if (n == 1) {
    if (k != 0) return;
    const int prim = sorted[0];
    const Slot leaf{make_float4(lo[3 * prim], lo[3 * prim + 1], lo[3 * prim + 2], __int_as_float(~prim)),
                    make_float4(hi[3 * prim], hi[3 * prim + 1], hi[3 * prim + 2], __int_as_float(0))};
    const Slot second{make_float4(3.4e38f, 3.4e38f, 3.4e38f, __int_as_float(~prim)), none.hi};
    nodes[0] = leaf.lo;
    nodes[1] = leaf.hi;
    nodes[2] = second.lo;
    nodes[3] = second.hi;
    put_wide_half(wide, 0, leaf, none);
    put_wide_half(wide, 1, second, none);  // a leaf code with an empty box: never hit
    return;
  }
  sarr[w][lane] = 0u;
  const int base = k & ~31;  // first leaf of this warp's block
  bool carry = k < n;        // holds a subtree not yet delivered to its parent
  float3 bl = make_float3(0.f, 0.f, 0.f), bh = bl;
  int code = 0, par = 0, last = k;  // last: largest leaf rank below the carried subtree
  if (carry) {
    const int prim = sorted[k];
    bl = make_float3(lo[3 * prim], lo[3 * prim + 1], lo[3 * prim + 2]);
    bh = make_float3(hi[3 * prim], hi[3 * prim + 1], hi[3 * prim + 2]);
    code = ~prim;
    par = parent[cap + k];
  }
  Slot c0 = none, c1 = none;  // the carried subtree's two slots (side order) when it is internal
  __syncwarp();
  // phase 1: the block-local nodes, in rounds over the whole warp (a block's
  // subtree has depth < 32, so 32 rounds finish it; the bound also ends the
  // loop on a corrupted parent array)
  bool wait = false;  // delivered to a block-local node whose other side has not been seen
  int wnode = 0, wside = 0, wpar = 0;  // wpar: the node's own parent entry, loaded on delivery
  for (int round = 0; round < 40; ++round) {
    int li = 32;
    if (carry && ((unsigned)par & kLocalParent)) li = (int)((((unsigned)par & ~kLocalParent) >> 1)) - base;
    const bool deliver = (unsigned)li < 32u;
    if (!__any_sync(full, deliver || wait)) break;
    if (deliver) {
      const int node = base + li, side = par & 1;
      if (side == 0 && node != 0) wpar = parent[node];  // needed if this lane carries the node on
      const Slot own{make_float4(bl.x, bl.y, bl.z, __int_as_float(code)),
                     make_float4(bh.x, bh.y, bh.z, __int_as_float(last))};
      __stcg(nodes + 4 * node + 2 * side, own.lo);
      __stcg(nodes + 4 * node + 2 * side + 1, own.hi);
      if (code < 0) put_wide_half(wide + 8 * (size_t)node, side, own, none);
      else put_wide_half(wide + 8 * (size_t)node, side, c0, c1);
      sslot[w][li][side] = own;
      atomicOr(&sarr[w][li], 1u << side);
      carry = false;
      wait = true;
      wnode = node;
      wside = side;
    }
    __syncwarp();
    if (wait && sarr[w][wnode - base] == 3u) {
      wait = false;
      if (wside == 0) {  // both sides are in: the side-0 lane carries the node up
        const Slot own{make_float4(bl.x, bl.y, bl.z, __int_as_float(code)),
                       make_float4(bh.x, bh.y, bh.z, __int_as_float(last))};
        const Slot sib = sslot[w][wnode - base][1];
        c0 = own;
        c1 = sib;
        last = __float_as_int(sib.hi.w);
        bl = make_float3(fminf(bl.x, sib.lo.x), fminf(bl.y, sib.lo.y), fminf(bl.z, sib.lo.z));
        bh = make_float3(fmaxf(bh.x, sib.hi.x), fmaxf(bh.y, sib.hi.y), fmaxf(bh.z, sib.hi.z));
        code = wnode;
        if (wnode != 0) {
          par = wpar;
          carry = true;
        }
      }
    }
    __syncwarp();
  }
  if (!carry) return;
  // phase 2: the nodes above the blocks.  Depth is bounded by the 30 Morton
  // bits plus 32 index bits of the tie-break; the loop bound only guards
  // against a corrupted parent array.
  // Per level only the slot the sibling reads is fenced; the parent entry is
  // loaded and the wide half written outside the fence -> atomic -> sibling
  // chain, which is the latency the climb to the root pays per level.
  for (int level = 0; level < 128; ++level) {
    const int node = (int)(((unsigned)par & ~kLocalParent) >> 1), side = par & 1;
    const int next = node != 0 ? parent[node] : 0;
    const Slot own{make_float4(bl.x, bl.y, bl.z, __int_as_float(code)),
                   make_float4(bh.x, bh.y, bh.z, __int_as_float(last))};
    __stcg(nodes + 4 * node + 2 * side, own.lo);
    __stcg(nodes + 4 * node + 2 * side + 1, own.hi);
    __threadfence();
    const unsigned old = atomicAdd(flags + node, 1u);
    if (code < 0) put_wide_half(wide + 8 * (size_t)node, side, own, none);
    else put_wide_half(wide + 8 * (size_t)node, side, c0, c1);
    if (old == 0) return;
    flags[node] = 0;
    const Slot sib{__ldcg(nodes + 4 * node + 2 * (1 - side)), __ldcg(nodes + 4 * node + 2 * (1 - side) + 1)};
    c0 = side == 0 ? own : sib;
    c1 = side == 0 ? sib : own;
    if (side == 0) last = __float_as_int(sib.hi.w);
    bl = make_float3(fminf(bl.x, sib.lo.x), fminf(bl.y, sib.lo.y), fminf(bl.z, sib.lo.z));
    bh = make_float3(fmaxf(bh.x, sib.hi.x), fmaxf(bh.y, sib.hi.y), fmaxf(bh.z, sib.hi.z));
    if (node == 0) return;
    code = node;
    par = next;
  }
}

inline size_t al256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_version(void) { return 1; }
#ifndef IPCB_ABI_HASH
#define IPCB_ABI_HASH "unknown"
#endif
const char* ipcb_abi_hash(void) { return IPCB_ABI_HASH; }
const char* ipcb_last_error(void) { return ipcb::last_error(); }

size_t ipcb_sort_workspace_u32(int n) { return sort::workspace_bytes<unsigned>(n < 1 ? 1 : n); }
size_t ipcb_sort_workspace_u64(int n) { return sort::workspace_bytes<unsigned long long>(n < 1 ? 1 : n); }

int ipcb_sort_pairs_u32(unsigned* keys, int* vals, int n, int end_bit, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (n < 0 || end_bit < 0 || end_bit > 32) return IPCB_E_ARG;
  if (n <= 1) return IPCB_OK;
  if (!keys || !vals || !ws || ws_bytes < sort::workspace_bytes<unsigned>(n)) return IPCB_E_ARG;
  sort::sort_pairs<unsigned>(keys, vals, n, end_bit, ws, ws_bytes, (cudaStream_t)s);
  return check_launch("ipcb_sort_pairs_u32");
}

int ipcb_sort_pairs_u64(unsigned long long* keys, int* vals, int n, int end_bit, void* ws, size_t ws_bytes,
                        ipcb_stream s) {
  if (n < 0 || end_bit < 0 || end_bit > 64) return IPCB_E_ARG;
  if (n <= 1) return IPCB_OK;
  if (!keys || !vals || !ws || ws_bytes < sort::workspace_bytes<unsigned long long>(n)) return IPCB_E_ARG;
  sort::sort_pairs<unsigned long long>(keys, vals, n, end_bit, ws, ws_bytes, (cudaStream_t)s);
  return check_launch("ipcb_sort_pairs_u64");
}

size_t ipcb_lbvh_bytes(int capacity) {
  if (capacity < 1) capacity = 1;
  size_t c = (size_t)capacity;
  size_t nn = c > 1 ? c - 1 : 1;
  return al256(nn * 4 * 16) + al256(2 * c * 4) + al256(c * 4) + al256(c * 4) + al256(c * 4) + al256(nn * 8 * 16);
}

int ipcb_lbvh_bind(ipcb_lbvh* bvh, void* mem, int capacity) {
  if (!bvh || !mem || capacity < 1) return IPCB_E_ARG;
  size_t c = (size_t)capacity;
  size_t nn = c > 1 ? c - 1 : 1;
  char* p = (char*)mem;
  bvh->n = 0;
  bvh->capacity = capacity;
  bvh->nodes = p;
  p += al256(nn * 4 * 16);
  bvh->parent = (int*)p;
  p += al256(2 * c * 4);
  bvh->sorted = (int*)p;
  p += al256(c * 4);
  bvh->keys = (unsigned*)p;
  p += al256(c * 4);
  bvh->flags = (unsigned*)p;
  p += al256(c * 4);
  bvh->wide = p;
  return IPCB_OK;
}

size_t ipcb_lbvh_build_workspace(int n) { return 256 + sort::workspace_bytes<unsigned>(n < 1 ? 1 : n); }

int ipcb_lbvh_build(ipcb_lbvh* bvh, const float* lower, const float* upper, int n, void* ws, size_t ws_bytes,
                    ipcb_stream s) {
  if (!bvh) return arg_error("ipcb_lbvh_build: no hierarchy");
  if (n < 0) return arg_error("ipcb_lbvh_build: n is negative");
  if (n > bvh->capacity) return arg_error("ipcb_lbvh_build: n exceeds the hierarchy's capacity");
  cudaStream_t st = (cudaStream_t)s;
  if (n == 0) {
    bvh->n = 0;
    return IPCB_OK;
  }
  if (!lower || !upper) return arg_error("ipcb_lbvh_build: null box array");
  if (!ws || ws_bytes < ipcb_lbvh_build_workspace(n))
    return arg_error("ipcb_lbvh_build: workspace missing or smaller than ipcb_lbvh_build_workspace(n)");
  bvh->n = n;
  unsigned* bounds = (unsigned*)ws;
  void* sws = (char*)ws + 256;
  cudaMemsetAsync(bounds, 0xff, 3 * sizeof(unsigned), st);
  cudaMemsetAsync(bounds + 3, 0x00, 3 * sizeof(unsigned), st);
  cudaMemsetAsync(bvh->flags, 0, (size_t)n * sizeof(unsigned), st);
  int nb = min(div_up(n, 256), 148 * 8);
  k_centre_bounds<<<nb, 256, 0, st>>>(lower, upper, n, bounds);
  k_morton<<<div_up(n, 256), 256, 0, st>>>(lower, upper, n, bounds, bvh->keys, bvh->sorted);
  sort::sort_pairs<unsigned>(bvh->keys, bvh->sorted, n, 30, sws, ws_bytes - 256, st);
  if (n > 1)
    k_karras<<<div_up(n - 1, 256), 256, 0, st>>>(bvh->keys, bvh->sorted, n, (float4*)bvh->nodes, bvh->parent,
                                                  bvh->capacity);
  k_refit<<<div_up(n, 32 * kRefitWarps), 32 * kRefitWarps, 0, st>>>(lower, upper, n, bvh->sorted, bvh->parent, bvh->capacity,
                                           (float4*)bvh->nodes, bvh->flags, (float4*)bvh->wide);
  return check_launch("ipcb_lbvh_build");
}

int ipcb_lbvh_refit(const ipcb_lbvh* bvh, const float* lower, const float* upper, ipcb_stream s) {
  if (!bvh || bvh->n < 0) return IPCB_E_ARG;
  if (bvh->n == 0) return IPCB_OK;
  if (!lower || !upper) return IPCB_E_ARG;
  k_refit<<<div_up(bvh->n, 32 * kRefitWarps), 32 * kRefitWarps, 0, (cudaStream_t)s>>>(lower, upper, bvh->n, bvh->sorted, bvh->parent,
                                                            bvh->capacity, (float4*)bvh->nodes, bvh->flags,
                                                            (float4*)bvh->wide);
  return check_launch("ipcb_lbvh_refit");
}

}  // extern "C"
