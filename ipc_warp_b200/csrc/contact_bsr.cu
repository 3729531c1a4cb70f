// BSR assembly of the contact Hessian straight from the contact lists and
// their 16 triplet blocks per record (the result of
// bsr_from_triplets(rows, cols, vals) at dynamic_contacts.py:290-296, all-zero
// blocks dropped).  The generic assembly (bsr.cu) buckets all 16 triplets of
// a record by row; here the unit is a (record, slot ii) quad: one row
// (vertex ii of the record) and 4 consecutive blocks (columns = the record's 4
// vertices).  A row's distinct columns are few (tens), so:
//   1. key every quad by its row; stable radix sort (order = (row, quad id))
//   2. pass A, warp per row: insert the columns of the non-zero blocks (the
//      narrow phase's per-record block masks) into a shared-memory hash, sort
//      the distinct columns, count them
//   3. scan the counts -> offsets
//   4. pass B, warp per row: the row's blocks 32 at a time, sorted by column
//      within the warp and reduced by segments (shuffles), one shared-memory
//      add per column and batch; a fixed order, so deterministic
// A row with more than kHash distinct columns sets IPCB_STATUS_ROW_OVERFLOW
// (the host then uses the generic assembly).
#include "common.cuh"
#include "scan.cuh"
#include "sort.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr int kHash = 128;     // distinct columns per row handled by one warp
constexpr int kOwn = kHash / 32;
constexpr int kWarps = 4;

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

IPCB_D int4 record_ids(const int* __restrict__ ee, int n_ee, const int* __restrict__ pt, int p) {
  return p < n_ee ? __ldg(reinterpret_cast<const int4*>(ee) + p) : __ldg(reinterpret_cast<const int4*>(pt) + (p - n_ee));
}
IPCB_D int comp(int4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

__global__ void k_quad_keys(int nq, const int* __restrict__ ee, int n_ee, const int* __restrict__ pt,
                            unsigned* __restrict__ keys, int* __restrict__ ids, int* __restrict__ row_cnt) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nq) return;
  int4 v = record_ids(ee, n_ee, pt, q >> 2);
  int row = comp(v, q & 3);
  keys[q] = (unsigned)row;
  ids[q] = q;
  atomicAdd(row_cnt + row, 1);
}

// insert c into the warp's open-addressing table (keys -1 = empty)
IPCB_D bool hash_insert(int* tab, int c) {
  unsigned h = ((unsigned)c * 2654435761u) & (kHash - 1);
  for (int probe = 0; probe < kHash; ++probe) {
    int old = atomicCAS(tab + h, -1, c);
    if (old == -1 || old == c) return true;
    h = (h + 1) & (kHash - 1);
  }
  return false;
}

__global__ void __launch_bounds__(kWarps * 32) k_row_columns(int nrow, const int* __restrict__ qstart,
                                                             const int* __restrict__ qids, const int* __restrict__ ee,
                                                             int n_ee, const int* __restrict__ pt,
                                                             const unsigned short* __restrict__ bmask,
                                                             int* __restrict__ tmpcols, int* __restrict__ row_nnz,
                                                             int* __restrict__ status) {
  __shared__ int tab[kWarps][kHash];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = blockIdx.x * kWarps + w;
  if (row >= nrow) return;
  int b = qstart[row], e = qstart[row + 1];
  if (b == e) {
    if (lane == 0) row_nnz[row] = 0;
    return;
  }
  for (int k = lane; k < kHash; k += 32) tab[w][k] = -1;
  __syncwarp();
  bool ok = true;
  for (int i = b + lane; i < e; i += 32) {
    int q = qids[i];
    int4 v = record_ids(ee, n_ee, pt, q >> 2);
    unsigned m = (bmask[q >> 2] >> (4 * (q & 3))) & 0xFu;  // blocks (ii, jj = 0..3)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj)
      if ((m >> jj) & 1u) ok &= hash_insert(tab[w], comp(v, jj));
  }
  __syncwarp();
  // compact the occupied slots to the front (stable), pad with INT_MAX, then
  // bitonic-sort the first P >= cnt entries
  const unsigned lt = (1u << lane) - 1u;
  int dest[kOwn], colv[kOwn];
  int cnt = 0;
#pragma unroll
  for (int r = 0; r < kOwn; ++r) {
    int c = tab[w][r * 32 + lane];
    unsigned m = __ballot_sync(0xffffffffu, c >= 0);
    dest[r] = c >= 0 ? cnt + __popc(m & lt) : -1;
    colv[r] = c;
    cnt += __popc(m);
  }
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kOwn; ++r) tab[w][r * 32 + lane] = 0x7fffffff;
  __syncwarp();
#pragma unroll
  for (int r = 0; r < kOwn; ++r)
    if (dest[r] >= 0) tab[w][dest[r]] = colv[r];
  __syncwarp();
  int P = 1;
  while (P < cnt) P <<= 1;
  for (int sz = 2; sz <= P; sz <<= 1)
    for (int st = sz >> 1; st > 0; st >>= 1) {
      for (int i = lane; i < P; i += 32) {
        int l = i ^ st;
        if (l > i) {
          int a = tab[w][i], c = tab[w][l];
          bool up = (i & sz) == 0;
          if ((a > c) == up) {
            tab[w][i] = c;
            tab[w][l] = a;
          }
        }
      }
      __syncwarp();
    }
  int base4 = 4 * b;  // the row may use up to 4 columns per quad
  for (int k = lane; k < cnt; k += 32) tmpcols[base4 + k] = tab[w][k];
  unsigned bad = __ballot_sync(0xffffffffu, !ok);
  if (lane == 0) {
    row_nnz[row] = cnt;
    if (bad) atomicOr(status, IPCB_STATUS_ROW_OVERFLOW);
  }
}

// pass B, warp per row: the row's sorted columns and one 9-value
// accumulator per column in shared memory.  The lanes load the row's blocks
// 32 at a time (block i = quad i / 4, column slot jj = i % 4), each finds its
// column's position by binary search, the warp sorts the 32 (position, lane)
// keys (bitonic, shuffles), gathers the values in that order and forms the
// segment sums of equal positions (shuffle-down scan); the first lane of each
// segment adds its sum to the column's accumulator.  Every sum runs in a
// fixed order (batches in input order, within a batch by lane), so the result
// is deterministic, and each column takes one shared-memory add per batch.
template <class S>
__global__ void __launch_bounds__(kWarps * 32) k_row_values(int nrow, const int* __restrict__ qstart,
                                                            const int* __restrict__ qids, const int* __restrict__ ee,
                                                            int n_ee, const int* __restrict__ pt,
                                                            const unsigned short* __restrict__ bmask,
                                                            const S* __restrict__ vals,
                                                            const int* __restrict__ tmpcols,
                                                            const int* __restrict__ offsets, int* __restrict__ columns,
                                                            S* __restrict__ values) {
  __shared__ int scol[kWarps][kHash];
  __shared__ S sacc[kWarps][kHash * 9];
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int row = blockIdx.x * kWarps + w;
  if (row >= nrow) return;
  int b = qstart[row], e = qstart[row + 1];
  if (b == e) return;
  const int out = offsets[row], cnt = min(offsets[row + 1] - out, kHash);
  for (int k = lane; k < cnt; k += 32) {
    scol[w][k] = tmpcols[4 * b + k];
#pragma unroll
    for (int t = 0; t < 9; ++t) sacc[w][9 * k + t] = S(0);
  }
  __syncwarp();
  const int nb = 4 * (e - b);
  constexpr int kNone = kHash;  // sorts after every real position
  for (int base = 0; base < nb; base += 32) {
    const int i = base + lane;
    int pos = kNone;
    S v[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) v[t] = S(0);
    if (i < nb) {
      const int q = __ldg(qids + b + (i >> 2)), jj = i & 3;
      if ((__ldg(bmask + (q >> 2)) >> (4 * (q & 3) + jj)) & 1u) {
        const int c = comp(record_ids(ee, n_ee, pt, q >> 2), jj);
        int lo = 0, hi = cnt - 1;
        while (lo <= hi) {
          const int mid = (lo + hi) >> 1, x = scol[w][mid];
          if (x == c) {
            pos = mid;
            break;
          }
          if (x < c) lo = mid + 1;
          else hi = mid - 1;
        }
        if (pos != kNone) {  // absent only when the row overflowed (status set in pass A)
          const S* src = vals + 36LL * q + 9 * jj;
#pragma unroll
          for (int t = 0; t < 9; ++t) v[t] = __ldg(src + t);
        }
      }
    }
    // bitonic sort of (pos, lane) over the warp
    int key = (pos << 5) | lane;
#pragma unroll
    for (int size = 2; size <= 32; size <<= 1)
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
        const int other = __shfl_xor_sync(full, key, stride);
        const bool up = (lane & size) == 0, lower = (lane & stride) == 0;
        key = (lower == up) ? min(key, other) : max(key, other);
      }
    const int src_lane = key & 31, p = key >> 5;
    S sv[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) sv[t] = __shfl_sync(full, v[t], src_lane);
    // segment sums toward the first lane of each run of equal positions
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
      const int op = __shfl_down_sync(full, p, off);
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const S o = __shfl_down_sync(full, sv[t], off);
        if (lane + off < 32 && op == p) sv[t] += o;
      }
    }
    const int prev = __shfl_up_sync(full, p, 1);
    if (p != kNone && (lane == 0 || prev != p)) {
#pragma unroll
      for (int t = 0; t < 9; ++t) sacc[w][9 * p + t] += sv[t];
    }
    __syncwarp();
  }
  for (int k = lane; k < cnt; k += 32) {
    columns[out + k] = scol[w][k];
#pragma unroll
    for (int t = 0; t < 9; ++t) values[9LL * (out + k) + t] = sacc[w][9 * k + t];
  }
}

__global__ void k_total(int nrow, int* __restrict__ offsets, const int* __restrict__ total, int* __restrict__ nnz) {
  offsets[nrow] = *total;
  *nnz = *total;
}

template <class S>
int assemble(int n_ee, int n_pt, int nv, const int* ee, const int* pt, const S* vals, const unsigned short* bmask,
             int* offsets, int* columns, S* values, int* nnz, int* status, void* ws, cudaStream_t st) {
  int P = n_ee + n_pt, nq = 4 * P;
  size_t NQ = (size_t)nq, R = (size_t)nv + 1;
  char* p = (char*)ws;
  unsigned* keys = (unsigned*)p; p += al(NQ * 4);
  int* ids = (int*)p; p += al(NQ * 4);
  int* qstart = (int*)p; p += al(R * 4);
  int* tmpcols = (int*)p; p += al(NQ * 4 * 4);
  int* total = (int*)p; p += 256;
  void* scratch = p; p += scan::scratch_bytes((int)R);
  void* sws = p;
  cudaMemsetAsync(qstart, 0, R * sizeof(int), st);
  k_quad_keys<<<div_up(nq, 256), 256, 0, st>>>(nq, ee, n_ee, pt, keys, ids, qstart);
  int bits = 1;
  while ((1LL << bits) < (long long)nv) ++bits;
  sort::sort_pairs<unsigned>(keys, ids, nq, bits, sws, sort::workspace_bytes<unsigned>(nq), st);
  scan::exclusive<int>(qstart, (int)R, scratch, total, st);
  int g = div_up(nv, kWarps);
  k_row_columns<<<g, kWarps * 32, 0, st>>>(nv, qstart, ids, ee, n_ee, pt, bmask, tmpcols, offsets, status);
  scan::exclusive<int>(offsets, nv, scratch, total, st);
  k_total<<<1, 1, 0, st>>>(nv, offsets, total, nnz);
  k_row_values<S><<<g, kWarps * 32, 0, st>>>(nv, qstart, ids, ee, n_ee, pt, bmask, vals, tmpcols, offsets, columns,
                                             values);
  return check_launch("ipcb_contact_bsr");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

size_t ipcb_contact_bsr_workspace(int n_records, int n_verts) {
  size_t NQ = 4 * (size_t)(n_records > 0 ? n_records : 1), R = (size_t)(n_verts > 0 ? n_verts : 0) + 1;
  return al(NQ * 4) * 2 + al(R * 4) + al(NQ * 16) + 256 + scan::scratch_bytes((int)R) +
         sort::workspace_bytes<unsigned>((int)NQ);
}

int ipcb_contact_bsr(const ipcb_contacts* ee, int n_ee, const ipcb_contacts* pt, int n_pt, int n_verts,
                     const void* vals, const unsigned short* block_mask, int fp64, int* offsets, int* columns,
                     void* values, int* nnz, int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!ee || !pt || n_ee < 0 || n_pt < 0 || n_verts < 0 || !offsets || !nnz || !status) return IPCB_E_ARG;
  if (n_ee > ee->capacity || n_pt > pt->capacity || (long long)4 * (n_ee + n_pt) > 0x7fffffff) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (n_ee + n_pt == 0 || n_verts == 0) {
    cudaMemsetAsync(offsets, 0, (size_t)(n_verts + 1) * sizeof(int), st);
    cudaMemsetAsync(nnz, 0, sizeof(int), st);
    return check_launch("ipcb_contact_bsr");
  }
  if (!vals || !block_mask || !columns || !values || !ws ||
      ws_bytes < ipcb_contact_bsr_workspace(n_ee + n_pt, n_verts))
    return IPCB_E_ARG;
  if (fp64)
    return assemble<double>(n_ee, n_pt, n_verts, ee->a1a2b1b2, pt->a1a2b1b2, (const double*)vals, block_mask,
                            offsets, columns, (double*)values, nnz, status, ws, st);
  return assemble<float>(n_ee, n_pt, n_verts, ee->a1a2b1b2, pt->a1a2b1b2, (const float*)vals, block_mask, offsets,
                         columns, (float*)values, nnz, status, ws, st);
}

}  // extern "C"
