// BSR assembly of the contact Hessian straight from the contact lists and
// their 16 triplet blocks per record (the result of
// bsr_from_triplets(rows, cols, vals) at dynamic_contacts.py:290-296, all-zero
// blocks dropped).  The generic assembly (bsr.cu) buckets all 16 triplets of
// a record by row; here the unit is a (record, slot ii) quad: one row
// (vertex ii of the record) and 4 consecutive blocks (columns = the record's 4
// vertices).  A row's distinct columns are few (tens), so:
//   1. thread per record: count the quads of each row and take each quad's
//      arrival slot in its row (atomics; a row's first arrival also appends
//      the row to the list of touched rows); scan the counts; scatter the
//      quad ids to their rows (arrival order)
//   2. pass A, warp per row: sort the row's quad ids (so the order, and every
//      sum below, is the same on every run), insert the columns of the
//      non-zero blocks (the narrow phase's per-record block masks) into a
//      shared-memory hash, sort the distinct columns, count them, and store
//      each quad's 4 column positions (one byte each)
//   3. scan the counts -> offsets
//   4. pass B, warp per row: the row's blocks 32 at a time, grouped by column
//      position within the warp and summed per group (shuffles), one
//      shared-memory add per column and batch; a fixed order, so deterministic
// Passes A and B run persistent warps that take the touched rows from a
// counter: most vertices of a large scene have no contact, and a launch over
// all rows would spend most of its blocks on empty ones.
// A row with more than kHash distinct columns sets IPCB_STATUS_ROW_OVERFLOW
// (the host then uses the generic assembly).
#include "common.cuh"
#include "scan.cuh"

#include <algorithm>

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr int kHash = 128;        // distinct columns per row handled by one warp
constexpr int kSmemQuads = 256;   // quads per row sorted in shared memory (longer rows: in global scratch)
constexpr unsigned kAbsent = 0xffu;  // column position of a zero block
constexpr int kOwn = kHash / 32;
constexpr int kWarps = 4;

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

IPCB_D int4 record_ids(const int* __restrict__ ee, int n_ee, const int* __restrict__ pt, int p) {
  return p < n_ee ? __ldg(reinterpret_cast<const int4*>(ee) + p) : __ldg(reinterpret_cast<const int4*>(pt) + (p - n_ee));
}
IPCB_D int comp(int4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : (k == 2 ? v.z : v.w)); }

// nrec = {EE records, PT records}: host values, or min(*cnt, capacity) of
// the lists read on the device (graph-capturable; no host read of the counts)
// nrec[2]: touched rows; nrec[3], nrec[4]: the work counters of passes A, B
__global__ void k_counts(const int* __restrict__ ee_cnt, int ee_n, const int* __restrict__ pt_cnt, int pt_n,
                         int* __restrict__ nrec) {
  nrec[0] = ee_cnt ? min(max(*ee_cnt, 0), ee_n) : ee_n;
  nrec[1] = pt_cnt ? min(max(*pt_cnt, 0), pt_n) : pt_n;
  nrec[2] = nrec[3] = nrec[4] = 0;
}

IPCB_D int arrive(int* __restrict__ row_cnt, int row, int* __restrict__ rows, int* __restrict__ nrows) {
  const int s = atomicAdd(row_cnt + row, 1);
  if (s == 0) rows[atomicAdd(nrows, 1)] = row;
  return s;
}

__global__ void k_rec_slots(int* __restrict__ nrec, const int* __restrict__ ee, const int* __restrict__ pt,
                            int4* __restrict__ slots, int* __restrict__ row_cnt, int* __restrict__ rows) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x, n_ee = nrec[0];
  if (p >= n_ee + nrec[1]) return;
  const int4 v = record_ids(ee, n_ee, pt, p);
  int4 s;
  s.x = arrive(row_cnt, v.x, rows, nrec + 2);
  s.y = arrive(row_cnt, v.y, rows, nrec + 2);
  s.z = arrive(row_cnt, v.z, rows, nrec + 2);
  s.w = arrive(row_cnt, v.w, rows, nrec + 2);
  slots[p] = s;
}

// the next touched row for this warp (one counter bump per row), -1 when done
IPCB_D int next_row(int* __restrict__ work, const int* __restrict__ rows, int nrows, int lane) {
  int r = 0;
  if (lane == 0) r = atomicAdd(work, 1);
  r = __shfl_sync(0xffffffffu, r, 0);
  return r < nrows ? __ldg(rows + r) : -1;
}

__global__ void k_rec_scatter(const int* __restrict__ nrec, const int* __restrict__ ee, const int* __restrict__ pt,
                              const int4* __restrict__ slots, const int* __restrict__ qstart, int* __restrict__ qids) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x, n_ee = nrec[0];
  if (p >= n_ee + nrec[1]) return;
  const int4 v = record_ids(ee, n_ee, pt, p), s = slots[p];
  qids[qstart[v.x] + s.x] = 4 * p;
  qids[qstart[v.y] + s.y] = 4 * p + 1;
  qids[qstart[v.z] + s.z] = 4 * p + 2;
  qids[qstart[v.w] + s.w] = 4 * p + 3;
}

// ascending bitonic sort of a[0, n) in one warp's shared memory, n a power of two
IPCB_D void warp_sort(int* a, int n, int lane) {
  for (int sz = 2; sz <= n; sz <<= 1)
    for (int st = sz >> 1; st > 0; st >>= 1) {
      for (int i = lane; i < n; i += 32) {
        const int l = i ^ st;
        if (l > i) {
          const int x = a[i], y = a[l];
          if ((x > y) == ((i & sz) == 0)) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncwarp();
    }
}

// ascending bitonic sort of 32 E values held E per lane (element e * 32 +
// lane in v[e]): strides below 32 exchange through shuffles, larger ones
// between a lane's own registers
template <int E>
IPCB_D void reg_sort(int (&v)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int sz = 2; sz <= N; sz <<= 1)
#pragma unroll
    for (int st = sz >> 1; st > 0; st >>= 1) {
      if (st >= 32) {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int f = e ^ (st >> 5);
          if (f > e) {
            const bool asc = ((e * 32 + lane) & sz) == 0;
            const int a = v[e], c = v[f];
            if (asc ? (a > c) : (a < c)) {
              v[e] = c;
              v[f] = a;
            }
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; ++e) {
          const int other = __shfl_xor_sync(0xffffffffu, v[e], st);
          const bool asc = ((e * 32 + lane) & sz) == 0, lower = (lane & st) == 0;
          v[e] = (lower == asc) ? min(v[e], other) : max(v[e], other);
        }
      }
    }
}

// sort the n (<= 32 E) ints at src (INT_MAX past n) in registers; the sorted
// values go to dst[0, 32 E) (shared memory) and, the first n, back to src
template <int E>
IPCB_D void sort_to(int* src, int n, int* dst, int lane) {
  int v[E];
#pragma unroll
  for (int e = 0; e < E; ++e) v[e] = e * 32 + lane < n ? src[e * 32 + lane] : 0x7fffffff;
  reg_sort<E>(v, lane);
#pragma unroll
  for (int e = 0; e < E; ++e) {
    dst[e * 32 + lane] = v[e];
    if (src != dst && e * 32 + lane < n) src[e * 32 + lane] = v[e];
  }
}

// insert c into the warp's open-addressing table (keys -1 = empty); returns
// the slot, or -1 when the table is full
IPCB_D int hash_insert(int* tab, int c) {
  unsigned h = ((unsigned)c * 2654435761u) & (kHash - 1);
  for (int probe = 0; probe < kHash; ++probe) {
    int old = atomicCAS(tab + h, -1, c);
    if (old == -1 || old == c) return (int)h;
    h = (h + 1) & (kHash - 1);
  }
  return -1;
}

IPCB_D int hash_find(const int* tab, int c) {
  unsigned h = ((unsigned)c * 2654435761u) & (kHash - 1);
  for (int probe = 0; probe < kHash; ++probe) {
    const int k = tab[h];
    if (k == c) return (int)h;
    if (k == -1) return -1;
    h = (h + 1) & (kHash - 1);
  }
  return -1;
}

IPCB_D unsigned quad_mask(const unsigned short* __restrict__ bmask, int q) {
  return (__ldg(bmask + (q >> 2)) >> (4 * (q & 3))) & 0xFu;  // blocks (ii = q & 3, jj = 0..3)
}

// pass A, warp per row.  The row's quad ids are sorted in shared memory (rows
// of more than kSmemQuads quads: in their own tmpcols range past the kHash
// column entries, 4 ints per quad reserved there), the distinct columns of
// the non-zero blocks go through a shared-memory hash, are compacted and
// sorted, and every quad gets its 4 column positions through a slot ->
// position table.
__global__ void __launch_bounds__(kWarps * 32, 12)
    k_row_columns(const int* __restrict__ rows, const int* __restrict__ qstart, int* __restrict__ qids,
                  const int* __restrict__ ee, int* __restrict__ nrec, const int* __restrict__ pt,
                  const unsigned short* __restrict__ bmask, int* __restrict__ tmpcols, unsigned* __restrict__ qpos,
                  int* __restrict__ row_nnz, int* __restrict__ status) {
  __shared__ int sq[kWarps][kSmemQuads];
  __shared__ int tab[kWarps][kHash];
  __shared__ int scol[kWarps][kHash];
  __shared__ unsigned char slot_pos[kWarps][kHash];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_ee = nrec[0], nrows = nrec[2];
  for (int row = next_row(nrec + 3, rows, nrows, lane); row >= 0; row = next_row(nrec + 3, rows, nrows, lane)) {
  __syncwarp();  // the previous row's shared-memory reads are done
  const int b = qstart[row], n = qstart[row + 1] - b;
  // the row's quads in quad-id order
  int nq2 = 32;
  while (nq2 < n) nq2 <<= 1;
  int* buf = n <= kSmemQuads ? sq[w] : tmpcols + 4LL * b + kHash;  // nq2 <= 2n <= 4n - kHash there
  for (int k = lane; k < kHash; k += 32) {
    tab[w][k] = -1;
    scol[w][k] = 0x7fffffff;
  }
  if (nq2 == 32) sort_to<1>(qids + b, n, buf, lane);
  else if (nq2 == 64) sort_to<2>(qids + b, n, buf, lane);
  else if (nq2 == 128) sort_to<4>(qids + b, n, buf, lane);
  else if (nq2 == 256) sort_to<8>(qids + b, n, buf, lane);
  else {
    for (int k = lane; k < nq2; k += 32) buf[k] = k < n ? qids[b + k] : 0x7fffffff;
    __syncwarp();
    warp_sort(buf, nq2, lane);
    for (int k = lane; k < n; k += 32) qids[b + k] = buf[k];
  }
  __syncwarp();
  // distinct columns, 32 quads at a time: lanes holding the same column
  // (__match_any_sync) let the lowest of them insert it and share its slot;
  // the first quad of each lane keeps its 4 slots
  bool ok = true;
  int slot0[4] = {-1, -1, -1, -1};
  for (int base = 0; base < n; base += 32) {
    const int k = base + lane;
    int4 v = make_int4(0, 0, 0, 0);
    unsigned m = 0;
    if (k < n) {
      const int q = buf[k];
      v = record_ids(ee, n_ee, pt, q >> 2);
      m = quad_mask(bmask, q);
    }
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const bool has = (m >> jj) & 1u;
      const int c = has ? comp(v, jj) : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, c);
      const int leader = __ffs(peers) - 1;
      int h = -1;
      if (has && lane == leader) h = hash_insert(tab[w], c);
      h = __shfl_sync(0xffffffffu, h, leader);
      if (has) {
        ok &= h >= 0;
        if (base == 0) slot0[jj] = h;
      }
    }
  }
  __syncwarp();
  // compact the occupied slots (stable) and sort them
  const unsigned lt = (1u << lane) - 1u;
  int cnt = 0;
#pragma unroll
  for (int r = 0; r < kOwn; ++r) {
    const int c = tab[w][r * 32 + lane];
    const unsigned m = __ballot_sync(0xffffffffu, c >= 0);
    if (c >= 0) scol[w][cnt + __popc(m & lt)] = c;
    cnt += __popc(m);
  }
  __syncwarp();
  if (cnt <= 32) sort_to<1>(scol[w], 32, scol[w], lane);
  else if (cnt <= 64) sort_to<2>(scol[w], 64, scol[w], lane);
  else sort_to<4>(scol[w], 128, scol[w], lane);
  __syncwarp();
  for (int k = lane; k < cnt; k += 32) slot_pos[w][hash_find(tab[w], scol[w][k])] = (unsigned char)k;
  __syncwarp();
  // each quad's 4 column positions (kAbsent for a zero block, or for a column
  // lost to a full table)
  for (int k = lane; k < n; k += 32) {
    unsigned packed = 0;
    if (k == lane) {
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) packed |= (slot0[jj] >= 0 ? (unsigned)slot_pos[w][slot0[jj]] : kAbsent) << (8 * jj);
    } else {
      const int q = buf[k];
      const int4 v = record_ids(ee, n_ee, pt, q >> 2);
      const unsigned m = quad_mask(bmask, q);
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) {
        const int h = (m >> jj) & 1u ? hash_find(tab[w], comp(v, jj)) : -1;
        packed |= (h >= 0 ? (unsigned)slot_pos[w][h] : kAbsent) << (8 * jj);
      }
    }
    qpos[b + k] = packed;
  }
  for (int k = lane; k < cnt; k += 32) tmpcols[4LL * b + k] = scol[w][k];
  const unsigned bad = __ballot_sync(0xffffffffu, !ok);
  if (lane == 0) {
    row_nnz[row] = cnt;
    if (bad) atomicOr(status, IPCB_STATUS_ROW_OVERFLOW);
  }
  }
}

// pass B, warp per row: one 9-value accumulator per column in shared memory.
// The lanes load the row's blocks 32 at a time (block i = quad i / 4, column
// slot jj = i % 4) with the column positions pass A stored, group equal
// positions (__match_any_sync), sum each group by pointer jumping over its
// lanes (shuffles), and the group's lowest lane adds the sum to the column's
// accumulator.  Every sum runs in a fixed order (batches in input order,
// within a batch a fixed tree over the group's lanes), so the result is
// deterministic, and each column takes one shared-memory add per batch.
template <class S>
__global__ void __launch_bounds__(kWarps * 32) k_row_values(const int* __restrict__ rows, int* __restrict__ nrec,
                                                            const int* __restrict__ qstart,
                                                            const int* __restrict__ qids,
                                                            const unsigned* __restrict__ qpos,
                                                            const S* __restrict__ vals,
                                                            const int* __restrict__ tmpcols,
                                                            const int* __restrict__ offsets, int* __restrict__ columns,
                                                            S* __restrict__ values) {
  __shared__ S sacc[kWarps][kHash * 9];
  // a batch's 8 quads (36 values each, contiguous per quad), loaded with
  // 16-byte vectors; lane l's block is then at 9 l (conflict-free: 9 is odd)
  __shared__ __align__(16) S sstage[kWarps][8 * 36];
  constexpr int kVec = 36 * (int)sizeof(S) / 16;  // 16-byte vectors per quad
  const unsigned full = 0xffffffffu;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nrows = nrec[2];
  for (int row = next_row(nrec + 4, rows, nrows, lane); row >= 0; row = next_row(nrec + 4, rows, nrows, lane)) {
  __syncwarp();  // the previous row's shared-memory reads are done
  int b = qstart[row], e = qstart[row + 1];
  const int out = offsets[row], cnt = min(offsets[row + 1] - out, kHash);
  if (cnt == 0) continue;  // a row whose blocks are all zero
  for (int k = lane; k < cnt; k += 32) {
#pragma unroll
    for (int t = 0; t < 9; ++t) sacc[w][9 * k + t] = S(0);
  }
  __syncwarp();
  const int nb = 4 * (e - b);
  constexpr int kNone = kHash;  // no block (past the row, or a zero block)
  for (int base = 0; base < nb; base += 32) {
    const int q0 = base >> 2, nq = min(8, (nb - base) >> 2);
    for (int u = lane; u < nq * kVec; u += 32) {
      const int kk = u / kVec, piece = u - kk * kVec;
      const int q = __ldg(qids + b + q0 + kk);
      reinterpret_cast<float4*>(&sstage[w][36 * kk])[piece] =
          __ldg(reinterpret_cast<const float4*>(vals + 36LL * q) + piece);
    }
    __syncwarp();
    const int i = base + lane;
    int pos = kNone;
    S v[9];
#pragma unroll
    for (int t = 0; t < 9; ++t) v[t] = S(0);
    if (i < nb) {
      const int k = i >> 2, jj = i & 3;
      const unsigned pk = (__ldg(qpos + b + k) >> (8 * jj)) & 0xffu;
      if ((int)pk < cnt) {  // kAbsent for a zero block
        pos = (int)pk;
        const S* src = &sstage[w][9 * lane];
#pragma unroll
        for (int t = 0; t < 9; ++t) v[t] = src[t];
      }
    }
    // lanes with the same position form a group (at most 8: a batch is 8
    // quads and a quad's 4 columns are distinct); each lane links to the next
    // higher lane of its group and three pointer-jumping steps leave the
    // group's sum, in a fixed order, in its lowest lane
    const unsigned peers = __match_any_sync(full, pos);
    const unsigned above = peers & ~((2u << lane) - 1u);
    int nxt = above ? __ffs(above) - 1 : -1;
#pragma unroll
    for (int step = 0; step < 3; ++step) {
      const int src = nxt >= 0 ? nxt : lane;
#pragma unroll
      for (int t = 0; t < 9; ++t) {
        const S o = __shfl_sync(full, v[t], src);
        if (nxt >= 0) v[t] += o;
      }
      const int n2 = __shfl_sync(full, nxt, src);
      nxt = nxt >= 0 ? n2 : -1;
    }
    if (pos != kNone && (peers & ((1u << lane) - 1u)) == 0) {
#pragma unroll
      for (int t = 0; t < 9; ++t) sacc[w][9 * pos + t] += v[t];
    }
    __syncwarp();
  }
  for (int k = lane; k < cnt; k += 32) {
    columns[out + k] = tmpcols[4LL * b + k];
#pragma unroll
    for (int t = 0; t < 9; ++t) values[9LL * (out + k) + t] = sacc[w][9 * k + t];
  }
  }
}

__global__ void k_total(int nrow, int* __restrict__ offsets, const int* __restrict__ total, int* __restrict__ nnz) {
  offsets[nrow] = *total;
  *nnz = *total;
}

template <class S>
int assemble(int n_ee, int n_pt, const int* ee_cnt, const int* pt_cnt, int nv, const int* ee, const int* pt,
             const S* vals, const unsigned short* bmask, int* offsets, int* columns, S* values, int* nnz, int* status,
             void* ws, cudaStream_t st) {
  const int P = n_ee + n_pt;  // records, or their bound when the counts are read on the device
  size_t NQ = 4 * (size_t)P, R = (size_t)nv + 1;
  char* p = (char*)ws;
  int4* slots = (int4*)p; p += al(NQ * 4);
  int* qids = (int*)p; p += al(NQ * 4);
  unsigned* qpos = (unsigned*)p; p += al(NQ * 4);
  int* qstart = (int*)p; p += al(R * 4);
  int* rows = (int*)p; p += al(R * 4);
  int* tmpcols = (int*)p; p += al(NQ * 4 * 4);
  int* total = (int*)p; p += 256;
  int* nrec = (int*)p; p += 256;
  void* scratch = p;
  cudaMemsetAsync(qstart, 0, R * sizeof(int), st);
  cudaMemsetAsync(offsets, 0, (size_t)nv * sizeof(int), st);  // rows without contact: no blocks
  k_counts<<<1, 1, 0, st>>>(ee_cnt, n_ee, pt_cnt, n_pt, nrec);
  k_rec_slots<<<div_up(P, 256), 256, 0, st>>>(nrec, ee, pt, slots, qstart, rows);
  scan::exclusive<int>(qstart, (int)R, scratch, total, st);
  k_rec_scatter<<<div_up(P, 256), 256, 0, st>>>(nrec, ee, pt, slots, qstart, qids);
  // persistent warps over the touched rows (at most min(nv, 4 P) of them)
  const long long max_rows = std::min<long long>(nv, NQ);
  const int ga = (int)std::min<long long>(148 * 12, div_up(max_rows, kWarps));
  const int gb = (int)std::min<long long>(148 * 8, div_up(max_rows, kWarps));
  k_row_columns<<<ga, kWarps * 32, 0, st>>>(rows, qstart, qids, ee, nrec, pt, bmask, tmpcols, qpos, offsets, status);
  scan::exclusive<int>(offsets, nv, scratch, total, st);
  k_total<<<1, 1, 0, st>>>(nv, offsets, total, nnz);
  k_row_values<S><<<gb, kWarps * 32, 0, st>>>(rows, nrec, qstart, qids, qpos, vals, tmpcols, offsets, columns,
                                              values);
  return check_launch("ipcb_contact_bsr");
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

size_t ipcb_contact_bsr_workspace(int n_records, int n_verts) {
  size_t NQ = 4 * (size_t)(n_records > 0 ? n_records : 1), R = (size_t)(n_verts > 0 ? n_verts : 0) + 1;
  return al(NQ * 4) * 3 + 2 * al(R * 4) + al(NQ * 16) + 512 + scan::scratch_bytes((int)R);
}

int ipcb_contact_bsr(const ipcb_contacts* ee, int n_ee, const ipcb_contacts* pt, int n_pt, int n_verts,
                     const void* vals, const unsigned short* block_mask, int fp64, int* offsets, int* columns,
                     void* values, int* nnz, int* status, void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!ee || !pt || n_verts < 0 || !offsets || !nnz || !status) return IPCB_E_ARG;
  // a negative count: min(*cnt, capacity) of that list, read on the device
  const int* ee_cnt = n_ee < 0 ? ee->cnt : nullptr;
  const int* pt_cnt = n_pt < 0 ? pt->cnt : nullptr;
  if ((n_ee < 0 && !ee_cnt) || (n_pt < 0 && !pt_cnt)) return IPCB_E_ARG;
  if (n_ee < 0) n_ee = ee->capacity;
  if (n_pt < 0) n_pt = pt->capacity;
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
    return assemble<double>(n_ee, n_pt, ee_cnt, pt_cnt, n_verts, ee->a1a2b1b2, pt->a1a2b1b2, (const double*)vals,
                            block_mask, offsets, columns, (double*)values, nnz, status, ws, st);
  return assemble<float>(n_ee, n_pt, ee_cnt, pt_cnt, n_verts, ee->a1a2b1b2, pt->a1a2b1b2, (const float*)vals,
                         block_mask, offsets, columns, (float*)values, nnz, status, ws, st);
}

}  // extern "C"
