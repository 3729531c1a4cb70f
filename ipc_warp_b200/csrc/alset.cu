// Hashed active set of the augmented-Lagrangian contact solver
// (augmented_lagrangian.py:105-198, 506-572): the per-vertex minimum time of
// impact of the intersection records, the filter that keeps a record when it
// is the earliest impact of one of its vertices, and a compact hash of
// constraints keyed by the primitive pair e0e1: bucket starts cell_start
// [table_size + 1] and the entries stored bucket by bucket.  Building one
// (count per bucket, exclusive scan, scatter with a per-bucket cursor) and
// merging a new set into an old one (old entries whose gamma stays >= 0.01
// plus new entries whose key the old set lacks) are one pass each.
#include "common.cuh"
#include "scan.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

constexpr double kToiFilterEps = 1.0e-12;
constexpr double kDecayThreshold = 0.01;

// hash_pos (augmented_lagrangian.py): (e0 * 73856093) xor (e1 * 19349663) in
// wrapping 32-bit arithmetic, made non-negative, modulo the table size
IPCB_D int hash_pos(int e0, int e1, int table_size) {
  int v = (int)(((unsigned)e0 * 73856093u) ^ ((unsigned)e1 * 19349663u));
  if (v < 0) v = -v;
  int r = v % table_size;
  return r < 0 ? r + table_size : r;  // only -2^31 stays negative above
}

template <class S>
struct Set {
  int T, cap;
  int* start;
  int4* ids;
  int2* key;
  S *l0, *alpha, *lam, *gamma, *slack, *moll, *d0;
  int* dtype;
  S* grad;
};

template <class S>
Set<S> view(const ipcb_al_set* a) {
  return Set<S>{a->table_size, a->capacity, a->cell_start, (int4*)a->a1a2b1b2, (int2*)a->e0e1, (S*)a->l0,
                (S*)a->alpha, (S*)a->lam, (S*)a->gamma, (S*)a->slack, (S*)a->mollifier, (S*)a->d0,
                a->distance_type, (S*)a->grad};
}

template <class S>
__global__ void k_vertex_toi(ipcb_contacts L, int n, S* __restrict__ vtoi) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 id = reinterpret_cast<const int4*>(L.a1a2b1b2)[i];
  const S a = static_cast<const S*>(L.alpha)[i];
  atomic_min_nonneg(vtoi + id.x, a);
  atomic_min_nonneg(vtoi + id.y, a);
  atomic_min_nonneg(vtoi + id.z, a);
  atomic_min_nonneg(vtoi + id.w, a);
}

template <class S>
IPCB_D bool filter_accept(int4 id, S a, const S* __restrict__ vtoi) {
  const S eps = S(kToiFilterEps);
  return a <= vtoi[id.x] + eps || a <= vtoi[id.y] + eps || a <= vtoi[id.z] + eps || a <= vtoi[id.w] + eps;
}

template <class S>
__global__ void k_create_count(ipcb_contacts L, int n, const S* __restrict__ vtoi, Set<S> H) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 id = reinterpret_cast<const int4*>(L.a1a2b1b2)[i];
  if (!filter_accept(id, static_cast<const S*>(L.alpha)[i], vtoi)) return;
  const int2 k = reinterpret_cast<const int2*>(L.e0e1)[i];
  atomicAdd(H.start + hash_pos(k.x, k.y, H.T), 1);
}

template <class S>
IPCB_D int claim(const Set<S>& H, int* __restrict__ cursor, int2 k) {
  const int b = hash_pos(k.x, k.y, H.T);
  return H.start[b] + atomicAdd(cursor + b, 1);
}

template <class S>
__global__ void k_create_register(ipcb_contacts L, int n, const S* __restrict__ vtoi, Set<S> H,
                                  int* __restrict__ cursor) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int4 id = reinterpret_cast<const int4*>(L.a1a2b1b2)[i];
  const S a = static_cast<const S*>(L.alpha)[i];
  if (!filter_accept(id, a, vtoi)) return;
  const int2 k = reinterpret_cast<const int2*>(L.e0e1)[i];
  const int p = claim(H, cursor, k);
  if (p >= H.cap) return;
  // to_al_constraint
  H.ids[p] = id;
  H.key[p] = k;
  H.l0[p] = static_cast<const S*>(L.l0)[i];
  H.alpha[p] = a;
  H.lam[p] = S(0);
  H.gamma[p] = S(1);
  H.slack[p] = S(0);
  H.moll[p] = S(1);
  H.dtype[p] = 0;
  H.d0[p] = S(0);
  for (int c = 0; c < 12; ++c) H.grad[12LL * p + c] = S(0);
}

template <class S>
IPCB_D bool in_set(const Set<S>& H, int2 k) {
  const int b = hash_pos(k.x, k.y, H.T);
  for (int i = H.start[b]; i < H.start[b + 1]; ++i) {
    const int2 o = H.key[i];
    if (o.x == k.x && o.y == k.y) return true;
  }
  return false;
}

// entry i of the merge input: old entries first, then new ones
template <class S>
IPCB_D bool merge_keep(const Set<S>& nw, const Set<S>& old, int n_old, int i, const Set<S>*& src, int& j) {
  if (i < n_old) {
    src = &old;
    j = i;
    return old.gamma[i] >= S(kDecayThreshold);
  }
  src = &nw;
  j = i - n_old;
  return !in_set(old, nw.key[j]);
}

template <class S>
__global__ void k_merge_count(Set<S> nw, Set<S> old, Set<S> dst, int n_old, int n_new) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_old + n_new) return;
  const Set<S>* src;
  int j;
  if (!merge_keep(nw, old, n_old, i, src, j)) return;
  const int2 k = src->key[j];
  atomicAdd(dst.start + hash_pos(k.x, k.y, dst.T), 1);
}

template <class S>
__global__ void k_merge_register(Set<S> nw, Set<S> old, Set<S> dst, int n_old, int n_new, int* __restrict__ cursor) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_old + n_new) return;
  const Set<S>* src;
  int j;
  if (!merge_keep(nw, old, n_old, i, src, j)) return;
  const int p = claim(dst, cursor, src->key[j]);
  if (p >= dst.cap) return;
  dst.ids[p] = src->ids[j];
  dst.key[p] = src->key[j];
  dst.l0[p] = src->l0[j];
  dst.alpha[p] = src->alpha[j];
  dst.lam[p] = src->lam[j];
  dst.gamma[p] = src->gamma[j];
  dst.slack[p] = src->slack[j];
  dst.moll[p] = src->moll[j];
  dst.dtype[p] = src->dtype[j];
  dst.d0[p] = src->d0[j];
  for (int c = 0; c < 12; ++c) dst.grad[12LL * p + c] = src->grad[12LL * j + c];
}

inline size_t al(size_t b) { return (b + 255) & ~(size_t)255; }

bool set_ok(const ipcb_al_set* a) {
  return a && a->table_size > 0 && a->capacity >= 0 && a->cell_start &&
         (a->capacity == 0 || (a->a1a2b1b2 && a->e0e1 && a->l0 && a->alpha && a->lam && a->gamma && a->slack &&
                                a->mollifier && a->d0 && a->distance_type && a->grad));
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_al_vertex_toi(int fp64, const ipcb_contacts* list, int n, void* vertex_toi, ipcb_stream s) {
  if (!list || n < 0 || n > list->capacity || !vertex_toi) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  if (!list->a1a2b1b2 || !list->alpha) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (fp64) k_vertex_toi<double><<<div_up(n, 256), 256, 0, st>>>(*list, n, (double*)vertex_toi);
  else k_vertex_toi<float><<<div_up(n, 256), 256, 0, st>>>(*list, n, (float*)vertex_toi);
  return check_launch("ipcb_al_vertex_toi");
}

size_t ipcb_al_workspace(int table_size) {
  if (table_size <= 0) return 0;
  return al((size_t)table_size * 4) + scan::scratch_bytes(table_size + 1);
}

int ipcb_al_create(int fp64, ipcb_al_set* set, const ipcb_contacts* list, int n, const void* vertex_toi, void* ws,
                   size_t ws_bytes, ipcb_stream s) {
  if (!set_ok(set) || !list || n < 0 || n > list->capacity || n > set->capacity || !ws ||
      ws_bytes < ipcb_al_workspace(set->table_size))
    return IPCB_E_ARG;
  if (n > 0 && (!vertex_toi || !list->a1a2b1b2 || !list->e0e1 || !list->alpha || !list->l0)) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int T = set->table_size;
  int* cursor = (int*)ws;
  void* scratch = (char*)ws + al((size_t)T * 4);
  cudaMemsetAsync(set->cell_start, 0, sizeof(int) * (T + 1), st);
  if (n == 0) return check_launch("ipcb_al_create");
  cudaMemsetAsync(cursor, 0, sizeof(int) * T, st);
  const int g = div_up(n, 256);
  if (fp64) {
    Set<double> H = view<double>(set);
    k_create_count<double><<<g, 256, 0, st>>>(*list, n, (const double*)vertex_toi, H);
    scan::exclusive<int>(set->cell_start, T + 1, scratch, nullptr, st);
    k_create_register<double><<<g, 256, 0, st>>>(*list, n, (const double*)vertex_toi, H, cursor);
  } else {
    Set<float> H = view<float>(set);
    k_create_count<float><<<g, 256, 0, st>>>(*list, n, (const float*)vertex_toi, H);
    scan::exclusive<int>(set->cell_start, T + 1, scratch, nullptr, st);
    k_create_register<float><<<g, 256, 0, st>>>(*list, n, (const float*)vertex_toi, H, cursor);
  }
  return check_launch("ipcb_al_create");
}

int ipcb_al_merge(int fp64, const ipcb_al_set* nw, const ipcb_al_set* old, ipcb_al_set* dst, int n_new, int n_old,
                  void* ws, size_t ws_bytes, ipcb_stream s) {
  if (!set_ok(nw) || !set_ok(old) || !set_ok(dst) || n_new < 0 || n_old < 0 || n_new > nw->capacity ||
      n_old > old->capacity || (long long)n_new + n_old > dst->capacity || !ws ||
      ws_bytes < ipcb_al_workspace(dst->table_size))
    return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  const int T = dst->table_size;
  int* cursor = (int*)ws;
  void* scratch = (char*)ws + al((size_t)T * 4);
  cudaMemsetAsync(dst->cell_start, 0, sizeof(int) * (T + 1), st);
  const int n = n_new + n_old;
  if (n == 0) return check_launch("ipcb_al_merge");
  cudaMemsetAsync(cursor, 0, sizeof(int) * T, st);
  const int g = div_up(n, 256);
  if (fp64) {
    Set<double> a = view<double>(nw), b = view<double>(old), c = view<double>(dst);
    k_merge_count<double><<<g, 256, 0, st>>>(a, b, c, n_old, n_new);
    scan::exclusive<int>(dst->cell_start, T + 1, scratch, nullptr, st);
    k_merge_register<double><<<g, 256, 0, st>>>(a, b, c, n_old, n_new, cursor);
  } else {
    Set<float> a = view<float>(nw), b = view<float>(old), c = view<float>(dst);
    k_merge_count<float><<<g, 256, 0, st>>>(a, b, c, n_old, n_new);
    scan::exclusive<int>(dst->cell_start, T + 1, scratch, nullptr, st);
    k_merge_register<float><<<g, 256, 0, st>>>(a, b, c, n_old, n_new, cursor);
  }
  return check_launch("ipcb_al_merge");
}

}  // extern "C"
