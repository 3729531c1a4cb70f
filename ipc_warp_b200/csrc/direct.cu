// Sparse Cholesky of the block Newton system on cuSOLVER's device csrchol
// (include/ipcb_direct.h).  The symbolic phase orders the block graph on the
// host, expands the permutation to scalars and builds the permuted scalar CSR
// together with a gather map from BSR value slots; the numeric phase gathers
// and factors on the device; the solve permutes b, runs the two triangular
// sweeps and scatters x back.
#include <cuda_runtime.h>
#include <cusolverSp.h>
#include <cusolverSp_LOWLEVEL_PREVIEW.h>
#include <cusparse.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "ipcb.h"
#include "ipcb_direct.h"

namespace {

thread_local std::string g_err;

int fail(int code, const char* what, int detail) {
  char buf[256];
  std::snprintf(buf, sizeof(buf), "%s (%d)", what, detail);
  g_err = buf;
  return code;
}

#define CU(x)                                                    \
  do {                                                           \
    cudaError_t e_ = (x);                                        \
    if (e_ != cudaSuccess) return fail(IPCB_E_CUDA, #x, (int)e_); \
  } while (0)
#define CS(x)                                                        \
  do {                                                               \
    cusolverStatus_t e_ = (x);                                       \
    if (e_ != CUSOLVER_STATUS_SUCCESS) return fail(IPCB_E_CUDA, #x, (int)e_); \
  } while (0)

struct Direct {
  cusolverSpHandle_t sp = nullptr;
  cusparseMatDescr_t descr = nullptr;
  csrcholInfo_t info = nullptr;
  int nb = 0, n = 0, nnz = 0, nnz_blocks = 0, fp64 = 0;
  int *rowptr = nullptr, *colind = nullptr, *map = nullptr, *perm = nullptr;
  void *vals = nullptr, *pb = nullptr, *px = nullptr, *buf = nullptr;
  size_t internal = 0, work = 0;
  bool analysed = false;

  void release() {
    cudaFree(rowptr); cudaFree(colind); cudaFree(map); cudaFree(perm);
    cudaFree(vals); cudaFree(pb); cudaFree(px); cudaFree(buf);
    rowptr = colind = map = perm = nullptr;
    vals = pb = px = buf = nullptr;
    if (info) cusolverSpDestroyCsrcholInfo(info);
    info = nullptr;
    analysed = false;
  }
};

template <class T>
__global__ void k_gather_values(const T* __restrict__ bsr, const int* __restrict__ map, int nnz, T* __restrict__ out) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < nnz) out[k] = bsr[map[k]];
}

// permuted[i] = src[perm[i]]  (perm: new scalar index -> old scalar index)
template <class T>
__global__ void k_permute(const T* __restrict__ src, const int* __restrict__ perm, int n, T* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[i] = src[perm[i]];
}

template <class T>
__global__ void k_unpermute(const T* __restrict__ src, const int* __restrict__ perm, int n, T* __restrict__ dst) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) dst[perm[i]] = src[i];
}

int grid(int n) { return (n + 255) / 256; }

}  // namespace

extern "C" {

const char* ipcb_direct_last_error(void) { return g_err.c_str(); }

int ipcb_direct_create(ipcb_direct_handle* out) {
  if (!out) return fail(IPCB_E_ARG, "null handle pointer", 0);
  Direct* d = new Direct();
  if (cusolverSpCreate(&d->sp) != CUSOLVER_STATUS_SUCCESS) {
    delete d;
    return fail(IPCB_E_CUDA, "cusolverSpCreate", 0);
  }
  cusparseCreateMatDescr(&d->descr);
  cusparseSetMatType(d->descr, CUSPARSE_MATRIX_TYPE_GENERAL);
  cusparseSetMatIndexBase(d->descr, CUSPARSE_INDEX_BASE_ZERO);
  *out = d;
  return 0;
}

int ipcb_direct_destroy(ipcb_direct_handle h) {
  Direct* d = static_cast<Direct*>(h);
  if (!d) return 0;
  d->release();
  if (d->descr) cusparseDestroyMatDescr(d->descr);
  if (d->sp) cusolverSpDestroy(d->sp);
  delete d;
  return 0;
}

int ipcb_direct_sizes(ipcb_direct_handle h, size_t* factor_bytes, size_t* work_bytes) {
  Direct* d = static_cast<Direct*>(h);
  if (!d || !d->analysed) return fail(IPCB_E_ARG, "not analysed", 0);
  if (factor_bytes) *factor_bytes = d->internal;
  if (work_bytes) *work_bytes = d->work;
  return 0;
}

int ipcb_direct_analyze(ipcb_direct_handle h, int n_blocks, int nnz_blocks, const int* offsets, const int* columns,
                        int fp64, int ordering, ipcb_direct_stream s) {
  Direct* d = static_cast<Direct*>(h);
  if (!d || n_blocks <= 0 || nnz_blocks < n_blocks || !offsets || !columns)
    return fail(IPCB_E_ARG, "bad pattern", n_blocks);
  if (ordering < IPCB_ORDER_NONE || ordering > IPCB_ORDER_METIS) return fail(IPCB_E_ARG, "bad ordering", ordering);
  cudaStream_t st = (cudaStream_t)s;
  d->release();
  std::vector<int> off(n_blocks + 1), col(nnz_blocks);
  CU(cudaMemcpyAsync(off.data(), offsets, sizeof(int) * (n_blocks + 1), cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(col.data(), columns, sizeof(int) * nnz_blocks, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  if (off[0] != 0 || off[n_blocks] != nnz_blocks) return fail(IPCB_E_ARG, "offsets do not match nnz", off[n_blocks]);
  for (int k = 0; k < nnz_blocks; ++k)
    if (col[k] < 0 || col[k] >= n_blocks) return fail(IPCB_E_ARG, "column out of range", col[k]);

  // block ordering p: new block i <- old block p[i]
  std::vector<int> p(n_blocks);
  std::iota(p.begin(), p.end(), 0);
  if (ordering != IPCB_ORDER_NONE) {
    if (ordering == IPCB_ORDER_SYMRCM)
      CS(cusolverSpXcsrsymrcmHost(d->sp, n_blocks, nnz_blocks, d->descr, off.data(), col.data(), p.data()));
    else if (ordering == IPCB_ORDER_SYMAMD)
      CS(cusolverSpXcsrsymamdHost(d->sp, n_blocks, nnz_blocks, d->descr, off.data(), col.data(), p.data()));
    else
      CS(cusolverSpXcsrmetisndHost(d->sp, n_blocks, nnz_blocks, d->descr, off.data(), col.data(), nullptr, p.data()));
  }
  std::vector<int> pinv(n_blocks);
  for (int i = 0; i < n_blocks; ++i) pinv[p[i]] = i;

  // permuted scalar CSR: row 3i+a holds, for each block (p[i], c) of the old
  // pattern in ascending new column pinv[c], the scalars 3 pinv[c] + 0..2
  const int n = 3 * n_blocks, nnz = 9 * nnz_blocks;
  std::vector<int> rowptr(n + 1), colind(nnz), map(nnz), perm(n);
  std::vector<std::pair<int, int>> row;  // (new block col, old block slot)
  int w = 0;
  for (int i = 0; i < n_blocks; ++i) {
    const int ob = p[i];
    row.clear();
    for (int k = off[ob]; k < off[ob + 1]; ++k) row.emplace_back(pinv[col[k]], k);
    std::sort(row.begin(), row.end());
    for (int a = 0; a < 3; ++a) {
      rowptr[3 * i + a] = w;
      perm[3 * i + a] = 3 * ob + a;
      for (const auto& e : row)
        for (int c = 0; c < 3; ++c) {
          colind[w] = 3 * e.first + c;
          map[w] = 9 * e.second + 3 * a + c;
          ++w;
        }
    }
  }
  rowptr[n] = w;

  d->nb = n_blocks;
  d->n = n;
  d->nnz = nnz;
  d->nnz_blocks = nnz_blocks;
  d->fp64 = fp64 ? 1 : 0;
  const size_t es = d->fp64 ? sizeof(double) : sizeof(float);
  CU(cudaMalloc(&d->rowptr, sizeof(int) * (n + 1)));
  CU(cudaMalloc(&d->colind, sizeof(int) * nnz));
  CU(cudaMalloc(&d->map, sizeof(int) * nnz));
  CU(cudaMalloc(&d->perm, sizeof(int) * n));
  CU(cudaMalloc(&d->vals, es * nnz));
  CU(cudaMalloc(&d->pb, es * n));
  CU(cudaMalloc(&d->px, es * n));
  CU(cudaMemcpyAsync(d->rowptr, rowptr.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d->colind, colind.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d->map, map.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(d->perm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  CU(cudaStreamSynchronize(st));  // host vectors go out of scope

  CS(cusolverSpSetStream(d->sp, st));
  CS(cusolverSpCreateCsrcholInfo(&d->info));
  CS(cusolverSpXcsrcholAnalysis(d->sp, n, nnz, d->descr, d->rowptr, d->colind, d->info));
  if (d->fp64)
    CS(cusolverSpDcsrcholBufferInfo(d->sp, n, nnz, d->descr, (const double*)d->vals, d->rowptr, d->colind, d->info,
                                    &d->internal, &d->work));
  else
    CS(cusolverSpScsrcholBufferInfo(d->sp, n, nnz, d->descr, (const float*)d->vals, d->rowptr, d->colind, d->info,
                                    &d->internal, &d->work));
  CU(cudaMalloc(&d->buf, std::max<size_t>(d->work, 256)));
  d->analysed = true;
  return 0;
}

int ipcb_direct_factor(ipcb_direct_handle h, const void* values, ipcb_direct_stream s) {
  Direct* d = static_cast<Direct*>(h);
  if (!d || !d->analysed || !values) return fail(IPCB_E_ARG, "not analysed", 0);
  cudaStream_t st = (cudaStream_t)s;
  CS(cusolverSpSetStream(d->sp, st));
  int singular = -1;
  if (d->fp64) {
    k_gather_values<double><<<grid(d->nnz), 256, 0, st>>>((const double*)values, d->map, d->nnz, (double*)d->vals);
    CU(cudaGetLastError());
    CS(cusolverSpDcsrcholFactor(d->sp, d->n, d->nnz, d->descr, (const double*)d->vals, d->rowptr, d->colind, d->info,
                                d->buf));
    CS(cusolverSpDcsrcholZeroPivot(d->sp, d->info, 0.0, &singular));
  } else {
    k_gather_values<float><<<grid(d->nnz), 256, 0, st>>>((const float*)values, d->map, d->nnz, (float*)d->vals);
    CU(cudaGetLastError());
    CS(cusolverSpScsrcholFactor(d->sp, d->n, d->nnz, d->descr, (const float*)d->vals, d->rowptr, d->colind, d->info,
                                d->buf));
    CS(cusolverSpScsrcholZeroPivot(d->sp, d->info, 0.0f, &singular));
  }
  if (singular >= 0) return fail(IPCB_E_SINGULAR, "non-positive pivot at scalar row", singular);
  return 0;
}

int ipcb_direct_solve(ipcb_direct_handle h, const void* b, void* x, ipcb_direct_stream s) {
  Direct* d = static_cast<Direct*>(h);
  if (!d || !d->analysed || !b || !x) return fail(IPCB_E_ARG, "not analysed", 0);
  cudaStream_t st = (cudaStream_t)s;
  CS(cusolverSpSetStream(d->sp, st));
  if (d->fp64) {
    k_permute<double><<<grid(d->n), 256, 0, st>>>((const double*)b, d->perm, d->n, (double*)d->pb);
    CS(cusolverSpDcsrcholSolve(d->sp, d->n, (const double*)d->pb, (double*)d->px, d->info, d->buf));
    k_unpermute<double><<<grid(d->n), 256, 0, st>>>((const double*)d->px, d->perm, d->n, (double*)x);
  } else {
    k_permute<float><<<grid(d->n), 256, 0, st>>>((const float*)b, d->perm, d->n, (float*)d->pb);
    CS(cusolverSpScsrcholSolve(d->sp, d->n, (const float*)d->pb, (float*)d->px, d->info, d->buf));
    k_unpermute<float><<<grid(d->n), 256, 0, st>>>((const float*)d->px, d->perm, d->n, (float*)x);
  }
  CU(cudaGetLastError());
  return 0;
}

}  // extern "C"
