// Tetrahedral FEM elastic term (fem/fem.py:22-34 compute_Dm, 139-203
// tet_kernel_sparse, time_integrator_base.py:124-137 compute_Psi) with the
// reference's three materials: stable Neo-Hookean (fem/snh.py), Neo-Hookean
// (fem/neo_hookean.py), St. Venant-Kirchhoff (fem/stvk.py).
//
// One thread per tet (the reference launches one per (tet, i, j) and
// recomputes F and P 16 times): F = Ds Bm, P(F), the 4 nodal forces
// H = -W P Bm^T (columns; the 4th is minus their sum), and the 16 3x3 blocks
// K_ij[:, k] from the 12 directional derivatives dP(F; dF) with the
// reference's dDs (columns -e_k for j < 3, +e_k in all three for j = 3).
// Triplets at tet*16 + i*4 + j, force atomically into b (when j == 0 in the
// reference; here once per node).  No PSD projection (as the reference).
#include "fem_impl.cuh"

namespace ipcb {
int check_launch(const char* where);

namespace {

template <class S>
__global__ void k_tet_dm(const S* __restrict__ xcs, const int4* __restrict__ tets, int n, S* __restrict__ Bm,
                         S* __restrict__ W) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  int4 t = tets[e];
  v3<S> x0 = load3(xcs, t.x), x1 = load3(xcs, t.y), x2 = load3(xcs, t.z), x3 = load3(xcs, t.w);
  M3<S> Dm = from_cols(x0 - x3, x1 - x3, x2 - x3);
  M3<S> B = inv3(Dm);
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) Bm[9 * e + 3 * i + j] = B.a[i][j];
  W[e] = fabs(det3(Dm)) / S(6);
}

// warps per block of k_tet_hessian: each warp stages 32 tets (145 values each)
template <class S> __host__ __device__ constexpr int tet_warps() { return sizeof(S) == 4 ? 2 : 1; }

template <class S>
__global__ void __launch_bounds__(64) k_tet_hessian(int mat, const S* __restrict__ x, const int4* __restrict__ tets,
                                                    int n, const S* __restrict__ Bm, const S* __restrict__ W, S mu,
                                                    S lam, int* __restrict__ rows, int* __restrict__ cols,
                                                    S* __restrict__ vals, S* __restrict__ b) {
  __shared__ S sm[tet_warps<S>()][32 * kTetStage];
  const int w = threadIdx.x >> 5;
  const int e0 = (blockIdx.x * tet_warps<S>() + w) * 32;
  if (e0 >= n) return;
  tet_hessian_warp<S>(mat, x, tets, e0, n, Bm, W, mu, lam, rows, cols, vals, b, sm[w]);
}

template <class S>
__global__ void k_tet_energy(int mat, const S* __restrict__ x, const int4* __restrict__ tets, int n,
                             const S* __restrict__ Bm, const S* __restrict__ W, S mu, S lam,
                             double* __restrict__ energy) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (e < n) {
    int4 t = tets[e];
    v3<S> p0 = load3(x, t.x), p1 = load3(x, t.y), p2 = load3(x, t.z), p3 = load3(x, t.w);
    M3<S> F = mmul(from_cols(p0 - p3, p1 - p3, p2 - p3), load_bm(Bm, e));
    v = (double)W[e] * (double)psi(mat, F, mu, lam);
  }
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __shared__ double s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s[k];
    atomicAdd(energy, t);
  }
}

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_tet_rest(int fp64, const void* xcs, const int* tets, int n_tets, void* Bm, void* W, ipcb_stream s) {
  if (n_tets < 0 || (n_tets && (!xcs || !tets || !Bm || !W))) return IPCB_E_ARG;
  if (n_tets == 0) return IPCB_OK;
  dim3 g(div_up(n_tets, 256));
  if (fp64)
    k_tet_dm<double><<<g, 256, 0, (cudaStream_t)s>>>((const double*)xcs, (const int4*)tets, n_tets, (double*)Bm,
                                                     (double*)W);
  else
    k_tet_dm<float><<<g, 256, 0, (cudaStream_t)s>>>((const float*)xcs, (const int4*)tets, n_tets, (float*)Bm,
                                                    (float*)W);
  return check_launch("ipcb_tet_rest");
}

int ipcb_tet_hessian(int material, int fp64, const void* x, const int* tets, int n_tets, const void* Bm, const void* W,
                     double mu, double lam, int* rows, int* cols, void* vals, void* b, ipcb_stream s) {
  if (material < 0 || material > 2 || n_tets < 0) return IPCB_E_ARG;
  if (n_tets == 0) return IPCB_OK;
  if (!x || !tets || !Bm || !W || !vals || !b || (!rows != !cols)) return IPCB_E_ARG;
  if (fp64)
    k_tet_hessian<double><<<div_up(n_tets, 32 * tet_warps<double>()), 32 * tet_warps<double>(), 0,
                            (cudaStream_t)s>>>(material, (const double*)x, (const int4*)tets, n_tets,
                                                          (const double*)Bm, (const double*)W, mu, lam, rows, cols,
                                                          (double*)vals, (double*)b);
  else
    k_tet_hessian<float><<<div_up(n_tets, 32 * tet_warps<float>()), 32 * tet_warps<float>(), 0,
                           (cudaStream_t)s>>>(material, (const float*)x, (const int4*)tets, n_tets,
                                                         (const float*)Bm, (const float*)W, (float)mu, (float)lam,
                                                         rows, cols, (float*)vals, (float*)b);
  return check_launch("ipcb_tet_hessian");
}

int ipcb_tet_energy(int material, int fp64, const void* x, const int* tets, int n_tets, const void* Bm, const void* W,
                    double mu, double lam, double* energy, ipcb_stream s) {
  if (material < 0 || material > 2 || n_tets < 0 || !energy) return IPCB_E_ARG;
  if (n_tets == 0) return IPCB_OK;
  dim3 g(div_up(n_tets, 256));
  if (fp64)
    k_tet_energy<double><<<g, 256, 0, (cudaStream_t)s>>>(material, (const double*)x, (const int4*)tets, n_tets,
                                                         (const double*)Bm, (const double*)W, mu, lam, energy);
  else
    k_tet_energy<float><<<g, 256, 0, (cudaStream_t)s>>>(material, (const float*)x, (const int4*)tets, n_tets,
                                                        (const float*)Bm, (const float*)W, (float)mu, (float)lam,
                                                        energy);
  return check_launch("ipcb_tet_energy");
}

}  // extern "C"
