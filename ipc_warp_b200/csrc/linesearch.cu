// Device-side backtracking line search (time_integrator_base.py:514-546): the
// trial state, the accept test and the step halving live in device memory, and
// the trial loop is a CUDA graph WHILE node whose body is one trial (x = x0 -
// alpha dx, BVH refit, DCD, the energies) followed by ipcb_ls_accept, which
// sets the loop condition.  One read of the state after the loop replaces the
// reference's one to three host reads per energy evaluation.
//
// Termination does not depend on the energies: every trial increments `it`,
// and the condition is cleared when the step is accepted, when alpha falls to
// eps * max(1, upper bound) (the reference's test), when `it` reaches max_it,
// or when a contact list overflowed (the host then reruns the search).
#include "common.cuh"

namespace ipcb {
int check_launch(const char* where);
void set_error(const char* where, cudaError_t e);

namespace {

template <class S>
__global__ void k_inertia(int n, const S* __restrict__ x, const S* __restrict__ x0, const S* __restrict__ xdot,
                          double gx, double gy, double gz, double h, const double* __restrict__ mass,
                          const unsigned char* __restrict__ fixed, const S* __restrict__ target, double k_att,
                          double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (i < n) {
    const double g[3] = {gx, gy, gz};
    const double m = mass[i];
    const bool fx = fixed && fixed[i];
    for (int k = 0; k < 3; ++k) {
      const double xi = (double)x[3 * i + k];
      const double xt = (double)x0[3 * i + k] + h * (double)xdot[3 * i + k] + h * h * g[k];
      const double d = xi - xt;
      e += 0.5 * m * d * d;
      if (fx) {
        const double r = xi - (double)target[3 * i + k];
        e += 0.5 * k_att * h * h * r * r;
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  __shared__ double s[8];
  if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += s[k];
    if (t != 0.0) atomicAdd(out, t);
  }
}

__global__ void k_ls_begin(ipcb_ls_state* st, const void* toi, int fp64, const int* __restrict__ status,
                           const double* __restrict__ acc, double h2, double eps, int max_it, ipcb_contacts ee,
                           ipcb_contacts pt) {
  const double t = fp64 ? *(const double*)toi : (double)*(const float*)toi;
  // a CCD query that ran out of stack, visits or root iterations may have
  // missed an earlier impact: its TOI is no bound, so no step is taken
  const int failed = status ? (*status & (IPCB_STATUS_STACK | IPCB_STATUS_ROOT_ITERS)) : 0;
  st->refused = failed;
  st->ub = failed ? 0.0 : (t < 1.0 ? 0.9 * t : 1.0);
  st->alpha = st->ub;
  st->eps = eps;
  st->E0 = h2 * (acc[0] + acc[1]) + acc[2];
  st->E1 = st->E0;
  st->alpha_accepted = 0.0;
  st->it = 0;
  st->max_it = max_it;
  st->accepted = 0;
  st->done = 0;
  // the lists of the E0 evaluation
  const int c_ee = ee.cnt ? *ee.cnt : 0, c_pt = pt.cnt ? *pt.cnt : 0;
  st->overflow = c_ee > ee.capacity || c_pt > pt.capacity;
  st->max_ee = c_ee;
  st->max_pt = c_pt;
}

template <class S>
__global__ void k_ls_trial(const ipcb_ls_state* __restrict__ st, int n3, const S* __restrict__ x_tmp,
                           const S* __restrict__ dx, S* __restrict__ x, double* __restrict__ acc) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const S a = (S)st->alpha;
  if (i < n3) x[i] = xsub(x_tmp[i], xmul(a, dx[i]));  // two roundings, as x_tmp - alpha * dx on the host
  if (i < 3) acc[i] = 0.0;
}

__global__ void k_ls_accept(ipcb_ls_state* st, const double* __restrict__ acc, double h2, ipcb_contacts ee,
                            ipcb_contacts pt, unsigned long long handle) {
  const int c_ee = ee.cnt ? *ee.cnt : 0, c_pt = pt.cnt ? *pt.cnt : 0;
  st->max_ee = max(st->max_ee, c_ee);
  st->max_pt = max(st->max_pt, c_pt);
  const bool over = c_ee > ee.capacity || c_pt > pt.capacity;
  const double E1 = h2 * (acc[0] + acc[1]) + acc[2];
  st->E1 = E1;
  st->it += 1;
  int cont = 0;
  if (st->refused) {
    // the CCD bound was refused: the one trial ran at alpha = 0, nothing is accepted
  } else if (over || st->overflow) {
    st->overflow = 1;
  } else if (isfinite(E1) && E1 < st->E0) {
    st->accepted = 1;
    st->alpha_accepted = st->alpha;
  } else {
    st->alpha *= 0.5;
    cont = st->alpha > st->eps * fmax(1.0, st->ub);
  }
  if (st->it >= st->max_it) cont = 0;
  st->done = !cont;
  if (handle) cudaGraphSetConditional((cudaGraphConditionalHandle)handle, cont ? 1u : 0u);
}

template <class S>
__global__ void k_ls_finish(const ipcb_ls_state* __restrict__ st, int n3, const S* __restrict__ x_tmp,
                            S* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n3 && !st->accepted) x[i] = x_tmp[i];
}

__global__ void k_acc_fold(double* acc, double* extra, int n) {
  double v = *acc;
  for (int i = 0; i < n; ++i) {
    v += extra[i];
    extra[i] = 0.0;
  }
  *acc = v;
}

struct WhileGraph {
  cudaGraph_t graph = nullptr;
  cudaGraph_t body = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
};

}  // namespace
}  // namespace ipcb

using namespace ipcb;

extern "C" {

int ipcb_ls_inertia(int fp64, int n, const void* x, const void* x0, const void* xdot, const double* gravity, double h,
                    const double* mass, const unsigned char* fixed, const void* target, double k_att, double* out,
                    ipcb_stream s) {
  if (n < 0 || !gravity || !out) return IPCB_E_ARG;
  if (n == 0) return IPCB_OK;
  if (!x || !x0 || !xdot || !mass || (fixed && !target)) return IPCB_E_ARG;
  cudaStream_t st = (cudaStream_t)s;
  if (fp64)
    k_inertia<double><<<div_up(n, 256), 256, 0, st>>>(n, (const double*)x, (const double*)x0, (const double*)xdot,
                                                      gravity[0], gravity[1], gravity[2], h, mass, fixed,
                                                      (const double*)target, k_att, out);
  else
    k_inertia<float><<<div_up(n, 256), 256, 0, st>>>(n, (const float*)x, (const float*)x0, (const float*)xdot,
                                                     gravity[0], gravity[1], gravity[2], h, mass, fixed,
                                                     (const float*)target, k_att, out);
  return check_launch("ipcb_ls_inertia");
}

int ipcb_ls_begin(ipcb_ls_state* st, const void* toi, int fp64, const int* status, const double* acc, double h2,
                  double eps, int max_it, const ipcb_contacts* ee, const ipcb_contacts* pt, ipcb_stream s) {
  if (!st || !toi || !acc || max_it <= 0 || !ee || !pt) return IPCB_E_ARG;
  k_ls_begin<<<1, 1, 0, (cudaStream_t)s>>>(st, toi, fp64, status, acc, h2, eps, max_it, *ee, *pt);
  return check_launch("ipcb_ls_begin");
}

int ipcb_ls_trial(const ipcb_ls_state* st, int fp64, int n_verts, const void* x_tmp, const void* dx, void* x,
                  double* acc, ipcb_stream s) {
  if (!st || n_verts <= 0 || !x_tmp || !dx || !x || !acc) return IPCB_E_ARG;
  const int n3 = 3 * n_verts;
  cudaStream_t str = (cudaStream_t)s;
  if (fp64)
    k_ls_trial<double><<<div_up(n3, 256), 256, 0, str>>>(st, n3, (const double*)x_tmp, (const double*)dx, (double*)x,
                                                         acc);
  else
    k_ls_trial<float><<<div_up(n3, 256), 256, 0, str>>>(st, n3, (const float*)x_tmp, (const float*)dx, (float*)x,
                                                        acc);
  return check_launch("ipcb_ls_trial");
}

int ipcb_ls_accept(ipcb_ls_state* st, const double* acc, double h2, const ipcb_contacts* ee, const ipcb_contacts* pt,
                   unsigned long long cond_handle, ipcb_stream s) {
  if (!st || !acc || !ee || !pt) return IPCB_E_ARG;
  k_ls_accept<<<1, 1, 0, (cudaStream_t)s>>>(st, acc, h2, *ee, *pt, cond_handle);
  return check_launch("ipcb_ls_accept");
}

int ipcb_ls_finish(const ipcb_ls_state* st, int fp64, int n_verts, const void* x_tmp, void* x, ipcb_stream s) {
  if (!st || n_verts <= 0 || !x_tmp || !x) return IPCB_E_ARG;
  const int n3 = 3 * n_verts;
  cudaStream_t str = (cudaStream_t)s;
  if (fp64) k_ls_finish<double><<<div_up(n3, 256), 256, 0, str>>>(st, n3, (const double*)x_tmp, (double*)x);
  else k_ls_finish<float><<<div_up(n3, 256), 256, 0, str>>>(st, n3, (const float*)x_tmp, (float*)x);
  return check_launch("ipcb_ls_finish");
}

int ipcb_acc_fold(double* acc, double* extra, int n, ipcb_stream s) {
  if (!acc || n < 0 || (n && !extra)) return IPCB_E_ARG;
  k_acc_fold<<<1, 1, 0, (cudaStream_t)s>>>(acc, extra, n);
  return check_launch("ipcb_acc_fold");
}

int ipcb_graph_while_begin(void** ctx, unsigned long long* handle, ipcb_stream s) {
  if (!ctx || !handle) return IPCB_E_ARG;
  WhileGraph* w = new WhileGraph();
  cudaError_t e = cudaGraphCreate(&w->graph, 0);
  if (e == cudaSuccess) e = cudaGraphConditionalHandleCreate(&w->handle, w->graph, 1u, cudaGraphCondAssignDefault);
  if (e == cudaSuccess) {
    cudaGraphNode_t node = nullptr;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = w->handle;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    e = cudaGraphAddNode(&node, w->graph, nullptr, 0, &p);
    if (e == cudaSuccess) w->body = p.conditional.phGraph_out[0];
  }
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph((cudaStream_t)s, w->body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
  if (e != cudaSuccess) {
    if (w->graph) cudaGraphDestroy(w->graph);
    delete w;
    *ctx = nullptr;
    set_error("ipcb_graph_while_begin", e);
    return IPCB_E_CUDA;
  }
  *ctx = w;
  *handle = (unsigned long long)w->handle;
  return IPCB_OK;
}

int ipcb_graph_while_end(void* ctx, ipcb_stream s) {
  if (!ctx) return IPCB_E_ARG;
  WhileGraph* w = (WhileGraph*)ctx;
  cudaGraph_t captured = nullptr;
  cudaError_t e = cudaStreamEndCapture((cudaStream_t)s, &captured);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&w->exec, w->graph, 0);
  if (e != cudaSuccess) {
    set_error("ipcb_graph_while_end", e);
    return IPCB_E_CUDA;
  }
  return IPCB_OK;
}

int ipcb_graph_launch(void* ctx, ipcb_stream s) {
  if (!ctx) return IPCB_E_ARG;
  WhileGraph* w = (WhileGraph*)ctx;
  if (!w->exec) return IPCB_E_ARG;
  const cudaError_t e = cudaGraphLaunch(w->exec, (cudaStream_t)s);
  if (e != cudaSuccess) {
    set_error("ipcb_graph_launch", e);
    return IPCB_E_CUDA;
  }
  return IPCB_OK;
}

void ipcb_graph_destroy(void* ctx) {
  if (!ctx) return;
  WhileGraph* w = (WhileGraph*)ctx;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  if (w->graph) cudaGraphDestroy(w->graph);
  delete w;
}

}  // extern "C"
