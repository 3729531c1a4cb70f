// LBVH build for callers that cannot allocate device memory.
//
// Some hosts cannot call cudaMalloc on the path that rebuilds a hierarchy:
// a simulation step that must not block (cudaMalloc may synchronise the
// device), a host framework that owns all device memory through its own pool
// and forbids other allocators, or a binding (JNI, FFI) that can hand over
// only the input and output buffers it already holds.  For them the build
// scratch (centroid bounds, radix-sort ping-pong buffers, digit table, scan
// totals) lives in one file-scope __device__ array below, sized for up to
// IPCB_LBVH_NOALLOC_MAX_PRIMS boxes.  Every GPU that loads this library holds
// that array until the process exits.
#include <mutex>

#include "common.cuh"
#include "sort.cuh"

namespace ipcb {
void set_error(const char* where, cudaError_t e);
void set_error_msg(const char* msg);
}  // namespace ipcb

namespace {

constexpr int kMaxPrims = IPCB_LBVH_NOALLOC_MAX_PRIMS;
// 256 B bounds + keys and values ping-pong + digit table [256][tiles] + scan
// totals, each rounded up to 256 B, plus slack
constexpr size_t kScratchBytes = 256 + 2 * (size_t)kMaxPrims * 4 +
                                 (size_t)256 * ((kMaxPrims + 2047) / 2048) * 4 + 4096;

static __device__ __align__(256) unsigned char g_lbvh_scratch[kScratchBytes];

// Device address of g_lbvh_scratch per device ordinal, as found by the last
// call made outside stream capture with that device current (in host code the
// symbol is only a host-side stand-in).  Calls outside capture look it up
// again, so the address follows the context that is current now (after a
// cudaDeviceReset, or in a context other than the primary one); a call inside
// capture takes the cached one.
constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

}  // namespace

extern "C" {

size_t ipcb_lbvh_build_noalloc_scratch_bytes(void) { return kScratchBytes; }

int ipcb_lbvh_build_noalloc(ipcb_lbvh* bvh, const float* lower, const float* upper, int n, ipcb_stream s) {
  if (n < 0) {
    ipcb::set_error_msg("ipcb_lbvh_build_noalloc: n is negative");
    return IPCB_E_ARG;
  }
  if (n > kMaxPrims) {
    ipcb::set_error_msg("ipcb_lbvh_build_noalloc: n exceeds IPCB_LBVH_NOALLOC_MAX_PRIMS (static scratch limit)");
    return IPCB_E_ARG;
  }
  if (!bvh || n > bvh->capacity) {
    ipcb::set_error_msg("ipcb_lbvh_build_noalloc: no hierarchy, or n exceeds its capacity");
    return IPCB_E_ARG;
  }
  if (ipcb_lbvh_build_workspace(n) > kScratchBytes) {
    ipcb::set_error_msg("ipcb_lbvh_build_noalloc: static scratch smaller than the build workspace");
    return IPCB_E_ARG;
  }
  if (n == 0) return ipcb_lbvh_build(bvh, lower, upper, 0, nullptr, 0, s);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    ipcb::set_error("ipcb_lbvh_build_noalloc: cudaGetDevice", e);
    return IPCB_E_CUDA;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing((cudaStream_t)s, &cs) != cudaSuccess) {
    cudaGetLastError();  // the query failed because capture is under way elsewhere: treat as capturing
    cs = cudaStreamCaptureStatusActive;
  }
  void* ws = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (cs == cudaStreamCaptureStatusNone) {
      e = cudaGetSymbolAddress(&ws, g_lbvh_scratch);
      if (e != cudaSuccess || !ws) {
        ipcb::set_error("ipcb_lbvh_build_noalloc: cudaGetSymbolAddress", e);
        return IPCB_E_CUDA;
      }
      if (dev < kMaxDevices) g_scratch_addr[dev] = ws;
    } else if (dev < kMaxDevices) {
      ws = g_scratch_addr[dev];
    }
  }
  if (!ws) {
    ipcb::set_error_msg(dev < kMaxDevices
                            ? "ipcb_lbvh_build_noalloc: first call on this device made inside stream capture; "
                              "call it once outside capture first"
                            : "ipcb_lbvh_build_noalloc: device ordinal >= 64 cannot be used inside stream capture");
    return IPCB_E_ARG;
  }
  return ipcb_lbvh_build(bvh, lower, upper, n, ws, kScratchBytes, s);
}

}  // extern "C"
