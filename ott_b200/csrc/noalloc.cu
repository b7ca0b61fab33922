// Sinkhorn solve for callers that cannot allocate device memory.
//
// Some callers own no allocator they may use at the point where they call
// the solver: a handler running inside a host framework that hands it only
// the input and output buffers (an XLA FFI handler gets its memory from
// XLA's allocator, and a cudaMalloc there would synchronise the device
// behind the framework's back), or a service that reserves its whole GPU
// memory budget once at start-up and must not grow it per request. For
// them ottb_sinkhorn_pointcloud_noalloc runs the same solve as
// ottb_sinkhorn_pointcloud with its workspace taken from a fixed array
// compiled into this library instead of from the caller.
//
// The array below lives in device memory of every GPU that loads the
// library, for as long as the process runs: OTTB_NOALLOC_SCRATCH_BYTES
// (16 MiB) per device.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/ott_b200.h"

static __device__ __align__(256) unsigned char g_noalloc_scratch[OTTB_NOALLOC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device. In host code
// the array's name is only a host-side stand-in, so the address must come
// from cudaGetSymbolAddress, with that device current. A call made outside
// stream capture looks it up again (cheap once the module is loaded), so a
// device reset, which reloads the module at a new address, never leaves a
// stale address behind; a call under capture uses the address of the last
// uncaptured call on that device, and fails without one.
int32_t scratch_address(cudaStream_t stream, void** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return OTTB_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return OTTB_ERR_NO_DEVICE;
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(stream, &cap) != cudaSuccess) return OTTB_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  if (cap == cudaStreamCaptureStatusNone) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return OTTB_ERR_CUDA;
    g_scratch_addr[dev] = p;
  } else if (g_scratch_addr[dev] == nullptr) {
    return OTTB_ERR_INVALID;  // first call on this device under capture
  }
  *out = g_scratch_addr[dev];
  return OTTB_OK;
}

}  // namespace

extern "C" int32_t ottb_sinkhorn_pointcloud_noalloc(const ottb_problem* problems,
                                                    int32_t num_problems, int32_t d,
                                                    const ottb_solver_cfg* cfg,
                                                    ottb_result* results, void* stream) {
  // Problems needing more scratch than the fixed array holds are refused
  // before anything is enqueued.
  const size_t need = ottb_sinkhorn_workspace_size(problems, num_problems, d, cfg);
  if (need > (size_t)OTTB_NOALLOC_SCRATCH_BYTES) return OTTB_ERR_WORKSPACE;
  void* scratch = nullptr;
  const int32_t st = scratch_address((cudaStream_t)stream, &scratch);
  if (st != OTTB_OK) return st;
  // The solve writes every word of its workspace it later reads (the call
  // header, and the split-arrival counters it clears with cudaMemsetAsync),
  // so what the previous call left in the array does not matter. Calls whose
  // work overlaps on the GPU share the array and race; the caller must order
  // them, e.g. by issuing them on one stream.
  return ottb_sinkhorn_pointcloud(problems, num_problems, d, cfg, results, scratch,
                                  (size_t)OTTB_NOALLOC_SCRATCH_BYTES, stream);
}
