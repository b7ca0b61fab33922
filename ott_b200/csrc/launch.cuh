// Host helper shared by the translation units: the dynamic shared-memory
// limit of a kernel, raised once per (device, kernel) under a mutex. The
// attribute belongs to the current device's context, so a process that
// launches on several GPUs sets it on each; the first call on a device
// must come before any stream capture that launches the kernel.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <utility>

namespace ottb {

inline bool ensure_dynamic_smem(const void* fn, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, fn})) return true;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) !=
      cudaSuccess)
    return false;
  done.insert({dev, fn});
  return true;
}

}  // namespace ottb
