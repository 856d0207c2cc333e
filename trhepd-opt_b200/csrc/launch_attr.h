// Per-device launch attributes (host side).
//
// cudaFuncSetAttribute(cudaFuncAttributeMaxDynamicSharedMemorySize) is a setting of
// the current device: a process with contexts on several GPUs must set it on each
// of them before its first launch there.  SmemOptIn remembers, per device, the
// largest byte count already set for one kernel.
#pragma once
#include <cuda_runtime.h>

#include <mutex>

namespace trhepd {

class SmemOptIn {
 public:
  static constexpr int kMaxDevices = 64;
  // Raise `func`'s dynamic shared-memory limit on the current device to `bytes`
  // (once per device and size).
  cudaError_t ensure(const void* func, size_t bytes) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices)
      return cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    std::lock_guard<std::mutex> g(m_);
    if (set_[dev] >= bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) set_[dev] = bytes;
    return e;
  }
  // The byte count set on `dev` (0 if none); for tests of the per-device keying.
  size_t bytes_on(int dev) {
    std::lock_guard<std::mutex> g(m_);
    return (dev >= 0 && dev < kMaxDevices) ? set_[dev] : 0;
  }

 private:
  std::mutex m_;
  size_t set_[kMaxDevices] = {};
};

}  // namespace trhepd
