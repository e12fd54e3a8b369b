// pcg_device.h — the GPU of a handle made current for one call of the C ABI.
#pragma once

#include <cuda_runtime.h>

namespace pcg {

// Makes `device` current and restores the caller's device on destruction,
// so that one host thread may drive handles on several GPUs.  device < 0
// leaves the current device alone.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int device) {
    int cur = 0;
    if (device >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != device && cudaSetDevice(device) == cudaSuccess)
      prev = cur;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope&) = delete;
  DeviceScope& operator=(const DeviceScope&) = delete;
};

}  // namespace pcg
