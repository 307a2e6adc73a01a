// Error reporting shared by every translation unit of libgbx_eri.
#pragma once
#include <cuda_runtime.h>

#include "gbx_eri.h"

namespace gbx {
int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
const char* gbx_last_error_str();  // message of the last failure on this thread

// Makes `dev` current for the scope, restoring the previous device.
struct DeviceGuardLite {
  int prev = -1;
  explicit DeviceGuardLite(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuardLite() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};
}  // namespace gbx
