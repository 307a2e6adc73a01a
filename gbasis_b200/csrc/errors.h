// Error reporting shared by every translation unit of libgbx_eri.
#pragma once
#include <cuda_runtime.h>

#include "gbx_eri.h"

namespace gbx {
int set_error(int code, const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
}  // namespace gbx
