// Reference-surface shim: the fatal CUDA check of src/core/cuda_check.hpp:7-39
// (print and exit 1), for driver code that calls the CUDA runtime itself.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#define WFE_CUDA_CHECK(call)                                                             \
  do {                                                                                   \
    cudaError_t wfe_e_ = (call);                                                         \
    if (wfe_e_ != cudaSuccess) {                                                         \
      std::fprintf(stderr, "CUDA error %s at %s:%d: %s\n", cudaGetErrorName(wfe_e_),     \
                   __FILE__, __LINE__, cudaGetErrorString(wfe_e_));                      \
      std::exit(1);                                                                      \
    }                                                                                    \
  } while (0)

namespace wfe {
// launches happen inside the library, which reports its own errors
inline void check_kernel(const char*) {}
}  // namespace wfe
