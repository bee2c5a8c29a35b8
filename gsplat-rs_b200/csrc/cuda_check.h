// CUDA runtime error check for host code: throws gsr::Error(Internal).
#pragma once

#include <cuda_runtime.h>
#include <string>

#include "gsr_host.h"

#define GSR_CUDA(expr)                                                                    \
  do {                                                                                    \
    cudaError_t err__ = (expr);                                                           \
    if (err__ != cudaSuccess)                                                             \
      throw ::gsr::Error(::gsr::Code::Internal, std::string("CUDA error: ") +             \
                                                    cudaGetErrorString(err__) + " (" #expr ")"); \
  } while (0)
