// gdlog/exception.cuh — checkCuda of the drop-in C++ API (same behaviour as
// the reference's include/exception.cuh:6-19: print, reset, exit).
#pragma once

#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

inline cudaError_t checkCuda(cudaError_t result) {
  if (result != cudaSuccess) {
    fprintf(stderr, "CUDA Runtime Error: %s\n", cudaGetErrorString(result));
    cudaDeviceReset();
    exit((int)result);
  }
  return result;
}
