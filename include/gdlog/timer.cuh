// gdlog/timer.cuh — KernelTimer of the drop-in C++ API (include/timer.cuh:5-30
// of the reference): a CUDA event pair on the legacy stream, in seconds.
#pragma once

#include <cuda_runtime.h>

struct KernelTimer {
  cudaEvent_t start, stop;
  KernelTimer() {
    cudaEventCreate(&start);
    cudaEventCreate(&stop);
  }
  ~KernelTimer() {
    cudaEventDestroy(start);
    cudaEventDestroy(stop);
  }
  void start_timer() { cudaEventRecord(start, 0); }
  void stop_timer() { cudaEventRecord(stop, 0); }
  float get_spent_time() {
    float ms = 0;
    cudaEventSynchronize(stop);
    cudaEventElapsedTime(&ms, start, stop);
    return ms / 1000.0f;
  }
};
