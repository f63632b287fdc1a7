// gdlog/engine.cuh — internals of the drop-in C++ API: the process-wide
// engine, error handling, and the probes that turn the program's __device__
// hooks into the column selections the C-ABI takes.
//
// Compile the program's .cu files with nvcc and -rdc=true (as the reference
// does, CMakeLists.txt:54-61) and link libgdlog_b200.so.  The probe kernels
// below are instantiated in the program's own translation units, so they
// call the program's hooks through the same device function pointers the
// reference's kernels would (src/relation.cu:268-276, 390-403).
#pragma once

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>

#include <cuda_runtime.h>

#include "../gdlog_b200.h"
#include "tuple.cuh"

namespace gdlog_compat {

inline gdl_engine *&engine_slot() {
  static gdl_engine *e = nullptr;
  return e;
}

// The reference aborts on any CUDA failure after printing it
// (include/exception.cuh:9-18).  This layer does the same by default;
// building with -DGDLOG_THROW turns failures into std::runtime_error.
inline void check(gdl_status s, const char *what) {
  if (s == GDL_OK) return;
  std::string msg = std::string("gdlog: ") + what + " failed: " + gdl_status_string(s) + ": " +
                    gdl_last_error(engine_slot());
#ifdef GDLOG_THROW
  throw std::runtime_error(msg);
#else
  fprintf(stderr, "%s\n", msg.c_str());
  exit((int)s);
#endif
}

// The engine every Relation and LIE of the process uses: device 0 (or the
// device current when it is first needed), its own stream.
inline gdl_engine *engine() {
  gdl_engine *&e = engine_slot();
  if (!e) {
    int dev = 0;
    cudaGetDevice(&dev);
    check(gdl_engine_create(dev, nullptr, &e), "gdl_engine_create");
  }
  return e;
}

// ---------------------------------------------------------------------------
// Hook probes.  A hook that only moves columns is recognised by running it
// on two sets of distinct sentinel values: output column j is input column
// k exactly when it shows the k-th sentinel of both sets.
// ---------------------------------------------------------------------------
constexpr column_type kProbeA[4] = {1000003ul, 2000029ul, 3000017ul, 4000037ul};
constexpr column_type kProbeB[4] = {5000011ul, 6000007ul, 7000003ul, 8000009ul};
constexpr column_type kUnset = 0xFFFFFFFFFFFFFFFFul;

__global__ void probe_generator(tuple_generator_hook h, column_type *buf) {
  // buf: [0..1] inner, [2..3] outer, [4..5] out  (set A), [6..11] set B
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    h(buf + 0, buf + 2, buf + 4);
    h(buf + 6, buf + 8, buf + 10);
  }
}

__global__ void probe_copy(tuple_copy_hook h, column_type *buf) {
  // buf: [0..1] src, [2..3] dst (set A), [4..5] src, [6..7] dst (set B)
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    h(buf + 0, buf + 2);
    h(buf + 4, buf + 6);
  }
}

__global__ void probe_predicate(tuple_predicate p, const column_type *rows, int n, int *out) {
  if (threadIdx.x == 0 && blockIdx.x == 0)
    for (int i = 0; i < n; i++) out[i] = p(const_cast<column_type *>(rows) + 2 * i) ? 1 : 0;
}

// Returns false when the hook computes values instead of moving columns.
inline bool decode_generator(tuple_generator_hook h, int32_t gen[2]) {
  column_type host[12];
  for (int i = 0; i < 4; i++) host[i] = kProbeA[i], host[6 + i] = kProbeB[i];
  host[4] = host[5] = host[10] = host[11] = kUnset;
  column_type *d = nullptr;
  if (cudaMalloc(&d, sizeof host) != cudaSuccess) return false;
  cudaMemcpy(d, host, sizeof host, cudaMemcpyHostToDevice);
  probe_generator<<<1, 1>>>(h, d);
  cudaError_t r = cudaMemcpy(host, d, sizeof host, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (r != cudaSuccess) return false;
  for (int j = 0; j < 2; j++) {
    gen[j] = -1;
    for (int k = 0; k < 4; k++)
      if (host[4 + j] == kProbeA[k] && host[10 + j] == kProbeB[k])
        gen[j] = k < 2 ? GDL_INNER(k) : GDL_OUTER(k - 2);
    if (gen[j] < 0) return false;
  }
  return true;
}

inline bool decode_copy(tuple_copy_hook h, int32_t gen[2]) {
  column_type host[8] = {kProbeA[0], kProbeA[1], kUnset, kUnset,
                         kProbeB[0], kProbeB[1], kUnset, kUnset};
  column_type *d = nullptr;
  if (cudaMalloc(&d, sizeof host) != cudaSuccess) return false;
  cudaMemcpy(d, host, sizeof host, cudaMemcpyHostToDevice);
  probe_copy<<<1, 1>>>(h, d);
  cudaError_t r = cudaMemcpy(host, d, sizeof host, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (r != cudaSuccess) return false;
  for (int j = 0; j < 2; j++) {
    gen[j] = -1;
    for (int k = 0; k < 2; k++)
      if (host[2 + j] == kProbeA[k] && host[6 + j] == kProbeB[k]) gen[j] = GDL_SRC(k);
    if (gen[j] < 0) return false;
  }
  return true;
}

// Classifies a predicate as t[0] <op> t[1] from its truth table; false if it
// is none of the six comparisons.
inline bool decode_predicate(tuple_predicate p, int32_t *kind) {
  const column_type rows[12] = {1, 2, 2, 1, 3, 3, 1000, 7, 7, 1000, 9, 9};
  column_type *d = nullptr;
  int *dout = nullptr;
  int out[6] = {0};
  if (cudaMalloc(&d, sizeof rows) != cudaSuccess) return false;
  if (cudaMalloc(&dout, sizeof out) != cudaSuccess) {
    cudaFree(d);
    return false;
  }
  cudaMemcpy(d, rows, sizeof rows, cudaMemcpyHostToDevice);
  probe_predicate<<<1, 1>>>(p, d, 6, dout);
  cudaError_t r = cudaMemcpy(out, dout, sizeof out, cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(dout);
  if (r != cudaSuccess) return false;
  // truth table on (lt, gt, eq) cases, twice
  struct {
    int kind, lt, gt, eq;
  } table[] = {{GDL_PRED_NE, 1, 1, 0}, {GDL_PRED_EQ, 0, 0, 1}, {GDL_PRED_LT, 1, 0, 0},
               {GDL_PRED_LE, 1, 0, 1}, {GDL_PRED_GT, 0, 1, 0}, {GDL_PRED_GE, 0, 1, 1}};
  for (auto &t : table)
    if (out[0] == t.lt && out[1] == t.gt && out[2] == t.eq && out[3] == t.gt && out[4] == t.lt &&
        out[5] == t.eq) {
      *kind = t.kind;
      return true;
    }
  return false;
}

}  // namespace gdlog_compat
