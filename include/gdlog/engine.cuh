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
// k exactly when it shows the k-th sentinel of both sets.  A join hook may
// also add a constant to a column (path_length's outer[2] + 1): output j is
// input k plus c when it shows sentinel k + c in both sets.
// ---------------------------------------------------------------------------
constexpr column_type kProbeA[4] = {1000003ul, 2000029ul, 3000017ul, 4000037ul};
constexpr column_type kProbeB[4] = {5000011ul, 6000007ul, 7000003ul, 8000009ul};
constexpr column_type kUnset = 0xFFFFFFFFFFFFFFFFul;

__global__ void probe_generator(tuple_generator_hook h, column_type *buf) {
  // buf: [0..2] inner, [3..5] outer, [6..8] out (set A), [9..17] set B
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    h(buf + 0, buf + 3, buf + 6);
    h(buf + 9, buf + 12, buf + 15);
  }
}

constexpr column_type kProbe3A[6] = {1000003ul, 2000029ul, 3000017ul,
                                     4000037ul, 5000011ul, 6000007ul};
constexpr column_type kProbe3B[6] = {7000003ul, 8000009ul, 9000011ul,
                                     10000019ul, 11000027ul, 12000017ul};

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

// gen[0..out_arity) for a join hook over tuples of in_arity (inner) and
// outer_arity columns.  Returns false when the hook computes anything but a
// column, or a column plus a small constant.
inline bool decode_generator(tuple_generator_hook h, int in_arity, int outer_arity, int out_arity,
                             int32_t *gen) {
  column_type host[18];
  for (int i = 0; i < 3; i++) {
    host[i] = kProbe3A[i], host[3 + i] = kProbe3A[3 + i], host[6 + i] = kUnset;
    host[9 + i] = kProbe3B[i], host[12 + i] = kProbe3B[3 + i], host[15 + i] = kUnset;
  }
  column_type *d = nullptr;
  if (cudaMalloc(&d, sizeof host) != cudaSuccess) return false;
  cudaMemcpy(d, host, sizeof host, cudaMemcpyHostToDevice);
  probe_generator<<<1, 1>>>(h, d);
  cudaError_t r = cudaMemcpy(host, d, sizeof host, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (r != cudaSuccess) return false;
  for (int j = 0; j < out_arity; j++) {
    gen[j] = -1;
    for (int k = 0; k < 6; k++) {
      if ((k < 3 && k >= in_arity) || (k >= 3 && k - 3 >= outer_arity)) continue;
      const column_type a = host[6 + j], b = host[15 + j];
      if (a < kProbe3A[k] || b < kProbe3B[k]) continue;
      const column_type c = a - kProbe3A[k];
      if (c != b - kProbe3B[k] || c >= 500000ul) continue;
      gen[j] = GDL_PLUS(k < 3 ? GDL_INNER(k) : GDL_OUTER(k - 3), (int32_t)c);
    }
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
