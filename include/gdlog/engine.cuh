// gdlog/engine.cuh — internals of the drop-in C++ API: the process-wide
// engine, error handling, the probes that turn the program's __device__
// hooks into the column selections the C-ABI takes, and the kernels that
// run any other hook through its function pointer.
//
// Compile the program's .cu files with nvcc and -rdc=true (as the reference
// does, CMakeLists.txt:54-61) and link libgdlog_b200.so.  The probe kernels
// and hook kernels below are instantiated in the program's own translation
// units, so they call the program's hooks through the same device function
// pointers the reference's kernels would (src/relation.cu:268-276, 390-403).
#pragma once

#include <cstdint>
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
// Hooks.  The reference calls a program's __device__ hooks through device
// function pointers once per candidate tuple (src/relation.cu:290-403).
// Most drivers' hooks only move columns (test/tc.cu:61-77, test/sg.cu:
// 58-88, test/cspa.cu:62-95), and the engine runs those as column
// selections in its own kernels, bitmaps included.  A hook is treated as a
// selection only if it agrees with one on every one of kProbeSamples
// randomised inputs (values across the whole 32-bit range, both orders of
// every pair of columns, equal columns, unwritten outputs filled with
// noise); a predicate likewise must agree with one comparison of two output
// columns on every sample.  Any other hook runs as the reference runs it:
// the engine hands each iteration's candidates to a kernel below,
// instantiated in the program's own translation unit, which calls the hook
// through its function pointer (gdl_lie_add_*_hooked).  GDLOG_EXACT_HOOKS=1
// sends every hook that way; GDLOG_HOOK_LOG=1 reports each decision.
// ---------------------------------------------------------------------------
constexpr int kProbeSamples = 256;

// Deterministic sample values: small, 20-bit, 32-bit and near 2^32, mixed
// per column (xorshift64*, Vigna 2016).
struct ProbeRng {
  uint64_t x = 0x9E3779B97F4A7C15ull;
  uint64_t next() {
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    return x * 0x2545F4914F6CDD1Dull;
  }
  column_type value() {
    const uint64_t r = next(), v = next();
    switch (r & 3) {
      case 0: return v % 64;
      case 1: return v % (1ull << 20);
      case 2: return v % (1ull << 32);
      default: return 0xFFFFFFFFull - v % 64;
    }
  }
};

namespace {

// buf: per sample 12 words: [0..3] inner / source, [4..7] outer, [8..11] out
__global__ void probe_join_hook(tuple_generator_hook h, column_type *buf, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h(buf + 12 * i, buf + 12 * i + 4, buf + 12 * i + 8);
}
__global__ void probe_copy_hook(tuple_copy_hook h, column_type *buf, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) h(buf + 12 * i, buf + 12 * i + 8);
}
__global__ void probe_pred_hook(tuple_predicate p, column_type *rows, int n, int *out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = p(rows + 4 * i) ? 1 : 0;
}

}  // namespace

// Runs the hook on the samples: buf is kProbeSamples x 12 words, filled by
// the caller; returns false on a CUDA error.
inline bool run_probe(bool join, void *hook, column_type *buf) {
  const size_t bytes = sizeof(column_type) * 12 * kProbeSamples;
  column_type *d = nullptr;
  if (cudaMalloc(&d, bytes) != cudaSuccess) return false;
  cudaMemcpy(d, buf, bytes, cudaMemcpyHostToDevice);
  if (join)
    probe_join_hook<<<(kProbeSamples + 127) / 128, 128>>>((tuple_generator_hook)hook, d,
                                                          kProbeSamples);
  else
    probe_copy_hook<<<(kProbeSamples + 127) / 128, 128>>>((tuple_copy_hook)hook, d,
                                                          kProbeSamples);
  const cudaError_t r = cudaMemcpy(buf, d, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  return r == cudaSuccess && cudaGetLastError() == cudaSuccess;
}

// Samples for a hook: column 0 of inner and outer equal (the join column;
// every candidate of a join has it), the rest independent; outputs noise.
inline void fill_samples(column_type *buf, ProbeRng &rng) {
  for (int i = 0; i < kProbeSamples; i++) {
    column_type *b = buf + 12 * i;
    for (int k = 0; k < 8; k++) b[k] = rng.value();
    b[4] = b[0];
    if (i % 8 == 1) b[5] = b[1];  // equal non-key columns now and then
    if (i % 8 == 2) b[1] = b[0];
    for (int k = 8; k < 12; k++) b[k] = rng.next();
  }
}

// Output column j as (input column, constant): src 0..3 inner / source,
// 16..19 outer.  -1 when no single column plus a constant below 2^23 fits
// every sample.
inline int32_t decode_column(const column_type *buf, int j, int in_arity, int outer_arity) {
  for (int side = 0; side < 2; side++) {
    const int arity = side ? outer_arity : in_arity;
    for (int k = 0; k < arity; k++) {
      const int off = side ? 4 + k : k;
      const column_type c = buf[8 + j] - buf[off];
      if (c >= (1ull << 23)) continue;
      bool all = true;
      for (int i = 1; i < kProbeSamples && all; i++)
        all = buf[12 * i + 8 + j] == buf[12 * i + off] + c;
      if (all) return GDL_PLUS(side ? GDL_OUTER(k) : GDL_INNER(k), (int32_t)c);
    }
  }
  return -1;
}

// gen[0..out_arity) for a join hook; false unless the hook is a column
// selection (plus constants) on every sample.
inline bool decode_generator(tuple_generator_hook h, int in_arity, int outer_arity, int out_arity,
                             int32_t *gen) {
  static column_type buf[12 * kProbeSamples];
  ProbeRng rng;
  fill_samples(buf, rng);
  if (!run_probe(true, (void *)h, buf)) return false;
  for (int j = 0; j < out_arity; j++)
    if ((gen[j] = decode_column(buf, j, in_arity, outer_arity)) < 0) return false;
  return true;
}

inline bool decode_copy(tuple_copy_hook h, int in_arity, int out_arity, int32_t *gen) {
  static column_type buf[12 * kProbeSamples];
  ProbeRng rng;
  fill_samples(buf, rng);
  if (!run_probe(false, (void *)h, buf)) return false;
  for (int j = 0; j < out_arity; j++)
    if ((gen[j] = decode_column(buf, j, in_arity, 0)) < 0) return false;
  return true;
}

// A predicate as t[a] <op> t[b] for two output columns; false if no single
// comparison agrees with it on every sample.
inline bool decode_predicate(tuple_predicate p, int arity, int32_t *kind, int32_t *pa,
                             int32_t *pb) {
  static column_type rows[4 * kProbeSamples];
  static int got[kProbeSamples];
  ProbeRng rng;
  for (int i = 0; i < kProbeSamples; i++) {
    column_type *t = rows + 4 * i;
    for (int k = 0; k < 4; k++) t[k] = rng.value();
    if (i % 4 == 1) t[1] = t[0];
    if (i % 8 == 2) t[2] = t[0];
    if (i % 8 == 3) t[2] = t[1];
  }
  column_type *d = nullptr;
  int *dout = nullptr;
  if (cudaMalloc(&d, sizeof rows) != cudaSuccess) return false;
  if (cudaMalloc(&dout, sizeof got) != cudaSuccess) {
    cudaFree(d);
    return false;
  }
  cudaMemcpy(d, rows, sizeof rows, cudaMemcpyHostToDevice);
  probe_pred_hook<<<(kProbeSamples + 127) / 128, 128>>>(p, d, kProbeSamples, dout);
  const cudaError_t r = cudaMemcpy(got, dout, sizeof got, cudaMemcpyDeviceToHost);
  cudaFree(d);
  cudaFree(dout);
  if (r != cudaSuccess || cudaGetLastError() != cudaSuccess) return false;
  for (int a = 0; a < arity; a++)
    for (int b = 0; b < arity; b++) {
      if (a == b) continue;
      for (int k = GDL_PRED_NE; k <= GDL_PRED_GE; k++) {
        bool all = true;
        for (int i = 0; i < kProbeSamples && all; i++) {
          const column_type x = rows[4 * i + a], y = rows[4 * i + b];
          const bool v = k == GDL_PRED_NE ? x != y : k == GDL_PRED_EQ ? x == y
                       : k == GDL_PRED_LT ? x < y : k == GDL_PRED_LE ? x <= y
                       : k == GDL_PRED_GT ? x > y : x >= y;
          all = v == (got[i] != 0);
        }
        if (all) {
          *kind = k;
          *pa = a;
          *pb = b;
          return true;
        }
      }
    }
  return false;
}

// -- the exact path: hooks through their function pointers ----------------

__device__ __forceinline__ void hook_unpack(uint64_t k, int arity, int k2, column_type *t) {
  t[0] = k >> 32;
  const uint64_t lo = k & 0xFFFFFFFFull;
  if (arity == 2) {
    t[1] = lo;
  } else if (arity == 3) {
    t[1] = lo >> k2;
    t[2] = lo & ((1ull << k2) - 1);
  } else {
    t[1] = lo;
  }
}

// The engine's packed key of an output tuple; false if a value does not
// fit its column.
__device__ __forceinline__ bool hook_pack(const column_type *t, int arity, int k2, uint64_t *key) {
  if (arity == 2) {
    if ((t[0] | t[1]) >> 32) return false;
    *key = t[0] << 32 | t[1];
    return true;
  }
  if ((t[0] >> 32) || (t[1] >> (32 - k2)) || (t[2] >> k2)) return false;
  *key = t[0] << 32 | t[1] << k2 | t[2];
  return true;
}

// Append the kept keys of a warp: one atomicAdd per warp reserves room.
__device__ __forceinline__ void hook_append(const gdl_hook_work &w, bool keep, uint64_t key) {
  const unsigned m = __ballot_sync(0xffffffffu, keep);
  if (!m) return;
  const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
  unsigned long long at = 0;
  if (lane == leader)
    at = atomicAdd(reinterpret_cast<unsigned long long *>(&w.state->written),
                   (unsigned long long)__popc(m));
  at = __shfl_sync(0xffffffffu, at, leader);
  if (keep) {
    const uint64_t pos = w.state->base + at + __popc(m & ((1u << lane) - 1u));
    if (pos < w.out->cap)
      w.out->ptr[pos] = key;
    else
      atomicOr(w.error, 128u);
  }
}

namespace {

// get_join_result (src/relation.cu:290-373): every candidate (inner row,
// outer row) through tp_gen, kept when tp_pred accepts the result.
__global__ void k_run_join_hooks(gdl_hook_work w, tuple_generator_hook gen,
                                 tuple_predicate pred) {
  if (w.state->skip) return;
  const uint64_t total = w.state->total, nrec = w.state->records;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t p0 = (uint64_t)blockIdx.x * blockDim.x; p0 < total; p0 += stride) {
    const uint64_t p = p0 + threadIdx.x;
    bool keep = false;
    uint64_t key = 0;
    if (p < total) {
      uint64_t lo = 0, hi = nrec;  // last record with rec_offset <= p
      while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (w.rec_offset[mid] <= p)
          lo = mid;
        else
          hi = mid;
      }
      column_type in[4] = {0, 0, 0, 0}, out_t[4] = {0, 0, 0, 0}, res[4] = {0, 0, 0, 0};
      hook_unpack(w.rows->ptr[w.rec_start[lo] + (p - w.rec_offset[lo])], w.in_arity, w.k2, in);
      hook_unpack(w.rec_key[lo], w.outer_arity, w.k2, out_t);
      gen(in, out_t, res);
      keep = pred == nullptr || pred(res);
      if (keep && !hook_pack(res, w.out_arity, w.k2, &key)) {
        atomicOr(w.error, 32768u);
        keep = false;
      }
    }
    hook_append(w, keep, key);
  }
}

// get_copy_result (src/relation.cu:390-403): every source row through the
// copy hook (the predicate is not applied, as in the reference).
__global__ void k_run_copy_hook(gdl_hook_work w, tuple_copy_hook h) {
  if (w.state->skip) return;
  const uint64_t total = w.state->total;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t p0 = (uint64_t)blockIdx.x * blockDim.x; p0 < total; p0 += stride) {
    const uint64_t p = p0 + threadIdx.x;
    bool keep = false;
    uint64_t key = 0;
    if (p < total) {
      column_type in[4] = {0, 0, 0, 0}, res[4] = {0, 0, 0, 0};
      hook_unpack(w.rows->ptr[p], w.in_arity, w.k2, in);
      h(in, res);
      keep = hook_pack(res, w.out_arity, w.k2, &key);
      if (!keep) atomicOr(w.error, 32768u);
    }
    hook_append(w, keep, key);
  }
}

}  // namespace

struct JoinHooks {
  tuple_generator_hook gen;
  tuple_predicate pred;
};

// gdl_hook_launch callbacks: enqueue the kernels above on the engine stream.
static inline void launch_join_hooks(void *ctx, const gdl_hook_work *w, void *stream) {
  const JoinHooks *h = static_cast<const JoinHooks *>(ctx);
  k_run_join_hooks<<<w->sms * 8, 256, 0, static_cast<cudaStream_t>(stream)>>>(*w, h->gen,
                                                                             h->pred);
}
static inline void launch_copy_hook(void *ctx, const gdl_hook_work *w, void *stream) {
  k_run_copy_hook<<<w->sms * 8, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      *w, *static_cast<const tuple_copy_hook *>(ctx));
}

inline bool exact_hooks() { return getenv("GDLOG_EXACT_HOOKS") != nullptr; }
inline void log_hook(const char *op, const char *how) {
  if (getenv("GDLOG_HOOK_LOG")) fprintf(stderr, "gdlog: %s hooks -> %s\n", op, how);
}

}  // namespace gdlog_compat
