// exchange.cuh — grouping rows by owning rank for the partitioned fixpoint.
//
// A partitioned fixpoint (one relation hash-partitioned over the ranks,
// id v owned by rank v % world) sends every candidate row to the owner of
// one of its columns once per pass.  These kernels group a device array of
// rows by destination, so that the collective (an all-to-all with one
// contiguous block per destination) reads them where they are:
//   k_part_count    per-destination counts (a shared histogram per block)
//   k_part_offsets  their exclusive prefix, the scatter cursors (one thread)
//   k_part_scatter  each row to its destination's block (a cursor per
//                   destination; the order inside a block is not kept —
//                   the receiver sorts and deduplicates)
#pragma once

#include "common.cuh"

namespace gdl {

constexpr int kPartMaxWorld = 1024;

__global__ void __launch_bounds__(256) k_part_count(const u64 *rows, u64 n, int col, u32 world,
                                                    u64 *counts) {
  __shared__ u32 s_cnt[kPartMaxWorld];
  for (u32 d = threadIdx.x; d < world; d += blockDim.x) s_cnt[d] = 0;
  __syncthreads();
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    atomicAdd(&s_cnt[rows[2 * i + col] % world], 1u);
  __syncthreads();
  for (u32 d = threadIdx.x; d < world; d += blockDim.x)
    if (s_cnt[d]) atomicAdd(reinterpret_cast<unsigned long long *>(&counts[d]), (u64)s_cnt[d]);
}

__global__ void k_part_offsets(const u64 *counts, u32 world, u64 *cursor) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  u64 acc = 0;
  for (u32 d = 0; d < world; d++) {
    cursor[d] = acc;
    acc += counts[d];
  }
}

__global__ void __launch_bounds__(256) k_part_scatter(const u64 *rows, u64 n, int col, u32 world,
                                                      u64 *cursor, u64 *out) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 c0 = rows[2 * i], c1 = rows[2 * i + 1];
    const u32 d = (u32)((col ? c1 : c0) % world);
    const u64 p = atomicAdd(reinterpret_cast<unsigned long long *>(&cursor[d]), 1ull);
    if (p < n) {
      out[2 * p] = c0;
      out[2 * p + 1] = c1;
    }
  }
}

}  // namespace gdl
