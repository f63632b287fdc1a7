// tma.cuh — the square-domain bitmap passes of pull.cuh (update step, fold)
// with tiles moved by the Tensor Memory Accelerator.
//
// A 256 x 256-bit tile is 256 rows of 32 bytes.  Read and written by
// threads, each 32-byte row piece costs the L1 a request of its own (a warp
// touches 32 lines per instruction); the LDG/STG kernels of pull.cuh are
// bound by those requests.  Here one thread moves whole tiles between global
// and shared memory with cp.async.bulk.tensor (2-D tensor maps over the
// bitmap, box = 8 words x 256 rows), so the threads only touch shared
// memory: the tile's rows are read 16 bytes at a time, transposed in
// registers (transpose32) and exchanged through a padded shared buffer.
//
// Pipeline per block (a persistent grid, tiles t = blockIdx.x + k*gridDim.x):
// the loads of tiles k+1 .. k+ns-1 are in flight in the other input stages
// while tile k is processed; tile k's outputs are written into one of two
// output slots and stored with one bulk group after the block's barrier;
// before that barrier the issuing thread waits until the group of tile k-1
// has read its slot, so tile k+1 may overwrite it.  Every mbarrier wait is bounded (Ctl::spin_limit
// polls): a wait that gives up raises Ctl::timeout, the block stores
// nothing more, waits (bounded) for its loads in flight and its stores, and
// returns.  No multicast, no cluster: every load reads this GPU's memory.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "dense.cuh"
#include "pull.cuh"

namespace gdl {

constexpr int kTmaTile = 256 * 32;  // bytes of one 256 x 256-bit tile

// Tensor maps of one update pass: NEWT's tile source (the transposed twin,
// or the rows), FULL, and the DELTA outputs (rows, transposed).
struct UpdMaps {
  CUtensorMap nsrc, f, dn, dt;
};
struct FoldMaps {
  CUtensorMap src, dst;
};

__device__ __forceinline__ u32 smem_addr(const void *p) {
  return (u32)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(u64 *bar, u32 count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(u64 *bar, u32 bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
// Wait for the phase of `parity` to complete, at most `limit` polls.
__device__ __forceinline__ bool mbar_wait(u64 *bar, u32 parity, u32 limit) {
  for (u32 i = 0; i < limit; i++) {
    u32 done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
__device__ __forceinline__ void tma_load(void *dst, const CUtensorMap *map, int x, int y,
                                         u64 *bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_addr(dst)),
      "l"(map), "r"(x), "r"(y), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_store(const CUtensorMap *map, int x, int y, const void *src) {
  asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.tile.bulk_group [%0, {%1, %2}], [%3];" ::
                   "l"(map),
               "r"(x), "r"(y), "r"(smem_addr(src))
               : "memory");
}
__device__ __forceinline__ void tma_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the committed store groups have finished reading shared memory
__device__ __forceinline__ void tma_wait_read() {
  asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}
// ... and their writes are done
__device__ __forceinline__ void tma_wait_done() {
  asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}
// shared-memory writes of this thread, before the async proxy reads them
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void lds8(const u32 *p, u32 *v) {
  const uint4 x = reinterpret_cast<const uint4 *>(p)[0], y = reinterpret_cast<const uint4 *>(p)[1];
  v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w, v[4] = y.x, v[5] = y.y, v[6] = y.z, v[7] = y.w;
}
__device__ __forceinline__ void sts8(u32 *p, const u32 *v) {
  reinterpret_cast<uint4 *>(p)[0] = make_uint4(v[0], v[1], v[2], v[3]);
  reinterpret_cast<uint4 *>(p)[1] = make_uint4(v[4], v[5], v[6], v[7]);
}
__device__ __forceinline__ bool any8(const u32 *v) {
  return (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) != 0u;
}

// Per-warp flags of a tile, ORed over the block after its barrier (the
// slot's entries are rewritten every second tile, after a barrier that
// follows every read of them).
__device__ __forceinline__ u32 block_flags(u32 *s_wf, u32 f, int wid) {
  const u32 w = __reduce_or_sync(0xffffffffu, f);
  if ((threadIdx.x & 31) == 0) s_wf[wid] = w;
  __syncthreads();
  u32 r = 0;
#pragma unroll
  for (int i = 0; i < kTrBlock / 32; i++) r |= s_wf[i];
  return r;
}

// Input stages: loads run ns - 1 tiles ahead of the tile being processed.
constexpr int kTmaMaxStages = 4;
// Shared memory: dynamic, 1024-byte aligned by hand.  Update pass: ns
// stages of (NEWT, FULL) tiles, 2 output slots of (FULL', DELTA rows[,
// DELTA^T]), one zero tile, alignment slack.
__host__ __device__ constexpr u32 upd_tma_smem(int ns, int has_dt) {
  return ns * 2 * kTmaTile + 2 * (has_dt ? 3 : 2) * kTmaTile + kTmaTile + 1024;
}
// Fold: ns stages of the source tile (and the destination's, unless it is
// overwritten), 2 output slots, one zero tile.
__host__ __device__ constexpr u32 fold_tma_smem(int ns, int overwrite) {
  return ns * (overwrite ? 1 : 2) * kTmaTile + 2 * kTmaTile + kTmaTile + 1024;
}
// Stages that keep two blocks of 256 threads on an SM (static shared memory
// about 10 KB a block) for the update pass, three for an overwriting fold.
__host__ __device__ constexpr int upd_tma_stages(int has_dt) { return has_dt ? 2 : 3; }
__host__ __device__ constexpr int fold_tma_stages(int overwrite) { return overwrite ? 4 : 3; }

enum UpdFlag : u32 { kFAnyN = 1, kFAnyG = 2, kFFail = 4 };

// k_bm_update_t (pull.cuh) with TMA tiles.  gt: NEWT is the transposed
// twin (m.nsrc over it; cleared where it has bits); else NEWT is the row
// bitmap G (m.nsrc over G; cleared where it has bits).  has_dn / has_dt:
// write DELTA's rows / DELTA transposed (every word).  ns input stages.
__global__ void __launch_bounds__(kTrBlock, 2)
    k_bm_update_tma(BmScanArgs a, const __grid_constant__ UpdMaps m, int dk, int gt, int has_dn,
                    int has_dt, int ns) {
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ u32 s_t[256][9];
  __shared__ u32 s_wf[2][kTrBlock / 32];
  __shared__ __align__(8) u64 s_bar[kTmaMaxStages];
  __shared__ unsigned long long s_cnt[2];
  __shared__ int s_skip;
  if (threadIdx.x == 0) s_skip = ctl_stop(a.ctl) || write_gate_closed(a);
  __syncthreads();
  if (s_skip) return;
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tma_smem_raw) + 1023) & ~uintptr_t(1023));
  // stage s: NEWT tile at 2s, FULL tile at 2s + 1; output slot o from tile
  // 2 ns + o nout on; then the zero tile
  const int nout = has_dt ? 3 : 2;
  auto tile_at = [&](int i) { return reinterpret_cast<u32 *>(base + i * kTmaTile); };
  auto in_n = [&](int st) { return tile_at(2 * st); };
  auto in_f = [&](int st) { return tile_at(2 * st + 1); };
  auto out_f = [&](int o) { return tile_at(2 * ns + o * nout); };
  auto out_dn = [&](int o) { return tile_at(2 * ns + o * nout + 1); };
  auto out_dt = [&](int o) { return tile_at(2 * ns + o * nout + 2); };
  u32 *zero = tile_at(2 * ns + 2 * nout);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const u64 per = 1ull << (dk - 8);
  const u64 tiles = per * per;
  const u32 limit = a.ctl->spin_limit;
  for (int i = tid; i < kTmaTile / 16; i += kTrBlock)
    reinterpret_cast<uint4 *>(zero)[i] = make_uint4(0, 0, 0, 0);
  fence_async_smem();
  if (tid == 0) {
    for (int i = 0; i < ns; i++) mbar_init(&s_bar[i], 1);
    s_cnt[0] = s_cnt[1] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // the block's j-th tile is blockIdx.x + j gridDim.x, in stage j % ns;
  // its NEWT tile is (tr, tc) of G, or (tc, tr) of the twin
  const u64 mine = tiles > blockIdx.x ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto issue = [&](u64 j) {
    const u64 t = blockIdx.x + j * gridDim.x;
    const int tr = (int)(t / per), tc = (int)(t % per), st = (int)(j % ns);
    mbar_expect_tx(&s_bar[st], 2 * kTmaTile);
    if (gt)
      tma_load(in_n(st), &m.nsrc, tr * 8, tc * 256, &s_bar[st]);
    else
      tma_load(in_n(st), &m.nsrc, tc * 8, tr * 256, &s_bar[st]);
    tma_load(in_f(st), &m.f, tc * 8, tr * 256, &s_bar[st]);
  };
  if (tid == 0)
    for (u64 j = 0; j + 1 < (u64)ns && j < mine; j++) issue(j);
  u64 n_delta = 0, n_newt = 0, moved = 0;
  bool failed = false;
  u64 k = 0;
  for (; k < mine; k++) {
    const u64 t = blockIdx.x + k * gridDim.x;
    const int st = (int)(k % ns), slot = (int)(k & 1);
    const int tr = (int)(t / per), tc = (int)(t % per);
    // (stage (k + ns - 1) % ns held tile k - 1, read before the last barrier)
    if (tid == 0 && k + ns - 1 < mine) issue(k + ns - 1);
    const bool ok = mbar_wait(&s_bar[st], (u32)(k / ns) & 1u, limit);
    u32 v[8], g[8], f[8], d[8];
    lds8(in_n(st) + tid * 8, v);
    const bool any_n = any8(v);
    if (gt) {
      // the twin's rows are NEWT's columns: transpose (lane j of warp w,
      // word i: NEWT row 32 i + j, word w), unless the whole tile is zero
      // (the barrier also orders the last tile's reads of s_t)
      if (__syncthreads_or(any_n)) {
#pragma unroll
        for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(v[i], lane);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) g[i] = s_t[tid][i];
      } else {
#pragma unroll
        for (int i = 0; i < 8; i++) g[i] = 0;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) g[i] = v[i];
    }
    lds8(in_f(st) + tid * 8, f);
    const bool any_g = any8(g);
    u32 nd = 0, ng = 0;  // (at most 256 bits a thread)
#pragma unroll
    for (int i = 0; i < 8; i++) {
      d[i] = g[i] & ~f[i];
      nd += __popc(d[i]);
      ng += __popc(g[i]);
      f[i] |= g[i];
    }
    n_delta += nd;
    n_newt += ng;
    sts8(out_f(slot) + tid * 8, f);
    if (has_dn) sts8(out_dn(slot) + tid * 8, d);
    if (has_dt) {
      // DELTA transposed: its rows are this tile's columns (the reads of
      // s_t above are behind this barrier)
      const bool any_d = __syncthreads_or(any8(d));
      if (any_d) {
#pragma unroll
        for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(d[i], lane);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) d[i] = s_t[tid][i];
      }
      sts8(out_dt(slot) + tid * 8, d);
    }
    fence_async_smem();
    // before the barrier: the stores of the tile before have read their slot
    if (tid == 0) tma_wait_read();
    const u32 fl = block_flags(s_wf[slot], (any_n ? kFAnyN : 0u) | (any_g ? kFAnyG : 0u) |
                                               (ok ? 0u : kFFail),
                               wid);
    if (fl & kFFail) {
      failed = true;
      break;
    }
    if (tid == 0) {
      // FULL' where NEWT had bits; DELTA's tiles always (every word of
      // them is written); NEWT's tile cleared where it had bits
      if (fl & kFAnyG) tma_store(&m.f, tc * 8, tr * 256, out_f(slot));
      if (has_dn) tma_store(&m.dn, tc * 8, tr * 256, out_dn(slot));
      if (has_dt) tma_store(&m.dt, tr * 8, tc * 256, out_dt(slot));
      if (fl & kFAnyN) {
        if (gt)
          tma_store(&m.nsrc, tr * 8, tc * 256, zero);
        else
          tma_store(&m.nsrc, tc * 8, tr * 256, zero);
      }
      tma_commit();
    }
    moved += 2 * 32 + ((fl & kFAnyG) ? 32 : 0) + (has_dn ? 32 : 0) + (has_dt ? 32 : 0) +
             ((fl & kFAnyN) ? 32 : 0);
  }
  if (failed && tid == 0) {
    atomicOr(&a.ctl->timeout, 1u);
    // loads that may still be in flight into this block's shared memory:
    // tile k (whose wait gave up) and the ones issued after it (bounded)
    for (u64 j = k; j < k + ns - 1 && j < mine; j++)
      mbar_wait(&s_bar[j % ns], (u32)(j / ns) & 1u, limit);
  }
  if (tid == 0) tma_wait_done();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_delta += __shfl_xor_sync(0xffffffffu, n_delta, o);
    n_newt += __shfl_xor_sync(0xffffffffu, n_newt, o);
    moved += __shfl_xor_sync(0xffffffffu, moved, o);
  }
  if (lane == 0) {
    if (n_delta) atomicAdd(&s_cnt[0], (unsigned long long)n_delta);
    if (n_newt) atomicAdd(&s_cnt[1], (unsigned long long)n_newt);
    prof_add(a.ctl, kPBitmap, moved);
  }
  __syncthreads();
  if (tid == 0) {
    if (s_cnt[0]) atomicAdd(reinterpret_cast<unsigned long long *>(&a.rec->total_a), s_cnt[0]);
    if (s_cnt[1]) atomicAdd(reinterpret_cast<unsigned long long *>(&a.rec->pop_g), s_cnt[1]);
  }
  if (launch_rec_finish(a.lrec) && tid == 0) {
    *a.count_a = a.rec->total_a;
    *a.pop_g_out = a.rec->pop_g;
    a.rec->total_a = 0;
    a.rec->pop_g = 0;
  }
}

// k_bm_fold_t (pull.cuh) with TMA tiles: dst |= transpose(src) (or, with
// overwrite, dst := transpose(src), every word stored), src cleared where it
// has bits, the dirty map of dst set for its non-zero rows.  ns input stages.
__global__ void __launch_bounds__(kTrBlock, 2)
    k_bm_fold_tma(const __grid_constant__ FoldMaps m, u8 *dirty, int dk, int overwrite, int ns,
                  Ctl *ctl) {
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ u32 s_t[256][9];
  __shared__ u32 s_wf[2][kTrBlock / 32];
  __shared__ __align__(8) u64 s_bar[kTmaMaxStages];
  if (ctl_stop(ctl)) return;
  unsigned char *base = reinterpret_cast<unsigned char *>(
      (reinterpret_cast<uintptr_t>(tma_smem_raw) + 1023) & ~uintptr_t(1023));
  // stage s: source tile at ni s, destination tile at ni s + 1 (ni = 2
  // unless overwriting); output slot o at ni ns + o; then the zero tile
  const int ni = overwrite ? 1 : 2;
  auto tile_at = [&](int i) { return reinterpret_cast<u32 *>(base + i * kTmaTile); };
  auto in_s = [&](int st) { return tile_at(ni * st); };
  auto in_d = [&](int st) { return tile_at(ni * st + 1); };
  auto out = [&](int o) { return tile_at(ni * ns + o); };
  u32 *zero = tile_at(ni * ns + 2);
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int rs = dk - 5;
  const u64 per = 1ull << (dk - 8);
  const u64 tiles = per * per;
  const u32 limit = ctl->spin_limit;
  for (int i = tid; i < kTmaTile / 16; i += kTrBlock)
    reinterpret_cast<uint4 *>(zero)[i] = make_uint4(0, 0, 0, 0);
  fence_async_smem();
  if (tid == 0) {
    for (int i = 0; i < ns; i++) mbar_init(&s_bar[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // the block's j-th tile: src tile (tr, tc), dst tile (tc, tr)
  const u64 mine = tiles > blockIdx.x ? (tiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  auto issue = [&](u64 j) {
    const u64 t = blockIdx.x + j * gridDim.x;
    const int tr = (int)(t / per), tc = (int)(t % per), st = (int)(j % ns);
    mbar_expect_tx(&s_bar[st], ni * kTmaTile);
    tma_load(in_s(st), &m.src, tc * 8, tr * 256, &s_bar[st]);
    if (!overwrite) tma_load(in_d(st), &m.dst, tr * 8, tc * 256, &s_bar[st]);
  };
  if (tid == 0)
    for (u64 j = 0; j + 1 < (u64)ns && j < mine; j++) issue(j);
  u64 moved = 0;
  bool failed = false;
  u64 k = 0;
  for (; k < mine; k++) {
    const u64 t = blockIdx.x + k * gridDim.x;
    const int st = (int)(k % ns), slot = (int)(k & 1);
    const int tr = (int)(t / per), tc = (int)(t % per);
    if (tid == 0 && k + ns - 1 < mine) issue(k + ns - 1);
    const bool ok = mbar_wait(&s_bar[st], (u32)(k / ns) & 1u, limit);
    u32 v[8], q[8];
    lds8(in_s(st) + tid * 8, v);
    const bool any_s = __syncthreads_or(any8(v));  // (block-uniform)
    bool any_q = false;
    if (any_s) {
#pragma unroll
      for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(v[i], lane);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < 8; i++) q[i] = s_t[tid][i];
      any_q = any8(q);
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) q[i] = 0;
    }
    if (!overwrite) {
      u32 dd[8];
      lds8(in_d(st) + tid * 8, dd);
#pragma unroll
      for (int i = 0; i < 8; i++) q[i] |= dd[i];
      if (any_q && dirty)
        dirty[((((u64)tc * 256 + (u64)tid) << rs) + (u64)tr * 8) / kBmChunkWords] = 1;
    }
    sts8(out(slot) + tid * 8, q);
    fence_async_smem();
    if (tid == 0) tma_wait_read();
    const u32 fl = block_flags(s_wf[slot], (any_q ? kFAnyG : 0u) | (ok ? 0u : kFFail), wid);
    if (fl & kFFail) {
      failed = true;
      break;
    }
    if (tid == 0) {
      if (overwrite || (fl & kFAnyG)) tma_store(&m.dst, tr * 8, tc * 256, out(slot));
      if (any_s) tma_store(&m.src, tc * 8, tr * 256, zero);
      tma_commit();
    }
    moved += 32 + (overwrite ? 32 : 32 + ((fl & kFAnyG) ? 32 : 0)) + (any_s ? 32 : 0);
  }
  if (failed && tid == 0) {
    atomicOr(&ctl->timeout, 1u);
    for (u64 j = k; j < k + ns - 1 && j < mine; j++)
      mbar_wait(&s_bar[j % ns], (u32)(j / ns) & 1u, limit);
  }
  if (tid == 0) tma_wait_done();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
  if (lane == 0) prof_add(ctl, kPBitmap, moved);
}

}  // namespace gdl
