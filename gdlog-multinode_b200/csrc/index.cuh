// index.cuh — open-addressing hash index over a sorted relation version.
//
// Replaces init_index_map + calculate_index_hash (src/relation.cu:12-80,
// 124-137).  The reference inserts every row and converges each slot, by
// CAS, to the smallest row index of its key run; a probe then walks the
// rows until the key changes (src/relation.cu:259-284).  Here only the
// first row of each run inserts, and the slot stores the whole run
// (start, len), found by a galloping search over the sorted keys, so a
// probe is one 16-byte load and the join's count pass never touches the
// inner rows.
//
// Slots are 16 bytes {c0, epoch, start, len}.  A slot is live only if its
// epoch equals the index's epoch; each build uses a fresh epoch, so the
// table is never cleared.  hash_mode 0 is the identity hash c0 & mask (used
// when the table holds a slot for every possible c0, i.e. no collisions at
// all); mode 1 is a 64-bit mixer with linear probing, inserted with a
// compare-and-swap on the (c0, epoch) word.  The table has at least twice
// as many slots as distinct keys, so probes always meet an empty slot.
#pragma once

#include "common.cuh"

namespace gdl {

constexpr int kIndexBlock = 256;

__device__ __forceinline__ u64 index_home(const Index &ix, u32 c0) {
  return ix.hash_mode == 0 ? ((u64)c0 & ix.mask) : (mix64((u64)c0) & ix.mask);
}

// Probe: returns len (0 when absent) and the run start.
__device__ __forceinline__ u32 index_probe(const Index &ix, u32 c0, u32 *start) {
  u64 h = index_home(ix, c0);
  for (u64 step = 0; step <= ix.mask; step++) {
    uint4 s = __ldg(reinterpret_cast<const uint4 *>(ix.slots) + h);
    if (s.y != ix.epoch) return 0;
    if (s.x == c0) {
      *start = s.z;
      return s.w;
    }
    if (ix.hash_mode == 0) return 0;
    h = (h + 1) & ix.mask;
  }
  return 0;
}

__device__ __forceinline__ void index_insert(const Index &ix, u32 epoch, u32 c0, u32 start,
                                             u32 len, Ctl *ctl) {
  u64 h = index_home(ix, c0);
  const unsigned long long mine = ((unsigned long long)epoch << 32) | c0;
  for (u64 step = 0; step <= ix.mask; step++) {
    unsigned long long *w = reinterpret_cast<unsigned long long *>(ix.slots + h);
    if (ix.hash_mode == 0) {
      ix.slots[h] = make_uint4(c0, epoch, start, len);
      return;
    }
    unsigned long long cur = *((volatile unsigned long long *)w);
    if ((u32)(cur >> 32) == epoch) {
      if ((u32)cur == c0) {  // same key, same build (a rerun of the iteration)
        ix.slots[h].z = start;
        ix.slots[h].w = len;
        return;
      }
      h = (h + 1) & ix.mask;
      continue;
    }
    unsigned long long old = atomicCAS(w, cur, mine);
    if (old == cur) {
      ix.slots[h].z = start;
      ix.slots[h].w = len;
      return;
    }
    // Lost the race for this slot: look at it again.
    step--;
  }
  atomicOr(&ctl->oob, 32u);  // table full: cannot happen at <= 1/2 load
}

// First position >= i whose c0 differs from c0(keys[i]) (keys sorted).
__device__ __forceinline__ u64 run_end(const u64 *keys, u64 n, u64 i) {
  const u32 c = key_c0(keys[i]);
  u64 lo = i + 1, step = 1;
  // Gallop to bracket the end, then binary search.
  u64 hi = lo;
  while (hi < n && key_c0(keys[hi]) == c) {
    lo = hi + 1;
    hi = i + (step <<= 1);
  }
  if (hi > n) hi = n;
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (key_c0(keys[mid]) == c)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Build `ix` over `arr` (sorted).  With only_if_nonempty set, the build is
// skipped when *only_if_nonempty == 0 (a FULL index is rebuilt only when
// the iteration produced a delta).
__global__ void __launch_bounds__(kIndexBlock) k_index_build(const DArr *arr, Index *ix,
                                                             const DArr *only_if_nonempty,
                                                             Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  if (only_if_nonempty && only_if_nonempty->n == 0) return;
  const u64 n = arr->n;
  const u32 epoch = (u32)(ctl->generation + 1);
  const Index local = *ix;
  if (blockIdx.x == 0 && threadIdx.x == 0) ix->epoch = epoch;
  const u64 *keys = arr->ptr;
  u32 inserted = 0;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    u64 k = keys[i];
    if (i == 0 || key_c0(keys[i - 1]) != key_c0(k)) {
      u64 e = run_end(keys, n, i);
      index_insert(local, epoch, key_c0(k), (u32)i, (u32)(e - i), ctl);
      inserted++;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) inserted += __shfl_xor_sync(0xffffffffu, inserted, o);
  if ((threadIdx.x & 31) == 0)
    prof_add(ctl, kPIndex, 16ull * inserted + (blockIdx.x == 0 && threadIdx.x == 0 ? 8 * n : 0));
}

}  // namespace gdl
