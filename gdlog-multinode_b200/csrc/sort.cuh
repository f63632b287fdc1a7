// sort.cuh — onesweep LSD radix sort of packed tuple keys.
//
// Replaces thrust::sort(tuple_indexed_less) on row-pointer arrays
// (src/relation.cu:576-578), which compares two dereferenced rows per step.
// Here the keys themselves are sorted, least-significant digit first, with
// the single-pass "onesweep" scheme (Adinets & Merrill 2022):
//   1. k_sort_hist reads the keys once and builds the digit histograms of
//      every pass; its last block turns them into bucket offsets.
//   2. k_sort_pass, once per digit, ranks a tile of keys in shared memory,
//      obtains the tile's global offset per digit with a decoupled look-back
//      over the preceding tiles, and scatters the tile in one go (read 8n,
//      write 8n per pass).
// Only the significant bits are sorted: with column values < 2^kbits the
// order of key (c0<<32|c1) equals the order of the 2*kbits-bit value
// (c0<<kbits|c1), so ceil(2*kbits/8) passes suffice.
// Sizes are device-resident (DArr::n); n must stay below 2^30 (the status
// word keeps 30 bits of count).  A single tile (n <= kSortTile) is sorted
// entirely in shared memory by block 0 of k_sort_hist.
#pragma once

#include "common.cuh"

namespace gdl {

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096 keys
constexpr int kSortWarps = kSortBlock / 32;
// Digit width: 8 bits by default (kRadix buckets); the kernels are
// templates over the width (6, 8 or 10 bits: 64, 256 or 1024 buckets), a
// tuning choice (fewer, wider passes against larger histograms).
constexpr int kRadixBits = 8;
constexpr int kRadix = 1 << kRadixBits;
constexpr int kMaxRadix = 1024;
constexpr int kMaxPasses = 8;

struct SortArgs {
  const DArr *keys;   // input keys; keys->ptr is also the even-pass buffer
  u64 *buf0;          // == keys->ptr at enqueue time
  u64 *buf1;          // scratch (odd-pass buffer)
  u64 cap;            // capacity of both buffers
  int kbits;
  int passes;
  u32 *offsets;       // [kMaxPasses][kRadix] bucket counts -> offsets
  u32 *status;        // [passes][max_tiles][kRadix]: [31:30] flag, [29:0] count
  u64 max_tiles;
  u32 *counters;      // [0..passes) tile counters, [kMaxPasses] done blocks
  Ctl *ctl;
};

template <int BITS>
__device__ __forceinline__ u32 sort_vkey_digit(u64 k, int kbits, int pass) {
  u64 mask = (kbits >= 32) ? 0xFFFFFFFFull : ((1ull << kbits) - 1);
  u64 v = ((k >> 32) << kbits) | (k & mask);
  return (u32)(v >> (BITS * pass)) & ((1u << BITS) - 1u);
}

// Stable rank of the keys a block holds, for one digit position.  Keys are
// held warp-striped: warp w, lane l, item i holds tile element
// w*32*ITEMS + i*32 + l, so (warp, item, lane) order is input order.
// Returns, per item, the key's position in the digit-sorted tile; also
// leaves per-digit tile counts in s_cnt and exclusive digit starts in
// s_start.  Invalid keys (past n) get digit kRadix and no position.
template <int RADIX>
struct RankSmem {
  u32 whist[kSortWarps][RADIX + 1];
  u32 cnt[RADIX + 1];
  u32 start[RADIX + 1];
  u64 scan_tmp[kSortWarps];
};

// Exclusive scan of n (<= kSortBlock * PER) counts in shared memory into
// `out`, each thread PER consecutive ones; out[n] = the total.
template <int PER>
__device__ __forceinline__ void scan_counts(const u32 *cnt, u32 *out, int n, u64 *scan_tmp) {
  u32 c[PER];
  u64 v = 0;
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const int d = threadIdx.x * PER + j;
    c[j] = d < n ? cnt[d] : 0u;
    v += c[j];
  }
  u64 total;
  u64 ex = block_excl_scan<kSortBlock>(v, scan_tmp, &total);
#pragma unroll
  for (int j = 0; j < PER; j++) {
    const int d = threadIdx.x * PER + j;
    if (d < n) out[d] = (u32)ex;
    ex += c[j];
  }
  if (threadIdx.x == 0) out[n] = (u32)total;
}

template <int ITEMS, int RADIX>
__device__ __forceinline__ void rank_tile(const u32 (&digit)[ITEMS], u32 (&pos)[ITEMS],
                                          RankSmem<RADIX> &sm) {
  constexpr int kRadix = RADIX;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int d = threadIdx.x; d < kSortWarps * (kRadix + 1); d += blockDim.x)
    (&sm.whist[0][0])[d] = 0;
  __syncthreads();
  u32 rank[ITEMS];
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    u32 d = digit[i];
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int leader = 31 - __clz(peers);
    u32 before = __popc(peers & ((1u << lane) - 1u));
    u32 base = sm.whist[warp][d];
    __syncwarp();
    if (lane == leader) sm.whist[warp][d] = base + __popc(peers);
    __syncwarp();
    rank[i] = base + before;
  }
  __syncthreads();
  // Per digit: exclusive offsets across warps, tile count.
  for (int d = threadIdx.x; d <= kRadix; d += blockDim.x) {
    u32 acc = 0;
#pragma unroll
    for (int w = 0; w < kSortWarps; w++) {
      u32 c = sm.whist[w][d];
      sm.whist[w][d] = acc;
      acc += c;
    }
    sm.cnt[d] = acc;
  }
  __syncthreads();
  // Exclusive scan of the digit counts (digit kRadix, past n, excluded).
  scan_counts<(kRadix + kSortBlock - 1) / kSortBlock>(sm.cnt, sm.start, kRadix, sm.scan_tmp);
  __syncthreads();
#pragma unroll
  for (int i = 0; i < ITEMS; i++) {
    u32 d = digit[i];
    pos[i] = sm.start[d] + sm.whist[warp][d] + rank[i];
  }
}

template <int RADIX>
struct SortSmem {
  RankSmem<RADIX> rk;
  u64 keys[kSortTile];
  u32 gbase[RADIX];
  long long tile;
};

__device__ __forceinline__ void load_tile_keys(const u64 *src, u64 n, long long tile,
                                               u64 (&k)[kSortItems], bool (&valid)[kSortItems]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u64 base = (u64)tile * kSortTile + (u64)warp * 32 * kSortItems + lane;
#pragma unroll
  for (int i = 0; i < kSortItems; i++) {
    u64 idx = base + (u64)i * 32;
    valid[i] = idx < n;
    k[i] = valid[i] ? src[idx] : 0ull;
  }
}

// Block 0 sorts a single tile entirely in shared memory.
template <int BITS>
__device__ void small_sort(const SortArgs &a, u64 n, SortSmem<1 << BITS> &sm) {
  constexpr int kRadix = 1 << BITS;
  u64 k[kSortItems];
  bool valid[kSortItems];
  load_tile_keys(a.buf0, n, 0, k, valid);
  for (int p = 0; p < a.passes; p++) {
    u32 d[kSortItems], pos[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; i++)
      d[i] = valid[i] ? sort_vkey_digit<BITS>(k[i], a.kbits, p) : kRadix;
    rank_tile<kSortItems, kRadix>(d, pos, sm.rk);
#pragma unroll
    for (int i = 0; i < kSortItems; i++)
      if (valid[i]) sm.keys[pos[i]] = k[i];
    __syncthreads();
    // Reload in warp-striped order for the next pass.
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < kSortItems; i++) {
      u64 idx = (u64)warp * 32 * kSortItems + (u64)i * 32 + lane;
      valid[i] = idx < n;
      k[i] = valid[i] ? sm.keys[idx] : 0ull;
    }
    __syncthreads();
  }
  u64 *dst = (a.passes & 1) ? a.buf1 : a.buf0;
  // Keys are now sorted in smem order (the last reload used that order).
  for (u64 i = threadIdx.x; i < n; i += blockDim.x) {
    if (i < a.cap)
      dst[i] = sm.keys[i];
    else
      atomicOr(&a.ctl->oob, 1u);
  }
}

template <int BITS>
__global__ void __launch_bounds__(kSortBlock) k_sort_hist(SortArgs a) {
  constexpr int kRadix = 1 << BITS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SortSmem<kRadix> &sm = *reinterpret_cast<SortSmem<kRadix> *>(smem_raw);
  __shared__ u32 s_hist[kMaxPasses][kRadix];
  if (ctl_stop(a.ctl)) return;
  const u64 n = a.keys->n;
  if (n == 0) return;
  if (blockIdx.x == 0 && threadIdx.x == 0)
    prof_add(a.ctl, kPSortHist, n <= (u64)kSortTile ? 16 * n : 8 * n);
  if (n <= (u64)kSortTile) {
    if (blockIdx.x == 0) small_sort<BITS>(a, n, sm);
    return;
  }
  const u64 tiles = (n + kSortTile - 1) / kSortTile;
  if (tiles > a.max_tiles || n >= (1ull << 30)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctl->oob, 2u);
    return;
  }
  // Clear the look-back status of every pass for the tiles in use.
  const u64 words = (u64)a.passes * a.max_tiles * kRadix;
  for (u64 p = 0; p < (u64)a.passes; p++)
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < tiles * kRadix;
         i += (u64)gridDim.x * blockDim.x)
      a.status[p * a.max_tiles * kRadix + i] = 0;
  (void)words;
  for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) (&s_hist[0][0])[i] = 0;
  __syncthreads();
  // four keys in flight per thread: their loads are issued together ahead
  // of the shared-memory counts
  const u64 stride = (u64)gridDim.x * blockDim.x;
  u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    u64 k[4];
#pragma unroll
    for (int j = 0; j < 4; j++) k[j] = a.buf0[i + j * stride];
#pragma unroll
    for (int j = 0; j < 4; j++)
      for (int p = 0; p < a.passes; p++)
        atomicAdd(&s_hist[p][sort_vkey_digit<BITS>(k[j], a.kbits, p)], 1u);
  }
  for (; i < n; i += stride) {
    const u64 k = a.buf0[i];
    for (int p = 0; p < a.passes; p++)
      atomicAdd(&s_hist[p][sort_vkey_digit<BITS>(k, a.kbits, p)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < a.passes * kRadix; i += blockDim.x) {
    u32 v = (&s_hist[0][0])[i];
    if (v) atomicAdd(&a.offsets[i], v);
  }
  // The last block turns the counts into exclusive bucket offsets.
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&a.counters[kMaxPasses], 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  for (int p = 0; p < a.passes; p++) {
    // (through shared memory: the counts, then their exclusive offsets)
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x)
      sm.rk.cnt[d] = *((volatile u32 *)&a.offsets[p * kRadix + d]);
    __syncthreads();
    scan_counts<(kRadix + kSortBlock - 1) / kSortBlock>(sm.rk.cnt, sm.rk.start, kRadix,
                                                        sm.rk.scan_tmp);
    __syncthreads();
    for (int d = threadIdx.x; d < kRadix; d += blockDim.x) a.offsets[p * kRadix + d] = sm.rk.start[d];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    for (int p = 0; p < kMaxPasses; p++) a.counters[p] = 0;
    a.counters[kMaxPasses] = 0;
    __threadfence();
  }
}

template <int BITS>
__global__ void __launch_bounds__(kSortBlock) k_sort_pass(SortArgs a, int pass) {
  constexpr int kRadix = 1 << BITS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SortSmem<kRadix> &sm = *reinterpret_cast<SortSmem<kRadix> *>(smem_raw);
  if (ctl_stop(a.ctl)) return;
  const u64 n = a.keys->n;
  if (n <= (u64)kSortTile) return;
  const u64 tiles = (n + kSortTile - 1) / kSortTile;
  if (tiles > a.max_tiles || n >= (1ull << 30)) return;
  const u64 *src = (pass & 1) ? a.buf1 : a.buf0;
  u64 *dst = (pass & 1) ? a.buf0 : a.buf1;
  u32 *status = a.status + (u64)pass * a.max_tiles * kRadix;
  const u32 *offs = a.offsets + pass * kRadix;
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(a.ctl, kPSortPass, 16 * n);
  while (true) {
    __syncthreads();
    if (threadIdx.x == 0) sm.tile = (long long)atomicAdd(&a.counters[pass], 1u);
    __syncthreads();
    const long long tile = sm.tile;
    if (tile >= (long long)tiles) break;
    u64 k[kSortItems];
    bool valid[kSortItems];
    load_tile_keys(src, n, tile, k, valid);
    u32 d[kSortItems], pos[kSortItems];
#pragma unroll
    for (int i = 0; i < kSortItems; i++)
      d[i] = valid[i] ? sort_vkey_digit<BITS>(k[i], a.kbits, pass) : kRadix;
    rank_tile<kSortItems, kRadix>(d, pos, sm.rk);
    // Publish this tile's per-digit count, look back for the prefix (a
    // thread per digit, or per kRadix / kSortBlock digits in turn).
    for (int dg = threadIdx.x; dg < kRadix; dg += blockDim.x) {
      const u32 c = sm.rk.cnt[dg];
      u32 *st = status + (u64)tile * kRadix + dg;
      if (tile == 0) {
        atomicExch(st, (2u << 30) | c);
        sm.gbase[dg] = offs[dg];
      } else {
        atomicExch(st, (1u << 30) | c);
        u32 prefix = 0, spins = 0;
        for (long long t = tile - 1; t >= 0;) {
          u32 w = *((volatile u32 *)(status + (u64)t * kRadix + dg));
          u32 f = w >> 30;
          if (f == 0) {
            if (++spins > a.ctl->spin_limit) {
              atomicOr(&a.ctl->timeout, 1u);
              break;
            }
            continue;
          }
          prefix += w & 0x3FFFFFFFu;
          if (f == 2) break;
          t--;
        }
        __threadfence();
        atomicExch(st, (2u << 30) | ((prefix + c) & 0x3FFFFFFFu));
        sm.gbase[dg] = offs[dg] + prefix;
      }
    }
#pragma unroll
    for (int i = 0; i < kSortItems; i++)
      if (valid[i]) sm.keys[pos[i]] = k[i];
    __syncthreads();
    const u64 in_tile = min((u64)kSortTile, n - (u64)tile * kSortTile);
    for (u32 i = threadIdx.x; i < in_tile; i += blockDim.x) {
      u64 key = sm.keys[i];
      u32 dg = sort_vkey_digit<BITS>(key, a.kbits, pass);
      u64 g = (u64)sm.gbase[dg] + (i - sm.rk.start[dg]);
      if (g < n && g < a.cap)
        dst[g] = key;
      else
        atomicOr(&a.ctl->oob, 4u);
    }
  }
  // The last block of the last pass leaves the bookkeeping clean.
  if (pass == a.passes - 1) {
    __shared__ int s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(&a.counters[kMaxPasses], 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (s_last) {
      for (int i = threadIdx.x; i < kMaxPasses * kRadix; i += blockDim.x) a.offsets[i] = 0;
      if (threadIdx.x == 0) {
        for (int p = 0; p < kMaxPasses; p++) a.counters[p] = 0;
        a.counters[kMaxPasses] = 0;
      }
      __threadfence();
    }
  }
}

template <int BITS>
constexpr size_t sort_smem_bytes() {
  return sizeof(SortSmem<1 << BITS>);
}
constexpr size_t kSortSmemBytes = sort_smem_bytes<kRadixBits>();

}  // namespace gdl
