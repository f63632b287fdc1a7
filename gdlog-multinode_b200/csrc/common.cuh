// common.cuh — device-side data layout and helpers of the fixpoint engine.
//
// Layout in HBM.  An arity-2 relation version (FULL, DELTA or NEWT) is one
// array of 64-bit keys, key = (c0 << 32) | c1.  For column values below
// 2^32 this is an order-isomorphism with the reference's unsigned
// lexicographic order over two u64 columns (include/tuple.cuh:106-126), so
// a sorted key array is exactly the reference's sorted tuple set, with no
// row-pointer indirection (the reference sorts arrays of row pointers with
// a dereferencing comparator, src/relation.cu:576-578).
//
// Every array lives behind a device-resident descriptor (DArr) whose count
// is read by the kernels themselves.  Nothing in an iteration needs a size
// on the host, so an iteration can be replayed from a CUDA graph with no
// host synchronisation.  Writes past a capacity are never made: the kernel
// records the capacity it needed and raises the overflow flag, the host
// grows the buffers and the iteration is run again from committed state.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gdl {

typedef unsigned long long u64;
typedef unsigned int u32;
typedef unsigned char u8;

constexpr int kWarp = 32;
constexpr int kMaxRels = 64;  // relations per engine (device table size)
constexpr u64 kNoTrace = ~0ull;

// ---------------------------------------------------------------------------
// Descriptors (device memory)
// ---------------------------------------------------------------------------
struct DArr {
  u64 *ptr;
  u64 n;    // elements present
  u64 cap;  // elements allocated
};

// Open-addressing index over one sorted key array: distinct c0 -> the run
// [start, start+len) of keys with that c0.  Replaces the reference's
// MEntity{hash, first row} table (include/relation.cuh:20-27,
// src/relation.cu:12-80), which stores only the run start and finds the run
// end by walking.  A slot is {c0, epoch, start, len}; it is live only when
// its epoch equals the index's epoch, so a rebuild never clears the table.
struct Index {
  uint4 *slots;
  u64 mask;       // slot count - 1 (power of two)
  u32 epoch;      // epoch of the entries that are live (0: never built)
  u32 hash_mode;  // 0: identity (c0 & mask), 1: 64-bit mixer
};

// Totals of one bitmap scan (dense.cuh).
struct BmScanRec {
  u64 total_a, total_b;  // list sizes
  u64 pop_g;             // popcount of NEWT (accumulated, reset by the write pass)
  u32 overflow;          // a list is too small
  u32 n_listed;          // dirty chunks listed by k_bm_dirty_chunks
};

// One instance of a batched LIE in the dense (bitmap) form: its rows start at
// word base_word, each 2^row_shift words long, n rows (= n local ids).
struct SegInfo {
  u64 base_word;
  u32 row_shift;
  u32 n;
};

// Device state of one relation.  `x` is committed state, `x_next` is what
// the running iteration builds; the commit kernel swaps them.
struct RelDev {
  DArr full, full_next;
  DArr delta, delta_next;
  DArr newt;  // NEWT accumulator: ops append, unsorted, may hold duplicates
  Index full_idx, full_idx_next;
  Index delta_idx, delta_idx_next;
  // tuple_counts visibility.  The reference zeroes a container's
  // tuple_counts in some early-exit paths (src/join.cu:38-45) while its rows
  // stay; ops see count * vis.  w_* are the working copies of an iteration.
  u32 full_vis, delta_vis;
  u32 w_full_vis, w_delta_vis;
  u64 c_newt_n;  // NEWT count seen by the last merge step (0: empty branch)
  u32 sorted_in_scratch;
  // set in an iteration where a join over static FULLs, skipped because an
  // earlier iteration of the LIE ran it, would have put tuples into this
  // NEWT (all of them already in FULL): NEWT counts as non-empty
  u32 newt_phantom;
  // Dense form (dense.cuh): FULL bitmap, NEWT bitmap and the dirty map of
  // NEWT (one bit per 64-word chunk), the tile counts / prefixes of this
  // relation's update scan and its record.
  u32 *bmF, *bmG;
  u8 *bmD;         // dirty map storage (one byte per 64-word chunk of bmG)
  u8 *dirty;       // bmD while the running LIE keeps a dirty map, else null
  u64 *tile_prefix;
  BmScanRec scan;
  u64 f_count;     // |FULL'| when the FULL list is not rebuilt every iteration
  u32 dense;       // the running LIE keeps this relation as bitmaps
  u32 full_lazy;   // FULL's list is materialised only when the LIE ends
  // Transposed bitmaps of pull-form joins (pull.cuh): DELTA (written by the
  // update step) and NEWT (written before the join that reads it), read as
  // outers; and NEWT's transposed twin that joins with a transposed output
  // write (folded into NEWT after each such join, zero between them).
  u32 *bmDT, *bmGT, *bmOT;
  // DELTA's rows as they are, for row-gather joins that read DELTA (pull.cuh)
  u32 *bmDN;
};

// Loop control of a running fixpoint (one per engine, device memory).
struct Ctl {
  u32 done;      // the LIE reached its fixpoint or max_iteration
  u32 pause;     // this launch batch reached its iteration budget
  u32 overflow;  // some capacity was too small; iteration not committed
  u32 timeout;   // a bounded wait gave up
  u32 oob;       // a write was dropped by a bounds check (must stay 0)
  u32 cond_set;  // graph conditional handle is valid
  u32 overflow_stage;  // 1: the overflow came from a dense update scan
  u32 pad_ctl;
  u32 spin_limit;  // polls a bounded wait makes before it gives up (timeout)
  u32 test_wait;   // nonzero: k_begin waits this many polls on `never` (tests)
  u32 never;       // a flag no kernel sets
  u32 pad_ctl2;
  u64 iteration;     // iteration_counter of the reference loop
  u64 stop_at;       // pause when iteration reaches this
  u64 max_iteration; // LIE::max_iteration
  u64 generation;    // monotonic build counter (index epochs)
  u64 trace_base;    // iteration number of trace row 0
  u64 trace_rows;    // capacity of the trace buffer in iterations
  unsigned long long cond_handle;  // cudaGraphConditionalHandle (while node)
  u64 need[3 * kMaxRels + 4];      // capacities needed after an overflow
  u64 prof[16];                    // algorithmic bytes moved, per ProfKind
};

// Kernel families for the per-kernel accounting.  Every kernel adds the
// algorithmic bytes of its launch (what the operation must read and write,
// not what this implementation happens to move) to Ctl::prof[kind].
enum ProfKind {
  kPSortHist = 0,  // k_sort_hist: 8n (16n when the whole sort is one tile)
  kPSortPass,      // k_sort_pass: 16n per digit pass
  kPMerge,         // k_merge_diff: 8(|NEWT|+|FULL|) read + 8(|U|+|D|) written
  kPIndex,         // k_index_build: 8n read + 16 per run inserted
  kPJoinCount,     // k_join_count: 8|outer| read + 16|outer| probe
  kPJoinMat,       // k_join_mat[_pred]: 16 per output + 24 per matched outer row
  kPCopy,          // k_copy: 16 per tuple; dense copies 8 per source tuple
  kPControl,       // k_begin / k_commit: 0
  kPBitmap,        // dense scans: bitmap words read/written + 8 per key listed
  kPKinds
};

__device__ __forceinline__ void prof_add(Ctl *c, int kind, u64 bytes) {
  if (bytes) atomicAdd(&c->prof[kind], bytes);
}

enum NeedSlot { kNeedNewt = 0, kNeedFull = 1, kNeedDelta = 2 };
__host__ __device__ inline int need_index(int rel, int kind) { return 3 * rel + kind; }

// ---------------------------------------------------------------------------
// Key helpers
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ u32 key_c0(u64 k) { return (u32)(k >> 32); }
__host__ __device__ __forceinline__ u32 key_c1(u64 k) { return (u32)k; }
__host__ __device__ __forceinline__ u64 make_key(u32 c0, u32 c1) {
  return ((u64)c0 << 32) | (u64)c1;
}

// splitmix64 finaliser (Steele, Lea, Flood 2014); also used by the digest.
__host__ __device__ __forceinline__ u64 mix64(u64 x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// Column selection (a tuple_generator_hook / tuple_copy_hook that only
// moves columns).  sel[j] indexes {inner.c0, inner.c1, outer.c0, outer.c1}
// for a join and {src.c0, src.c1} for a copy.
struct Sel2 {
  int s0, s1;
};
__device__ __forceinline__ u32 pick4(int s, u64 a, u64 b) {
  return s == 0 ? key_c0(a) : s == 1 ? key_c1(a) : s == 2 ? key_c0(b) : key_c1(b);
}
__device__ __forceinline__ u64 gen_join(Sel2 g, u64 inner, u64 outer) {
  return make_key(pick4(g.s0, inner, outer), pick4(g.s1, inner, outer));
}

// Arity 3 (a third, dependent column such as a path length; the reference's
// test/path_length.cu).  A tuple (c0, c1, c2) is the key
// c0 << 32 | c1 << k2 | c2: column 0 keeps the high half, so index builds
// and join probes read it as for arity 2, and keys still sort in the
// lexicographic order of the tuples (include/tuple.cuh:106-126) when
// c1 < 2^(32-k2) and c2 < 2^k2.
__host__ __device__ __forceinline__ u32 key_col(u64 k, int arity, int j, int k2) {
  if (j == 0) return (u32)(k >> 32);
  const u32 lo = (u32)k;
  if (arity == 2) return lo;
  return j == 1 ? (lo >> k2) : (lo & ((1u << k2) - 1u));
}

// General tuple generator: output column j is column src[j] of the inner /
// source tuple (0..2) or of the outer tuple (16..18), plus add[j] (hooks
// such as path_length's outer[2] + 1, recognised as a column plus a
// constant).
struct GenSpec {
  int src[3];
  u32 add[3];
  int out_arity, in_arity, outer_arity;
  int k2;  // bits of column 2 in arity-3 keys
};

// The key of the generated tuple; a value that does not fit its column
// sets Ctl::oob bit 32768 (the fixpoint then fails) and yields key 0.
__device__ __forceinline__ u64 gen_spec(const GenSpec &g, u64 inner, u64 outer, u32 *oob) {
  u64 v[3] = {0, 0, 0};
  for (int j = 0; j < g.out_arity; j++) {
    const int s = g.src[j];
    const u64 x = s < 16 ? key_col(inner, g.in_arity, s, g.k2)
                         : key_col(outer, g.outer_arity, s - 16, g.k2);
    v[j] = x + g.add[j];
  }
  bool fits;
  u64 k;
  if (g.out_arity == 2) {
    fits = ((v[0] | v[1]) >> 32) == 0;
    k = (v[0] << 32) | v[1];
  } else {
    fits = (v[0] >> 32) == 0 && (v[1] >> (32 - g.k2)) == 0 && (v[2] >> g.k2) == 0;
    k = (v[0] << 32) | (v[1] << g.k2) | v[2];
  }
  if (!fits) {
    atomicOr(oob, 32768u);
    return 0;
  }
  return k;
}

// Predicate on the generated tuple (tuple_predicate): t[a] op t[b].
struct Pred {
  int kind, a, b;
};
__device__ __forceinline__ bool pred_ok(Pred p, u64 t) {
  if (p.kind == 0) return true;
  u32 x = p.a == 0 ? key_c0(t) : key_c1(t);
  u32 y = p.b == 0 ? key_c0(t) : key_c1(t);
  switch (p.kind) {
    case 1: return x != y;
    case 2: return x == y;
    case 3: return x < y;
    case 4: return x <= y;
    case 5: return x > y;
    default: return x >= y;
  }
}

__device__ __forceinline__ bool ctl_stop(const Ctl *c) {
  return c->done | c->pause | c->overflow | c->timeout;
}

// ---------------------------------------------------------------------------
// Decoupled look-back (Merrill & Garland 2016) for one u64 value per tile.
// A tile publishes its aggregate, later its inclusive prefix, each in its
// own slot, then a flag word [31:2] launch generation, [1:0] state (1
// aggregate, 2 inclusive).  Words of another generation read as "not
// ready", so the arrays are never cleared.  Every wait is bounded: after
// ctl->spin_limit polls (default kSpinLimit) the waiter raises ctl->timeout
// and returns, and every
// scatter that uses the result is bounds-checked, so a stuck predecessor
// cannot hang or fault the GPU.
// ---------------------------------------------------------------------------
constexpr u32 kSpinLimit = 1u << 22;

struct Lb {
  u32 *flag;
  u64 *agg;
  u64 *inc;
};

__device__ __forceinline__ void lb_publish(Lb lb, long long tile, u32 gen, bool inclusive, u64 v) {
  if (inclusive)
    lb.inc[tile] = v;
  else
    lb.agg[tile] = v;
  __threadfence();
  atomicExch(&lb.flag[tile], ((gen & 0x3FFFFFFFu) << 2) | (inclusive ? 2u : 1u));
}

// Warp-cooperative look-back by the calling warp (all 32 lanes) for tile
// `tile`; returns the exclusive prefix to every lane.
__device__ __forceinline__ u64 lb_warp_prefix(Lb lb, long long tile, u32 gen, Ctl *ctl) {
  const int lane = threadIdx.x & 31;
  const u32 g = gen & 0x3FFFFFFFu;
  u64 prefix = 0;
  long long base = tile - 1;
  u32 spins = 0;
  while (base >= 0) {
    long long t = base - lane;
    u32 f = 0;
    bool ready = true;
    if (t >= 0) {
      f = *((volatile u32 *)&lb.flag[t]);
      ready = (f >> 2) == g && (f & 3u);
    }
    if (__all_sync(0xffffffffu, ready) == 0) {
      if (++spins > ctl->spin_limit) {
        if (lane == 0) atomicOr(&ctl->timeout, 1u);
        return prefix;
      }
      continue;
    }
    __threadfence();
    bool inc = t >= 0 && (f & 2u);
    unsigned incmask = __ballot_sync(0xffffffffu, inc);
    int first_inc = incmask ? __ffs(incmask) - 1 : 32;  // nearest inclusive
    u64 v = 0;
    if (t >= 0 && lane <= first_inc)
      v = inc ? *((volatile u64 *)&lb.inc[t]) : *((volatile u64 *)&lb.agg[t]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    prefix += v;
    if (incmask) break;
    base -= 32;
  }
  return prefix;
}

// Per-launch bookkeeping of a look-back kernel: dynamic tile counter,
// finished-block counter and the generation tag.  The last block to finish
// resets the counters and bumps the generation for the next launch.
struct LaunchRec {
  u32 tile_ctr;
  u32 done_ctas;
  u32 gen;
  u32 pad;
};

__device__ __forceinline__ bool launch_rec_finish(LaunchRec *r) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    u32 prev = atomicAdd(&r->done_ctas, 1u);
    s_last = prev == gridDim.x - 1;
    if (s_last) {
      r->tile_ctr = 0;
      r->done_ctas = 0;
      r->gen = r->gen + 1;
      __threadfence();
    }
  }
  __syncthreads();
  return s_last;
}

// Grab the next tile for this block (thread 0 grabs, all threads get it).
__device__ __forceinline__ long long grab_tile(LaunchRec *r, long long *s_slot) {
  __syncthreads();
  if (threadIdx.x == 0) *s_slot = (long long)atomicAdd(&r->tile_ctr, 1u);
  __syncthreads();
  return *s_slot;
}

// Block-wide exclusive scan of one u64 per thread (BLOCK threads).
template <int BLOCK>
__device__ __forceinline__ u64 block_excl_scan(u64 v, u64 *s_warp, u64 *total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u64 x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    u64 y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    u64 w = lane < BLOCK / 32 ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      u64 y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    if (lane < BLOCK / 32) s_warp[lane] = w;  // inclusive per warp
  }
  __syncthreads();
  u64 warp_excl = warp ? s_warp[warp - 1] : 0;
  *total = s_warp[BLOCK / 32 - 1];
  __syncthreads();
  return warp_excl + x - v;
}

}  // namespace gdl
