// dense.cuh — bitmap form of relation versions over a small key domain.
//
// When every column value is below 2^dk with 2*dk <= 32, the whole key
// domain of an arity-2 relation is 2^(2dk) bits (at most 512 MB), and a
// version of the relation can be held as a bitmap whose bit (c0, c1) sits in
// row c0.  Bit order is the reference's tuple order (include/tuple.cuh:
// 106-126), so compacting a bitmap gives the sorted, deduplicated tuple list
// directly.  This replaces, for such domains, the sort -> unique ->
// set_difference -> merge sequence of the reference's update step
// (src/lie.cu:122-185, src/relation.cu:405-521, src/join.cu:160-225):
//   * joins and copies set bits of the output relation's NEWT bitmap G with
//     fire-and-forget atomicOr (no return value, so no round trip), plus a
//     bit in a small dirty map (one bit per 64-word chunk of G);
//   * the update step reads only the dirty chunks of G: DELTA = G & ~F as a
//     sorted list, FULL |= G in place, G cleared.  A relation whose FULL
//     list is read during the loop also gets FULL' = F | G as a sorted list
//     and its run index from per-row popcounts (a full pass over F).
// A scan is three kernels: k_bm_tilecount (per 2048-word tile, clean tiles
// skipped by their dirty word), k_bm_scan (exclusive prefix of the tile
// counts, totals, capacity check) and k_bm_write.  All update relations are
// counted and checked before any of them is written (the write passes'
// capacity gate), so a
// capacity overflow leaves every bitmap untouched and the update step can
// simply run again after the lists grow.
//
// Batched form.  Many independent instances of one program can share one
// LIE: instance i owns the ids (i << S) | local, local < n_i, and its
// tuples keep both columns inside its own range.  The bitmap is then block
// diagonal: instance i has n_i rows of 2^row_shift words (the power of two
// at or above n_i / 32), starting at a tile-aligned word.  A DenseMap
// describes either layout; the square domain is the one-instance case.
#pragma once

#include "common.cuh"
#include "index.cuh"
#include "join.cuh"

namespace gdl {

constexpr int kBmBlock = 256;
constexpr int kBmWordsPerThread = 8;
constexpr int kBmTileWords = kBmBlock * kBmWordsPerThread;  // 2048 words = 65536 keys
constexpr int kBmChunkWords = 64;                          // dirty granularity (256 B)
constexpr int kDenseMaxDomainBits = 32;  // ids below 2^16: a row is one scan tile
constexpr int kMaxInstanceNodes = 1 << 16;  // a row is at most one scan tile

// Where a key lives in the bitmap: the tuple (c0, c1) of instance
// i = c0 >> seg_shift is bit (c1 & 31) of word
//   seg[i].base_word + (local(c0) << seg[i].row_shift) + (local(c1) >> 5).
struct DenseMap {
  const SegInfo *seg;     // one entry per instance
  const u32 *tile_inst;   // instance of each scan tile (null: all instance 0)
  u32 n_inst;
  int seg_shift;          // 31 for the square domain (every id is local)
  u64 words;              // total bitmap words (a multiple of kBmTileWords)
};

__device__ __forceinline__ bool dm_locate(const DenseMap &m, u64 key, u64 *word, u32 *bit) {
  const u32 c0 = key_c0(key), c1 = key_c1(key);
  const u32 i = c0 >> m.seg_shift;
  if (i >= m.n_inst || (c1 >> m.seg_shift) != i) return false;
  const u32 mask = (1u << m.seg_shift) - 1u;
  const u32 lx = c0 & mask, lz = c1 & mask;
  const SegInfo s = m.seg[i];
  if (lx >= s.n || lz >= s.n) return false;
  *word = s.base_word + ((u64)lx << s.row_shift) + (lz >> 5);
  *bit = lz & 31u;
  return true;
}

__device__ __forceinline__ u32 dm_tile_inst(const DenseMap &m, u64 tile) {
  return m.tile_inst ? m.tile_inst[tile] : 0u;
}

// The key of bit b of word w, w inside instance inst.
__device__ __forceinline__ u64 dm_key(const DenseMap &m, u32 inst, const SegInfo &s, u64 w, int b) {
  const u64 wl = w - s.base_word;
  const u32 lx = (u32)(wl >> s.row_shift);
  const u32 lz = (u32)(((wl & ((1ull << s.row_shift) - 1)) << 5) + (u64)b);
  const u32 hi = m.seg_shift >= 31 ? 0u : (inst << m.seg_shift);
  return make_key(hi | lx, hi | lz);
}

// The dirty map has one byte per 64-word chunk of NEWT, set with a plain
// store (no read-modify-write, so no contention between the many threads
// that touch one chunk).  It is only kept for large bitmaps; without it
// (null) every chunk counts as dirty.
__device__ __forceinline__ void bm_mark(u32 *bm, u8 *dirty, u64 w, u32 b) {
  // A reduction (red), not an atomic: the old value is never needed, so
  // the L2 does the OR without sending anything back.
  asm volatile("red.global.or.b32 [%0], %1;" ::"l"(bm + w), "r"(1u << b) : "memory");
  if (dirty) dirty[w / kBmChunkWords] = 1;
}

// Set the bit of one key; keys outside their instance's range are dropped
// and recorded in Ctl::oob instead of being written.
__device__ __forceinline__ void dm_set(const DenseMap &m, u32 *bm, u8 *dirty, u64 key, Ctl *ctl) {
  u64 w;
  u32 b;
  if (dm_locate(m, key, &w, &b) && w < m.words)
    bm_mark(bm, dirty, w, b);
  else
    atomicOr(&ctl->oob, 8192u);
}

// Warp-aggregated bit-sets: every lane of the warp holds at most one
// candidate (w = ~0: none); lanes whose bits fall in the same word OR them
// in shared memory first (s: this warp's 32 slots), and one lane per
// distinct word sends the reduction.  All 32 lanes must call it.  Pays when
// a warp's candidates share words (the batched DAG closures: one row, one
// layer); costs a match and two warp barriers per 32 candidates otherwise.
__device__ __forceinline__ void warp_set_bits(u32 *bm, u8 *dirty, u64 w, u32 bit, u32 *s) {
  const int lane = threadIdx.x & 31;
  const unsigned same = __match_any_sync(0xffffffffu, w);
  const int leader = __ffs(same) - 1;
  s[lane] = 0u;
  __syncwarp();
  if (bit) atomicOr(&s[leader], bit);
  __syncwarp();
  if (lane == leader && w != ~0ull) {
    asm volatile("red.global.or.b32 [%0], %1;" ::"l"(bm + w), "r"(s[lane]) : "memory");
    if (dirty) dirty[w / kBmChunkWords] = 1;
  }
  __syncwarp();
}

// The word and bit of one candidate for warp_set_bits (w = ~0 when it fails
// the predicate, or lies outside its instance: then recorded in Ctl::oob).
__device__ __forceinline__ void dm_word(const DenseMap &m, u64 key, Ctl *ctl, u64 *w, u32 *bit) {
  u32 b;
  if (dm_locate(m, key, w, &b) && *w < m.words) {
    *bit = 1u << b;
  } else {
    atomicOr(&ctl->oob, 8192u);
    *w = ~0ull;
    *bit = 0u;
  }
}

// Dirty byte of the chunk thread `tid` reads in scan tile `tile` (8 words
// per thread, 8 threads per chunk); 1 when no map is kept.
__device__ __forceinline__ u8 chunk_dirty(const u8 *dirty, u64 tile, int tid) {
  return dirty ? dirty[tile * (kBmTileWords / kBmChunkWords) + tid / (kBmChunkWords / 8)] : 1;
}

// Expressions a scan can compact, over the word pair (g, f).
enum BmExpr { kBmNone = 0, kBmDelta = 1, kBmUnion = 2 };
__device__ __forceinline__ u32 bm_eval(int ex, u32 g, u32 f) {
  return ex == kBmDelta ? (g & ~f) : ex == kBmUnion ? (f | g) : 0u;
}

struct BmScanArgs {
  const u32 *g;    // NEWT bitmap (may be null: all zero)
  u32 *f;          // FULL bitmap (may be null: all zero)
  // If set, g / f / dirty are this relation's bmG / bmF / dirty map, read
  // from the device descriptor when the kernel starts.
  const RelDev *rd;
  u8 *dirty;       // dirty map of g (null: every chunk may hold bits)
  int skip_clean;  // read only dirty chunks (every expression is 0 where g is)
  int inplace;     // write pass: f |= g, g := 0 and dirty := 0 in dirty chunks
  DenseMap map;
  int ex_a, ex_b;  // expressions for list a and list b
  DArr *list_a;    // output lists (sorted keys); null when not wanted
  DArr *list_b;
  Index *idx_b;    // if set: run index of list b
  u64 *count_a;    // if set: receives total_a (a count without a list)
  u64 *count_b;    // if set: receives total_b (a count without a list)
  u64 *pop_g_out;  // if set: receives popcount(g) (NEWT size)
  u64 *inst_delta; // if set: per-instance count of list a is added here
  int need_a, need_b;  // need slots to raise on overflow (-1: none)
  // Gated write pass: before writing anything, every update relation's
  // count pass is checked (gate_rels[gate_update[0 .. gate_n)]); one list
  // too small anywhere raises the overflow and no bitmap is touched.
  int gated;
  const RelDev *gate_rels;
  const int *gate_update;
  int gate_n;
  u64 *tile_prefix;    // [tiles] tile counts, then their exclusive prefix (a << 32 | b)
  // Group mode (no index built): a warp per group of kGroupChunks 64-word
  // chunks, tile_prefix holding one entry per group.  chunk_list: [chunks]
  // the dirty chunks in order (listed mode, with a dirty map); null: every
  // chunk, group g = words 256 g .. 256 g + 255.
  int grouped;
  u32 *chunk_list;
  BmScanRec *rec;
  LaunchRec *lrec;
  Lb lb;
  Ctl *ctl;
};

__device__ __forceinline__ u64 bm_tiles(u64 words) {
  return (words + kBmTileWords - 1) / kBmTileWords;
}

__device__ __forceinline__ void scan_bind(BmScanArgs &a) {
  if (a.rd) {
    a.g = a.rd->bmG;
    a.f = a.rd->bmF;
    a.dirty = a.rd->dirty;
  }
}

// Listed mode.  A large NEWT bitmap touched in few places (the batched form:
// a fraction of every active instance's rows each iteration) is scanned by
// its dirty chunks only.  Pass 0 lists the dirty chunks in order; the count
// and write passes then give each warp a group of kGroupChunks listed chunks
// (8 words per lane), with warp shuffles instead of block barriers, and the
// scan pass (k_bm_scan) runs over the group counts.
constexpr int kScanItems = 8;
constexpr int kScanChunk = kBmBlock * kScanItems;
constexpr int kGroupChunks = 32 * 8 / kBmChunkWords;  // 4
constexpr int kDirtyItems = 16;                       // dirty bytes per thread (one uint4)
constexpr int kDirtyUnit = kBmBlock * kDirtyItems;    // chunks per look-back unit

// Chunks a group-mode pass covers: the listed ones, or all of them.
__device__ __forceinline__ u64 group_chunks(const BmScanArgs &a) {
  return a.chunk_list ? (u64)a.rec->n_listed : a.map.words / kBmChunkWords;
}

__device__ __forceinline__ u64 scan_items(const BmScanArgs &a) {
  return a.grouped ? (group_chunks(a) + kGroupChunks - 1) / kGroupChunks : bm_tiles(a.map.words);
}

// Pass 0 (listed mode): the ordered list of dirty chunks (decoupled
// look-back over units of kDirtyUnit chunks).
__global__ void __launch_bounds__(kBmBlock) k_bm_dirty_chunks(BmScanArgs a) {
  __shared__ u64 s_scan[kBmBlock / 32];
  __shared__ long long s_unit;
  __shared__ u64 s_base;
  if (ctl_stop(a.ctl)) return;
  scan_bind(a);
  const u64 chunks = a.map.words / kBmChunkWords;  // words: whole tiles, so a multiple of 32
  const u64 units = (chunks + kDirtyUnit - 1) / kDirtyUnit;
  const u32 gen = a.lrec->gen;
  while (true) {
    const long long c = grab_tile(a.lrec, &s_unit);
    if (c >= (long long)units) break;
    const u64 c0 = (u64)c * kDirtyUnit + (u64)threadIdx.x * kDirtyItems;
    u32 bits = 0;
    if (c0 < chunks) {
      if (a.dirty) {
        const uint4 v = *reinterpret_cast<const uint4 *>(a.dirty + c0);
        const u32 q[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int i = 0; i < kDirtyItems; i++)
          if ((q[i >> 2] >> (8 * (i & 3))) & 0xFFu) bits |= 1u << i;
      } else {
        bits = (1u << kDirtyItems) - 1u;
      }
    }
    u64 tot;
    const u64 ex = block_excl_scan<kBmBlock>((u64)__popc(bits), s_scan, &tot);
    if (threadIdx.x < 32) {
      u64 prefix = 0;
      if (c == 0) {
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, true, tot);
      } else {
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, false, tot);
        prefix = lb_warp_prefix(a.lb, c, gen, a.ctl);
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, true, prefix + tot);
      }
      if (threadIdx.x == 0) {
        s_base = prefix;
        if ((u64)c == units - 1) a.rec->n_listed = (u32)(prefix + tot);
      }
    }
    __syncthreads();
    u64 pos = s_base + ex;
    while (bits) {
      const int i = __ffs(bits) - 1;
      bits &= bits - 1;
      if (pos < chunks) a.chunk_list[pos] = (u32)(c0 + i);
      pos++;
    }
  }
  launch_rec_finish(a.lrec);
}

// The listed chunk and the 8 words a lane covers in group gi (false past the list).
__device__ __forceinline__ bool group_words(const BmScanArgs &a, u64 n_listed, u64 gi, int lane,
                                            u64 *chunk, u64 *w0) {
  const u64 li = gi * kGroupChunks + (u64)(lane >> 3);
  if (li >= n_listed) return false;
  *chunk = a.chunk_list ? a.chunk_list[li] : li;
  *w0 = *chunk * kBmChunkWords + (u64)(lane & 7) * 8;
  return true;
}

__device__ __forceinline__ void load8(const u32 *p, u32 *v) {
  const uint4 x = reinterpret_cast<const uint4 *>(p)[0], y = reinterpret_cast<const uint4 *>(p)[1];
  v[0] = x.x;
  v[1] = x.y;
  v[2] = x.z;
  v[3] = x.w;
  v[4] = y.x;
  v[5] = y.y;
  v[6] = y.z;
  v[7] = y.w;
}

// Pass 1 (group mode): packed (a, b) counts of every group, a warp per group.
__global__ void __launch_bounds__(kBmBlock) k_bm_groupcount(BmScanArgs a) {
  if (ctl_stop(a.ctl)) return;
  scan_bind(a);
  const u64 n_listed = group_chunks(a);
  const u64 groups = (n_listed + kGroupChunks - 1) / kGroupChunks;
  const int lane = threadIdx.x & 31;
  const u64 nw = (u64)gridDim.x * (kBmBlock / 32);
  u64 my_g = 0;
  for (u64 gi = ((u64)blockIdx.x * kBmBlock + threadIdx.x) >> 5; gi < groups; gi += nw) {
    u64 ch, w0;
    u32 ca = 0, cb = 0;
    if (group_words(a, n_listed, gi, lane, &ch, &w0)) {
      u32 g[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      if (a.g) load8(a.g + w0, g);
      const bool any_g = (g[0] | g[1] | g[2] | g[3] | g[4] | g[5] | g[6] | g[7]) != 0u;
      // f matters where g has bits (delta), or everywhere for a union
      if (a.f && (any_g || a.ex_a == kBmUnion || a.ex_b == kBmUnion)) load8(a.f + w0, f);
#pragma unroll
      for (int i = 0; i < 8; i++) {
        ca += __popc(bm_eval(a.ex_a, g[i], f[i]));
        cb += __popc(bm_eval(a.ex_b, g[i], f[i]));
        my_g += __popc(g[i]);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ca += __shfl_xor_sync(0xffffffffu, ca, o);
      cb += __shfl_xor_sync(0xffffffffu, cb, o);
    }
    if (lane == 0) a.tile_prefix[gi] = ((u64)ca << 32) | cb;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_g += __shfl_xor_sync(0xffffffffu, my_g, o);
  if (lane == 0 && my_g) atomicAdd(&a.rec->pop_g, my_g);
}

// Pass 1: packed (a, b) counts of every tile, one block per tile; a tile
// whose chunks are all clean is skipped when allowed.
__global__ void __launch_bounds__(kBmBlock) k_bm_tilecount(BmScanArgs a) {
  __shared__ u32 s_red[2][kBmBlock / 32];
  if (ctl_stop(a.ctl)) return;
  scan_bind(a);
  const u64 tiles = bm_tiles(a.map.words);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u64 my_g = 0;
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const bool read = !a.skip_clean || chunk_dirty(a.dirty, tile, threadIdx.x);
    if (!__syncthreads_or(read)) {
      if (threadIdx.x == 0) a.tile_prefix[tile] = 0;
      continue;
    }
    const u64 w0 = tile * kBmTileWords + (u64)threadIdx.x * kBmWordsPerThread;
    u32 ca = 0, cb = 0;
    if (read) {
#pragma unroll
      for (int i = 0; i < kBmWordsPerThread; i++) {
        const u64 w = w0 + i;
        const u32 g = a.g ? a.g[w] : 0u, f = a.f ? a.f[w] : 0u;
        ca += __popc(bm_eval(a.ex_a, g, f));
        cb += __popc(bm_eval(a.ex_b, g, f));
        my_g += __popc(g);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      ca += __shfl_xor_sync(0xffffffffu, ca, o);
      cb += __shfl_xor_sync(0xffffffffu, cb, o);
    }
    if (lane == 0) {
      s_red[0][warp] = ca;
      s_red[1][warp] = cb;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      u64 ta = 0, tb = 0;
      for (int w = 0; w < kBmBlock / 32; w++) {
        ta += s_red[0][w];
        tb += s_red[1][w];
      }
      a.tile_prefix[tile] = (ta << 32) | tb;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_g += __shfl_xor_sync(0xffffffffu, my_g, o);
  if (lane == 0 && my_g) atomicAdd(&a.rec->pop_g, my_g);
}

// Pass 2: exclusive prefix of the tile (listed mode: group) counts in place
// (decoupled look-back over chunks of 2048 entries), totals and the
// capacity check.
__global__ void __launch_bounds__(kBmBlock) k_bm_scan(BmScanArgs a) {
  __shared__ u64 s_scan[kBmBlock / 32];
  __shared__ long long s_tile;
  __shared__ u64 s_base;
  if (ctl_stop(a.ctl)) return;
  const u64 tiles = scan_items(a);
  // at least one chunk, so that the totals are written when nothing is listed
  const u64 chunks = max((tiles + kScanChunk - 1) / kScanChunk, (u64)1);
  const u32 gen = a.lrec->gen;
  while (true) {
    const long long c = grab_tile(a.lrec, &s_tile);
    if (c >= (long long)chunks) break;
    const u64 t0 = (u64)c * kScanChunk + (u64)threadIdx.x * kScanItems;
    u64 v[kScanItems], sum = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      v[i] = t0 + i < tiles ? a.tile_prefix[t0 + i] : 0;
      sum += v[i];
    }
    u64 tot;
    const u64 ex = block_excl_scan<kBmBlock>(sum, s_scan, &tot);
    if (threadIdx.x < 32) {
      u64 prefix = 0;
      if (c == 0) {
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, true, tot);
      } else {
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, false, tot);
        prefix = lb_warp_prefix(a.lb, c, gen, a.ctl);
        if (threadIdx.x == 0) lb_publish(a.lb, c, gen, true, prefix + tot);
      }
      if (threadIdx.x == 0) {
        s_base = prefix;
        if ((u64)c == chunks - 1) {
          const u64 ta = (prefix + tot) >> 32, tb = (prefix + tot) & 0xFFFFFFFFull;
          a.rec->total_a = ta;
          a.rec->total_b = tb;
          bool over = false;
          if (a.list_a && ta > a.list_a->cap) {
            over = true;
            if (a.need_a >= 0) atomicMax(&a.ctl->need[a.need_a], ta);
          }
          if (a.list_b && tb > a.list_b->cap) {
            over = true;
            if (a.need_b >= 0) atomicMax(&a.ctl->need[a.need_b], tb);
          }
          a.rec->overflow = over;
        }
      }
    }
    __syncthreads();
    u64 run = s_base + ex;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
      if (t0 + i < tiles) a.tile_prefix[t0 + i] = run;
      run += v[i];
    }
  }
  launch_rec_finish(a.lrec);
}

// The capacity gate of a write pass (after the count and scan passes of
// every update relation): true when some relation's list is too small.
// The block that sees it closed first raises the overflow (stage 1: the
// joins' bits are kept, only the update step reruns); every block returns
// without writing.
__device__ __forceinline__ bool write_gate_closed(const BmScanArgs &a) {
  if (!a.gated) return a.rec->overflow != 0;
  bool closed = false;
  for (int i = 0; i < a.gate_n; i++) {
    const RelDev &r = a.gate_rels[a.gate_update[i]];
    closed |= r.dense && r.scan.overflow;
  }
  if (closed && blockIdx.x == 0 && threadIdx.x == 0) {
    a.rec->pop_g = 0;
    a.ctl->overflow_stage = 1;
    atomicExch(&a.ctl->overflow, 1u);
  }
  return closed;
}

// The block that finishes a write pass last publishes the list sizes.
// `bytes`: this thread's bitmap traffic (words of G and F examined, F
// words updated and G words cleared), added to the scan family's
// algorithmic bytes with one global atomic per block.
__device__ __forceinline__ void write_finish(const BmScanArgs &a, u64 bytes) {
  __shared__ unsigned long long s_bytes;
  if (threadIdx.x == 0) s_bytes = 0;
  __syncthreads();
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
  if ((threadIdx.x & 31) == 0 && bytes) atomicAdd(&s_bytes, (unsigned long long)bytes);
  __syncthreads();
  if (threadIdx.x == 0) prof_add(a.ctl, kPBitmap, s_bytes);
  if (launch_rec_finish(a.lrec) && threadIdx.x == 0) {
    if (a.list_a) a.list_a->n = a.rec->total_a;
    if (a.list_b) a.list_b->n = a.rec->total_b;
    if (a.count_a) *a.count_a = a.rec->total_a;
    if (a.count_b) *a.count_b = a.rec->total_b;
    if (a.pop_g_out) *a.pop_g_out = a.rec->pop_g;
    a.rec->pop_g = 0;
    prof_add(a.ctl, kPBitmap, 8 * (a.rec->total_a + a.rec->total_b));
  }
}

// Pass 3: write list a, list b (+ its index), update f in place and clear g
// in the dirty chunks (every chunk without a dirty map).  One block per tile.
// Listing the set bits of the 256 words a warp holds (8 consecutive words
// per lane, lane-major) in bit order: key r goes to lane r % 32, so keys are
// stored in coalesced runs and no lane waits on another lane's denser words.
// Each lane finds its word by an 8-step search over the words' exclusive
// bit offsets and its bit by a 5-step popcount search.
struct WarpBits {
  u32 w[256];  // the warp's words
  u32 p[256];  // exclusive bit offsets of the words within the warp
};

__device__ __forceinline__ u32 nth_set_bit(u32 x, u32 n) {
  u32 pos = 0;
#pragma unroll
  for (int h = 16; h > 0; h >>= 1) {
    const u32 low = __popc(x & ((1u << h) - 1u));
    if (n >= low) {
      n -= low;
      x >>= h;
      pos += h;
    }
  }
  return pos;
}

// emit(r, k, b): key r of the warp is bit b of the warp's word k.
// lane_excl: bits held by lower lanes; total: bits of the whole warp.
template <class Emit>
__device__ __forceinline__ void warp_list_bits(const u32 *e, u32 lane_excl, u32 total,
                                               WarpBits &s, Emit emit) {
  const int lane = threadIdx.x & 31;
  u32 run = lane_excl;
#pragma unroll
  for (int i = 0; i < 8; i++) {
    s.w[lane * 8 + i] = e[i];
    s.p[lane * 8 + i] = run;
    run += __popc(e[i]);
  }
  __syncwarp();
  for (u32 r = lane; r < total; r += 32) {
    u32 k = 0;
#pragma unroll
    for (u32 h = 128; h > 0; h >>= 1)
      if (s.p[k + h] <= r) k += h;
    emit(r, k, nth_set_bit(s.w[k], r - s.p[k]));
  }
  __syncwarp();
}

struct BmWriteSmem {
  u32 off_b[kBmTileWords + 1];  // exclusive offsets of list b per word
  u64 scan_tmp[kBmBlock / 32];
  WarpBits bits[kBmBlock / 32];
};

__global__ void __launch_bounds__(kBmBlock, 3) k_bm_write(BmScanArgs a) {
  __shared__ BmWriteSmem sm;
  if (ctl_stop(a.ctl)) return;
  if (write_gate_closed(a)) {
    if (!a.gated && blockIdx.x == 0 && threadIdx.x == 0) {
      a.rec->pop_g = 0;
      atomicExch(&a.ctl->overflow, 1u);
    }
    return;
  }
  scan_bind(a);
  const u64 words = a.map.words;
  const u64 tiles = bm_tiles(words);
  const u32 epoch = (u32)(a.ctl->generation + 1);
  const Index ix = a.idx_b ? *a.idx_b : Index{};
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.idx_b) a.idx_b->epoch = epoch;
  u64 *la = a.list_a ? a.list_a->ptr : nullptr;
  u64 *lb = a.list_b ? a.list_b->ptr : nullptr;
  const u64 cap_a = a.list_a ? a.list_a->cap : 0, cap_b = a.list_b ? a.list_b->cap : 0;
  u64 moved = 0;  // bitmap bytes examined / updated by this thread
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const u8 db = chunk_dirty(a.dirty, tile, threadIdx.x);
    const bool read = !a.skip_clean || db;
    if (!__syncthreads_or(read)) continue;
    const bool clr = a.inplace && db;
    if (read) moved += kBmWordsPerThread * ((a.g ? 4 : 0) + (a.f ? 4 : 0));
    const u64 prefix = a.tile_prefix[tile];
    const u64 wt = tile * kBmTileWords;
    const u32 inst = dm_tile_inst(a.map, tile);
    const SegInfo seg = a.map.seg[inst];
    const u64 w0 = wt + (u64)threadIdx.x * kBmWordsPerThread;
    u32 ea[kBmWordsPerThread], eb[kBmWordsPerThread];
    u32 ca = 0, cb = 0;
#pragma unroll
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u64 w = w0 + i;
      u32 g = 0, f = 0;
      if (read) {
        g = a.g ? a.g[w] : 0u;
        f = a.f ? a.f[w] : 0u;
        if (clr && g) {
          a.f[w] = f | g;
          const_cast<u32 *>(a.g)[w] = 0u;
          moved += 8;
        }
      }
      ea[i] = bm_eval(a.ex_a, g, f);
      eb[i] = bm_eval(a.ex_b, g, f);
      ca += __popc(ea[i]);
      cb += __popc(eb[i]);
    }
    if (clr && a.dirty && (threadIdx.x % (kBmChunkWords / 8)) == 0)
      a.dirty[tile * (kBmTileWords / kBmChunkWords) + threadIdx.x / (kBmChunkWords / 8)] = 0;
    u64 tot;
    const u64 ex = block_excl_scan<kBmBlock>(((u64)ca << 32) | cb, sm.scan_tmp, &tot);
    if (threadIdx.x == 0 && a.inst_delta && (tot >> 32)) atomicAdd(&a.inst_delta[inst], tot >> 32);
    if (a.idx_b) {
      u32 ob = (u32)(ex & 0xFFFFFFFFull);
#pragma unroll
      for (int i = 0; i < kBmWordsPerThread; i++) {
        sm.off_b[threadIdx.x * kBmWordsPerThread + i] = ob;
        ob += __popc(eb[i]);
      }
    }
    // the keys, warp by warp (warp wid holds words wt + 256 wid ...)
    {
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
      const u64 ex0 = __shfl_sync(0xffffffffu, ex, 0);
      const u64 end = __shfl_sync(0xffffffffu, ex + (((u64)ca << 32) | cb), 31);
      const u64 ww = wt + (u64)wid * 256;
      if (la) {
        const u64 base = (prefix >> 32) + (ex0 >> 32);
        warp_list_bits(ea, (u32)((ex >> 32) - (ex0 >> 32)), (u32)((end >> 32) - (ex0 >> 32)),
                       sm.bits[wid], [&](u32 r, u32 k, u32 b) {
                         const u64 pos = base + r;
                         if (pos < cap_a)
                           la[pos] = dm_key(a.map, inst, seg, ww + k, (int)b);
                         else
                           atomicOr(&a.ctl->oob, 2048u);
                       });
      }
      if (lb) {
        const u64 lo0 = ex0 & 0xFFFFFFFFull;
        const u64 base = (prefix & 0xFFFFFFFFull) + lo0;
        warp_list_bits(eb, (u32)((ex & 0xFFFFFFFFull) - lo0), (u32)((end & 0xFFFFFFFFull) - lo0),
                       sm.bits[wid], [&](u32 r, u32 k, u32 b) {
                         const u64 pos = base + r;
                         if (pos < cap_b)
                           lb[pos] = dm_key(a.map, inst, seg, ww + k, (int)b);
                         else
                           atomicOr(&a.ctl->oob, 4096u);
                       });
      }
      (void)lane;
    }
    if (a.idx_b) {
      if (threadIdx.x == 0) sm.off_b[kBmTileWords] = (u32)(tot & 0xFFFFFFFFull);
      __syncthreads();
      // One slot per non-empty row of the tile: {c0, epoch, start, len}.
      // Rows are 2^row_shift words, at most one tile, aligned in the tile.
      const u32 rs = seg.row_shift;
      const u64 row_words = 1ull << rs;
      const u64 rows = kBmTileWords >> rs;
      const u32 hi = a.map.seg_shift >= 31 ? 0u : (inst << a.map.seg_shift);
      for (u64 r = threadIdx.x; r < rows; r += blockDim.x) {
        const u64 lw = r << rs;  // first word of the row in the tile
        if (wt + lw >= words || wt + lw < seg.base_word) break;
        const u64 row = (wt + lw - seg.base_word) >> rs;
        if (row >= seg.n) break;
        const u32 len = sm.off_b[lw + row_words] - sm.off_b[lw];
        if (len) {
          const u32 start = (u32)((prefix & 0xFFFFFFFFull) + sm.off_b[lw]);
          index_insert(ix, epoch, hi | (u32)row, start, len, a.ctl);
        }
      }
      __syncthreads();
    }
  }
  write_finish(a, moved);
}

// Pass 3 (group mode): as k_bm_write, a warp per group of chunks.  No
// index is built in this mode (it needs whole rows).
struct GroupWriteSmem {
  WarpBits bits[kBmBlock / 32];
  u64 w0[kBmBlock / 32][32];   // first word of each lane
  u32 inst[kBmBlock / 32][32]; // instance of each lane's chunk
};

__global__ void __launch_bounds__(kBmBlock) k_bm_groupwrite(BmScanArgs a) {
  __shared__ GroupWriteSmem sm;
  if (ctl_stop(a.ctl)) return;
  if (write_gate_closed(a)) {
    if (!a.gated && blockIdx.x == 0 && threadIdx.x == 0) {
      a.rec->pop_g = 0;
      atomicExch(&a.ctl->overflow, 1u);
    }
    return;
  }
  scan_bind(a);
  const u64 n_listed = group_chunks(a);
  const u64 groups = (n_listed + kGroupChunks - 1) / kGroupChunks;
  const int lane = threadIdx.x & 31;
  const u64 nw = (u64)gridDim.x * (kBmBlock / 32);
  u64 *la = a.list_a ? a.list_a->ptr : nullptr;
  u64 *lb = a.list_b ? a.list_b->ptr : nullptr;
  const u64 cap_a = a.list_a ? a.list_a->cap : 0, cap_b = a.list_b ? a.list_b->cap : 0;
  u64 moved = 0;  // bitmap bytes examined / updated by this lane
  for (u64 gi = ((u64)blockIdx.x * kBmBlock + threadIdx.x) >> 5; gi < groups; gi += nw) {
    u64 ch = 0, w0 = 0;
    u32 ea[8], eb[8];
    u32 ca = 0, cb = 0;
    const bool on = group_words(a, n_listed, gi, lane, &ch, &w0);
    u32 g[8] = {0, 0, 0, 0, 0, 0, 0, 0}, f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (on) {
      if (a.g) load8(a.g + w0, g);
      const bool any_g = (g[0] | g[1] | g[2] | g[3] | g[4] | g[5] | g[6] | g[7]) != 0u;
      if (a.f && (any_g || a.ex_a == kBmUnion || a.ex_b == kBmUnion)) load8(a.f + w0, f);
      moved += a.g ? 32 : 0;
      if (a.f && (any_g || a.ex_a == kBmUnion || a.ex_b == kBmUnion)) moved += 32;
      if (a.inplace && any_g) moved += 64;
      if (a.inplace && any_g) {
        uint4 *pf = reinterpret_cast<uint4 *>(a.f + w0);
        pf[0] = make_uint4(f[0] | g[0], f[1] | g[1], f[2] | g[2], f[3] | g[3]);
        pf[1] = make_uint4(f[4] | g[4], f[5] | g[5], f[6] | g[6], f[7] | g[7]);
        uint4 *pg = reinterpret_cast<uint4 *>(const_cast<u32 *>(a.g) + w0);
        pg[0] = make_uint4(0, 0, 0, 0);
        pg[1] = make_uint4(0, 0, 0, 0);
      }
      if (a.inplace && a.dirty && (lane & 7) == 0) a.dirty[ch] = 0;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) {
      ea[i] = bm_eval(a.ex_a, g[i], f[i]);
      eb[i] = bm_eval(a.ex_b, g[i], f[i]);
      ca += __popc(ea[i]);
      cb += __popc(eb[i]);
    }
    // warp exclusive scan of the packed counts
    const u64 mine = ((u64)ca << 32) | cb;
    u64 inc = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    const u64 prefix = a.tile_prefix[gi];
    // per-instance count of list a: one atomic per chunk (its 8 lanes summed)
    u32 c8 = ca;
#pragma unroll
    for (int o = 1; o < 8; o <<= 1) c8 += __shfl_xor_sync(0xffffffffu, c8, o);
    const int wid = threadIdx.x >> 5;
    const u32 inst = on ? dm_tile_inst(a.map, w0 / kBmTileWords) : 0u;
    if (on && a.inst_delta && (lane & 7) == 0 && c8) atomicAdd(&a.inst_delta[inst], (u64)c8);
    sm.w0[wid][lane] = w0;
    sm.inst[wid][lane] = inst;
    const u64 end = __shfl_sync(0xffffffffu, inc, 31);
    // the keys of the group, key r by lane r % 32 (lanes past the list hold
    // no bits)
    if (la) {
      const u64 base = prefix >> 32;
      warp_list_bits(ea, (u32)((inc - mine) >> 32), (u32)(end >> 32), sm.bits[wid],
                     [&](u32 r, u32 k, u32 b) {
                       const u32 in = sm.inst[wid][k >> 3];
                       const SegInfo sg = a.map.seg[in];
                       const u64 pos = base + r;
                       if (pos < cap_a)
                         la[pos] = dm_key(a.map, in, sg, sm.w0[wid][k >> 3] + (k & 7), (int)b);
                       else
                         atomicOr(&a.ctl->oob, 2048u);
                     });
    }
    if (lb) {
      const u64 base = prefix & 0xFFFFFFFFull;
      warp_list_bits(eb, (u32)((inc - mine) & 0xFFFFFFFFull), (u32)(end & 0xFFFFFFFFull),
                     sm.bits[wid], [&](u32 r, u32 k, u32 b) {
                       const u32 in = sm.inst[wid][k >> 3];
                       const SegInfo sg = a.map.seg[in];
                       const u64 pos = base + r;
                       if (pos < cap_b)
                         lb[pos] = dm_key(a.map, in, sg, sm.w0[wid][k >> 3] + (k & 7), (int)b);
                       else
                         atomicOr(&a.ctl->oob, 4096u);
                     });
    }
  }
  write_finish(a, moved);
}

// Zero a NEWT bitmap in its dirty chunks (all of it without a dirty map)
// and clear the dirty map.  One block per tile.
// ---------------------------------------------------------------------------
// Listing of a square-domain bitmap (ids below 2^dk, rows of 2^(dk-5)
// words) as its sorted key list, in three passes over 2048-word tiles:
// k_bm_list_count (a popcount per tile, streaming), k_bm_list_offsets (one
// block: the tiles' output offsets and the list's size) and k_bm_list_write
// (a block per tile with keys, the keys written at their offset with
// coalesced stores and no search per key; an empty tile costs one read of
// its count).  Replaces the sort of the flattened FULL at the end of a LIE
// (src/lie.cu:219-254).
//
// Thread t holds words i * 256 + t of the tile (i = 0..7, "segment" i).  A
// segment is 256 words, 8192 bit positions, so the keys of one segment
// always fit one staging buffer.
// ---------------------------------------------------------------------------
constexpr int kListScanBlock = 1024;

__global__ void __launch_bounds__(kBmBlock) k_bm_list_count(const u32 *bm, u64 tiles, u32 *cnt,
                                                            Ctl *ctl) {
  __shared__ u32 s_w[kBmBlock / 32];
  if (ctl_stop(ctl)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    // words 4 t' .. 4 t' + 3 and 1024 + 4 t' .. of the tile (t' = thread)
    const uint4 *p = reinterpret_cast<const uint4 *>(bm + t * kBmTileWords);
    const uint4 x = p[threadIdx.x], y = p[kBmBlock + threadIdx.x];
    u32 c = __popc(x.x) + __popc(x.y) + __popc(x.z) + __popc(x.w) + __popc(y.x) + __popc(y.y) +
            __popc(y.z) + __popc(y.w);
    c = __reduce_add_sync(0xffffffffu, c);
    if (lane == 0) s_w[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
      u32 sum = 0;
#pragma unroll
      for (int i = 0; i < kBmBlock / 32; i++) sum += s_w[i];
      cnt[t] = sum;
    }
    __syncthreads();
  }
}

// One block: off[t] = keys of the tiles before t; out->n = the total
// (within the list's capacity).  check_n: out->n on entry is the bit count
// the loop kept for this version, and another total raises the bounds flag
// (a load's listing has no such count).
__global__ void __launch_bounds__(kListScanBlock) k_bm_list_offsets(const u32 *cnt, u64 tiles,
                                                                    u64 *off, DArr *out,
                                                                    int check_n, Ctl *ctl) {
  __shared__ u64 s_warp[kListScanBlock / 32];
  if (ctl_stop(ctl)) return;
  u64 carry = 0;
  for (u64 c0 = 0; c0 < tiles; c0 += kListScanBlock * 4) {
    const u64 b = c0 + 4ull * threadIdx.x;
    u32 v[4];
#pragma unroll
    for (int i = 0; i < 4; i++) v[i] = b + i < tiles ? cnt[b + i] : 0u;
    const u64 local = (u64)v[0] + v[1] + v[2] + v[3];
    u64 tot;
    u64 ex = block_excl_scan<kListScanBlock>(local, s_warp, &tot) + carry;
    carry += tot;
#pragma unroll
    for (int i = 0; i < 4; i++)
      if (b + i < tiles) {
        off[b + i] = ex;
        ex += v[i];
      }
  }
  if (threadIdx.x == 0) {
    const u64 expect_n = out->n, cap = out->cap;
    out->n = carry <= cap ? carry : cap;
    if (carry > cap || (check_n && carry != expect_n)) atomicOr(&ctl->oob, 16384u);
  }
}

constexpr int kListStage = kBmBlock * 32;  // 8192 positions per segment

struct ListSmem {
  unsigned short stage[2][kListStage];
  u32 wtot[kBmWordsPerThread][kBmBlock / 32];  // per segment: warp totals, then offsets
  u32 seg_tot[kBmWordsPerThread];
  u32 seg_off[kBmWordsPerThread];
  long long tile;
};

// Keys leave through a shared-memory window: each segment's keys are staged
// as their 13-bit positions in the segment (2 bytes; the row and column are
// rebuilt at the copy-out), each thread expanding its own word, then copied
// out in one coalesced pass.  Two buffers alternate between the segments
// that hold keys, so one barrier per segment separates a buffer's expansion
// from its copy-out and the copy-out from the buffer's next expansion.
// Tiles are taken from a counter (dense tiles cluster at the low ids of
// skewed graphs); a tile's offset comes from k_bm_list_offsets.
__global__ void __launch_bounds__(kBmBlock) k_bm_list_write(const u32 *bm, u64 tiles, int rs,
                                                            const u32 *cnt, const u64 *off,
                                                            DArr *out, LaunchRec *rec, Ctl *ctl) {
  __shared__ ListSmem sm;
  if (ctl_stop(ctl)) return;
  const u64 row_mask = (1ull << rs) - 1;
  u64 *dst = out->ptr;
  const u64 cap = out->cap;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u64 moved = 0;
  u32 nbuf = 0;  // segments with keys staged so far (buffer parity)
  while (true) {
    const long long tl = grab_tile(rec, &sm.tile);
    if (tl >= (long long)tiles) break;
    const u64 t = (u64)tl;
    if (cnt[t] == 0) continue;  // (block-uniform)
    const u64 w0 = t * kBmTileWords;
    u32 v[kBmWordsPerThread], ex[kBmWordsPerThread];
#pragma unroll
    for (int i = 0; i < kBmWordsPerThread; i++) {
      v[i] = bm[w0 + (u64)i * kBmBlock + threadIdx.x];
      const u32 c = __popc(v[i]);
      u32 x = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
      }
      ex[i] = x - c;
      if (lane == 31) sm.wtot[i][warp] = x;
    }
    __syncthreads();
    if (threadIdx.x < kBmWordsPerThread) {
      // per segment: exclusive warp offsets and the segment's total
      u32 acc = 0;
      for (int w = 0; w < kBmBlock / 32; w++) {
        const u32 x = sm.wtot[threadIdx.x][w];
        sm.wtot[threadIdx.x][w] = acc;
        acc += x;
      }
      sm.seg_tot[threadIdx.x] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      u32 a = 0;
      for (int i = 0; i < kBmWordsPerThread; i++) {
        sm.seg_off[i] = a;
        a += sm.seg_tot[i];
      }
    }
    __syncthreads();
    const u64 base = off[t];
    moved += 4 * kBmWordsPerThread;
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u32 st = sm.seg_tot[i];  // block-uniform
      if (st == 0) continue;
      unsigned short *stg = sm.stage[nbuf++ & 1];
      // expand this thread's word: its keys' positions in the segment
      u32 x = v[i];
      u32 p = sm.wtot[i][warp] + ex[i];
      const u32 q0 = threadIdx.x * 32;
      while (x) {
        stg[p++] = (unsigned short)(q0 + (u32)(__ffs(x) - 1));
        x &= x - 1;
      }
      __syncthreads();
      // copy-out: position q of segment word ws = q / 32, bit q % 32
      const u64 ws = w0 + (u64)i * kBmBlock;
      const u64 pos0 = base + sm.seg_off[i];
      u64 *o = dst + pos0;
      moved += 8 * (u64)(threadIdx.x == 0 ? st : 0);
      if (pos0 + st <= cap && rs >= 8) {
        // rows of 256 words or more: the segment lies in one row, so its
        // keys are the segment's first key plus their positions
        const u64 kb = ((ws >> rs) << 32) | ((ws & row_mask) << 5);
        for (u32 j = threadIdx.x; j < st; j += kBmBlock) o[j] = kb + stg[j];
      } else if (pos0 + st <= cap) {
        for (u32 j = threadIdx.x; j < st; j += kBmBlock) {
          const u32 q = stg[j];
          const u64 w = ws + (q >> 5);
          o[j] = ((w >> rs) << 32) | ((w & row_mask) << 5) | (q & 31u);
        }
      } else {
        for (u32 j = threadIdx.x; j < st; j += kBmBlock) {
          const u32 q = stg[j];
          const u64 w = ws + (q >> 5);
          if (pos0 + j < cap)
            o[j] = ((w >> rs) << 32) | ((w & row_mask) << 5) | (q & 31u);
          else
            atomicOr(&ctl->oob, 16384u);
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
  if (lane == 0) prof_add(ctl, kPBitmap, moved);
  launch_rec_finish(rec);
}

__device__ __forceinline__ void clear_newt_tiles(u32 *G, u8 *D, u64 words) {
  const u64 tiles = bm_tiles(words);
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    if (!chunk_dirty(D, tile, threadIdx.x)) continue;
    uint4 *p = reinterpret_cast<uint4 *>(G + tile * kBmTileWords + threadIdx.x * 8);
    p[0] = make_uint4(0, 0, 0, 0);
    p[1] = make_uint4(0, 0, 0, 0);
    if (D && (threadIdx.x % (kBmChunkWords / 8)) == 0)
      D[tile * (kBmTileWords / kBmChunkWords) + threadIdx.x / (kBmChunkWords / 8)] = 0;
  }
}

__global__ void __launch_bounds__(256) k_bm_clear_dirty(const RelDev *rd, DenseMap map, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  clear_newt_tiles(rd->bmG, rd->dirty, map.words);
}

// Set the bits of a key list (FULL at the start of a LIE; no dirty map).
__global__ void __launch_bounds__(256) k_bm_from_list(const DArr *list, u32 *bm, DenseMap map,
                                                      Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 n = list->n;
  const u64 *k = list->ptr;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    dm_set(map, bm, nullptr, k[i], ctl);
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPBitmap, 8 * n);
}

// load_relation's sort + unique over a small square domain (ids below
// 2^dk): every row sets its bit (c0, c1) of a zeroed bitmap, word
// c0 * 2^(dk-5) + c1 / 32, and the listing passes read the bitmap back in
// key order, each tuple once.  A key outside the domain is dropped and
// raises the bounds flag (the host sizes dk from the largest value).
__global__ void __launch_bounds__(256) k_bm_set_keys(const u64 *keys, u64 n, u32 *bm, int dk,
                                                     Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u32 lim = 1u << dk;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 k = keys[i];
    const u32 c0 = key_c0(k), c1 = key_c1(k);
    if (c0 >= lim || c1 >= lim) {
      atomicOr(&ctl->oob, 65536u);
      continue;
    }
    const u64 bit = ((u64)c0 << dk) | c1;
    atomicOr(&bm[bit >> 5], 1u << (bit & 31));
  }
}

// RelationalJoin materialisation into the output's NEWT bitmap.  Balanced
// over candidate positions as k_join_mat: a block owns kMatTile consecutive
// positions, each thread kMatPer consecutive ones, found with one binary
// search over the tile's records and then walked forward.  A candidate is one
// inner read, the column move, the predicate and two fire-and-forget
// atomicOr (the bit and its chunk's dirty bit).
constexpr int kMatPer = kMatTile / kMatBlock;  // positions per thread

__global__ void __launch_bounds__(kMatBlock) k_join_mat_bm(JoinArgs a, const RelDev *out_rd,
                                                           DenseMap map) {
  __shared__ MatSmem sm;
  if (ctl_stop(a.ctl)) return;
  const u64 total = a.op->total;
  const u64 nc = a.op->nc;
  if (total == 0) return;
  u32 *G = out_rd->bmG;
  u8 *D = out_rd->dirty;
  const u64 *inner = a.inner->ptr;
  const u64 tiles = (total + kMatTile - 1) / kMatTile;
  for (u64 batch = blockIdx.x; batch < tiles; batch += (u64)gridDim.x * kMatBlock) {
    __syncthreads();
    mat_batch_starts(a.crow_off, nc, tiles, batch, sm.tile_k0);
    for (u32 j = 0; j < kMatBlock; j++) {
      const u64 tile = batch + (u64)j * gridDim.x;
      if (tile >= tiles) break;
      const u64 p0 = tile * kMatTile;
      const u64 p1 = min(p0 + kMatTile, total);
      __syncthreads();
      const u32 m = mat_stage_tile(a, nc, sm.tile_k0[j], sm);
      __syncthreads();
      u64 p = p0 + (u64)threadIdx.x * kMatPer;
      if (p < p1) {
        u32 r = find_rec(sm.off, m, p);
        u64 next = sm.off[r + 1];
        const u64 pe = min(p + kMatPer, p1);
        for (; p < pe; p++) {
          while (p >= next) {
            r++;
            next = sm.off[r + 1];
          }
          const u64 t = gen_join(a.sel, inner[sm.start[r] + (p - sm.off[r])], sm.key[r]);
          if (pred_ok(a.pred, t)) dm_set(map, G, D, t, a.ctl);
        }
      }
    }
  }
  if (launch_rec_finish(a.rec) && threadIdx.x == 0)
    prof_add(a.ctl, kPJoinMat, 16 * total + 24 * nc);
}

// Dense joins in one pass (src/join.cu:12-158 with a bitmap output).  No
// output position is needed when results are bits, so the count pass of
// the list form (k_join_count's counts and record compaction, then
// k_join_mat_bm balanced by output position) is replaced by probe and
// expand: a warp takes 32 outer rows, probes the inner index for each and
// expands their runs together, 32 candidates per step (lane p takes
// candidate base + p of the warp's concatenated runs, found by a 5-step
// search over the runs' offsets).  A run longer than kHeavyRun is cut into
// pieces of kHeavyPiece candidates, appended to the record buffer
// (crow_key / crow_start / crow_len, count in op->nc), and expanded by
// k_join_heavy_bm, a block per piece, so no key can hold one warp long.
constexpr int kFuseBlock = 256;
constexpr int kFuseCtasPerSm = 6;
constexpr u32 kHeavyRun = 128;
constexpr u32 kHeavyPiece = 2048;
// Row-OR pieces: a run at least as long as its row has words (one reduction
// per word then replaces one per candidate, and the row is 4 bytes a word
// instead of 8 per candidate) is ORed from the inner's FULL bitmap in
// pieces of kRowPiece words.  A row piece's record: crow_key = first output
// word, crow_off = first inner word, crow_start = 0, crow_len = kRowFlag |
// words.
constexpr u32 kRowPiece = 256;
constexpr u32 kRowFlag = 0x80000000u;

// The block size is a tuning choice (128, 256 or 512 threads; the same
// warps per SM at each).
template <int BLOCK>
struct FuseSmem {
  u64 row[BLOCK / 32][32];
  u64 excl[BLOCK / 32][32];
  u32 start[BLOCK / 32][32];
  u32 agg[BLOCK / 32][32];  // warp_set_bits slots
};

template <bool AGG, int BLOCK>
__global__ void __launch_bounds__(BLOCK, kFuseCtasPerSm * kFuseBlock / BLOCK)
    k_join_bm(JoinArgs a, const RelDev *out_rd, DenseMap map) {
  constexpr int kFuseBlock = BLOCK;
  __shared__ FuseSmem<BLOCK> sm;
  if (ctl_stop(a.ctl)) return;
  const u64 n_outer = eff_count(a.outer, a.outer_vis);
  const u64 n_inner = eff_count(a.inner, a.inner_vis);
  if (n_outer == 0 || n_inner == 0) {
    join_empty_side(a, n_outer);
    return;
  }
  if (a.once) {
    // a join over static FULLs that an earlier iteration ran with both
    // sides non-empty: the same tuples, all in the output's FULL already
    if (*a.once) {
      if (blockIdx.x == 0 && threadIdx.x == 0 && *a.produced) *a.phantom = 1;
      return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.once_pending = 1;
  }
  u32 *G = out_rd->bmG;
  u8 *D = out_rd->dirty;
  const Index ix = *a.inner_idx;
  const u64 *inner = a.inner->ptr;
  const u64 *outer = a.outer->ptr;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const u64 chunks = (n_outer + 31) / 32;
  const u64 nw = (u64)gridDim.x * (kFuseBlock / 32);
  u64 cand = 0;  // candidates expanded by this warp
  bool emitted = false;
  for (u64 c = (u64)blockIdx.x * (kFuseBlock / 32) + wid; c < chunks; c += nw) {
    const u64 i = c * 32 + lane;
    u64 row = 0;
    u32 s = 0, l = 0;
    if (i < n_outer) {
      row = outer[i];
      l = index_probe(ix, key_c0(row), &s);
    }
    if (l > kHeavyRun) {
      // output row x (from the outer row) and inner row z (the join key)
      u64 xw = 0, zw = 0;
      u32 rw = 0;
      if (a.row_or) {
        // ids of instance i are (i << seg_shift) | local; the square
        // domain is one instance of every id
        const bool square = map.seg_shift >= 31;
        const u32 x = pick4(a.sel.s0, 0, row), z = key_c0(row);
        const u32 xi = square ? 0u : x >> map.seg_shift, zi = square ? 0u : z >> map.seg_shift;
        const u32 base = square ? 0u : xi << map.seg_shift;
        u32 bx, bz;
        if (xi == zi && dm_locate(map, make_key(x, base), &xw, &bx) &&
            dm_locate(map, make_key(z, base), &zw, &bz)) {
          rw = 1u << map.seg[xi].row_shift;
          if (l < rw) rw = 0;  // shorter than its row: expand it
        }
      }
      const u32 np = rw ? (rw + kRowPiece - 1) / kRowPiece : (l + kHeavyPiece - 1) / kHeavyPiece;
      const u64 pos = atomicAdd(reinterpret_cast<unsigned long long *>(&a.op->nc), (u64)np);
      if (pos + np <= a.crow_cap) {
        for (u32 k = 0; k < np; k++) {
          if (rw) {
            a.crow_key[pos + k] = xw + (u64)k * kRowPiece;
            a.crow_off[pos + k] = zw + (u64)k * kRowPiece;
            a.crow_start[pos + k] = 0;
            a.crow_len[pos + k] = kRowFlag | min(kRowPiece, rw - k * kRowPiece);
          } else {
            a.crow_key[pos + k] = row;
            a.crow_start[pos + k] = s + k * kHeavyPiece;
            a.crow_len[pos + k] = min(kHeavyPiece, l - k * kHeavyPiece);
          }
        }
        l = 0;
      }  // else: no room, the warp expands the run itself
    }
    u64 inc = l;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const u64 y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    const u64 total = __shfl_sync(0xffffffffu, inc, 31);
    sm.row[wid][lane] = row;
    sm.start[wid][lane] = s;
    sm.excl[wid][lane] = inc - l;
    __syncwarp();
    for (u64 base = 0; base < total; base += 32) {
      const u64 p = base + lane;
      u64 w = ~0ull;
      u32 bit = 0u;
      if (p < total) {
        // the last run starting at or before p (an empty run shares its
        // offset with the next one, so it is never the last)
        int r = 0;
#pragma unroll
        for (int h = 16; h > 0; h >>= 1)
          if (sm.excl[wid][r + h] <= p) r += h;
        const u64 t = gen_join(a.sel, inner[sm.start[wid][r] + (p - sm.excl[wid][r])],
                               sm.row[wid][r]);
        if (pred_ok(a.pred, t)) {
          emitted = true;
          if (AGG)
            dm_word(map, t, a.ctl, &w, &bit);
          else
            dm_set(map, G, D, t, a.ctl);
        }
      }
      if (AGG) warp_set_bits(G, D, w, bit, sm.agg[wid]);
    }
    __syncwarp();
    cand += total;
  }
  // (run pieces appended for k_join_heavy_bm report from there)
  if (a.produced && __any_sync(0xffffffffu, emitted) && lane == 0) *a.produced = 1;
  if (lane == 0) prof_add(a.ctl, kPJoinMat, cand * 12);
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(a.ctl, kPJoinMat, n_outer * 16);
}

// The pieces of long runs appended by k_join_bm, a block per piece; the
// last block empties the piece list for the next launch (so does block 0
// of a stopped launch, which expands nothing).
template <bool AGG, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_join_heavy_bm(JoinArgs a, const RelDev *out_rd,
                                                        DenseMap map) {
  __shared__ u32 s_agg[BLOCK / 32][32];
  if (ctl_stop(a.ctl)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) a.op->nc = 0;
    return;
  }
  const u64 np = min(a.op->nc, a.crow_cap);
  u32 *G = out_rd->bmG;
  u8 *D = out_rd->dirty;
  const u64 *inner = a.inner->ptr;
  u64 cand = 0;
  const u32 *F = a.row_or ? a.inner_rd->bmF : nullptr;
  u64 row_bytes = 0;
  bool emitted = false;
  for (u64 k = blockIdx.x; k < np; k += gridDim.x) {
    const u64 row = a.crow_key[k];
    const u32 s = a.crow_start[k], l = a.crow_len[k];
    if (l & kRowFlag) {
      // a row piece: OR the inner row's words into the output row
      const u32 nw = l & ~kRowFlag;
      const u64 zw = a.crow_off[k];
      for (u32 j = threadIdx.x; j < nw; j += blockDim.x) {
        const u32 v = F[zw + j];
        if (v) {
          emitted = true;
          asm volatile("red.global.or.b32 [%0], %1;" ::"l"(G + row + j), "r"(v) : "memory");
          if (D) D[(row + j) / kBmChunkWords] = 1;
        }
      }
      row_bytes += 8 * (u64)nw;  // a word read and a word reduced
      continue;
    }
    for (u32 j0 = 0; j0 < l; j0 += blockDim.x) {  // rounds uniform over the block
      const u32 j = j0 + threadIdx.x;
      u64 w = ~0ull;
      u32 bit = 0u;
      if (j < l) {
        const u64 t = gen_join(a.sel, inner[s + j], row);
        if (pred_ok(a.pred, t)) {
          emitted = true;
          if (AGG)
            dm_word(map, t, a.ctl, &w, &bit);
          else
            dm_set(map, G, D, t, a.ctl);
        }
      }
      if (AGG) warp_set_bits(G, D, w, bit, s_agg[threadIdx.x >> 5]);
    }
    cand += l;
  }
  if (a.produced && __any_sync(0xffffffffu, emitted) && (threadIdx.x & 31) == 0) *a.produced = 1;
  if (threadIdx.x == 0) prof_add(a.ctl, kPJoinMat, cand * 12 + row_bytes);
  if (launch_rec_finish(a.rec) && threadIdx.x == 0) {
    a.op->nc = 0;
    prof_add(a.ctl, kPJoinMat, np * 24);
  }
}

// RelationalCopy into the destination's NEWT bitmap (src/copy.cu:12-95).  An
// empty source empties the destination NEWT (src/copy.cu:24-27): that case
// is handled by a k_bm_clear_dirty launched conditionally before.
__global__ void __launch_bounds__(256) k_copy_bm(CopyArgs c, const RelDev *dest_rd, DenseMap map) {
  if (ctl_stop(c.ctl)) return;
  if (c.once && *c.once) return;
  const u64 n = eff_count(c.src, c.src_vis);
  if (n == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0 && c.once_pending) *c.once_pending = 1;
    return;
  }
  u32 *G = dest_rd->bmG;
  u8 *D = dest_rd->dirty;
  const u64 *src = c.src->ptr;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    dm_set(map, G, D, gen_join(c.sel, src[i], 0), c.ctl);
  if (launch_rec_finish(c.rec) && threadIdx.x == 0) {
    if (c.once_pending) *c.once_pending = 1;
    prof_add(c.ctl, kPCopy, 8 * n);
  }
}

// Empties the destination NEWT of a Copy whose source is empty (launched
// just before k_copy_bm; a no-op otherwise or for a FULL source already
// copied).
__global__ void __launch_bounds__(256) k_copy_empty_clear(CopyArgs c, const RelDev *dest_rd,
                                                          DenseMap map) {
  if (ctl_stop(c.ctl)) return;
  if (c.once && *c.once) return;
  if (eff_count(c.src, c.src_vis) != 0) return;
  clear_newt_tiles(dest_rd->bmG, dest_rd->dirty, map.words);
}

// RelationalACopy (src/acopy.cu:12-50): dest NEWT := sel(src NEWT).  The
// destination NEWT was cleared by k_bm_clear_dirty just before; the source
// NEWT bitmap is read in its dirty chunks only.  One block per tile.
__global__ void __launch_bounds__(256) k_acopy_bm(const RelDev *src_rd, Sel2 sel,
                                                  const RelDev *dest_rd, DenseMap map, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u32 *S = src_rd->bmG;
  const u8 *SD = src_rd->dirty;
  u32 *G = dest_rd->bmG;
  u8 *D = dest_rd->dirty;
  const u64 tiles = bm_tiles(map.words);
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    if (!chunk_dirty(SD, tile, threadIdx.x)) continue;
    const u32 inst = dm_tile_inst(map, tile);
    const SegInfo seg = map.seg[inst];
    const u64 w0 = tile * kBmTileWords + threadIdx.x * 8;
    for (int i = 0; i < 8; i++) {
      u32 x = S[w0 + i];
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        dm_set(map, G, D, gen_join(sel, dm_key(map, inst, seg, w0 + i, b), 0), ctl);
      }
    }
  }
}

// Batched form: an instance whose update relations produced new tuples in
// this iteration records it (inst_last = iteration + 1), so that its own
// loop-pass count is known when the shared loop ends.
__global__ void k_inst_track(u64 *inst_delta, u64 *inst_last, u32 n_inst, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 it = ctl->iteration;
  for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n_inst; i += gridDim.x * blockDim.x) {
    if (inst_delta[i]) {
      inst_last[i] = it + 1;
      inst_delta[i] = 0;
    }
  }
}

// Per-instance size and digest of a FULL bitmap, in each instance's local
// ids (the digest gdl_relation_digest gives for the instance run alone).
// Pass 1: popcount per tile.
__global__ void __launch_bounds__(256) k_inst_tile_pop(const u32 *bm, DenseMap map, u32 *tile_pop) {
  __shared__ u32 s_sum;
  const u64 tiles = bm_tiles(map.words);
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    if (threadIdx.x == 0) s_sum = 0;
    __syncthreads();
    u32 c = 0;
    for (u64 w = t * kBmTileWords + threadIdx.x; w < min((t + 1) * kBmTileWords, map.words);
         w += blockDim.x)
      c += __popc(bm[w]);
    atomicAdd(&s_sum, c);
    __syncthreads();
    if (threadIdx.x == 0) tile_pop[t] = s_sum;
    __syncthreads();
  }
}

// Pass 2 (after a per-instance exclusive scan of tile_pop into tile_rank):
// digest terms of every tuple, summed per instance.
__global__ void __launch_bounds__(256) k_inst_digest(const u32 *bm, DenseMap map,
                                                     const u64 *tile_rank, u64 *acc) {
  // Thread t holds words i * 256 + t of a tile (segments i = 0..7).  Each
  // thread expands its word's bits into the segment's staging buffer at
  // their ranks (per-segment prefix sums: no per-tuple search), as 13-bit
  // positions in the segment; then all threads hash the staged tuples
  // together, so the hash chain, the costly part, runs without divergence.
  // Two buffers alternate between segments with tuples (one barrier each).
  __shared__ unsigned short s_stage[2][kBmBlock * 32];
  __shared__ u32 s_wtot[kBmWordsPerThread][kBmBlock / 32];
  __shared__ u32 s_seg_tot[kBmWordsPerThread];
  __shared__ u32 s_seg_off[kBmWordsPerThread];
  __shared__ u64 s_red[kBmBlock / 32];
  const u64 tiles = bm_tiles(map.words);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  u32 nbuf = 0;
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    const u32 inst = dm_tile_inst(map, t);
    const SegInfo seg = map.seg[inst];
    const u64 row_mask = (1ull << seg.row_shift) - 1;
    const u64 w0 = t * kBmTileWords;
    u32 x[kBmWordsPerThread], ex[kBmWordsPerThread];
#pragma unroll
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u64 w = w0 + (u64)i * kBmBlock + threadIdx.x;
      x[i] = w < map.words ? bm[w] : 0u;
      const u32 c = __popc(x[i]);
      u32 v = c;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const u32 y = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += y;
      }
      ex[i] = v - c;
      if (lane == 31) s_wtot[i][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < kBmWordsPerThread) {
      u32 a = 0;
      for (int w = 0; w < kBmBlock / 32; w++) {
        const u32 v = s_wtot[threadIdx.x][w];
        s_wtot[threadIdx.x][w] = a;
        a += v;
      }
      s_seg_tot[threadIdx.x] = a;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      u32 a = 0;
      for (int i = 0; i < kBmWordsPerThread; i++) {
        s_seg_off[i] = a;
        a += s_seg_tot[i];
      }
    }
    __syncthreads();
    u64 h_sum = 0;
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u32 st = s_seg_tot[i];  // block-uniform
      if (st == 0) continue;
      unsigned short *stg = s_stage[nbuf++ & 1];
      u32 bits = x[i];
      u32 p = s_wtot[i][warp] + ex[i];
      const u32 q0 = threadIdx.x * 32;
      while (bits) {
        stg[p++] = (unsigned short)(q0 + (u32)(__ffs(bits) - 1));
        bits &= bits - 1;
      }
      __syncthreads();
      // staged position j holds the tuple of rank r0 + j
      const u64 r0 = tile_rank[t] + s_seg_off[i];
      const u64 wl0 = w0 + (u64)i * kBmBlock - seg.base_word;
      for (u32 j = threadIdx.x; j < st; j += kBmBlock) {
        const u32 q = stg[j];
        const u64 wl = wl0 + (q >> 5);
        const u64 lx = wl >> seg.row_shift;
        const u64 lz = ((wl & row_mask) << 5) | (q & 31u);
        h_sum += mix64(mix64(mix64(r0 + j) ^ lx) ^ lz);
      }
    }
    // one atomic per tile: the tile's terms summed over the block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) h_sum += __shfl_xor_sync(0xffffffffu, h_sum, o);
    if (lane == 0) s_red[warp] = h_sum;
    __syncthreads();
    if (threadIdx.x == 0) {
      u64 tot = 0;
      for (int w = 0; w < kBmBlock / 32; w++) tot += s_red[w];
      if (tot) atomicAdd(&acc[inst], tot);
    }
    __syncthreads();
  }
}

}  // namespace gdl
