// dense.cuh — bitmap form of relation versions over a small key domain.
//
// When every column value is below 2^dk with 2*dk <= 30, the whole key
// domain of an arity-2 relation is 2^(2dk) bits (at most 128 MB), and a
// version of the relation can be held as a bitmap whose bit (c0, c1) sits in
// row c0.  Bit order is the reference's tuple order (include/tuple.cuh:
// 106-126), so compacting a bitmap gives the sorted, deduplicated tuple list
// directly.  This replaces, for such domains, the sort -> unique ->
// set_difference -> merge sequence of the reference's update step
// (src/lie.cu:122-185, src/relation.cu:405-521, src/join.cu:160-225):
//   * joins and copies test-and-set bits of the output relation's NEWT
//     bitmap G (atomicOr), so the raw join output -- often tens of times
//     larger than its distinct tuples -- is never written to memory;
//   * one streaming pass over (G, F) per relation then yields DELTA =
//     G & ~F and FULL' = F | G as sorted lists, the next FULL bitmap, and
//     the run index of FULL' from per-row popcounts.
// Each scan is two kernels: k_bm_count computes per-tile counts and their
// exclusive prefixes (decoupled look-back) and checks the output
// capacities; k_bm_write writes.  Nothing but idempotent bit-sets happens
// before a capacity check, so an iteration that overflows can be re-run.
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
constexpr int kDenseMaxDomainBits = 30;
constexpr int kMaxInstanceNodes = 1 << 16;  // a row is at most one scan tile

// Where a key lives in the bitmap: the tuple (c0, c1) of instance
// i = c0 >> seg_shift is bit (c1 & 31) of word
//   seg[i].base_word + (local(c0) << seg[i].row_shift) + (local(c1) >> 5).
struct DenseMap {
  const SegInfo *seg;     // one entry per instance
  const u32 *tile_inst;   // instance of each scan tile (null: all instance 0)
  u32 n_inst;
  int seg_shift;          // 31 for the square domain (every id is local)
  u64 words;              // total bitmap words
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

// Set the bit of one key; keys outside their instance's range are dropped
// and recorded in Ctl::oob instead of being written.
__device__ __forceinline__ void dm_set(const DenseMap &m, u32 *bm, u64 key, Ctl *ctl) {
  u64 w;
  u32 b;
  if (dm_locate(m, key, &w, &b) && w < m.words)
    atomicOr(bm + w, 1u << b);
  else
    atomicOr(&ctl->oob, 8192u);
}

// Expressions a scan can compact, over the word pair (g, f).
enum BmExpr { kBmNone = 0, kBmDelta = 1, kBmUnion = 2 };
__device__ __forceinline__ u32 bm_eval(int ex, u32 g, u32 f) {
  return ex == kBmDelta ? (g & ~f) : ex == kBmUnion ? (f | g) : 0u;
}

struct BmScanRec {
  u64 total_a, total_b;  // list sizes
  u64 pop_g;             // popcount of g (accumulated, reset by k_bm_write)
  u32 overflow;
  u32 pad;
};

struct BmScanArgs {
  const u32 *g;    // NEWT bitmap (may be null: all zero)
  const u32 *f;    // FULL bitmap (may be null: all zero)
  u32 *f_next;     // if set: receives f | g
  // If set, g / f / f_next are this relation's bmG / bmF / bmF_next, read
  // from the device descriptor when the kernel starts: k_commit swaps bmF
  // and bmF_next on the device, so pointers captured in a graph would go
  // stale.
  const RelDev *rd;
  DenseMap map;
  int ex_a, ex_b;  // expressions for list a and list b
  DArr *list_a;    // output lists (sorted keys); null when not wanted
  DArr *list_b;
  Index *idx_b;    // if set: run index of list b
  u64 *count_b;    // if set: receives total_b (FULL count without a list)
  u64 *pop_g_out;  // if set: receives popcount(g) (NEWT size)
  u64 *inst_delta; // if set: per-instance count of list a is added here
  int need_a, need_b;  // need slots to raise on overflow (-1: none)
  int update_stage;    // an update-step scan: its overflow can be resumed
  u64 *tile_prefix;    // [tiles] packed exclusive prefix (a << 32 | b)
  u64 tiles_cap;
  BmScanRec *rec;
  LaunchRec *lrec;
  Lb lb;
  Ctl *ctl;
};

__device__ __forceinline__ u64 bm_tiles(u64 words) {
  return (words + kBmTileWords - 1) / kBmTileWords;
}

// Pass 1: per-tile counts, exclusive prefixes by decoupled look-back, and
// the capacity check (recorded in rec->overflow for k_bm_write to raise).
__global__ void __launch_bounds__(kBmBlock) k_bm_count(BmScanArgs a) {
  __shared__ u64 s_scan[kBmBlock / 32];
  __shared__ long long s_tile;
  if (ctl_stop(a.ctl)) return;
  const u64 words = a.map.words;
  const u64 tiles = bm_tiles(words);
  if (tiles > a.tiles_cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(&a.ctl->oob, 1024u);
    return;
  }
  if (a.rd) {
    a.g = a.rd->bmG;
    a.f = a.rd->bmF;
    a.f_next = a.rd->bmF_next;
  }
  const u32 gen = a.lrec->gen;
  u64 my_g = 0;
  while (true) {
    const long long tile = grab_tile(a.lrec, &s_tile);
    if (tile >= (long long)tiles) break;
    const u64 w0 = (u64)tile * kBmTileWords + (u64)threadIdx.x * kBmWordsPerThread;
    u32 ca = 0, cb = 0;
#pragma unroll
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u64 w = w0 + i;
      if (w < words) {
        const u32 g = a.g ? a.g[w] : 0u, f = a.f ? a.f[w] : 0u;
        ca += __popc(bm_eval(a.ex_a, g, f));
        cb += __popc(bm_eval(a.ex_b, g, f));
        my_g += __popc(g);
      }
    }
    u64 tot;
    block_excl_scan<kBmBlock>(((u64)ca << 32) | cb, s_scan, &tot);
    if (threadIdx.x < 32) {
      u64 prefix = 0;
      if (tile == 0) {
        if (threadIdx.x == 0) lb_publish(a.lb, tile, gen, true, tot);
      } else {
        if (threadIdx.x == 0) lb_publish(a.lb, tile, gen, false, tot);
        prefix = lb_warp_prefix(a.lb, tile, gen, a.ctl);
        if (threadIdx.x == 0) lb_publish(a.lb, tile, gen, true, prefix + tot);
      }
      if (threadIdx.x == 0) {
        a.tile_prefix[tile] = prefix;
        if ((u64)tile == tiles - 1) {
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
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) my_g += __shfl_xor_sync(0xffffffffu, my_g, o);
  if ((threadIdx.x & 31) == 0 && my_g) atomicAdd(&a.rec->pop_g, my_g);
  launch_rec_finish(a.lrec);
}

// Pass 2: write list a, list b (+ its index) and f_next.
struct BmWriteSmem {
  u32 off_b[kBmTileWords + 1];  // exclusive offsets of list b per word
  u64 scan_tmp[kBmBlock / 32];
};

__global__ void __launch_bounds__(kBmBlock) k_bm_write(BmScanArgs a) {
  __shared__ BmWriteSmem sm;
  if (ctl_stop(a.ctl)) return;
  if (a.rec->overflow) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      a.rec->pop_g = 0;
      if (a.update_stage) a.ctl->overflow_stage = 1;
      atomicExch(&a.ctl->overflow, 1u);
    }
    return;
  }
  const u64 words = a.map.words;
  const u64 tiles = bm_tiles(words);
  if (tiles > a.tiles_cap) return;
  if (a.rd) {
    a.g = a.rd->bmG;
    a.f = a.rd->bmF;
    a.f_next = a.rd->bmF_next;
  }
  const u32 epoch = (u32)(a.ctl->generation + 1);
  const Index ix = a.idx_b ? *a.idx_b : Index{};
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.idx_b) a.idx_b->epoch = epoch;
  u64 *la = a.list_a ? a.list_a->ptr : nullptr;
  u64 *lb = a.list_b ? a.list_b->ptr : nullptr;
  const u64 cap_a = a.list_a ? a.list_a->cap : 0, cap_b = a.list_b ? a.list_b->cap : 0;
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
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
      if (w < words) {
        g = a.g ? a.g[w] : 0u;
        f = a.f ? a.f[w] : 0u;
        if (a.f_next) a.f_next[w] = f | g;
      }
      ea[i] = bm_eval(a.ex_a, g, f);
      eb[i] = bm_eval(a.ex_b, g, f);
      ca += __popc(ea[i]);
      cb += __popc(eb[i]);
    }
    u64 tot;
    const u64 ex = block_excl_scan<kBmBlock>(((u64)ca << 32) | cb, sm.scan_tmp, &tot);
    if (threadIdx.x == 0 && a.inst_delta && (tot >> 32)) atomicAdd(&a.inst_delta[inst], tot >> 32);
    u64 pa = (prefix >> 32) + (ex >> 32);
    u64 pb = (prefix & 0xFFFFFFFFull) + (ex & 0xFFFFFFFFull);
    u32 ob = (u32)(ex & 0xFFFFFFFFull);
#pragma unroll
    for (int i = 0; i < kBmWordsPerThread; i++) {
      if (a.idx_b) sm.off_b[threadIdx.x * kBmWordsPerThread + i] = ob;
      ob += __popc(eb[i]);
      u32 x = la ? ea[i] : 0u;
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        if (pa < cap_a)
          la[pa] = dm_key(a.map, inst, seg, w0 + i, b);
        else
          atomicOr(&a.ctl->oob, 2048u);
        pa++;
      }
      x = lb ? eb[i] : 0u;
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        if (pb < cap_b)
          lb[pb] = dm_key(a.map, inst, seg, w0 + i, b);
        else
          atomicOr(&a.ctl->oob, 4096u);
        pb++;
      }
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
    }
    __syncthreads();
  }
  if (launch_rec_finish(a.lrec) && threadIdx.x == 0) {
    if (a.list_a) a.list_a->n = a.rec->total_a;
    if (a.list_b) a.list_b->n = a.rec->total_b;
    if (a.count_b) *a.count_b = a.rec->total_b;
    if (a.pop_g_out) *a.pop_g_out = a.rec->pop_g;
    a.rec->pop_g = 0;
    prof_add(a.ctl, kPBitmap,
             words * 4 * ((a.g ? 2 : 0) + (a.f ? 2 : 0) + (a.f_next ? 1 : 0)) +
                 8 * (a.rec->total_a + a.rec->total_b));
  }
}

// Zero a bitmap (words a multiple of 4).
__global__ void __launch_bounds__(256) k_bm_clear(u32 *bm, u64 words, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  uint4 *p = reinterpret_cast<uint4 *>(bm);
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < words / 4;
       i += (u64)gridDim.x * blockDim.x)
    p[i] = make_uint4(0, 0, 0, 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPBitmap, words * 4);
}

// Set the bits of a key list (FULL at the start of a LIE).
__global__ void __launch_bounds__(256) k_bm_from_list(const DArr *list, u32 *bm, DenseMap map,
                                                      Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 n = list->n;
  const u64 *k = list->ptr;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
    dm_set(map, bm, k[i], ctl);
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPBitmap, 8 * n);
}

// Emission.  A relation whose FULL list is not read during the loop
// (kEmitDelta) or whose NEWT is read as a list (kEmitNewt, tmp relations)
// gets its new keys listed by the ops themselves: the first thread to set a
// key's NEWT bit appends the key, so the update step works on the list and
// never scans the bitmap.  kEmitDelta skips keys already in FULL, so its
// list is DELTA itself.  A full list raises Ctl::overflow; the host then
// clears the NEWT bitmaps and runs the iteration again with larger lists.
struct EmitTarget {
  u32 *g;          // NEWT bitmap
  const u32 *f;    // FULL bitmap for kEmitDelta (keys in FULL are skipped)
  DArr *list;      // delta_next or newt; null: bits only (scan path)
  u64 *ptr;        // list storage and capacity, read once
  u64 cap;
  u64 *gen;        // tuples generated (kEmitDelta: is NEWT empty?)
  int need_slot;
};

__device__ __forceinline__ EmitTarget emit_target(RelDev *rd, int rel) {
  EmitTarget t;
  t.g = rd->bmG;
  t.f = rd->emit == kEmitDelta ? rd->bmF : nullptr;
  t.list = rd->emit == kEmitDelta ? &rd->delta_next : rd->emit == kEmitNewt ? &rd->newt : nullptr;
  t.ptr = t.list ? t.list->ptr : nullptr;
  t.cap = t.list ? t.list->cap : 0;
  t.gen = &rd->gen_count;
  t.need_slot = need_index(rel, rd->emit == kEmitDelta ? kNeedDelta : kNeedNewt);
  return t;
}

// Append `key` at position pos of the target list (bounds-checked).
__device__ __forceinline__ void emit_store(const EmitTarget &T, u64 pos, u64 key, Ctl *ctl) {
  if (pos < T.cap) {
    T.ptr[pos] = key;
  } else {
    atomicMax(&ctl->need[T.need_slot], pos + 1);
    atomicExch(&ctl->overflow, 1u);
  }
}

// Set one key's NEWT bit; true if this thread set it first (and it is not
// in FULL when the target checks FULL).
__device__ __forceinline__ bool emit_set(const DenseMap &m, const EmitTarget &T, u64 key, Ctl *ctl) {
  u64 w;
  u32 b;
  if (!dm_locate(m, key, &w, &b) || w >= m.words) {
    atomicOr(&ctl->oob, 8192u);
    return false;
  }
  if (T.f && ((T.f[w] >> b) & 1u)) return false;
  const u32 old = atomicOr(T.g + w, 1u << b);
  return !(old & (1u << b));
}

// Warp-synchronous emission of one candidate per lane (all 32 lanes call).
__device__ __forceinline__ void emit_warp(const DenseMap &m, const EmitTarget &T, bool valid,
                                          u64 key, Ctl *ctl) {
  const int lane = threadIdx.x & 31;
  const unsigned vm = __ballot_sync(0xffffffffu, valid);
  if (T.list && lane == 0 && vm) atomicAdd(T.gen, (u64)__popc(vm));
  const bool first = valid && emit_set(m, T, key, ctl);
  if (!T.list) return;
  const unsigned fm = __ballot_sync(0xffffffffu, first);
  if (!fm) return;
  const int leader = __ffs(fm) - 1;
  u64 base = 0;
  if (lane == leader) base = atomicAdd(&T.list->n, (u64)__popc(fm));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (first) emit_store(T, base + __popc(fm & ((1u << lane) - 1u)), key, ctl);
}

// The same for one thread alone.
__device__ __forceinline__ void emit_one(const DenseMap &m, const EmitTarget &T, u64 key, Ctl *ctl) {
  if (T.list) atomicAdd(T.gen, 1ull);
  if (emit_set(m, T, key, ctl) && T.list) emit_store(T, atomicAdd(&T.list->n, 1ull), key, ctl);
}

// RelationalJoin materialisation into the output's NEWT bitmap.  Balanced
// over candidate positions as k_join_mat: a block owns kMatTile consecutive
// positions, each thread kMatPer consecutive ones, found with one binary
// search over the tile's records and then walked forward.  A candidate is one
// inner read, the column move, the predicate and one atomicOr (outputs of
// different outer rows rarely share a bitmap word, so no warp aggregation of
// the bits; only list appends are aggregated).
constexpr int kMatPer = kMatTile / kMatBlock;  // positions per thread

__global__ void __launch_bounds__(kMatBlock) k_join_mat_bm(JoinArgs a, RelDev *out_rd,
                                                           DenseMap map) {
  __shared__ MatSmem sm;
  if (ctl_stop(a.ctl)) return;
  const u64 total = a.op->total;
  const u64 nc = a.op->nc;
  if (total == 0) return;
  const EmitTarget T = emit_target(out_rd, a.out_rel);
  const u64 *inner = a.inner->ptr;
  const u64 tiles = (total + kMatTile - 1) / kMatTile;
  for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
    const u64 p0 = tile * kMatTile;
    const u64 p1 = min(p0 + kMatTile, total);
    __syncthreads();
    if (threadIdx.x == 0) {
      u64 lo = 0, hi = nc;
      while (hi - lo > 1) {
        u64 mid = (lo + hi) >> 1;
        if (a.crow_off[mid] <= p0)
          lo = mid;
        else
          hi = mid;
      }
      sm.k0 = lo;
      sm.nrec = (u32)min((u64)kMatTile, nc - lo);
    }
    __syncthreads();
    const u64 k0 = sm.k0;
    const u32 m = sm.nrec;
    for (u32 i = threadIdx.x; i <= m; i += blockDim.x) {
      sm.off[i] = a.crow_off[k0 + i];
      if (i < m) {
        sm.start[i] = a.crow_start[k0 + i];
        sm.key[i] = a.crow_key[k0 + i];
      }
    }
    __syncthreads();
    u64 p = p0 + (u64)threadIdx.x * kMatPer;
    u32 r = 0;
    u64 next = 0;
    if (p < p1) {
      r = find_rec(sm.off, m, p);
      next = sm.off[r + 1];
    }
#pragma unroll
    for (int j = 0; j < kMatPer; j++, p++) {
      bool valid = p < p1;
      u64 t = 0;
      if (valid) {
        while (p >= next) {
          r++;
          next = sm.off[r + 1];
        }
        t = gen_join(a.sel, inner[sm.start[r] + (p - sm.off[r])], sm.key[r]);
        valid = pred_ok(a.pred, t);
      }
      emit_warp(map, T, valid, t, a.ctl);
    }
  }
  if (launch_rec_finish(a.rec) && threadIdx.x == 0)
    prof_add(a.ctl, kPJoinMat, 16 * total + 24 * nc);
}

// Clear one relation's NEWT: bitmap and emission list (ACopy replaces the
// destination's NEWT, src/acopy.cu:37-43).
__global__ void __launch_bounds__(256) k_newt_reset(RelDev *rd, DenseMap map, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  uint4 *p = reinterpret_cast<uint4 *>(rd->bmG);
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < map.words / 4;
       i += (u64)gridDim.x * blockDim.x)
    p[i] = make_uint4(0, 0, 0, 0);
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    if (rd->emit == kEmitDelta) rd->delta_next.n = 0;
    if (rd->emit == kEmitNewt) rd->newt.n = 0;
    rd->gen_count = 0;
    prof_add(ctl, kPBitmap, map.words * 4);
  }
}

// RelationalCopy into the destination's NEWT (src/copy.cu:12-95).  An empty
// source empties the destination NEWT (src/copy.cu:24-27).
__global__ void __launch_bounds__(256) k_copy_bm(CopyArgs c, RelDev *dest_rd, DenseMap map) {
  if (ctl_stop(c.ctl)) return;
  if (c.once && *c.once) return;
  const u64 n = eff_count(c.src, c.src_vis);
  if (n == 0) {
    uint4 *p = reinterpret_cast<uint4 *>(dest_rd->bmG);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < map.words / 4;
         i += (u64)gridDim.x * blockDim.x)
      p[i] = make_uint4(0, 0, 0, 0);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      if (c.once_pending) *c.once_pending = 1;
      if (dest_rd->emit == kEmitDelta) dest_rd->delta_next.n = 0;
      if (dest_rd->emit == kEmitNewt) dest_rd->newt.n = 0;
      dest_rd->gen_count = 0;
    }
    return;
  }
  const EmitTarget T = emit_target(dest_rd, c.dest_rel);
  const u64 *src = c.src->ptr;
  for (u64 i0 = (u64)blockIdx.x * blockDim.x; i0 < n; i0 += (u64)gridDim.x * blockDim.x) {
    const u64 i = i0 + threadIdx.x;
    const bool valid = i < n;
    emit_warp(map, T, valid, valid ? gen_join(c.sel, src[i], 0) : 0, c.ctl);
  }
  if (launch_rec_finish(c.rec) && threadIdx.x == 0) {
    if (c.once_pending) *c.once_pending = 1;
    prof_add(c.ctl, kPCopy, 8 * n);
  }
}

// RelationalACopy (src/acopy.cu:12-50): dest NEWT := sel(src NEWT); the
// destination was reset by k_newt_reset just before.  The source NEWT is
// its list when it has one, else its bitmap.
__global__ void __launch_bounds__(256) k_acopy_bm(const RelDev *src_rd, Sel2 sel, RelDev *dest_rd,
                                                  int dest_rel, DenseMap map, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const EmitTarget T = emit_target(dest_rd, dest_rel);
  if (src_rd->emit == kEmitNewt) {
    const u64 n = src_rd->newt.n;
    const u64 *src = src_rd->newt.ptr;
    for (u64 i0 = (u64)blockIdx.x * blockDim.x; i0 < n; i0 += (u64)gridDim.x * blockDim.x) {
      const u64 i = i0 + threadIdx.x;
      const bool valid = i < n;
      emit_warp(map, T, valid, valid ? gen_join(sel, src[i], 0) : 0, ctl);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPCopy, 8 * n);
    return;
  }
  const u32 *src_bm = src_rd->bmG;
  for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < map.words;
       w += (u64)gridDim.x * blockDim.x) {
    u32 x = src_bm[w];
    if (!x) continue;
    const u32 inst = dm_tile_inst(map, w / kBmTileWords);
    const SegInfo seg = map.seg[inst];
    while (x) {
      const int b = __ffs(x) - 1;
      x &= x - 1;
      emit_one(map, T, gen_join(sel, dm_key(map, inst, seg, w, b), 0), ctl);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPCopy, map.words * 4);
}

// Update step of an emitting relation.  kEmitDelta: delta_next already is
// DELTA; kEmitNewt: DELTA = the NEWT keys not in FULL.  Then FULL |= DELTA
// in place and the NEWT bitmap is cleared word by word from the list (its
// bits are exactly the listed keys).  With inst_delta set, each instance
// that gained a key is flagged.
__global__ void __launch_bounds__(256) k_emit_update(RelDev *rd, int rel, DenseMap map,
                                                     u64 *inst_delta, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const bool from_newt = rd->emit == kEmitNewt;
  const DArr &L = from_newt ? rd->newt : rd->delta_next;
  const u64 n = L.n;
  const u64 *keys = L.ptr;
  u32 *F = rd->bmF, *G = rd->bmG;
  DArr *D = &rd->delta_next;
  u64 *dptr = D->ptr;
  const u64 dcap = D->cap;
  const int lane = threadIdx.x & 31;
  for (u64 i0 = (u64)blockIdx.x * blockDim.x; i0 < n; i0 += (u64)gridDim.x * blockDim.x) {
    const u64 i = i0 + threadIdx.x;
    bool add = false;
    u64 key = 0, w = 0;
    u32 b = 0;
    if (i < n) {
      key = keys[i];
      if (dm_locate(map, key, &w, &b) && w < map.words) {
        G[w] = 0;
        add = !from_newt || !((F[w] >> b) & 1u);
      } else {
        atomicOr(&ctl->oob, 8192u);
      }
    }
    if (add) {
      atomicOr(F + w, 1u << b);
      if (inst_delta) inst_delta[key_c0(key) >> map.seg_shift] = 1;
    }
    if (from_newt) {
      const unsigned am = __ballot_sync(0xffffffffu, add);
      if (am) {
        const int leader = __ffs(am) - 1;
        u64 base = 0;
        if (lane == leader) base = atomicAdd(&D->n, (u64)__popc(am));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (add) {
          const u64 pos = base + __popc(am & ((1u << lane) - 1u));
          if (pos < dcap) {
            dptr[pos] = key;
          } else {
            atomicMax(&ctl->need[need_index(rel, kNeedDelta)], pos + 1);
            atomicOr(&ctl->oob, 16384u);  // cannot happen: delta_next >= newt
          }
        }
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPBitmap, 16 * n);
}

// Clear a NEWT bitmap word by word from its list (tmp relations at the end
// of an iteration).
__global__ void __launch_bounds__(256) k_newt_unset(RelDev *rd, DenseMap map, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 n = rd->newt.n;
  const u64 *keys = rd->newt.ptr;
  u32 *G = rd->bmG;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    u64 w;
    u32 b;
    if (dm_locate(map, keys[i], &w, &b) && w < map.words) G[w] = 0;
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
  __shared__ u32 s_off[257];
  const u64 tiles = bm_tiles(map.words);
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    const u32 inst = dm_tile_inst(map, t);
    const SegInfo seg = map.seg[inst];
    const u64 w0 = t * kBmTileWords + (u64)threadIdx.x * kBmWordsPerThread;
    u32 cnt = 0;
    for (int i = 0; i < kBmWordsPerThread; i++)
      if (w0 + i < map.words) cnt += __popc(bm[w0 + i]);
    // exclusive scan of cnt over the block (small, via shared memory)
    s_off[threadIdx.x] = cnt;
    __syncthreads();
    if (threadIdx.x == 0) {
      u32 run = 0;
      for (int k = 0; k < 256; k++) {
        const u32 v = s_off[k];
        s_off[k] = run;
        run += v;
      }
    }
    __syncthreads();
    u64 rank = tile_rank[t] + s_off[threadIdx.x];
    u64 h_sum = 0;
    for (int i = 0; i < kBmWordsPerThread; i++) {
      const u64 w = w0 + i;
      if (w >= map.words) break;
      u32 x = bm[w];
      while (x) {
        const int b = __ffs(x) - 1;
        x &= x - 1;
        const u64 wl = w - seg.base_word;
        const u64 lx = wl >> seg.row_shift;
        const u64 lz = ((wl & ((1ull << seg.row_shift) - 1)) << 5) + (u64)b;
        u64 h = mix64(rank);
        h = mix64(h ^ lx);
        h = mix64(h ^ lz);
        h_sum += h;
        rank++;
      }
    }
    if (h_sum) atomicAdd(&acc[inst], h_sum);
    __syncthreads();
  }
}

}  // namespace gdl
