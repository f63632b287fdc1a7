// pull.cuh — joins into bitmaps gathered by output row ("pull" form).
//
// A join whose output tuple is (outer column 1, inner column 1), joined on
// column 0 of both sides, makes output row r the union of the inner runs
// I[k] over the keys k with (k, r) in the outer.  Same generation's two
// recursive rules have this shape (test/sg.cu:165-175):
//   tmp(b, x) :- sg(a, b), edge(a, x)       sg(x, y) :- tmp(b, x), edge(b, y)
// and so do CSPA's joins (test/cspa.cu:279-352).  The push form
// (k_join_bm, dense.cuh) walks the outer in key order and sends one L2
// reduction per candidate tuple, and the candidates of one output row
// repeat each other many times over: on R-MAT graphs 35-49 candidates fall
// on each distinct output word.  Here the outer is read transposed — bit
// (r, k) of OT is outer tuple (k, r) — so that one block sees a run of a
// row's keys together, gathers the row in shared memory and sends one
// reduction per nonzero word.
//
//   k_bm_transpose  OT := transpose(g) or transpose(g & ~f) (the DELTA that
//                   the next update step lists), in 256 x 256-bit tiles:
//                   each 32 x 32 block is transposed in registers with five
//                   shuffle rounds and written out through shared memory
//                   as whole 32-byte sectors.  Optionally counts the bits
//                   (the size of a NEWT outer, whose list is not built).
//   k_join_pull_bm  a block per unit of 256 OT words (part of one row, or
//                   several short rows), taken from a work counter (an
//                   empty unit costs one barrier after the grab): lists
//                   the unit's keys into shared memory (each thread those
//                   of its word), takes them 256 at a time, probes the
//                   inner index (one 16-byte slot per key), expands the
//                   runs balanced over the block into the shared row (2
//                   consecutive candidates per thread, so a run is read in
//                   16-byte pieces), then ORs the row's nonzero words into
//                   the output.  A long run whose inner is a FULL kept as
//                   a bitmap is ORed from that bitmap's row instead.
//   k_bm_update_t   the update step of a relation whose DELTA only these
//                   joins read, in one pass that also writes DELTA
//                   transposed.
//   k_bm_fold_t     for a join whose output is (inner column 1, outer
//                   column 1): the same kernel gathers by the outer's
//                   column 1 into a transposed twin of the output NEWT,
//                   which this pass ORs into NEWT transposed and clears.
//
// The square domain only (ids below 2^dk, 8 <= dk <= 16; one instance).
#pragma once

#include "common.cuh"
#include "dense.cuh"
#include "index.cuh"
#include "join.cuh"

namespace gdl {

constexpr int kTrBlock = 256;
constexpr int kPullBlock = 256;
constexpr int kPullUnit = 256;   // OT words per unit of work (a word per thread): 8192 keys
constexpr int kPullPer = 2;      // consecutive candidates per thread and step
constexpr int kPullMinBits = 8;  // a transposed tile is 256 ids square
constexpr int kPullAutoBits = 10;  // the pull form by default from 2^10 ids on

// Lane l holds row l of a 32 x 32 bit block (bit j = column j); afterwards
// lane j holds column j (bit l = row l).  Each round swaps the off-diagonal
// quarters of the blocks of side 2s between lane pairs l, l ^ s.
// A lane keeps the bits of `keep` (m in the lower lane of a pair, ~m in
// the upper) and takes the others from its partner's word rotated into
// place: left by s in the lower lane, right by s in the upper.  The bits
// that wrap around in the rotation fall outside the taken mask (m = ~m >> s
// and ~m = m << s for these masks), so one funnel shift and one select do
// a round.
__device__ __forceinline__ u32 transpose32(u32 x, int lane) {
  const u32 masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int i = 0; i < 5; i++) {
    const int s = 16 >> i;
    const bool up = (lane & s) != 0;
    const u32 keep = up ? ~masks[i] : masks[i];
    const u32 y = __shfl_xor_sync(0xffffffffu, x, s);
    const u32 r = __funnelshift_l(y, y, up ? 32 - s : s);
    x = (x & keep) | (r & ~keep);
  }
  return x;
}

struct TransposeArgs {
  const u32 *g;   // source bitmap
  const u32 *f;   // if set: the source is g & ~f
  u32 *dst;       // transposed bitmap (every word written)
  int dk;         // 2^dk ids, rows of 2^(dk-5) words
  DArr *count_to; // if set: receives the number of bits as its n
  u64 *count_acc; // zero between launches
  LaunchRec *lrec;
  Ctl *ctl;
};

__global__ void __launch_bounds__(kTrBlock) k_bm_transpose(TransposeArgs a) {
  __shared__ u32 s_t[256][9];  // the transposed tile; row pitch 9 avoids bank conflicts
  __shared__ unsigned long long s_bits;
  if (ctl_stop(a.ctl)) return;
  const int rs = a.dk - 5;
  const u64 per = 1ull << (a.dk - 8);  // tiles per side
  const u64 tiles = per * per;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u64 bits = 0, moved = 0;
  for (u64 t = blockIdx.x; t < tiles; t += gridDim.x) {
    const u64 tr = t / per, tc = t % per;
    // this thread's input row: tile row tr, row threadIdx.x of the tile
    // (warp wid holds rows 32 wid .. 32 wid + 31), words 8 tc .. 8 tc + 7
    const u64 src = ((tr * 256 + (u64)threadIdx.x) << rs) + tc * 8;
    u32 v[8];
    load8(a.g + src, v);
    bool any = (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) != 0u;
    moved += 32;
    if (a.f && any) {
      u32 w[8];
      load8(a.f + src, w);
      moved += 32;
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] &= ~w[i];
      any = (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) != 0u;
    }
#pragma unroll
    for (int i = 0; i < 8; i++) bits += __popc(v[i]);
    // (a tile's reads of s_t are ordered before the next tile's writes by
    // the next tile's __syncthreads_or)
    const bool tile_any = __syncthreads_or(any);
    uint4 *d = reinterpret_cast<uint4 *>(a.dst + ((tc * 256 + (u64)threadIdx.x) << rs) + tr * 8);
    if (tile_any) {
#pragma unroll
      for (int i = 0; i < 8; i++) {
        // lane j: input column 32 (8 tc + i) + j = output row, its bits
        // the input rows 256 tr + 32 wid + l = output word 8 tr + wid
        s_t[i * 32 + lane][wid] = transpose32(v[i], lane);
      }
      __syncthreads();
      const u32 *q = s_t[threadIdx.x];
      d[0] = make_uint4(q[0], q[1], q[2], q[3]);
      d[1] = make_uint4(q[4], q[5], q[6], q[7]);
    } else {
      d[0] = make_uint4(0, 0, 0, 0);
      d[1] = make_uint4(0, 0, 0, 0);
    }
    moved += 32;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    bits += __shfl_xor_sync(0xffffffffu, bits, o);
    moved += __shfl_xor_sync(0xffffffffu, moved, o);
  }
  if (lane == 0) prof_add(a.ctl, kPBitmap, moved);
  if (!a.count_to) return;
  if (threadIdx.x == 0) s_bits = 0;
  __syncthreads();
  if (lane == 0 && bits) atomicAdd(&s_bits, (unsigned long long)bits);
  __syncthreads();
  if (threadIdx.x == 0 && s_bits) atomicAdd(reinterpret_cast<unsigned long long *>(a.count_acc), s_bits);
  if (launch_rec_finish(a.lrec) && threadIdx.x == 0) {
    a.count_to->n = *a.count_acc;
    *a.count_acc = 0;
  }
}

// The update step of a relation whose DELTA only pull-form joins read and
// whose FULL is not read as a list during the loop, in one pass over the
// 256 x 256-bit tiles (instead of count, scan, write and transpose passes):
// DELTA = G & ~F counted and written transposed into dt, F |= G and G
// cleared where G has bits, NEWT's size counted.  Behind the write passes'
// capacity gate: when another relation's list is too small nothing is
// written and the update step runs again after the lists grow.  gt: when
// every join that writes the relation has a transposed output and nothing
// reads its NEWT during the iteration, NEWT is only that transposed twin
// (never folded): it is read transposed, tile by tile, and cleared.
__global__ void __launch_bounds__(kTrBlock, 4) k_bm_update_t(BmScanArgs a, u32 *dt, int dk, u32 *gt,
                                                          u32 *dn) {
  __shared__ u32 s_t[256][9];
  __shared__ unsigned long long s_cnt[2];
  if (ctl_stop(a.ctl)) return;
  if (write_gate_closed(a)) return;
  scan_bind(a);
  u32 *G = const_cast<u32 *>(a.g);
  u32 *F = a.f;
  const int rs = dk - 5;
  const u64 per = 1ull << (dk - 8);
  const u64 tiles = per * per;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (threadIdx.x < 2) s_cnt[threadIdx.x] = 0;
  // the loop below may have no barrier (no transposed output): order the
  // zeroing before any warp's atomicAdd into s_cnt
  __syncthreads();
  u64 n_delta = 0, n_newt = 0, moved = 0;
  // NEWT's words of a tile: from G (row-major, at `src`) or from gt (the
  // transposed twin, at the mirrored tile).  Software-pipelined: the next
  // tile's NEWT words load while this tile is processed.
  auto newt_at = [&](u64 tt) {
    const u64 r = tt / per, c = tt % per;
    return gt ? ((c * 256 + (u64)threadIdx.x) << rs) + r * 8
              : ((r * 256 + (u64)threadIdx.x) << rs) + c * 8;
  };
  const u32 *nsrc = gt ? gt : G;
  u64 t = blockIdx.x;
  u32 nx[8];
  if (t < tiles) load8(nsrc + newt_at(t), nx);
  // A tile's reads of s_t are ordered before the next writes of s_t by the
  // __syncthreads_or that precedes every write.
  for (; t < tiles; t += gridDim.x) {
    const u64 tr = t / per, tc = t % per;
    const u64 src = ((tr * 256 + (u64)threadIdx.x) << rs) + tc * 8;
    u32 g[8], d[8], cur[8], f[8];
#pragma unroll
    for (int i = 0; i < 8; i++) cur[i] = nx[i];
    if (t + gridDim.x < tiles) load8(nsrc + newt_at(t + gridDim.x), nx);
    bool have_f = false;
    if (gt) {
      // NEWT's tile (tr, tc) is the transpose of gt's tile (tc, tr)
      const u64 tsrc = ((tc * 256 + (u64)threadIdx.x) << rs) + tr * 8;
      const bool any_v = (cur[0] | cur[1] | cur[2] | cur[3] | cur[4] | cur[5] | cur[6] | cur[7]) != 0u;
      moved += 32;
      if (any_v) {
        uint4 *pv = reinterpret_cast<uint4 *>(gt + tsrc);
        pv[0] = make_uint4(0, 0, 0, 0);
        pv[1] = make_uint4(0, 0, 0, 0);
        moved += 32;
      }
      if (__syncthreads_or(any_v)) {
        // FULL's words of the tile load while it is transposed
        load8(F + src, f);
        have_f = true;
        moved += 32;
#pragma unroll
        for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(cur[i], lane);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 8; i++) g[i] = s_t[threadIdx.x][i];
      } else {
#pragma unroll
        for (int i = 0; i < 8; i++) g[i] = 0;
      }
    } else {
#pragma unroll
      for (int i = 0; i < 8; i++) g[i] = cur[i];
      moved += 32;
    }
    const bool any_g = (g[0] | g[1] | g[2] | g[3] | g[4] | g[5] | g[6] | g[7]) != 0u;
    bool any = false;
#pragma unroll
    for (int i = 0; i < 8; i++) d[i] = 0;
    if (any_g) {
      if (!have_f) {
        load8(F + src, f);
        moved += 32;
      }
      uint4 *pf = reinterpret_cast<uint4 *>(F + src);
      pf[0] = make_uint4(f[0] | g[0], f[1] | g[1], f[2] | g[2], f[3] | g[3]);
      pf[1] = make_uint4(f[4] | g[4], f[5] | g[5], f[6] | g[6], f[7] | g[7]);
      moved += 32;
      if (!gt) {
        uint4 *pg = reinterpret_cast<uint4 *>(G + src);
        pg[0] = make_uint4(0, 0, 0, 0);
        pg[1] = make_uint4(0, 0, 0, 0);
        moved += 32;
      }
#pragma unroll
      for (int i = 0; i < 8; i++) {
        d[i] = g[i] & ~f[i];
        n_delta += __popc(d[i]);
        n_newt += __popc(g[i]);
        any |= d[i] != 0u;
      }
    }
    if (dn) {
      // DELTA's rows as they are, for row-gather joins (every word written)
      uint4 *pn = reinterpret_cast<uint4 *>(dn + src);
      pn[0] = make_uint4(d[0], d[1], d[2], d[3]);
      pn[1] = make_uint4(d[4], d[5], d[6], d[7]);
      moved += 32;
    }
    if (dt) {  // (uniform over the launch)
      const bool tile_any = __syncthreads_or(any);
      uint4 *o = reinterpret_cast<uint4 *>(dt + ((tc * 256 + (u64)threadIdx.x) << rs) + tr * 8);
      if (tile_any) {
#pragma unroll
        for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(d[i], lane);
        __syncthreads();
        const u32 *q = s_t[threadIdx.x];
        o[0] = make_uint4(q[0], q[1], q[2], q[3]);
        o[1] = make_uint4(q[4], q[5], q[6], q[7]);
      } else {
        o[0] = make_uint4(0, 0, 0, 0);
        o[1] = make_uint4(0, 0, 0, 0);
      }
      moved += 32;
    }
  }
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
  if (threadIdx.x == 0) {
    if (s_cnt[0]) atomicAdd(reinterpret_cast<unsigned long long *>(&a.rec->total_a), s_cnt[0]);
    if (s_cnt[1]) atomicAdd(reinterpret_cast<unsigned long long *>(&a.rec->pop_g), s_cnt[1]);
  }
  if (launch_rec_finish(a.lrec) && threadIdx.x == 0) {
    *a.count_a = a.rec->total_a;
    *a.pop_g_out = a.rec->pop_g;
    a.rec->total_a = 0;
    a.rec->pop_g = 0;
  }
}

// Shared state of k_join_pull_bm.  The row accumulator is the dynamic
// shared memory: pull_acc_words(dk) words.
struct PullSmem {
  unsigned short keys[kPullUnit * 32];  // the unit's keys in order: word << 5 | bit
  u32 off[kPullBlock];      // exclusive candidate offsets of the round's keys
  u32 start[kPullBlock];    // inner run start of each key
  u32 arow[kPullBlock];     // accumulator offset of each key's output row
  u32 row_key[kPullBlock];  // the round's keys ORed as inner bitmap rows
  u32 row_arow[kPullBlock];
  u32 n_rows;
  u64 scan_tmp[kPullBlock / 32];
  long long unit;
};

// The accumulator holds the unit's rows, and at least one whole row (the
// output columns of a key can be anywhere in its row): max(256, 2^(dk-5)).
__host__ __device__ __forceinline__ u32 pull_acc_words(int dk) {
  return 1u << (dk - 5 > 8 ? dk - 5 : 8);
}

// G / D: the output bitmap and its dirty map (or null): the output
// relation's NEWT, or its transposed twin for a join whose output is
// (inner column 1, outer column 1).
__global__ void __launch_bounds__(kPullBlock, 8) k_join_pull_bm(JoinArgs a, u32 *G, u8 *D,
                                                               const u32 *OT, int dk) {
  __shared__ PullSmem sm;
  extern __shared__ u32 acc[];
  if (ctl_stop(a.ctl)) return;
  const u64 n_outer = eff_count(a.outer, a.outer_vis);
  const u64 n_inner = eff_count(a.inner, a.inner_vis);
  if (n_outer == 0 || n_inner == 0) {
    join_empty_side(a, n_outer);
    return;
  }
  const Index ix = *a.inner_idx;
  const u64 *inner = a.inner->ptr;
  const int tid = threadIdx.x;
  const int rs = dk - 5;
  const u32 row_mask = (1u << rs) - 1;
  const u32 acc_words = pull_acc_words(dk);
  const u32 units = (u32)((1ull << (2 * dk - 5)) / kPullUnit);
  const u32 n_ids = 1u << dk;
  // Row-OR (the inner is a FULL kept as a bitmap): a run of at least a
  // quarter of a row is ORed from the inner's bitmap row instead of being
  // expanded, 4 bytes a word read coalesced instead of a search, 8 bytes
  // and a shared atomic per candidate.
  const u32 *F = a.row_or ? a.inner_rd->bmF : nullptr;
  const u32 row_min = max(64u, (1u << rs) >> 2);
  for (u32 i = tid; i < acc_words; i += kPullBlock) acc[i] = 0;
  if (tid == 0) sm.n_rows = 0;
  u64 cand = 0, keys = 0, flushed = 0, row_words = 0;
  while (true) {
    const long long g = grab_tile(a.rec, &sm.unit);
    if (g >= (long long)units) break;
    const u32 u = (u32)g;
    const u32 w0 = u * kPullUnit;  // below 2^27
    const u32 wv = OT[w0 + tid];
    if (!__syncthreads_or(wv != 0u)) continue;  // an empty unit: one barrier
    u64 tot64;
    u32 pos = (u32)block_excl_scan<kPullBlock>((u64)__popc(wv), sm.scan_tmp, &tot64);
    const u32 tot = (u32)tot64;
    if (tot == 0) continue;  // block-uniform
    // each thread lists its own word's keys in place (the unit's keys in
    // order: word-major, then bit)
    for (u32 x = wv; x; x &= x - 1) sm.keys[pos++] = (unsigned short)((tid << 5) | (__ffs(x) - 1));
    __syncthreads();
    keys += tot;
    const u32 r0 = w0 >> rs;  // first output row of the unit
    for (u32 q0 = 0; q0 < tot; q0 += kPullBlock) {
      const u32 q = q0 + tid;
      u32 len = 0, st = 0, arow = 0;
      if (q < tot) {
        const u32 kb = sm.keys[q];
        const u32 b = kb & 31u;
        const u32 ow = w0 + (kb >> 5);  // OT word: row ow >> rs, keys 32 (ow & row_mask) ..
        arow = ((ow >> rs) - r0) << rs;
        const u32 key = ((ow & row_mask) << 5) + b;
        len = index_probe(ix, key, &st);
        if (F && len >= row_min) {
          const u32 slot = atomicAdd(&sm.n_rows, 1u);
          sm.row_key[slot] = key;
          sm.row_arow[slot] = arow;
          len = 0;
        }
      }
      u64 ctot64;
      sm.off[tid] = (u32)block_excl_scan<kPullBlock>((u64)len, sm.scan_tmp, &ctot64);
      const u32 ctot = (u32)ctot64;  // at most 256 runs of at most 2^16
      sm.start[tid] = st;
      sm.arow[tid] = arow;
      __syncthreads();
      // kPullPer consecutive candidates per thread: one search for the
      // first (the last key whose offset is <= p; an empty run shares its
      // offset with the next key, so it is never the last), then walked
      // forward; the loads are issued before the ORs
      for (u32 p0 = tid * kPullPer; p0 < ctot; p0 += kPullBlock * kPullPer) {
        u32 j = 0;
#pragma unroll
        for (u32 h = kPullBlock / 2; h > 0; h >>= 1)
          if (sm.off[j + h] <= p0) j += h;
        u32 jend = j + 1 < kPullBlock ? sm.off[j + 1] : ctot;
        u32 col[kPullPer], ar[kPullPer];
#pragma unroll
        for (int i = 0; i < kPullPer; i++) {
          const u32 p = p0 + i;
          col[i] = ~0u;
          if (p < ctot) {
            while (p >= jend) {  // next non-empty run
              j++;
              jend = j + 1 < kPullBlock ? sm.off[j + 1] : ctot;
            }
            col[i] = key_c1(inner[sm.start[j] + (p - sm.off[j])]);
            ar[i] = sm.arow[j];
          }
        }
#pragma unroll
        for (int i = 0; i < kPullPer; i++) {
          if (col[i] == ~0u) continue;
          if (col[i] < n_ids)
            atomicOr(&acc[ar[i] + (col[i] >> 5)], 1u << (col[i] & 31));
          else
            atomicOr(&a.ctl->oob, 8192u);
        }
      }
      cand += ctot;
      __syncthreads();
      if (F) {
        // the round's row keys, after its candidates (plain ORs: each
        // word of the shared row belongs to one thread)
        const u32 nr = sm.n_rows;
        __syncthreads();  // every thread has read the count
        for (u32 i = 0; i < nr; i++) {
          const u32 *src = F + ((u64)sm.row_key[i] << rs);
          u32 *dst = acc + sm.row_arow[i];
          for (u32 w = tid; w < (1u << rs); w += kPullBlock) {
            const u32 v = src[w];
            if (v) dst[w] |= v;
          }
        }
        row_words += (u64)nr << rs;
        if (tid == 0) sm.n_rows = 0;
        __syncthreads();  // rows ORed, count reset before the next round's probes
      }
    }
    // flush the unit's rows: one reduction per nonzero word
    for (u32 i = tid; i < acc_words; i += kPullBlock) {
      const u32 v = acc[i];
      if (v) {
        const u64 gw = ((u64)r0 << rs) + i;
        asm volatile("red.global.or.b32 [%0], %1;" ::"l"(G + gw), "r"(v) : "memory");
        if (D) D[gw / kBmChunkWords] = 1;
        acc[i] = 0;
        flushed++;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) flushed += __shfl_xor_sync(0xffffffffu, flushed, o);
  // algorithmic bytes: 4 per OT word, 16 per key (its index slot), 8 per
  // candidate (the inner tuple), 4 per inner bitmap word of a row-OR key,
  // 4 per word reduced into the output
  if ((tid & 31) == 0) prof_add(a.ctl, kPJoinMat, 4 * flushed);
  if (tid == 0) prof_add(a.ctl, kPJoinMat, 16 * keys + 8 * cand + 4 * row_words);
  if (launch_rec_finish(a.rec) && tid == 0) prof_add(a.ctl, kPJoinMat, 4ull * units * kPullUnit);
}

// ---------------------------------------------------------------------------
// Row-gather joins.  The same joins as k_join_pull_bm, computed the other
// way round: output column y (an inner column-1 value) is the union of the
// outer's bitmap ROWS O[k] over the inner's in-edges (k, y):
//     Out^T[y] = OR over k in inner^T[y] of O[k].
// Its work is |inner| bitmap rows of 2^(dk-5) words, read coalesced,
// whatever the number of candidate tuples (which the pull form expands one
// shared-memory atomic each: 4-8x more work on same generation's dense
// iterations).  It fits a small inner kept static through the LIE (an edge
// relation): its in-edges are listed once (k_inv_*) and kept until the
// relation is loaded again or a LIE updates it.  The output is
// the transpose of the pull form's, so the two forms swap the roles of the
// output's NEWT and its transposed twin.
// ---------------------------------------------------------------------------
constexpr int kRowsMinBits = 12;   // a bitmap row is at least 32 uint4 (one per lane)
constexpr unsigned long long kRowsBudget = 256ull << 20;  // |inner| x row bytes, auto mode

// In-edges of a sorted key list (k << 32 | y): counts per y.
__global__ void __launch_bounds__(256) k_inv_count(const DArr *list, u32 *cnt, int dk, Ctl *ctl) {
  const u64 n = list->n;
  const u32 lim = 1u << dk;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u32 y = key_c1(list->ptr[i]);
    if (y < lim && key_c0(list->ptr[i]) < lim)
      atomicAdd(&cnt[y], 1u);
    else
      atomicOr(&ctl->oob, 8192u);
  }
}

// Scatter: the in-edges of y at [off[y], off[y+1]), each edge's source in
// keys and its y in ys (the order inside a y does not matter: the gather
// ORs).
__global__ void __launch_bounds__(256) k_inv_fill(const DArr *list, u32 *cur, u32 *keys, u32 *ys,
                                                  int dk) {
  const u64 n = list->n;
  const u32 lim = 1u << dk;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u64 kk = list->ptr[i];
    const u32 y = key_c1(kk), k = key_c0(kk);
    if (y >= lim || k >= lim) continue;
    const u32 pos = atomicAdd(&cur[y], 1u);
    keys[pos] = k;
    ys[pos] = y;
  }
}

constexpr int kInvBlock = 1024;
constexpr int kInvPer = 8;  // consecutive ids per thread and chunk

// One block: from the in-degree counts cnt[y] (2^dk of them), the edge
// offsets off[0..2^dk] and the fill cursors cur (a copy; cur may be cnt).
// Chunks of kInvBlock x kInvPer ids, each thread kInvPer consecutive ones
// read and written as 16-byte vectors.
__global__ void __launch_bounds__(kInvBlock) k_inv_offsets(const u32 *cnt, u32 *off, u32 *cur,
                                                           int dk) {
  __shared__ u64 s_warp[kInvBlock / 32];
  const u32 n = 1u << dk;  // a multiple of kInvPer
  u64 carry = 0;           // edges of the chunks before
  for (u32 c0 = 0; c0 < n; c0 += kInvBlock * kInvPer) {
    const u32 b = c0 + kInvPer * threadIdx.x;
    u32 v[kInvPer];
    if (b < n) {
      const uint4 x = reinterpret_cast<const uint4 *>(cnt + b)[0];
      const uint4 y = reinterpret_cast<const uint4 *>(cnt + b)[1];
      v[0] = x.x, v[1] = x.y, v[2] = x.z, v[3] = x.w;
      v[4] = y.x, v[5] = y.y, v[6] = y.z, v[7] = y.w;
    } else {
#pragma unroll
      for (int i = 0; i < kInvPer; i++) v[i] = 0;
    }
    u64 local = 0;
#pragma unroll
    for (int i = 0; i < kInvPer; i++) local += v[i];
    u64 tot;
    const u64 ex = block_excl_scan<kInvBlock>(local, s_warp, &tot) + carry;
    carry += tot;
    if (b >= n) continue;
    u32 e = (u32)ex;
    u32 o[kInvPer];
#pragma unroll
    for (int i = 0; i < kInvPer; i++) {
      o[i] = e;
      e += v[i];
    }
    uint4 *po4 = reinterpret_cast<uint4 *>(off + b), *pc4 = reinterpret_cast<uint4 *>(cur + b);
    po4[0] = make_uint4(o[0], o[1], o[2], o[3]);
    po4[1] = make_uint4(o[4], o[5], o[6], o[7]);
    pc4[0] = make_uint4(o[0], o[1], o[2], o[3]);
    pc4[1] = make_uint4(o[4], o[5], o[6], o[7]);
  }
  if (threadIdx.x == 0) off[n] = (u32)carry;
}

struct RowsArgs {
  JoinArgs j;          // outer / inner descriptors (emptiness rules), ctl, launch record,
                       // the run-once flags of a join over static FULLs
  const u32 *O;        // the outer's rows: DELTA (non-transposed copy), a tmp NEWT, or a
                       // static FULL's bitmap
  u32 *outer_clear;    // bitmap to clear if an empty inner zeroes a NEWT outer
  const u32 *inv_keys;  // in-edge sources, grouped by y
  const u32 *inv_ys;    // the y of each in-edge
  const u32 *inv_off;   // inv_off[2^dk]: the number of in-edges
  u32 unit;             // in-edges per unit of work (8, 16 or 32)
  u32 *dst;            // output rows y (the output's NEWT or its transposed twin)
  u8 *dirty;           // dirty map of dst, or null
  int dst_zero;        // dst is all zero when the launch starts
  int clear_diag;      // predicate t[0] != t[1]: bit (y, y) dropped from row y
  int dk;
};

// One output row's words held by a warp: lane l holds uint4 number
// j * 32 + l of the row (so each load instruction reads 512 contiguous
// bytes).  V = 2^(dk-5) / 128 uint4 per lane.
template <int V>
__device__ __forceinline__ void rows_flush(const RowsArgs &a, u32 y, bool whole, uint4 *acc,
                                           u64 &words_out) {
  const int lane = threadIdx.x & 31;
  const int rs = a.dk - 5;
  uint4 *d = reinterpret_cast<uint4 *>(a.dst + ((u64)y << rs));
  if (a.clear_diag) {
    // word y / 32 of the row is component (y / 32) % 4 of uint4 y / 128,
    // held by lane (y / 128) % 32 as its entry (y / 128) / 32
    const u32 q = y >> 7, c = (y >> 5) & 3u, m = ~(1u << (y & 31));
#pragma unroll
    for (int j = 0; j < V; j++)
      if (q == (u32)(j * 32 + lane)) {
        if (c == 0) acc[j].x &= m;
        else if (c == 1) acc[j].y &= m;
        else if (c == 2) acc[j].z &= m;
        else acc[j].w &= m;
      }
  }
#pragma unroll
  for (int j = 0; j < V; j++) {
    const uint4 v = acc[j];
    if ((v.x | v.y | v.z | v.w) == 0u) continue;
    const u32 q = (u32)j * 32 + lane;
    if (whole && a.dst_zero) {
      // this warp owns row y in this launch, and the row is zero: a store
      d[q] = v;
    } else if (whole) {
      // this warp owns row y in this launch: plain read-OR-write
      uint4 o = d[q];
      o.x |= v.x;
      o.y |= v.y;
      o.z |= v.z;
      o.w |= v.w;
      d[q] = o;
    } else {
      u32 *w = reinterpret_cast<u32 *>(d + q);
      if (v.x) asm volatile("red.global.or.b32 [%0], %1;" ::"l"(w + 0), "r"(v.x) : "memory");
      if (v.y) asm volatile("red.global.or.b32 [%0], %1;" ::"l"(w + 1), "r"(v.y) : "memory");
      if (v.z) asm volatile("red.global.or.b32 [%0], %1;" ::"l"(w + 2), "r"(v.z) : "memory");
      if (v.w) asm volatile("red.global.or.b32 [%0], %1;" ::"l"(w + 3), "r"(v.w) : "memory");
    }
    if (a.dirty) a.dirty[(((u64)y << rs) + 4ull * q) / kBmChunkWords] = 1;
    words_out += 4;
  }
}

template <int V>
__global__ void __launch_bounds__(256) k_join_rows_bm(RowsArgs a) {
  if (ctl_stop(a.j.ctl)) return;
  if (eff_count(a.j.inner, a.j.inner_vis) == 0) {
    // src/join.cu:42-45: an empty inner zeroes the outer's count
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      if (a.j.outer_vis)
        *a.j.outer_vis = 0;
      else
        ((DArr *)a.j.outer)->n = 0;
    }
    if (a.outer_clear) {
      uint4 *p = reinterpret_cast<uint4 *>(a.outer_clear);
      const u64 n4 = (1ull << (2 * a.dk - 5)) / 4;
      for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
           i += (u64)gridDim.x * blockDim.x)
        p[i] = make_uint4(0, 0, 0, 0);
    }
    return;
  }
  // a DELTA outer zeroed earlier in the iteration reads as empty
  if (a.j.outer_vis && eff_count(a.j.outer, a.j.outer_vis) == 0) return;
  if (a.j.once) {
    // a join over static FULLs that an earlier iteration ran with both
    // sides non-empty: the same tuples, all in the output's FULL already
    if (*a.j.once) {
      if (blockIdx.x == 0 && threadIdx.x == 0 && *a.j.produced) *a.j.phantom = 1;
      return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.j.once_pending = 1;
  }
  const int lane = threadIdx.x & 31;
  const int rs = a.dk - 5;
  // the in-edges actually listed (values outside the domain are skipped by
  // k_inv_fill and reported by the fixpoint)
  const u32 n_edges = a.inv_off[1u << a.dk];
  u64 words_out = 0, edges = 0;
  // Units are runs of U consecutive in-edges (grouped by y, so a unit holds
  // the in-edges of a few consecutive y's), taken round robin: every warp
  // reads the same number of rows, kFly at a time, and flushes its
  // accumulator where y changes.  A y none of whose in-edges lie just
  // before or just after the unit has them all here: its row is this
  // warp's alone.  The next unit's ids load while this unit's rows are read.
  // U follows from the edge count: each warp takes k units of U <= a.unit
  // edges (k = ceil(edges per warp / a.unit)), so no warp takes one unit
  // more than the others (that unit would be the launch's tail).  U stays
  // at least a.unit / 2: shorter units would cut most y's in-edges apart,
  // and a y split between units is written with reductions.
  const u32 nw = (gridDim.x * blockDim.x) >> 5;
  const u32 per_warp = (n_edges + nw - 1) / nw;
  const u32 k_units = max(1u, (per_warp + a.unit - 1) / a.unit);
  const u32 U = max(max(1u, a.unit / 2), (per_warp + k_units - 1) / k_units);
  const u32 n_units = (n_edges + U - 1) / U;
  const uint4 none = make_uint4(0, 0, 0, 0);
  constexpr int kFly = V <= 4 ? 4 : 2;
  u32 u = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  u32 my_k = 0, my_y = ~0u;
  if (u < n_units && u * U + lane < n_edges && lane < (int)U) {
    my_k = a.inv_keys[u * U + lane];
    my_y = a.inv_ys[u * U + lane];
  }
  while (u < n_units) {
    const u32 base = u * U;
    const u32 m = min(U, n_edges - base);
    // the y's of the edges just before and just after this unit
    u32 edge_y = ~0u;
    if (lane == 0 && base > 0) edge_y = a.inv_ys[base - 1];
    if (lane == 1 && base + m < n_edges) edge_y = a.inv_ys[base + m];
    // the next unit's ids
    const u32 un = u + nw;
    u32 nk = 0, ny = ~0u;
    if (un < n_units && un * U + lane < n_edges && lane < (int)U) {
      nk = a.inv_keys[un * U + lane];
      ny = a.inv_ys[un * U + lane];
    }
    const u32 y_before = __shfl_sync(0xffffffffu, edge_y, 0);
    const u32 y_after = __shfl_sync(0xffffffffu, edge_y, 1);
    uint4 acc[V];
#pragma unroll
    for (int j = 0; j < V; j++) acc[j] = none;
    u32 cur_y = __shfl_sync(0xffffffffu, my_y, 0);
    for (u32 i = 0; i < m; i += kFly) {
      // kFly rows in flight: all their loads issued before the ORs (a slot
      // past the unit's end reads row 0, inside the bitmap, and is unused)
      uint4 b[kFly][V];
#pragma unroll
      for (int f = 0; f < kFly; f++) {
        const u32 k = __shfl_sync(0xffffffffu, my_k, (int)((i + f) & 31u));
        const uint4 *row = reinterpret_cast<const uint4 *>(a.O + ((u64)(i + f < m ? k : 0u) << rs));
#pragma unroll
        for (int j = 0; j < V; j++) b[f][j] = row[j * 32 + lane];
      }
#pragma unroll
      for (int f = 0; f < kFly; f++) {
        const u32 yf = __shfl_sync(0xffffffffu, my_y, (int)((i + f) & 31u));
        if (i + f >= m) break;
        if (yf != cur_y) {
          rows_flush<V>(a, cur_y, cur_y != y_before && cur_y != y_after, acc, words_out);
#pragma unroll
          for (int j = 0; j < V; j++) acc[j] = none;
          cur_y = yf;
        }
#pragma unroll
        for (int j = 0; j < V; j++) {
          acc[j].x |= b[f][j].x;
          acc[j].y |= b[f][j].y;
          acc[j].z |= b[f][j].z;
          acc[j].w |= b[f][j].w;
        }
      }
    }
    rows_flush<V>(a, cur_y, cur_y != y_before && cur_y != y_after, acc, words_out);
    edges += m;
    u = un;
    my_k = nk;
    my_y = ny;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) words_out += __shfl_xor_sync(0xffffffffu, words_out, o);
  // algorithmic bytes: a row of the outer and an (edge, y) pair per
  // in-edge, and each output word written (read and written back)
  if (lane == 0)
    prof_add(a.j.ctl, kPJoinMat, edges * ((4ull << rs) + 8) + 8 * words_out);
  if (lane == 0 && words_out && a.j.produced) *a.j.produced = 1;
  launch_rec_finish(a.j.rec);
}

// dst |= transpose(src), src cleared: the transposed output of the joins
// whose output is (inner column 1, outer column 1), folded into the output
// relation's NEWT (and its dirty map) after each such join.  Every word of
// dst comes from one tile of src, so the ORs need no atomics.  overwrite:
// dst := transpose(src), every word written and none read (the first
// writer of a tmp relation's NEWT in an iteration, without a dirty map: what
// dst held before is not part of this iteration's NEWT).
__global__ void __launch_bounds__(kTrBlock) k_bm_fold_t(u32 *src, u32 *dst, u8 *dirty, int dk,
                                                        int overwrite, Ctl *ctl) {
  __shared__ u32 s_t[256][9];
  if (ctl_stop(ctl)) return;
  const int rs = dk - 5;
  const u64 per = 1ull << (dk - 8);
  const u64 tiles = per * per;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  u64 moved = 0;
  // Software-pipelined over the block's tiles: the next tile's source words
  // and this tile's destination words are loaded before this tile's
  // barriers, so the two memory round trips of a tile overlap.  A tile's
  // reads of s_t are ordered before the next tile's writes by that tile's
  // __syncthreads_or.
  u64 t = blockIdx.x;
  u32 v[8];
  if (t < tiles) load8(src + ((((t / per) * 256 + (u64)threadIdx.x) << rs) + (t % per) * 8), v);
  for (; t < tiles; t += gridDim.x) {
    const u64 tr = t / per, tc = t % per;
    const u64 at = ((tr * 256 + (u64)threadIdx.x) << rs) + tc * 8;
    const u64 dw = ((tc * 256 + (u64)threadIdx.x) << rs) + tr * 8;
    const u64 tn = t + gridDim.x;
    u32 vn[8], d[8];
    if (tn < tiles)
      load8(src + ((((tn / per) * 256 + (u64)threadIdx.x) << rs) + (tn % per) * 8), vn);
    if (!overwrite) load8(dst + dw, d);
    const bool any = (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) != 0u;
    moved += 4 * 8;
    if (any) {
      uint4 *ps = reinterpret_cast<uint4 *>(src + at);
      ps[0] = make_uint4(0, 0, 0, 0);
      ps[1] = make_uint4(0, 0, 0, 0);
      moved += 4 * 8;
    }
    uint4 *pd = reinterpret_cast<uint4 *>(dst + dw);
    if (__syncthreads_or(any)) {  // block-uniform
#pragma unroll
      for (int i = 0; i < 8; i++) s_t[i * 32 + lane][wid] = transpose32(v[i], lane);
      __syncthreads();
      const u32 *q = s_t[threadIdx.x];
      if (overwrite) {
        pd[0] = make_uint4(q[0], q[1], q[2], q[3]);
        pd[1] = make_uint4(q[4], q[5], q[6], q[7]);
        moved += 4 * 8;
      } else if ((q[0] | q[1] | q[2] | q[3] | q[4] | q[5] | q[6] | q[7]) != 0u) {
        pd[0] = make_uint4(d[0] | q[0], d[1] | q[1], d[2] | q[2], d[3] | q[3]);
        pd[1] = make_uint4(d[4] | q[4], d[5] | q[5], d[6] | q[6], d[7] | q[7]);
        if (dirty) dirty[dw / kBmChunkWords] = 1;
        moved += 4 * 8;
      }
    } else if (overwrite) {
      pd[0] = make_uint4(0, 0, 0, 0);
      pd[1] = make_uint4(0, 0, 0, 0);
      moved += 4 * 8;
    }
    if (!overwrite) moved += 4 * 8;
    if (tn < tiles) {
#pragma unroll
      for (int i = 0; i < 8; i++) v[i] = vn[i];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
  if (lane == 0) prof_add(ctl, kPBitmap, moved);
}

// Set the transposed bits (c1, c0) of a key list (DELTA at the start of a
// LIE), square domain of 2^dk ids.
__global__ void __launch_bounds__(256) k_bm_from_list_t(const DArr *list, u32 *bm, int dk, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 n = list->n;
  const u64 *k = list->ptr;
  const u32 lim = 1u << dk;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
    const u32 c0 = key_c0(k[i]), c1 = key_c1(k[i]);
    if (c0 < lim && c1 < lim)
      atomicOr(bm + (((u64)c1 << (dk - 5)) + (c0 >> 5)), 1u << (c0 & 31));
    else
      atomicOr(&ctl->oob, 8192u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) prof_add(ctl, kPBitmap, 8 * n);
}

}  // namespace gdl
