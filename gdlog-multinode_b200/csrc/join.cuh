// join.cuh — two-pass hash join, projection copy and ACopy kernels.
//
// RelationalJoin (src/join.cu:12-270) counts (get_join_result_size,
// src/relation.cu:221-288), reduces and scans the counts with Thrust
// (src/join.cu:77-102), then materialises with one thread per outer row
// (get_join_result, src/relation.cu:290-373), walking the inner run twice.
// Here:
//   * k_join_count stages a tile of outer rows in shared memory, probes the
//     inner index once per row (one 16-byte load gives the whole run), and
//     in the same kernel scans the counts with a decoupled look-back and
//     compacts the rows that match anything into (output offset, run start,
//     run length, outer key) records.
//   * k_join_mat is load-balanced over OUTPUT positions: each block owns a
//     contiguous range of outputs, finds the records covering it by binary
//     search, and each thread writes two adjacent output tuples with one
//     16-byte store, so writes are coalesced whatever the skew of the runs.
//   * joins with a predicate use k_join_mat_pred: a warp per record, the
//     lanes test candidates 32 at a time and compact the survivors with a
//     ballot.
// Output is appended to the NEWT accumulator of the output relation.  Every
// append is rounded up to an even count (the pad repeats the last tuple of
// the op, which the later deduplication removes), so every append starts
// 16-byte aligned.
#pragma once

#include "common.cuh"
#include "index.cuh"

namespace gdl {

constexpr int kJoinBlock = 256;
constexpr int kJoinItems = 4;
constexpr int kJoinTile = kJoinBlock * kJoinItems;  // outer rows per tile
constexpr int kMatBlock = 256;
constexpr int kMatTile = 2 * kMatBlock * 2;  // outputs per block tile (2 pairs/thread)

struct JoinRec {
  u64 total;     // output tuples of the op (before padding)
  u64 nc;        // compacted records
  u64 base;      // append position in NEWT
  u64 overflow;  // the output does not fit NEWT (raised by the next kernel)
  u64 written;   // hooked ops: rows the caller's kernel appended
  u64 skip;      // hooked ops: nothing to do this iteration
};

struct JoinArgs {
  const DArr *outer;
  u32 *outer_vis;  // working tuple_counts visibility; NULL for a NEWT outer
  const DArr *inner;
  const u32 *inner_vis;
  const Index *inner_idx;
  DArr *out_newt;
  Sel2 sel;
  Pred pred;
  JoinRec *op;
  LaunchRec *rec;
  Lb lb_cnt, lb_nz;
  u64 *crow_off;    // [nc + 1] output offsets
  u32 *crow_start;  // [nc] inner run start
  u32 *crow_len;    // [nc] inner run length
  u64 *crow_key;    // [nc] outer key
  u64 crow_cap;
  Ctl *ctl;
  int out_rel;
  // Dense output (dense.cuh): count every candidate (the predicate is
  // applied when bits are set) and skip the NEWT capacity check.  A NEWT
  // outer emptied by an empty inner (src/join.cu:38-45) also has its bitmap
  // cleared.
  int dense;
  u32 *outer_bm;
  u64 outer_bm_words;
  // Row-OR joins (dense.cuh, k_join_bm): the inner is a FULL kept as a
  // bitmap (inner_rd->bmF) and the output is (an outer column, inner
  // column 1), so a long run is its bitmap row, ORed into the output row.
  const RelDev *inner_rd;
  int row_or;
  // arity 3 or computed columns: tuples come from gen (list form only)
  int generic;
  GenSpec gen;
  // A join over static FULLs (push form, dense): `once` = ran in an earlier
  // iteration of this fixpoint, `once_pending` = ran in this one, `produced`
  // = that run set a tuple, `phantom` = the output's RelDev::newt_phantom.
  const u32 *once;
  u32 *once_pending;
  u32 *produced;
  u32 *phantom;
};

__device__ __forceinline__ u64 join_out(const JoinArgs &a, u64 inner, u64 outer) {
  return a.generic ? gen_spec(a.gen, inner, outer, &a.ctl->oob) : gen_join(a.sel, inner, outer);
}

__device__ __forceinline__ u64 eff_count(const DArr *a, const u32 *vis) {
  return (vis && *vis == 0) ? 0 : a->n;
}

// src/join.cu:38-45: either side empty -> no output, and the OUTER's
// tuple_counts is set to 0 (a real change only when the inner is empty).
// Every block of the launch calls this.
__device__ __forceinline__ void join_empty_side(const JoinArgs &a, u64 n_outer) {
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.op->total = 0;
    a.op->nc = 0;
    a.op->overflow = 0;
    if (n_outer != 0) {
      if (a.outer_vis)
        *a.outer_vis = 0;
      else
        ((DArr *)a.outer)->n = 0;
    }
  }
  if (n_outer != 0 && !a.outer_vis && a.outer_bm) {
    uint4 *p = reinterpret_cast<uint4 *>(a.outer_bm);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < a.outer_bm_words / 4;
         i += (u64)gridDim.x * blockDim.x)
      p[i] = make_uint4(0, 0, 0, 0);
  }
}

struct JoinSmem {
  u64 keys[kJoinTile];
  u64 scan_tmp[kJoinBlock / 32];
  u64 cnt_base, nz_base;
  long long tile;
};

__global__ void __launch_bounds__(kJoinBlock) k_join_count(JoinArgs a) {
  __shared__ JoinSmem sm;
  if (ctl_stop(a.ctl)) return;
  const u64 n_outer = eff_count(a.outer, a.outer_vis);
  const u64 n_inner = eff_count(a.inner, a.inner_vis);
  if (n_outer == 0 || n_inner == 0) {
    join_empty_side(a, n_outer);
    return;
  }
  const u64 tiles = (n_outer + kJoinTile - 1) / kJoinTile;
  const u32 gen = a.rec->gen;
  const Index ix = *a.inner_idx;
  const u64 *inner = a.inner->ptr;
  const u64 *outer = a.outer->ptr;
  while (true) {
    const long long tile = grab_tile(a.rec, &sm.tile);
    if (tile >= (long long)tiles) break;
    const u64 r0 = (u64)tile * kJoinTile;
    const u64 rn = min((u64)kJoinTile, n_outer - r0);
    for (u64 i = threadIdx.x; i < rn; i += blockDim.x) sm.keys[i] = outer[r0 + i];
    __syncthreads();
    u32 start[kJoinItems], len[kJoinItems];
    u64 cnt[kJoinItems];
    u64 my_cnt = 0, my_nz = 0;
#pragma unroll
    for (int k = 0; k < kJoinItems; k++) {
      const u64 i = (u64)threadIdx.x * kJoinItems + k;
      start[k] = 0;
      len[k] = 0;
      cnt[k] = 0;
      if (i < rn) {
        const u64 row = sm.keys[i];
        u32 s = 0;
        u32 l = index_probe(ix, key_c0(row), &s);
        start[k] = s;
        len[k] = l;
        if (a.pred.kind == 0 || a.dense) {
          cnt[k] = l;
        } else {
          u64 c = 0;
          for (u32 j = 0; j < l; j++) c += pred_ok(a.pred, join_out(a, inner[s + j], row));
          cnt[k] = c;
        }
        my_cnt += cnt[k];
        my_nz += cnt[k] != 0;
      }
    }
    u64 tot_cnt, tot_nz;
    const u64 ex_cnt = block_excl_scan<kJoinBlock>(my_cnt, sm.scan_tmp, &tot_cnt);
    const u64 ex_nz = block_excl_scan<kJoinBlock>(my_nz, sm.scan_tmp, &tot_nz);
    // Warp 0 looks back for the count prefix, warp 1 for the record prefix.
    const int warp = threadIdx.x >> 5;
    if (warp < 2) {
      const Lb lb = warp == 0 ? a.lb_cnt : a.lb_nz;
      const u64 agg = warp == 0 ? tot_cnt : tot_nz;
      u64 prefix = 0;
      if (tile == 0) {
        if ((threadIdx.x & 31) == 0) lb_publish(lb, tile, gen, true, agg);
      } else {
        if ((threadIdx.x & 31) == 0) lb_publish(lb, tile, gen, false, agg);
        prefix = lb_warp_prefix(lb, tile, gen, a.ctl);
        if ((threadIdx.x & 31) == 0) lb_publish(lb, tile, gen, true, prefix + agg);
      }
      if ((threadIdx.x & 31) == 0) {
        if (warp == 0)
          sm.cnt_base = prefix;
        else
          sm.nz_base = prefix;
      }
    }
    __syncthreads();
    u64 off = sm.cnt_base + ex_cnt, rec = sm.nz_base + ex_nz;
#pragma unroll
    for (int k = 0; k < kJoinItems; k++) {
      const u64 i = (u64)threadIdx.x * kJoinItems + k;
      if (i < rn && cnt[k]) {
        if (rec < a.crow_cap) {
          a.crow_off[rec] = off;
          a.crow_start[rec] = start[k];
          a.crow_len[rec] = len[k];
          a.crow_key[rec] = sm.keys[i];
        } else {
          atomicOr(&a.ctl->oob, 64u);
        }
        off += cnt[k];
        rec++;
      }
    }
    if ((u64)tile == tiles - 1 && threadIdx.x == 0) {
      const u64 total = sm.cnt_base + tot_cnt, nc = sm.nz_base + tot_nz;
      a.op->total = total;
      a.op->nc = nc;
      prof_add(a.ctl, kPJoinCount, 24 * n_outer);
      if (nc < a.crow_cap + 1) a.crow_off[nc] = total;
      // The overflow is recorded in the op and raised by the next kernel:
      // ctl flags must not change while blocks of this launch may still
      // test them on entry.
      const u64 need = a.out_newt->n + ((total + 1) & ~1ull);
      a.op->overflow = !a.dense && need > a.out_newt->cap;
      if (a.op->overflow) atomicMax(&a.ctl->need[need_index(a.out_rel, kNeedNewt)], need);
    }
  }
  launch_rec_finish(a.rec);
}

// Record covering output position p: largest k with off[k] <= p.
__device__ __forceinline__ u32 find_rec(const u64 *off, u32 n, u64 p) {
  u32 lo = 0, hi = n;  // off[lo] <= p < off[hi] (off[n] = end of range)
  while (hi - lo > 1) {
    u32 mid = (lo + hi) >> 1;
    if (off[mid] <= p)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

struct MatSmem {
  u64 off[kMatTile + 1];
  u32 start[kMatTile];
  u64 key[kMatTile];
  u64 tile_k0[kMatBlock];  // first record of each tile of the current batch
};

// Materialisation tiles are handed out round-robin (tile = blockIdx.x +
// j * gridDim.x).  A block finds the first records of its next kMatBlock
// tiles at once, one binary search over crow_off per thread, so the
// dependent global loads of the searches overlap instead of stalling the
// block before every tile.
__device__ __forceinline__ void mat_batch_starts(const u64 *crow_off, u64 nc, u64 tiles,
                                                 u64 batch, u64 *tile_k0) {
  const u64 t = batch + (u64)threadIdx.x * gridDim.x;
  if (t >= tiles) return;
  const u64 p0 = t * kMatTile;
  u64 lo = 0, hi = nc;  // largest k with crow_off[k] <= p0
  while (hi - lo > 1) {
    const u64 mid = (lo + hi) >> 1;
    if (crow_off[mid] <= p0)
      lo = mid;
    else
      hi = mid;
  }
  tile_k0[threadIdx.x] = lo;
}

// Stage the records of one tile (k0 .. k0+m-1 cover its positions; each
// record holds >= 1 output) in shared memory.
__device__ __forceinline__ u32 mat_stage_tile(const JoinArgs &a, u64 nc, u64 k0, MatSmem &sm) {
  const u32 m = (u32)min((u64)kMatTile, nc - k0);
  for (u32 i = threadIdx.x; i <= m; i += blockDim.x) {
    sm.off[i] = a.crow_off[k0 + i];
    if (i < m) {
      sm.start[i] = a.crow_start[k0 + i];
      sm.key[i] = a.crow_key[k0 + i];
    }
  }
  return m;
}

__global__ void __launch_bounds__(kMatBlock) k_join_mat(JoinArgs a) {
  __shared__ MatSmem sm;
  if (ctl_stop(a.ctl)) return;
  if (a.op->overflow) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&a.ctl->overflow, 1u);
    return;
  }
  const u64 total = a.op->total;
  const u64 nc = a.op->nc;
  const u64 base = a.out_newt->n;
  if (total == 0) return;
  const u64 *inner = a.inner->ptr;
  u64 *out = a.out_newt->ptr + base;
  const u64 cap_left = a.out_newt->cap - base;
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
      // Two rounds of one 16-byte store (two tuples) per thread.
      for (u64 q = threadIdx.x; q < (u64)kMatTile / 2; q += blockDim.x) {
        const u64 p = p0 + 2 * q;
        if (p >= p1) break;
        u32 r = find_rec(sm.off, m, p);
        u64 o0 = join_out(a, inner[sm.start[r] + (p - sm.off[r])], sm.key[r]);
        u64 o1 = o0;
        if (p + 1 < total) {
          if (p + 1 >= sm.off[r + 1]) r++;
          o1 = join_out(a, inner[sm.start[r] + (p + 1 - sm.off[r])], sm.key[r]);
        }
        if (p + 1 < cap_left)
          reinterpret_cast<ulonglong2 *>(out)[p >> 1] = make_ulonglong2(o0, o1);
        else
          atomicOr(&a.ctl->oob, 128u);
      }
    }
  }
  // The last block to finish publishes the new NEWT count.
  if (launch_rec_finish(a.rec) && threadIdx.x == 0) {
    a.op->base = base;
    a.out_newt->n = base + ((total + 1) & ~1ull);
    prof_add(a.ctl, kPJoinMat, 16 * total + 24 * nc);
  }
}

// Predicate joins: a warp per record; survivors compacted with a ballot.
__global__ void __launch_bounds__(kMatBlock) k_join_mat_pred(JoinArgs a) {
  if (ctl_stop(a.ctl)) return;
  if (a.op->overflow) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicExch(&a.ctl->overflow, 1u);
    return;
  }
  const u64 total = a.op->total;
  const u64 nc = a.op->nc;
  const u64 base = a.out_newt->n;
  if (total == 0) return;
  const u64 *inner = a.inner->ptr;
  u64 *out = a.out_newt->ptr + base;
  const u64 cap_left = a.out_newt->cap - base;
  const int lane = threadIdx.x & 31;
  const u64 warps = (u64)gridDim.x * (blockDim.x / 32);
  for (u64 k = (u64)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5); k < nc; k += warps) {
    const u64 off = a.crow_off[k];
    const u32 s = a.crow_start[k], l = a.crow_len[k];
    const u64 row = a.crow_key[k];
    u64 written = 0;
    for (u32 j0 = 0; j0 < l; j0 += 32) {
      const u32 j = j0 + lane;
      u64 t = 0;
      bool ok = false;
      if (j < l) {
        t = join_out(a, inner[s + j], row);
        ok = pred_ok(a.pred, t);
      }
      unsigned m = __ballot_sync(0xffffffffu, ok);
      if (ok) {
        u64 pos = off + written + __popc(m & ((1u << lane) - 1u));
        if (pos < cap_left)
          out[pos] = t;
        else
          atomicOr(&a.ctl->oob, 256u);
      }
      written += __popc(m);
    }
  }
  if (launch_rec_finish(a.rec) && threadIdx.x == 0) {
    if (total & 1) {
      __threadfence();
      if (total < cap_left) out[total] = *((volatile u64 *)&out[total - 1]);
    }
    a.op->base = base;
    a.out_newt->n = base + ((total + 1) & ~1ull);
    prof_add(a.ctl, kPJoinMat, 16 * total + 24 * nc);
  }
}

// RelationalCopy (src/copy.cu:12-95) / projection kernel get_copy_result
// (src/relation.cu:390-403): dest NEWT += sel(src).  A FULL-source copy runs
// once per LIE (src/lie.cu:69-75): `once` points at the committed "copied"
// flag and `once_pending` at the flag this iteration sets.
struct CopyArgs {
  const DArr *src;
  const u32 *src_vis;
  DArr *dest;
  Sel2 sel;
  const u32 *once;
  u32 *once_pending;
  LaunchRec *rec;
  Ctl *ctl;
  int dest_rel;
  int replace;  // ACopy: dest := sel(src) instead of appending
  int generic;  // arity 3 or computed columns: tuples come from gen
  GenSpec gen;
};

__device__ __forceinline__ u64 copy_out(const CopyArgs &c, u64 src) {
  return c.generic ? gen_spec(c.gen, src, 0, &c.ctl->oob) : gen_join(c.sel, src, 0);
}

__global__ void __launch_bounds__(kMatBlock) k_copy(CopyArgs c) {
  if (ctl_stop(c.ctl)) return;
  if (c.once && *c.once) return;
  const u64 n = eff_count(c.src, c.src_vis);
  if (n == 0) {
    // src/copy.cu:24-27 (dest NEWT count := 0); src/acopy.cu:14-18.
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      c.dest->n = 0;
      if (c.once_pending) *c.once_pending = 1;
    }
    return;
  }
  const u64 base = c.replace ? 0 : c.dest->n;
  const u64 need = base + ((n + 1) & ~1ull);
  if (need > c.dest->cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      atomicMax(&c.ctl->need[need_index(c.dest_rel, kNeedNewt)], need);
      atomicExch(&c.ctl->overflow, 1u);
    }
    return;
  }
  const u64 *src = c.src->ptr;
  u64 *out = c.dest->ptr + base;
  const u64 pairs = (n + 1) / 2;
  for (u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x; q < pairs;
       q += (u64)gridDim.x * blockDim.x) {
    const u64 p = 2 * q;
    u64 o0 = copy_out(c, src[p]);
    u64 o1 = p + 1 < n ? copy_out(c, src[p + 1]) : o0;
    reinterpret_cast<ulonglong2 *>(out)[q] = make_ulonglong2(o0, o1);
  }
  if (launch_rec_finish(c.rec) && threadIdx.x == 0) {
    c.dest->n = need;
    if (c.once_pending) *c.once_pending = 1;
    prof_add(c.ctl, kPCopy, 16 * n);
  }
}

// ---------------------------------------------------------------------------
// Operators whose per-tuple work is the caller's kernel (gdl_lie_add_*_hooked,
// the reference's device-function-pointer hooks, src/relation.cu:290-403).
// The engine brackets that kernel: the begin kernel decides whether the
// operator runs this iteration and where its rows go, the end kernel
// publishes NEWT's count.  JoinRec doubles as the caller-visible
// gdl_hook_state.
// ---------------------------------------------------------------------------

// Join: after k_join_count (which applied src/join.cu:38-45 and checked NEWT
// capacity for every candidate).
__global__ void k_hook_join_begin(JoinArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  JoinRec *r = a.op;
  r->written = 0;
  r->skip = 1;
  if (ctl_stop(a.ctl)) return;
  if (r->overflow) {
    atomicExch(&a.ctl->overflow, 1u);
    return;
  }
  if (r->total == 0) return;
  r->base = a.out_newt->n;
  r->skip = 0;
}

// Appends are rounded up to an even count as everywhere else: an odd tail
// repeats the last row the operator wrote (the update step deduplicates).
__device__ __forceinline__ void hook_publish(DArr *out, JoinRec *r) {
  const u64 w = r->written;
  u64 *p = out->ptr + r->base;
  if (w & 1) p[w] = p[w - 1];
  out->n = r->base + ((w + 1) & ~1ull);
}

__global__ void k_hook_join_end(JoinArgs a) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  JoinRec *r = a.op;
  if (r->skip || ctl_stop(a.ctl)) return;
  hook_publish(a.out_newt, r);
  prof_add(a.ctl, kPJoinMat, 16 * r->total + 24 * r->nc);
}

// Copy / ACopy: src/copy.cu:12-95, src/acopy.cu:12-50, as k_copy does them.
__global__ void k_hook_copy_begin(CopyArgs c, JoinRec *r) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  r->written = 0;
  r->skip = 1;
  if (ctl_stop(c.ctl)) return;
  if (c.once && *c.once) return;
  const u64 n = eff_count(c.src, c.src_vis);
  if (n == 0) {  // src/copy.cu:24-27 (dest NEWT count := 0); src/acopy.cu:14-18
    c.dest->n = 0;
    if (c.once_pending) *c.once_pending = 1;
    return;
  }
  const u64 base = c.replace ? 0 : c.dest->n;
  const u64 need = base + ((n + 1) & ~1ull);
  if (need > c.dest->cap) {
    atomicMax(&c.ctl->need[need_index(c.dest_rel, kNeedNewt)], need);
    atomicExch(&c.ctl->overflow, 1u);
    return;
  }
  r->total = n;
  r->nc = 0;
  r->base = base;
  r->skip = 0;
}

__global__ void k_hook_copy_end(CopyArgs c, JoinRec *r) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  if (r->skip || ctl_stop(c.ctl)) return;
  if (c.replace && r->written == 0) {
    c.dest->n = 0;
  } else if (r->written) {
    hook_publish(c.dest, r);
  }
  if (c.once_pending) *c.once_pending = 1;
  prof_add(c.ctl, kPCopy, 16 * r->total);
}

}  // namespace gdl
