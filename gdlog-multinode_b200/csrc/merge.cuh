// merge.cuh — merge-path union / difference of a sorted NEWT into FULL.
//
// One pass replaces three reference steps of the per-relation update
// (src/lie.cu:122-185): thrust::set_difference(newt, full) -> delta, the
// deduplication of NEWT (thrust::unique, src/join.cu:193-195), and
// flush_delta's thrust::merge(full, delta) (src/relation.cu:484-487).
//
// Input A: sorted keys, duplicates allowed (the radix-sorted NEWT).
// Input B: sorted, unique keys (committed FULL).
// Output U = B ∪ A (sorted, unique) -> FULL of the next iteration.
// Output D = A \ B (sorted, unique) -> DELTA of the next iteration.
// The merged sequence takes B first on ties, so an A key is new exactly
// when it differs from the key merged just before it.  Tiles of the merged
// sequence are found with merge-path searches (Green, McColl, Bader 2012);
// the output offsets of each tile come from a decoupled look-back on the
// packed pair (|D| << 32 | |U|).  Reads 8(|A|+|B|) bytes, writes
// 8(|U|+|D|) bytes.
#pragma once

#include "common.cuh"

namespace gdl {

constexpr int kMergeBlock = 256;
constexpr int kMergeItems = 8;
constexpr int kMergeTile = kMergeBlock * kMergeItems;  // 2048 merged keys

struct MergeArgs {
  const DArr *newt;   // count of A (A's data is `a`, the sorted NEWT)
  const u64 *a;
  const DArr *full;   // B
  DArr *full_next;    // U
  DArr *delta_next;   // D
  u64 *c_newt_n;      // RelDev::c_newt_n of the relation
  LaunchRec *rec;
  Lb lb;
  u64 *parts;     // [tiles + 1] A-split of every tile boundary (k_merge_partition)
  u64 parts_cap;
  Ctl *ctl;
  int rel;
};

// Number of A keys among the first d keys of the merged sequence.
__device__ __forceinline__ u64 merge_path(const u64 *A, u64 na, const u64 *B, u64 nb, u64 d) {
  u64 lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
  while (lo < hi) {
    u64 mid = (lo + hi) >> 1;
    if (A[mid] < B[d - mid - 1])
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// Dependent columns (Relation::dependent_column_size): the set difference
// NEWT \ FULL of the update step compares only the first arity - dep
// columns (src/lie.cu:131-138), while unique and merge compare whole
// tuples.  Before the merge, every sorted NEWT key whose prefix (the key
// with its dependent bits, low_mask, cleared) is already in FULL is replaced
// by the first FULL key with that prefix.  NEWT stays sorted, the merge sees
// those keys tie with FULL (not new, nothing added), and DELTA and FULL'
// come out as set_difference then merge give them.
__global__ void k_dep_mask(u64 *a, const DArr *newt, const DArr *full, u64 low_mask, Ctl *ctl) {
  if (ctl_stop(ctl)) return;
  const u64 na = newt->n, nb = full->n;
  const u64 *B = full->ptr;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < na;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 p = a[i] & ~low_mask;
    u64 lo = 0, hi = nb;  // first FULL key >= p
    while (lo < hi) {
      const u64 mid = (lo + hi) >> 1;
      if (B[mid] < p)
        lo = mid + 1;
      else
        hi = mid;
    }
    if (lo < nb && (B[lo] & ~low_mask) == p) a[i] = B[lo];
  }
}

__device__ __forceinline__ bool merge_fits(const MergeArgs &m, u64 na, u64 nb) {
  return na + nb <= m.full_next->cap && na <= m.delta_next->cap;
}

// Split points of the merged sequence at every tile boundary, one thread
// per boundary, so that no CTA of k_merge_diff waits on a serial search
// through global memory.
__global__ void __launch_bounds__(256) k_merge_partition(MergeArgs m) {
  if (ctl_stop(m.ctl)) return;
  const u64 na = m.newt->n, nb = m.full->n;
  if (na == 0 || !merge_fits(m, na, nb)) return;  // k_merge_diff handles both
  const u64 total = na + nb;
  const u64 tiles = (total + kMergeTile - 1) / kMergeTile;
  for (u64 t = (u64)blockIdx.x * blockDim.x + threadIdx.x; t <= tiles;
       t += (u64)gridDim.x * blockDim.x) {
    if (t < m.parts_cap)
      m.parts[t] = merge_path(m.a, na, m.full->ptr, nb, min(t * (u64)kMergeTile, total));
    else
      atomicOr(&m.ctl->oob, 512u);
  }
}

struct MergeSmem {
  u64 ab[kMergeTile];  // A segment then B segment; reused for U output
  u64 dbuf[kMergeTile];
  u64 scan_tmp[kMergeBlock / 32];
  u64 prev;
  long long tile;
  u64 a0, a1, b0, b1;
  u64 u_base, d_base;
  int has_prev;
};

__global__ void __launch_bounds__(kMergeBlock) k_merge_diff(MergeArgs m) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  MergeSmem &sm = *reinterpret_cast<MergeSmem *>(smem_raw);
  if (ctl_stop(m.ctl)) return;
  const u64 na = m.newt->n;
  const u64 nb = m.full->n;
  if (na == 0) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      m.delta_next->n = 0;
      *m.c_newt_n = 0;
    }
    return;
  }
  if (!merge_fits(m, na, nb)) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      atomicMax(&m.ctl->need[need_index(m.rel, kNeedFull)], na + nb);
      atomicMax(&m.ctl->need[need_index(m.rel, kNeedDelta)], na);
      atomicExch(&m.ctl->overflow, 1u);
    }
    return;
  }
  const u64 *A = m.a;
  const u64 *B = m.full->ptr;
  u64 *U = m.full_next->ptr;
  u64 *D = m.delta_next->ptr;
  const u64 total = na + nb;
  const u64 tiles = (total + kMergeTile - 1) / kMergeTile;
  const u32 gen = m.rec->gen;
  while (true) {
    const long long tile = grab_tile(m.rec, &sm.tile);
    if (tile >= (long long)tiles) break;
    const u64 d0 = (u64)tile * kMergeTile;
    const u64 d1 = min(d0 + kMergeTile, total);
    if (threadIdx.x == 0) {
      const bool ok = (u64)tile + 1 < m.parts_cap;
      u64 i0 = ok ? m.parts[tile] : merge_path(A, na, B, nb, d0);
      u64 i1 = ok ? m.parts[tile + 1] : merge_path(A, na, B, nb, d1);
      sm.a0 = i0;
      sm.a1 = i1;
      sm.b0 = d0 - i0;
      sm.b1 = d1 - i1;
      u64 j0 = d0 - i0;
      bool ha = i0 > 0, hb = j0 > 0;
      sm.has_prev = ha || hb;
      u64 pa = ha ? A[i0 - 1] : 0, pb = hb ? B[j0 - 1] : 0;
      sm.prev = ha && hb ? max(pa, pb) : (ha ? pa : pb);
    }
    __syncthreads();
    const u64 a0 = sm.a0, a1 = sm.a1, b0 = sm.b0, b1 = sm.b1;
    const u64 sna = a1 - a0, snb = b1 - b0;
    for (u64 i = threadIdx.x; i < sna + snb; i += blockDim.x)
      sm.ab[i] = i < sna ? A[a0 + i] : B[b0 + (i - sna)];
    __syncthreads();
    const u64 *sA = sm.ab, *sB = sm.ab + sna;
    // This thread's slice of the tile's merged sequence.
    const u64 dd = min((u64)threadIdx.x * kMergeItems, sna + snb);
    u64 ia = merge_path(sA, sna, sB, snb, dd);
    u64 ib = dd - ia;
    bool has_prev;
    u64 prev;
    if (ia == 0 && ib == 0) {
      has_prev = sm.has_prev;
      prev = sm.prev;
    } else {
      has_prev = true;
      u64 pa = ia ? sA[ia - 1] : 0, pb = ib ? sB[ib - 1] : 0;
      prev = (ia && ib) ? max(pa, pb) : (ia ? pa : pb);
    }
    u64 val[kMergeItems];
    u32 ku = 0, kd = 0;  // bit masks: item kept in U / in D
    const u64 cnt = min((u64)kMergeItems, sna + snb - dd);
#pragma unroll
    for (int k = 0; k < kMergeItems; k++) {
      if ((u64)k < cnt) {
        bool takeB = ib < snb && (ia >= sna || sB[ib] <= sA[ia]);
        u64 e = takeB ? sB[ib++] : sA[ia++];
        bool fresh = takeB || !(has_prev && e == prev);
        val[k] = e;
        if (fresh) ku |= 1u << k;
        if (fresh && !takeB) kd |= 1u << k;
        prev = e;
        has_prev = true;
      }
    }
    const u64 nu = __popc(ku), nd = __popc(kd);
    u64 tot_u, tot_d;
    const u64 ex_u = block_excl_scan<kMergeBlock>(nu, sm.scan_tmp, &tot_u);
    const u64 ex_d = block_excl_scan<kMergeBlock>(nd, sm.scan_tmp, &tot_d);
    // Tile offsets: look back on the packed pair (|D| << 32 | |U|).
    if (threadIdx.x < 32) {
      const u64 agg = (tot_d << 32) | tot_u;
      u64 prefix = 0;
      if (tile == 0) {
        if (threadIdx.x == 0) lb_publish(m.lb, tile, gen, true, agg);
      } else {
        if (threadIdx.x == 0) lb_publish(m.lb, tile, gen, false, agg);
        prefix = lb_warp_prefix(m.lb, tile, gen, m.ctl);
        if (threadIdx.x == 0) lb_publish(m.lb, tile, gen, true, prefix + agg);
      }
      if (threadIdx.x == 0) {
        sm.u_base = prefix & 0xFFFFFFFFull;
        sm.d_base = prefix >> 32;
        if ((u64)tile == tiles - 1) {
          m.full_next->n = (prefix & 0xFFFFFFFFull) + tot_u;
          m.delta_next->n = (prefix >> 32) + tot_d;
          *m.c_newt_n = na;
          prof_add(m.ctl, kPMerge,
                   8 * (na + nb) + 8 * ((prefix & 0xFFFFFFFFull) + tot_u + (prefix >> 32) + tot_d));
        }
      }
    }
    __syncthreads();  // sm.ab no longer read: reuse it for U
    {
      u32 pu = (u32)ex_u, pd = (u32)ex_d;
#pragma unroll
      for (int k = 0; k < kMergeItems; k++) {
        if (ku & (1u << k)) sm.ab[pu++] = val[k];
        if (kd & (1u << k)) sm.dbuf[pd++] = val[k];
      }
    }
    __syncthreads();
    const u64 ub = sm.u_base, db = sm.d_base;
    for (u64 i = threadIdx.x; i < tot_u; i += blockDim.x) {
      u64 g = ub + i;
      if (g < m.full_next->cap)
        U[g] = sm.ab[i];
      else
        atomicOr(&m.ctl->oob, 8u);
    }
    for (u64 i = threadIdx.x; i < tot_d; i += blockDim.x) {
      u64 g = db + i;
      if (g < m.delta_next->cap)
        D[g] = sm.dbuf[i];
      else
        atomicOr(&m.ctl->oob, 16u);
    }
  }
  launch_rec_finish(m.rec);
}

constexpr size_t kMergeSmemBytes = sizeof(MergeSmem);

// Commit of a load (the end of load_relation, src/relation.cu:815-838):
// FULL' becomes FULL, NEWT and the merge's DELTA output are emptied.  A
// failed device check is kept in a sticky word instead, for the host to
// report at its next read of the relation table.
__global__ void k_load_commit(RelDev *r, const Ctl *ctl, u32 *err) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const u32 bad = (ctl->timeout ? 1u : 0u) | (ctl->oob ? 2u : 0u) | (ctl->overflow ? 4u : 0u);
  if (bad) {
    atomicOr(err, bad);
    return;
  }
  const DArr t = r->full;
  r->full = r->full_next;
  r->full_next = t;
  r->newt.n = 0;
  r->delta_next.n = 0;
  r->c_newt_n = 0;
}

}  // namespace gdl
