// control.cuh — per-iteration bookkeeping kernels of the device-side loop,
// plus the load-path helpers (pack, digest).
//
// LIE::fixpoint_loop (src/lie.cu:26-274) drives the loop from the host with
// a cudaDeviceSynchronize after almost every step.  Here the loop state is
// on the device: k_begin opens an iteration, k_commit closes it (swaps the
// rebuilt FULL/DELTA in, writes the per-iteration log line, decides
// termination exactly as src/lie.cu:208-215 does) and, when the iteration
// runs inside a CUDA graph while-node, sets the node's condition.
#pragma once

#include "common.cuh"

namespace gdl {

constexpr int kMaxOps = 64;

struct LieDev {
  int n_update, n_static, n_tmp, n_ops;
  int update[kMaxRels];
  int statics[kMaxRels];
  int tmps[kMaxRels];
  // Joins whose inner and outer are FULLs of static relations derive the
  // same tuples in every iteration: after one iteration that ran them with
  // both sides non-empty they add nothing new (semi-naive evaluation runs
  // such a rule once).  Per fixpoint call: ran (committed), ran this
  // iteration, and whether the run set any tuple.
  u32 jonce[kMaxOps];
  u32 jonce_pending[kMaxOps];
  u32 produced[kMaxOps];
  u32 once[kMaxOps];          // RelationalCopy::copied (committed)
  u32 once_pending[kMaxOps];  // set by this iteration's copies
  u64 *trace;                 // [trace rows][n_update][3]
};

// A lane's entries of the LIE's lists (entries lane and lane + 32; every
// list holds at most kMaxRels = 64), read once with all their loads in
// flight together: the control kernels are one warp whose time is its
// chains of dependent loads.
constexpr int kListPerLane = kMaxRels / 32;
static_assert(kMaxOps <= kMaxRels, "ops per lane");
struct LaneLists {
  int nu, ns, nt, no;
  int upd[kListPerLane], sta[kListPerLane], tmp[kListPerLane];
};
__device__ __forceinline__ LaneLists lane_lists(const LieDev *L, int lane) {
  LaneLists x;
  x.nu = L->n_update;
  x.ns = L->n_static;
  x.nt = L->n_tmp;
  x.no = L->n_ops;
#pragma unroll
  for (int j = 0; j < kListPerLane; j++) {
    // (every slot is inside the arrays; slots past a list's length unused)
    x.upd[j] = L->update[lane + 32 * j];
    x.sta[j] = L->statics[lane + 32 * j];
    x.tmp[j] = L->tmps[lane + 32 * j];
  }
  return x;
}

// Open an iteration: working visibilities from the committed ones, NEWT
// emptied, this iteration's Copy-once flags cleared.  Run by one warp, lane
// l taking entries l and l + 32 of each list (each relation is in one
// list; k_commit gives every entry to the same lane).
__device__ __forceinline__ void begin_iteration(RelDev *rels, LieDev *L, const LaneLists &x,
                                                int lane) {
#pragma unroll
  for (int j = 0; j < kListPerLane; j++) {
    const int i = lane + 32 * j;
    if (i < x.nu) {
      RelDev &r = rels[x.upd[j]];
      r.w_full_vis = r.full_vis;
      r.w_delta_vis = r.delta_vis;
      r.newt.n = 0;
    }
    if (i < x.ns) {
      RelDev &r = rels[x.sta[j]];
      r.w_full_vis = r.full_vis;
      r.w_delta_vis = r.delta_vis;
    }
    if (i < x.nt) {
      RelDev &r = rels[x.tmp[j]];
      r.w_full_vis = r.full_vis;
      r.w_delta_vis = r.delta_vis;
      r.newt.n = 0;
    }
    if (i < x.no) {
      L->once_pending[i] = 0;
      L->jonce_pending[i] = 0;
    }
  }
}

// One warp.
__global__ void k_begin(RelDev *rels, LieDev *L, Ctl *ctl) {
  const int lane = threadIdx.x;
  if (lane >= 32 || ctl_stop(ctl)) return;
  int ok = 1;
  if (lane == 0 && ctl->test_wait) {
    // gdl_engine_test_timeout: a bounded wait on a flag that nothing sets
    u32 polls = 0;
    while (!*((volatile u32 *)&ctl->never)) {
      if (++polls > ctl->test_wait) {
        atomicOr(&ctl->timeout, 1u);
        ok = 0;
        break;
      }
    }
  }
  if (!__shfl_sync(0xffffffffu, ok, 0)) return;
  begin_iteration(rels, L, lane_lists(L, lane), lane);
}

template <class T>
__device__ __forceinline__ void dswap(T &a, T &b) {
  T t = a;
  a = b;
  b = t;
}

// begin_next: when the loop goes on, also open the next iteration (the
// graph body then needs no k_begin of its own; the host launches one
// before each graph launch).  One warp: lane l commits entries l, l + 32,
// ... of each list; the loop-level decisions are warp-uniform.
__global__ void k_commit(RelDev *rels, LieDev *L, Ctl *ctl, int begin_next) {
  const int lane = threadIdx.x;
  if (lane >= 32) return;
  // the control words and the lists, all loads in flight together
  bool stop = ctl->done | ctl->pause | ctl->overflow | ctl->timeout;
  const u64 it = ctl->iteration, trace_base = ctl->trace_base;
  const u64 trace_rows = ctl->trace_rows, max_it = ctl->max_iteration, stop_at = ctl->stop_at;
  const u32 cond_set = ctl->cond_set;
  const unsigned long long cond_handle = ctl->cond_handle;
  const LaneLists x = lane_lists(L, lane);
  u64 *trace = L->trace;
  if (!stop) {
    const u64 row = it - trace_base;
    const int nu = x.nu;
    bool grew = false;
#pragma unroll
    for (int j = 0; j < kListPerLane; j++) {
      const int i = lane + 32 * j;
      if (i >= nu) continue;
      RelDev &r = rels[x.upd[j]];
      u64 *tr = (trace && row < trace_rows) ? trace + (row * nu + i) * 3 : 0;
      // (Dense form: the update scan has already merged NEWT into the FULL
      // bitmap in place, dense.cuh.)
      if (r.c_newt_n == 0 && !r.newt_phantom) {
        // src/lie.cu:114-121: no new tuple -> a fresh, empty DELTA.
        r.delta.n = 0;
        r.delta_vis = 1;
        r.full_vis = r.w_full_vis;
        if (tr) {
          tr[0] = kNoTrace;
          tr[1] = 0;
          tr[2] = r.full.n;
        }
      } else {
        dswap(r.delta, r.delta_next);
        dswap(r.delta_idx, r.delta_idx_next);
        r.delta_vis = 1;
        if (r.delta.n) {
          // flush_delta (src/relation.cu:405-521): FULL := FULL ∪ DELTA.
          if (r.dense && r.full_lazy) {
            r.full.n += r.delta.n;  // the list is written when the LIE ends
          } else {
            dswap(r.full, r.full_next);
            dswap(r.full_idx, r.full_idx_next);
          }
          r.full_vis = 1;
          grew = true;
        } else {
          r.full_vis = r.w_full_vis;
        }
        if (tr) {
          tr[0] = r.delta.n;
          tr[1] = r.delta.n;
          tr[2] = r.full.n;
        }
      }
      r.newt.n = 0;
      r.c_newt_n = 0;
      r.newt_phantom = 0;
    }
    const bool fixpoint = !__any_sync(0xffffffffu, grew);
#pragma unroll
    for (int j = 0; j < kListPerLane; j++) {
      const int i = lane + 32 * j;
      if (i < x.ns) {
        RelDev &r = rels[x.sta[j]];
        r.full_vis = r.w_full_vis;
        r.delta_vis = r.w_delta_vis;
      }
      if (i < x.nt) rels[x.tmp[j]].newt.n = 0;  // src/lie.cu:85-87
      if (i < x.no) {
        L->once[i] |= L->once_pending[i];
        L->jonce[i] |= L->jonce_pending[i];
      }
    }
    const u64 next = it + 1;
    const bool done = fixpoint || next > max_it;
    const bool pause = !done && next >= stop_at;
    if (lane == 0) {
      ctl->iteration = next;
      ctl->generation = ctl->generation + 1;
      if (done)
        ctl->done = 1;
      else if (pause)
        ctl->pause = 1;
    }
    stop = done || pause;
    __syncwarp();
    if (begin_next && !stop) begin_iteration(rels, L, x, lane);
    __threadfence();
  }
  if (lane == 0 && cond_set)
    cudaGraphSetConditional((cudaGraphConditionalHandle)cond_handle, stop ? 0u : 1u);
}

// Point the control block at a graph's while-node condition: the loop's
// first iteration ran on the stream, the graph runs the ones after it.
__global__ void k_arm_graph(Ctl *ctl, unsigned long long handle) {
  if (threadIdx.x != 0) return;
  ctl->cond_handle = handle;
  ctl->cond_set = 1;
}

// After a loop batch, when the loop reached its fixpoint (or max_iteration)
// with no error: clear `done`, so that the listings enqueued behind the
// loop run.  Otherwise set `pause`, so that they return at once (the host
// reads the loop's state from a copy taken before this, and writes the
// control block again before the next batch).
__global__ void k_ctl_resume(Ctl *ctl) {
  if (threadIdx.x != 0) return;
  if (ctl->done && !ctl->pause && !ctl->overflow && !ctl->timeout && !ctl->oob)
    ctl->done = 0;
  else
    ctl->pause = 1;  // (the host restores the control block before the next batch)
}

// Pack host-layout rows (two u64 columns) into keys; raise bit 0 of *bad if
// a column does not fit 32 bits.  *maxv receives the largest column value.
__global__ void k_pack_rows(const u64 *rows, u64 n, u64 *keys, u64 *maxv, u32 *bad) {
  u64 m = 0;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    u64 c0 = rows[2 * i], c1 = rows[2 * i + 1];
    if ((c0 | c1) >> 32) atomicOr(bad, 1u);
    keys[i] = make_key((u32)c0, (u32)c1);
    m = max(m, max(c0, c1));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m) atomicMax(maxv, m);
}

// Unpack keys into host-layout rows.
__global__ void k_unpack_rows(const u64 *keys, u64 n, u64 *rows) {
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    u64 k = keys[i];
    rows[2 * i] = key_c0(k);
    rows[2 * i + 1] = key_c1(k);
  }
}

// Digest of sorted keys: sum over i of a hash of (i, c0, c1).
__device__ __forceinline__ u64 digest_term(u64 i, u64 k) {
  return mix64(mix64(mix64(i) ^ (u64)key_c0(k)) ^ (u64)key_c1(k));
}
__global__ void k_digest(const u64 *keys, u64 n, u64 *acc) {
  u64 s = 0;
  const u64 stride = (u64)gridDim.x * blockDim.x;
  u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
  // four keys in flight per thread (the hash chain is long; the loads are
  // issued together ahead of it)
  for (; i + 3 * stride < n; i += 4 * stride) {
    const u64 k0 = keys[i], k1 = keys[i + stride], k2 = keys[i + 2 * stride],
              k3 = keys[i + 3 * stride];
    s += digest_term(i, k0) + digest_term(i + stride, k1) + digest_term(i + 2 * stride, k2) +
         digest_term(i + 3 * stride, k3);
  }
  for (; i < n; i += stride) s += digest_term(i, keys[i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(acc, s);
}

}  // namespace gdl
