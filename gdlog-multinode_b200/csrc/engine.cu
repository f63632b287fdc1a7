// engine.cu — host side of the B200 fixpoint engine and its C-ABI
// (include/gdlog_b200.h).
//
// The engine mirrors the reference's object model (Relation with
// FULL/DELTA/NEWT, LIE with update/static/tmp relations and an ordered list
// of RA operators; include/relation.cuh:257-300, include/lie.cuh:11-65) but
// runs a LIE's semi-naive loop as a fixed sequence of kernels per iteration
// whose sizes are all device-resident:
//
//   k_begin                      open the iteration (working counts)
//   per op:  k_join_count + k_join_mat[_pred]   (RelationalJoin)
//            k_copy                             (RelationalCopy / ACopy)
//   per update relation:
//            k_sort_hist + k_sort_pass x P      (onesweep radix sort NEWT)
//            k_merge_diff                       (dedup, NEWT \ FULL, FULL ∪ Δ)
//            k_index_build (FULL, DELTA)        (only indexes some op probes)
//   k_commit                     swap in, log, decide termination (and,
//                                in the graph, open the next iteration)
//
// (In the dense form the per-relation dedup is a bitmap scan instead, and
// joins set bits: dense.cuh.)
//
// That sequence is captured once into a CUDA graph as the body of a
// conditional while-node; k_commit sets the node's condition, so a whole
// batch of iterations runs from one graph launch with no host round trip.
// The host looks at the loop state only between batches: to grow buffers
// after a capacity overflow (the iteration is then rerun from committed
// state) or to finish.
#include "../../include/gdlog_b200.h"

#include "common.cuh"
#include "control.cuh"
#include "dense.cuh"
#include "index.cuh"
#include "join.cuh"
#include "merge.cuh"
#include "pull.cuh"
#include "sort.cuh"
#include "tma.cuh"
#include "exchange.cuh"

#include <algorithm>
#include <condition_variable>
#include <thread>
#include <map>
#include <unordered_map>
#include <chrono>
#include <cstdarg>
#include <cstddef>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

using namespace gdl;

namespace {

constexpr u64 kMinCap = 1ull << 16;
constexpr int kIdentityMaxBits = 22;
constexpr u64 kMaxRows = (1ull << 30) - 4096;  // sort status keeps 30 bits
// Loads over ids below 2^this deduplicate through a domain bitmap (128 MB
// at 15 bits); wider ids use the radix sort.
constexpr int kLoadBitmapMaxBits = 15;
constexpr u64 kTraceRows = 256;  // iterations a loop batch logs (one device buffer)

u64 round_up(u64 x, u64 m) { return (x + m - 1) / m * m; }
double host_ms_since(std::chrono::steady_clock::time_point t) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t).count();
}
u64 next_pow2(u64 x) {
  u64 p = 1;
  while (p < x) p <<= 1;
  return p;
}
int bits_for(u64 v) {
  int b = 1;
  while (b < 64 && (v >> b)) b++;
  return b;
}

// Launch accounting of one enqueue: kernels per ProfKind.
struct Counts {
  int total = 0;
  int kind[kPKinds] = {};
  void add(int k) {
    total++;
    kind[k]++;
  }
};

struct OpHost {
  int kind;  // 0 join, 1 copy, 2 acopy
  int inner = -1, inner_ver = GDL_FULL, outer = -1, outer_ver = GDL_DELTA, out = -1;
  Sel2 sel{0, 1};
  Pred pred{0, 0, 0};
  bool generic = false;  // arity 3 or a computed column: tuples from gen
  GenSpec gen{};
  // The caller's kernel does the per-tuple work (gdl_lie_add_*_hooked).
  gdl_hook_launch hook = nullptr;
  void *hook_ctx = nullptr;
};

struct LieHost {
  std::vector<int> update, statics, tmps;
  std::vector<OpHost> ops;
  long long max_iteration = 2147483647LL;  // include/lie.cuh:30 (INT_MAX)
  bool reload_full = true;                 // include/lie.cuh:29
  bool trace_on = true;
  LieDev *d_lie = nullptr;
  LieDev hdr{};                  // host copy of the header fields (not the copy-once flags)
  u64 *d_trace = nullptr;        // the device trace rows
  JoinRec *d_joinrec = nullptr;  // [kMaxOps]
  std::vector<uint64_t> trace;   // 5 words per record
  double ms = 0;
  u64 kernels = 0, iterations = 0, retries = 0, graph_launches = 0;
  // host wall milliseconds of the last fixpoint: setup, capacity growth
  // (including re-runs), graph capture + instantiation
  double setup_ms = 0, grow_ms = 0, graph_ms = 0;
  cudaGraphExec_t gexec = nullptr;
  unsigned long long cond_handle = 0;
  int gslot = -1;             // gexec's entry in the engine's executable cache
  bool graph_reused = false;  // the last fixpoint's executable came from it
  bool graph_dirty = true;
  Counts per_iter;  // launches of one enqueued iteration
  // Dense form of the running fixpoint (dense.cuh): bits per column (square
  // domain) and the bitmap layout.
  bool dense = false;
  int dk = 0;
  DenseMap map{};
  // Batched form: per-instance new-tuple counts of the running iteration and
  // the last iteration (+1) in which each instance produced new tuples.
  u64 *d_inst_delta = nullptr, *d_inst_last = nullptr;
  u32 n_inst = 0;
};

struct RelHost {
  std::string name;
  int arity = 2, icols = 1, dep = 0;
  bool index_flag = true, tmp_flag = false;
  // FULL's raw buffer in load order (the reference's data_raw); the first
  // |FULL| rows of it become DELTA at the start of a LIE
  // (copy_relation_container, src/relation.cu:764-795).
  u64 *raw = nullptr;
  u64 raw_n = 0;
  bool raw_is_full = true;
  bool delta_sorted = true;
  u64 bm_words = 0;  // size of this relation's bitmaps (dense form), words
  bool bm_valid = false;       // bmF holds FULL (set by a dense LIE)
  bool full_resident = false;  // FULL exists only as bmF (batched form, or too large)
  int bm_dk = 0;               // square domain bits of that bitmap (plain form)
  // In-edges of this relation's FULL (column-1 value -> column-0 values),
  // built at the start of a LIE whose row-gather joins read it as inner.
  // A load committed on the device that the host mirror has not read back
  // (its FULL count is known on the device only).
  bool stale = false;
  u32 *inv_off = nullptr, *inv_cur = nullptr;
  u32 *inv_keys = nullptr, *inv_ys = nullptr;  // per in-edge: source, y
  u64 inv_cap = 0;
  int inv_dk = 0;
  // the in-edge lists hold FULL's current rows (inv_n of them, 2^inv_dk
  // ids): cleared by a load and when a LIE updates the relation
  bool inv_ready = false;
  u64 inv_n = 0;
};

}  // namespace

struct gdl_engine {
  int device = 0;
  int sms = 148;
  cudaStream_t s = nullptr;
  bool own_stream = false;
  std::string err;
  std::vector<RelHost> rels;
  std::vector<RelDev> h;  // host mirror of the device relation table
  RelDev *d_rels = nullptr;
  Ctl *d_ctl = nullptr;
  Ctl *h_ctl = nullptr;  // pinned
  // Pinned copies taken behind a loop batch before its one host wait: the
  // control block after the listings enqueued behind the loop, the batch's
  // trace rows and the relation table.
  Ctl *h_ctl2 = nullptr;
  u64 *h_trace = nullptr;  // [kTraceRows][kMaxRels][3]
  RelDev *h_rels_pin = nullptr;
  int kbits = 1;         // bits of the largest column value loaded
  // Arity 3 (common.cuh, key_col): once a relation of arity 3 exists every
  // sort covers the whole low half of the keys; k2 = bits of column 2, fixed
  // by the first arity-3 load (32 - bits of the ids loaded until then).
  bool wide = false;
  int k2 = 0;
  u64 max_value = 0;
  std::vector<LieHost> lies;
  // scratch
  u64 *sort_buf = nullptr;
  u64 sort_cap = 0;
  u32 *sort_offsets = nullptr, *sort_counters = nullptr, *sort_status = nullptr;
  u64 sort_status_tiles = 0;
  int sort_status_passes = 0;
  int sort_status_radix = 0;
  // Tuned shapes (gdl_tuning): radix sort digit width, block size of the
  // probe-and-expand join (k_join_bm), in-edges per unit of work of a
  // row-gather join (k_join_rows_bm).
  int radix_bits = kRadixBits;
  int join_block = 256;
  int rows_piece = 32;
  // launches of this engine's kernels outside the loop's counted ones (LIE
  // setup, listings): a fixpoint adds those in its span to its kernel count
  u64 aux_launches = 0;
  int load_dedup = 2;  // loads: 1 radix sort + merge, 2 bitmap listing where it fits
  u64 *crow_off = nullptr, *crow_key = nullptr;
  u32 *crow_start = nullptr, *crow_len = nullptr;
  u64 crow_cap = 0;
  Lb lb_cnt{}, lb_nz{}, lb_merge{};
  u64 *merge_parts = nullptr;  // [lb_merge_tiles + 1]
  // Dense scans: look-back state of the tile-count scan.
  Lb lb_bm{};
  u64 lb_bm_tiles = 0;
  Lb lb_list{};  // listings (k_bm_list_*): per 2048-word tile its count (flag) and offset (agg)
  u64 lb_list_tiles = 0;
  // Graph executables of dropped LIEs: destroyed by a worker thread of the
  // engine (destroying one takes ~0.1 ms of host time that the caller's
  // next program need not wait for; none of them can be running).
  // Tensor maps of the square-domain bitmaps for the TMA passes (tma.cuh),
  // by (base address, domain bits); tma_ok: the driver's encoder was found
  // (GDLOG_NO_TMA=1 keeps the LDG/STG passes of pull.cuh).
  bool tma_ok = false;
  void *tma_encode = nullptr;
  std::map<std::pair<const void *, int>, CUtensorMap> tmaps;
  std::vector<cudaGraphExec_t> graveyard;
  std::mutex reap_mu;
  std::condition_variable reap_cv;
  std::vector<cudaGraphExec_t> reap_list;  // handed to the worker
  std::thread reaper;
  bool reap_stop = false;
  // dalloc / dfree: bytes of each live block, and freed blocks for reuse
  std::unordered_map<void *, size_t> alloc_size;
  std::multimap<size_t, void *> spare;
  std::unordered_map<void *, std::multimap<size_t, void *>::iterator> spare_at;
  size_t spare_bytes = 0;
  // The blocks the program before the last gdl_engine_clear got, per
  // request size in request order (replayed by dalloc), and this program's.
  std::unordered_map<size_t, std::vector<void *>> replay, alloc_log;
  std::unordered_map<size_t, size_t> replay_seen;
  // Executables of iteration graphs, kept across programs (build_graph).
  struct CachedGraph {
    cudaGraph_t graph = nullptr;  // the loop graph (owns body)
    cudaGraph_t body = nullptr;   // the iteration as captured, for comparison
    cudaGraphExec_t exec = nullptr;
    unsigned long long handle = 0;
    Counts per_iter;
    size_t nodes = 0;
    u64 sig = 0;  // graph_signature of body
    bool in_use = false;
    u64 used = 0;  // last use, for eviction
  };
  std::vector<CachedGraph> gcache;
  u64 gcache_clock = 0;
  std::unordered_map<const void *, std::vector<size_t>> param_sizes;
  // Largest 2*bits domain kept as bitmaps (GDLOG_DENSE_MAX_BITS), and the
  // dedup path: 0 chosen by domain size, 1 always sort/merge, 2 always
  // bitmaps where the domain allows (GDLOG_DEDUP=auto|sort|dense).
  int dense_max_bits = kDenseMaxDomainBits;
  int dedup_mode = 0;
  int join_ctas_per_sm = 8;   // gdl_tuning
  int count_ctas_per_sm = 4;
  int index_slots_per_key = 2;
  int dirty_min_log2_words = 24;
  int dense_join_passes = 1;
  int join_aggregate = 1;  // 1: one reduction per candidate, 2: warp-aggregated by word
  bool row_or_joins = true;  // GDLOG_ROW_OR=0 turns row-OR joins off
  // 1: push form only, 2: pull form where eligible from 2^kPullAutoBits ids,
  // 3: pull form where eligible (pull.cuh)
  int pull_joins = 2;
  int row_gather = 2;
  u32 spin_limit = kSpinLimit;  // polls of a bounded device wait
  u32 test_wait = 0;            // gdl_engine_test_timeout (next fixpoint only)
  u64 *d_pull_count = nullptr;  // bit count of a transposed NEWT (zero between launches)
  // Device memory in bytes, read once at creation: cudaMemGetInfo can take
  // tens of milliseconds on a busy host, so the fixpoint sizes its lists
  // from this and asks for free memory only after an allocation failed.
  u64 total_mem = 0;
  // Batched form (gdl_engine_set_instances): the block-diagonal layout.
  bool instances = false;
  std::vector<SegInfo> segs;
  int seg_shift = 31;
  u64 seg_words = 0;
  SegInfo *d_segs = nullptr;
  u32 *d_tile_inst = nullptr;
  SegInfo *d_square_seg = nullptr;  // the one segment of the square domain
  u64 lb_cnt_tiles = 0, lb_nz_tiles = 0, lb_merge_tiles = 0;
  LaunchRec *recs = nullptr;  // [0] join count, [1] join mat, [2] merge, [3] copy,
                              // [4] [5] bitmap scans, [6] pull join, [7] transpose,
                              // [8] bitmap listing
  DArr *d_tmp = nullptr;      // [4] temporary descriptors for loads
  void *d_count = nullptr;    // gdl_join_count's scratch (CountScratch)
  void *d_part = nullptr;     // gdl_partition_rows: counts and cursors per destination
  u64 *d_u64 = nullptr;       // [4] small device scalars
  u32 *d_u32 = nullptr;       // [4]: [0] pack check, [3] device checks of async loads (sticky)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Graph capture runs on its own stream, so that the engine stream can run
  // a loop's first iteration meanwhile; ev_first marks that iteration's end.
  cudaStream_t cap_s = nullptr;
  cudaEvent_t ev_first = nullptr;
  u64 kernels_launched = 0;
  bool broken = false;  // a bounded wait gave up or a bounds check fired
  // The control block's build generation (index epochs), tracked on the
  // host: set by reset_ctl and by every read of the control block after a
  // loop ran, so setting up a loop needs no read-back.
  u64 generation = 0;
  // The host mirror `h` equals the device relation table: set by a pull and
  // by the last push of a load or a fixpoint, cleared before the kernels
  // that change the table run, so reads need no round trip when it is set.
  bool mirror_fresh = false;
  // Per-kernel accounting of fixpoint loops (gdl_engine_profile).  With
  // `profile` set, loops run launch by launch with an event pair around
  // every kernel instead of from the captured graph.
  bool profile = false;
  double prof_ms[kPKinds] = {};
  u64 prof_launches[kPKinds] = {};
  u64 prof_bytes[kPKinds] = {};
  std::vector<cudaEvent_t> ev_pool;
  struct Pending {
    int kind;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
};

namespace {

gdl_status fail(gdl_engine *e, gdl_status code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  e->err = buf;
  return code;
}

#define CK(e, call)                                                                   \
  do {                                                                                \
    cudaError_t _r = (call);                                                          \
    if (_r != cudaSuccess)                                                            \
      return fail((e), _r == cudaErrorMemoryAllocation ? GDL_E_NOMEM : GDL_E_CUDA,    \
                  "%s failed: %s (%s:%d)", #call, cudaGetErrorString(_r), __FILE__, \
                  __LINE__);                                                          \
  } while (0)

#define TRY(x)                     \
  do {                             \
    gdl_status _s = (x);           \
    if (_s != GDL_OK) return _s;   \
  } while (0)

// Device blocks are recycled inside the engine: a freed block joins a spare
// list (up to a quarter of the device's memory) and a later request of at
// most its size, and at least half of it, takes it back, stream-ordered on
// the engine stream like the pool's own reuse.  A program run after
// gdl_engine_clear therefore makes no allocation calls once the first run
// has sized everything.
//
// The same program run again gets the same blocks: the j-th request of a
// given size takes back, when it is spare, the block the j-th request of
// that size got in the program before the last gdl_engine_clear.  Device
// addresses in the program's kernel arguments then repeat, and its
// iteration graphs are found in the executable cache (build_graph).
void *take_spare(gdl_engine *e, std::multimap<size_t, void *>::iterator it) {
  void *p = it->second;
  e->spare_bytes -= it->first;
  e->alloc_size[p] = it->first;
  e->spare_at.erase(p);
  e->spare.erase(it);
  return p;
}
void drop_spare(gdl_engine *e) {
  for (auto &kv : e->spare) cudaFreeAsync(kv.second, e->s);
  e->spare.clear();
  e->spare_at.clear();
  e->spare_bytes = 0;
}
gdl_status dalloc(gdl_engine *e, void **p, size_t bytes) {
  *p = nullptr;
  bytes = round_up(std::max<size_t>(bytes, 16), 256);
  const size_t j = e->replay_seen[bytes]++;
  auto rp = e->replay.find(bytes);
  if (rp != e->replay.end() && j < rp->second.size()) {
    auto at = e->spare_at.find(rp->second[j]);
    if (at != e->spare_at.end()) *p = take_spare(e, at->second);
  }
  if (!*p) {
    auto it = e->spare.lower_bound(bytes);
    if (it != e->spare.end() && it->first <= 2 * bytes) *p = take_spare(e, it);
  }
  if (!*p) {
    cudaError_t r = cudaMallocAsync(p, bytes, e->s);
    if (r == cudaErrorMemoryAllocation && !e->spare.empty()) {
      // give the spare blocks back and try once more
      cudaGetLastError();
      drop_spare(e);
      r = cudaMallocAsync(p, bytes, e->s);
    }
    CK(e, r);
    e->alloc_size[*p] = bytes;
  }
  e->alloc_log[bytes].push_back(*p);
  return GDL_OK;
}
void dfree(gdl_engine *e, void *p) {
  if (!p) return;
  auto it = e->alloc_size.find(p);
  if (it == e->alloc_size.end()) {
    cudaFreeAsync(p, e->s);
    return;
  }
  const size_t b = it->second;
  e->alloc_size.erase(it);
  if (e->spare_bytes + b > e->total_mem / 4) {
    cudaFreeAsync(p, e->s);
    return;
  }
  e->spare_at[p] = e->spare.emplace(b, p);
  e->spare_bytes += b;
}

// Grow array `a` to hold at least `need` elements; keep its contents.
gdl_status ensure_arr(gdl_engine *e, DArr &a, u64 need, bool keep) {
  if (a.cap >= need && a.ptr) return GDL_OK;
  u64 cap = std::max<u64>({need, kMinCap, a.cap + a.cap / 2});
  cap = round_up(cap, 2);
  if (cap > kMaxRows) cap = std::max<u64>(need, kMaxRows);
  if (need > kMaxRows)
    return fail(e, GDL_E_UNSUPPORTED, "relation of %llu tuples exceeds the %llu-tuple limit",
                (unsigned long long)need, (unsigned long long)kMaxRows);
  u64 *p = nullptr;
  TRY(dalloc(e, (void **)&p, cap * sizeof(u64)));
  if (keep && a.n) CK(e, cudaMemcpyAsync(p, a.ptr, a.n * sizeof(u64), cudaMemcpyDeviceToDevice, e->s));
  dfree(e, a.ptr);
  a.ptr = p;
  a.cap = cap;
  if (!keep) a.n = std::min(a.n, cap);
  return GDL_OK;
}

// Size an index for arrays of capacity `cap`.
gdl_status ensure_index(gdl_engine *e, Index &ix, u64 cap) {
  u32 mode;
  u64 slots;
  if (e->kbits <= kIdentityMaxBits) {
    mode = 0;
    slots = 1ull << e->kbits;
  } else {
    mode = 1;
    u64 distinct = std::min<u64>(cap, 1ull << std::min(e->kbits, 40));
    slots = next_pow2(std::max<u64>((u64)e->index_slots_per_key * distinct, 1024));
  }
  if (ix.slots && ix.hash_mode == mode && ix.mask + 1 >= slots) return GDL_OK;
  dfree(e, ix.slots);
  TRY(dalloc(e, (void **)&ix.slots, slots * sizeof(uint4)));
  CK(e, cudaMemsetAsync(ix.slots, 0, slots * sizeof(uint4), e->s));
  ix.mask = slots - 1;
  ix.hash_mode = mode;
  ix.epoch = 0;
  return GDL_OK;
}

// Hand the executables of dropped LIEs to the engine's worker thread, which
// destroys them (none of them can be running: the stream was synchronised
// when they were dropped).
void reap_graphs(gdl_engine *e) {
  if (e->graveyard.empty()) return;
  {
    std::lock_guard<std::mutex> lock(e->reap_mu);
    if (!e->reaper.joinable()) {
      const int dev = e->device;
      e->reaper = std::thread([e, dev] {
        cudaSetDevice(dev);
        std::unique_lock<std::mutex> lk(e->reap_mu);
        while (true) {
          e->reap_cv.wait(lk, [e] { return e->reap_stop || !e->reap_list.empty(); });
          std::vector<cudaGraphExec_t> work;
          work.swap(e->reap_list);
          lk.unlock();
          for (cudaGraphExec_t x : work) cudaGraphExecDestroy(x);
          lk.lock();
          if (e->reap_stop && e->reap_list.empty()) return;
        }
      });
    }
    e->reap_list.insert(e->reap_list.end(), e->graveyard.begin(), e->graveyard.end());
  }
  e->graveyard.clear();
  e->reap_cv.notify_one();
}

gdl_status pull(gdl_engine *e) {
  if (e->rels.empty()) return GDL_OK;
  u32 load_err = 0;
  CK(e, cudaMemcpyAsync(e->h.data(), e->d_rels, e->rels.size() * sizeof(RelDev),
                        cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaMemcpyAsync(&load_err, e->d_u32 + 3, sizeof load_err, cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  e->mirror_fresh = true;
  for (RelHost &rh : e->rels) rh.stale = false;
  if (load_err) {
    e->broken = true;
    return fail(e, GDL_E_TIMEOUT,
                "a relation load failed its device checks (timeout %u, dropped write %u, "
                "capacity %u)", load_err & 1u, (load_err >> 1) & 1u, (load_err >> 2) & 1u);
  }
  return GDL_OK;
}
// pull() unless the mirror is known to equal the device table.
gdl_status refresh(gdl_engine *e) { return e->mirror_fresh ? GDL_OK : pull(e); }
// pull() only if relation r's mirror entry waits for a load's result.
gdl_status refresh_rel(gdl_engine *e, int r) { return e->rels[r].stale ? pull(e) : GDL_OK; }
// One relation's mirror entry to the device (the others stay as they are
// there: an asynchronous load may have changed them).
gdl_status push_rel(gdl_engine *e, int r) {
  CK(e, cudaMemcpyAsync(e->d_rels + r, &e->h[r], sizeof(RelDev), cudaMemcpyHostToDevice, e->s));
  return GDL_OK;
}
// The host mirror to the device, stream-ordered: a copy from pageable
// memory is staged when the call returns, so the mirror may change at once.
gdl_status push(gdl_engine *e) {
  if (e->rels.empty()) return GDL_OK;
  CK(e, cudaMemcpyAsync(e->d_rels, e->h.data(), e->rels.size() * sizeof(RelDev),
                        cudaMemcpyHostToDevice, e->s));
  return GDL_OK;
}

// The 2-D tensor map of a square-domain bitmap (2^dk rows of 2^(dk-5)
// words) with a box of one 256 x 256-bit tile; null if it cannot be made.
const CUtensorMap *bm_tmap(gdl_engine *e, const u32 *bm, int dk) {
  if (!e->tma_ok || !bm || dk < 8) return nullptr;
  auto key = std::make_pair((const void *)bm, dk);
  auto it = e->tmaps.find(key);
  if (it != e->tmaps.end()) return &it->second;
  using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                              const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                              const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
  CUtensorMap m;
  const cuuint64_t dims[2] = {1ull << (dk - 5), 1ull << dk};
  const cuuint64_t strides[1] = {(1ull << (dk - 5)) * 4};
  const cuuint32_t box[2] = {8, 256};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = reinterpret_cast<Encode>(e->tma_encode)(
      &m, CU_TENSOR_MAP_DATA_TYPE_UINT32, 2, const_cast<u32 *>(bm), dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return nullptr;
  return &(e->tmaps[key] = m);
}

int grid_for(gdl_engine *e, u64 work, u64 per_block, int per_sm) {
  u64 g = (work + per_block - 1) / per_block;
  u64 lim = (u64)e->sms * per_sm;
  if (g > lim) g = lim;
  if (g < 1) g = 1;
  return (int)g;
}

// Sorts radix the significant bits only: column 0's kbits and the low half's
// kbits (arity 2) or all 32 (once arity-3 keys exist).
int sort_lo_bits(const gdl_engine *e) { return e->wide ? 32 : e->kbits; }
// Digit width of the radix sort: the tuned one (6, 8 or 10 bits) unless it
// would take more than kMaxPasses passes over the significant bits.
int sort_bits(const gdl_engine *e) {
  const int b = e->radix_bits, bits = e->kbits + sort_lo_bits(e);
  return (bits + b - 1) / b <= kMaxPasses ? b : kRadixBits;
}
int sort_passes(const gdl_engine *e) {
  const int b = sort_bits(e);
  return std::max(1, (e->kbits + sort_lo_bits(e) + b - 1) / b);
}

// The key bits of a relation's dependent columns (cleared to compare the
// set difference's prefix, merge.cuh k_dep_mask); 0 without any.
u64 dep_low_mask(const gdl_engine *e, const RelHost &h) {
  if (h.dep == 0) return 0;
  if (h.arity == 3 && h.dep == 1) return (1ull << e->k2) - 1;
  return 0xFFFFFFFFull;  // columns 1.. of the low half
}

cudaEvent_t take_event(gdl_engine *e) {
  cudaEvent_t ev = nullptr;
  if (!e->ev_pool.empty()) {
    ev = e->ev_pool.back();
    e->ev_pool.pop_back();
  } else if (cudaEventCreate(&ev) != cudaSuccess) {
    ev = nullptr;
  }
  return ev;
}

// Event pair around one launch when profiling (no-op otherwise).
cudaEvent_t prof_begin(gdl_engine *e) {
  if (!e->profile) return nullptr;
  cudaEvent_t a = take_event(e);
  if (a) cudaEventRecord(a, e->s);
  return a;
}
void prof_end(gdl_engine *e, int kind, cudaEvent_t a) {
  if (!a) return;
  cudaEvent_t b = take_event(e);
  if (!b) {
    e->ev_pool.push_back(a);
    return;
  }
  cudaEventRecord(b, e->s);
  e->pending.push_back({kind, a, b});
}
// After a stream synchronize: fold the recorded pairs into prof_ms.
void prof_collect(gdl_engine *e) {
  for (auto &p : e->pending) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) e->prof_ms[p.kind] += ms;
    e->ev_pool.push_back(p.a);
    e->ev_pool.push_back(p.b);
  }
  e->pending.clear();
}

#define PLAUNCH(cnt, kind, ...)                \
  do {                                         \
    cudaEvent_t _pe = prof_begin(e);           \
    __VA_ARGS__;                               \
    prof_end(e, (kind), _pe);                  \
    (cnt)->add(kind);                          \
  } while (0)

// ---------------------------------------------------------------------------
// Scratch sizing
// ---------------------------------------------------------------------------
gdl_status ensure_lb(gdl_engine *e, Lb &lb, u64 &have, u64 tiles) {
  if (have >= tiles) return GDL_OK;
  tiles = std::max<u64>(tiles + tiles / 2, 1024);
  dfree(e, lb.flag);
  dfree(e, lb.agg);
  dfree(e, lb.inc);
  TRY(dalloc(e, (void **)&lb.flag, tiles * sizeof(u32)));
  TRY(dalloc(e, (void **)&lb.agg, tiles * sizeof(u64)));
  TRY(dalloc(e, (void **)&lb.inc, tiles * sizeof(u64)));
  CK(e, cudaMemsetAsync(lb.flag, 0, tiles * sizeof(u32), e->s));
  have = tiles;
  return GDL_OK;
}

gdl_status ensure_scratch(gdl_engine *e) {
  u64 max_cap = 0, max_full = 0, max_newt = 0;
  for (size_t i = 0; i < e->rels.size(); i++) {
    const RelDev &r = e->h[i];
    max_cap = std::max({max_cap, r.full.cap, r.delta.cap, r.newt.cap, r.delta_next.cap});
    max_full = std::max({max_full, r.full.cap, r.full_next.cap});
    max_newt = std::max({max_newt, r.newt.cap});
  }
  max_newt = std::max(max_newt, e->sort_cap);
  // sort
  if (e->sort_cap < max_newt || !e->sort_buf) {
    dfree(e, e->sort_buf);
    e->sort_cap = std::max<u64>(max_newt, kMinCap);
    TRY(dalloc(e, (void **)&e->sort_buf, e->sort_cap * sizeof(u64)));
  }
  const u64 tiles = e->sort_cap / kSortTile + 2;
  const int passes = std::max(sort_passes(e), 1);
  const int radix = 1 << sort_bits(e);
  if (tiles > e->sort_status_tiles || passes > e->sort_status_passes ||
      radix > e->sort_status_radix || !e->sort_status) {
    dfree(e, e->sort_status);
    e->sort_status_tiles = tiles;
    e->sort_status_passes = std::max(passes, 4);
    e->sort_status_radix = std::max(radix, kRadix);
    TRY(dalloc(e, (void **)&e->sort_status,
               (u64)e->sort_status_passes * tiles * e->sort_status_radix * sizeof(u32)));
  }
  if (!e->sort_offsets) {
    TRY(dalloc(e, (void **)&e->sort_offsets, kMaxPasses * kMaxRadix * sizeof(u32)));
    TRY(dalloc(e, (void **)&e->sort_counters, (kMaxPasses + 1) * sizeof(u32)));
    CK(e, cudaMemsetAsync(e->sort_offsets, 0, kMaxPasses * kMaxRadix * sizeof(u32), e->s));
    CK(e, cudaMemsetAsync(e->sort_counters, 0, (kMaxPasses + 1) * sizeof(u32), e->s));
  }
  // join records
  if (e->crow_cap < max_cap || !e->crow_off) {
    u64 c = std::max<u64>(max_cap, kMinCap);
    dfree(e, e->crow_off);
    dfree(e, e->crow_key);
    dfree(e, e->crow_start);
    dfree(e, e->crow_len);
    TRY(dalloc(e, (void **)&e->crow_off, (c + 1) * sizeof(u64)));
    TRY(dalloc(e, (void **)&e->crow_key, c * sizeof(u64)));
    TRY(dalloc(e, (void **)&e->crow_start, c * sizeof(u32)));
    TRY(dalloc(e, (void **)&e->crow_len, c * sizeof(u32)));
    e->crow_cap = c;
  }
  TRY(ensure_lb(e, e->lb_cnt, e->lb_cnt_tiles, e->crow_cap / kJoinTile + 2));
  TRY(ensure_lb(e, e->lb_nz, e->lb_nz_tiles, e->crow_cap / kJoinTile + 2));
  const u64 had = e->lb_merge_tiles;
  TRY(ensure_lb(e, e->lb_merge, e->lb_merge_tiles, (max_full + max_newt) / kMergeTile + 2));
  if (!e->merge_parts || had != e->lb_merge_tiles) {
    dfree(e, e->merge_parts);
    TRY(dalloc(e, (void **)&e->merge_parts, (e->lb_merge_tiles + 1) * sizeof(u64)));
  }
  return GDL_OK;
}

// Scan scratch of a relation kept as bitmaps of `words` words: one u64 per
// tile or per group of kGroupChunks chunks (more of the latter), then the
// dirty-chunk list (u32 per chunk).
u64 scan_scratch_bytes(u64 words) {
  const u64 chunks = words / kBmChunkWords;
  return chunks / kGroupChunks * sizeof(u64) + chunks * sizeof(u32);
}

// Bitmaps of one relation in dense form: NEWT always, FULL and its next
// version for update relations.
gdl_status ensure_bitmaps(gdl_engine *e, int r, u64 words, bool with_full) {
  RelHost &rh = e->rels[r];
  RelDev &h = e->h[r];
  if (rh.bm_words != words) {
    for (u32 **p : {&h.bmF, &h.bmG, &h.bmDT, &h.bmGT, &h.bmOT, &h.bmDN}) {
      dfree(e, *p);
      *p = nullptr;
    }
    dfree(e, h.bmD);
    h.bmD = nullptr;
    dfree(e, h.tile_prefix);
    h.tile_prefix = nullptr;
    rh.bm_words = words;
  }
  if (!h.bmG) TRY(dalloc(e, (void **)&h.bmG, words * 4));
  if (!h.bmD) TRY(dalloc(e, (void **)&h.bmD, words / kBmChunkWords));
  // tile (or chunk-group) counts / prefixes, then the dirty-chunk list
  if (!h.tile_prefix) TRY(dalloc(e, (void **)&h.tile_prefix, scan_scratch_bytes(words)));
  if (with_full && !h.bmF) TRY(dalloc(e, (void **)&h.bmF, words * 4));
  memset(&h.scan, 0, sizeof h.scan);
  return GDL_OK;
}

// The FULL bitmap of a static relation read as a row-gather join's outer
// (its FULL does not change during the LIE): that bitmap alone, sized as
// ensure_bitmaps sizes them.
gdl_status ensure_static_bitmap(gdl_engine *e, int r, u64 words) {
  RelHost &rh = e->rels[r];
  RelDev &h = e->h[r];
  if (rh.bm_words != words) {
    for (u32 **p : {&h.bmF, &h.bmG, &h.bmDT, &h.bmGT, &h.bmOT, &h.bmDN}) {
      dfree(e, *p);
      *p = nullptr;
    }
    dfree(e, h.bmD);
    h.bmD = nullptr;
    dfree(e, h.tile_prefix);
    h.tile_prefix = nullptr;
    rh.bm_words = words;
  }
  if (!h.bmF) TRY(dalloc(e, (void **)&h.bmF, words * 4));
  return GDL_OK;
}

gdl_status ensure_dense_scratch(gdl_engine *e, u64 words) {
  // look-back units: tiles / kScanChunk, or in listed mode dirty chunks /
  // kDirtyUnit and chunk groups / kScanChunk (the largest of the three)
  const u64 chunks = words / kBmChunkWords;
  const u64 units = std::max({words / kBmTileWords / kScanChunk, chunks / kDirtyUnit,
                              chunks / kGroupChunks / kScanChunk}) + 2;
  TRY(ensure_lb(e, e->lb_bm, e->lb_bm_tiles, units));
  return GDL_OK;
}

// Put the device control block in a runnable state (no stop flags, no
// graph condition) keeping the build generation.
gdl_status reset_ctl(gdl_engine *e) {
  Ctl c;
  memset(&c, 0, sizeof c);
  c.generation = ++e->generation;
  c.max_iteration = ~0ull;
  c.stop_at = ~0ull;
  c.spin_limit = e->spin_limit;
  CK(e, cudaMemcpyAsync(e->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, e->s));
  return GDL_OK;
}

// ---------------------------------------------------------------------------
// Kernel launchers
// ---------------------------------------------------------------------------
void launch_sort(gdl_engine *e, const DArr *d_keys, u64 *buf0, u64 cap, Counts *kc) {
  SortArgs a;
  memset(&a, 0, sizeof a);
  a.keys = d_keys;
  a.buf0 = buf0;
  a.buf1 = e->sort_buf;
  a.cap = std::min(cap, e->sort_cap);
  a.kbits = sort_lo_bits(e);
  a.passes = sort_passes(e);
  a.offsets = e->sort_offsets;
  a.status = e->sort_status;
  a.max_tiles = e->sort_status_tiles;
  a.counters = e->sort_counters;
  a.ctl = e->d_ctl;
  int gh = grid_for(e, cap, (u64)kSortTile, 2);
  int gp = grid_for(e, cap, kSortTile, 4);
  switch (sort_bits(e)) {
#define GDL_SORT(B)                                                                         \
  case B:                                                                                   \
    PLAUNCH(kc, kPSortHist,                                                                 \
            k_sort_hist<B><<<gh, kSortBlock, sort_smem_bytes<B>(), e->s>>>(a));             \
    for (int p = 0; p < a.passes; p++)                                                      \
      PLAUNCH(kc, kPSortPass,                                                               \
              k_sort_pass<B><<<gp, kSortBlock, sort_smem_bytes<B>(), e->s>>>(a, p));       \
    break;
    GDL_SORT(6)
    GDL_SORT(10)
    default:
    GDL_SORT(8)
#undef GDL_SORT
  }
}

u64 *sorted_location(gdl_engine *e, u64 *buf0) { return (sort_passes(e) & 1) ? e->sort_buf : buf0; }

// FULL := unique(sort(keys[0..n))) for a load; DELTA/NEWT cleared.  The
// load is committed on the device (k_load_commit) without a round trip: the
// host mirror of this relation is marked stale and read back at the next
// point that needs it, where the load's device checks are reported too.
// Only this relation's entry is written to the device table.
gdl_status launch_list(gdl_engine *e, const u32 *bm, u64 words, int rs, DArr *out,
                       int check_n);

gdl_status load_keys(gdl_engine *e, int rel, const u64 *keys_dev, u64 n) {
  RelHost &rh = e->rels[rel];
  TRY(refresh_rel(e, rel));
  RelDev &r = e->h[rel];
  rh.bm_valid = false;
  rh.full_resident = false;
  rh.inv_ready = false;
  // raw := keys in load order
  if (rh.raw && !rh.raw_is_full) dfree(e, rh.raw);
  rh.raw = nullptr;
  rh.raw_n = n;
  rh.raw_is_full = false;
  if (n) {
    TRY(dalloc(e, (void **)&rh.raw, n * sizeof(u64)));
    CK(e, cudaMemcpyAsync(rh.raw, keys_dev, n * sizeof(u64), cudaMemcpyDeviceToDevice, e->s));
  }
  r.full.n = 0;
  r.delta.n = 0;
  r.newt.n = 0;
  r.full_vis = r.delta_vis = r.w_full_vis = r.w_delta_vis = 1;
  r.full_idx.epoch = r.full_idx_next.epoch = r.delta_idx.epoch = r.delta_idx_next.epoch = 0;
  TRY(ensure_arr(e, r.full, n, false));
  TRY(ensure_arr(e, r.full_next, n, false));
  const int ldk = std::max(e->kbits, kPullMinBits);
  // the bitmap's bytes are streamed twice (cleared, then counted): worth it
  // up to 32 MB, or with at least one row per KB of bitmap (measured: 40,000
  // rows over 2^14 ids load faster this way; 20,000-60,000 over 2^15 ids,
  // 128 MB, slower)
  const u64 bm_bytes = 1ull << (2 * ldk - 3);
  if (n > (u64)kSortTile && e->load_dedup == 2 && !e->wide && rh.arity == 2 &&
      ldk <= kLoadBitmapMaxBits && (bm_bytes <= (32ull << 20) || n >= bm_bytes / 1024)) {
    // Sort + unique through a bitmap over the key domain (2^(2 ldk) bits,
    // at most 128 MB): the rows' bits set, then listed in key order into
    // full_next, which k_load_commit swaps in.  Five streaming launches in
    // place of the radix sort's and merge's latency-bound passes.
    const u64 words = 1ull << (2 * ldk - 5);
    u32 *bm = nullptr;
    TRY(dalloc(e, (void **)&bm, words * sizeof(u32)));
    CK(e, cudaMemsetAsync(bm, 0, words * sizeof(u32), e->s));
    TRY(push_rel(e, rel));
    TRY(reset_ctl(e));
    k_bm_set_keys<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(keys_dev, n, bm, ldk, e->d_ctl);
    TRY(launch_list(e, bm, words, ldk - 5, &e->d_rels[rel].full_next, 0));
    k_load_commit<<<1, 32, 0, e->s>>>(&e->d_rels[rel], e->d_ctl, e->d_u32 + 3);
    CK(e, cudaGetLastError());
    dfree(e, bm);  // stream-ordered behind the listing
    std::swap(r.full, r.full_next);
    r.newt.n = 0;
    r.delta_next.n = 0;
    r.c_newt_n = 0;
    rh.stale = true;
    e->mirror_fresh = false;
    return GDL_OK;
  }
  if (n) {
    // sort a copy in the NEWT buffer, then dedup it into FULL
    TRY(ensure_arr(e, r.newt, n, false));
    TRY(ensure_arr(e, r.delta_next, n, false));
    TRY(ensure_scratch(e));
    CK(e, cudaMemcpyAsync(r.newt.ptr, keys_dev, n * sizeof(u64), cudaMemcpyDeviceToDevice, e->s));
    r.newt.n = n;
    TRY(push_rel(e, rel));
    TRY(reset_ctl(e));
    Counts kc;
    launch_sort(e, &e->d_rels[rel].newt, r.newt.ptr, r.newt.cap, &kc);
    MergeArgs m;
    memset(&m, 0, sizeof m);
    m.newt = &e->d_rels[rel].newt;
    m.a = sorted_location(e, r.newt.ptr);
    // B = empty FULL
    m.full = &e->d_rels[rel].full;
    m.full_next = &e->d_rels[rel].full_next;
    m.delta_next = &e->d_rels[rel].delta_next;
    m.c_newt_n = &e->d_rels[rel].c_newt_n;
    m.rec = &e->recs[2];
    m.lb = e->lb_merge;
    m.parts = e->merge_parts;
    m.parts_cap = e->lb_merge_tiles + 1;
    m.ctl = e->d_ctl;
    m.rel = rel;
    k_merge_partition<<<grid_for(e, n / kMergeTile + 2, 256, 8), 256, 0, e->s>>>(m);
    k_merge_diff<<<grid_for(e, n, kMergeTile, 4), kMergeBlock, kMergeSmemBytes, e->s>>>(m);
    k_load_commit<<<1, 32, 0, e->s>>>(&e->d_rels[rel], e->d_ctl, e->d_u32 + 3);
    CK(e, cudaGetLastError());
    // the mirror as the device now has it, but for FULL's count
    std::swap(r.full, r.full_next);
    r.newt.n = 0;
    r.delta_next.n = 0;
    r.c_newt_n = 0;
    rh.stale = true;
    e->mirror_fresh = false;
    return GDL_OK;
  }
  TRY(push_rel(e, rel));
  return GDL_OK;
}

// ---------------------------------------------------------------------------
// One iteration of a LIE
// ---------------------------------------------------------------------------
struct Plan {
  std::vector<char> full_idx, delta_idx;  // per relation: index needed
  std::vector<char> full_list;            // FULL read as a list by some op
  std::vector<char> newt_list;            // NEWT read as a join outer
  std::vector<char> acopy_src;            // NEWT read by an ACopy
  std::vector<char> pull;                 // per op: pull form (pull.cuh)
  std::vector<char> pull_t;               // per op: pull form with a transposed output
  std::vector<char> out_t;                // per relation: written by such an op
  std::vector<char> fold_late;            // per relation: its transposed twin is its NEWT
  std::vector<char> delta_t, newt_t;      // per relation: transposed DELTA / NEWT read
  std::vector<char> delta_list;           // per relation: DELTA read as a list by some op
  std::vector<char> rows;                 // per op: row-gather form (pull.cuh, k_join_rows_bm)
  std::vector<char> delta_n;              // per relation: DELTA rows kept non-transposed too
  // per op: writes the output's transposed twin (pull form with output
  // (inner column 1, outer column 1), or row-gather form with output
  // (outer column 1, inner column 1))
  std::vector<char> out_twin;
  // per relation: DELTA is never read as a list, so the update step is one
  // fused pass (k_bm_update_t) that writes DELTA as bitmaps only
  std::vector<char> fused;
  // per op: its fold (k_bm_fold_t) is the first thing of the iteration to
  // touch the output, a tmp relation, so it may overwrite that NEWT bitmap
  // instead of ORing into it (when the bitmap has no dirty map); per tmp
  // relation: its first op is such a fold, so its NEWT needs no clearing
  // after the operators (k_bm_clear_dirty)
  std::vector<char> fold_over, tmp_overwritten;
  // per op: a join over FULLs of static relations into an update relation
  // whose NEWT no op reads (run once per fixpoint in the dense push form,
  // k_join_bm)
  std::vector<char> static_once;
  // per op: a row-gather join whose output bitmap (a transposed twin) is
  // all zero when it starts (pull.cuh, RowsArgs::dst_zero)
  std::vector<char> twin_zero;
  // per op: a row-gather join writing an update relation's NEWT directly,
  // first of the iteration's ops to write that relation (the update step
  // leaves NEWT zero, so its rows are zero when the join starts)
  std::vector<char> g_zero;
};

Plan make_plan(gdl_engine *e, const LieHost &L) {
  Plan p;
  const size_t n = e->rels.size();
  p.full_idx.assign(n, 0);
  p.delta_idx.assign(n, 0);
  p.full_list.assign(n, 0);
  p.newt_list.assign(n, 0);
  p.acopy_src.assign(n, 0);
  p.pull.assign(L.ops.size(), 0);
  p.pull_t.assign(L.ops.size(), 0);
  p.out_t.assign(n, 0);
  p.fold_late.assign(n, 0);
  p.delta_t.assign(n, 0);
  p.newt_t.assign(n, 0);
  p.delta_list.assign(n, 0);
  p.rows.assign(L.ops.size(), 0);
  p.delta_n.assign(n, 0);
  p.out_twin.assign(L.ops.size(), 0);
  p.fused.assign(n, 0);
  p.fold_over.assign(L.ops.size(), 0);
  p.tmp_overwritten.assign(n, 0);
  p.static_once.assign(L.ops.size(), 0);
  p.twin_zero.assign(L.ops.size(), 0);
  p.g_zero.assign(L.ops.size(), 0);
  {
    std::vector<char> is_static(n, 0), is_update(n, 0), newt_read(n, 0);
    for (int r : L.statics) is_static[r] = 1;
    for (int r : L.update) is_update[r] = 1;
    for (const OpHost &op : L.ops) {
      if (op.kind == 0 && op.outer_ver == GDL_NEWT) newt_read[op.outer] = 1;
      if (op.kind == 2 || (op.kind == 1 && op.inner_ver == GDL_NEWT)) newt_read[op.inner] = 1;
    }
    for (size_t oi = 0; oi < L.ops.size(); oi++) {
      const OpHost &op = L.ops[oi];
      p.static_once[oi] = op.kind == 0 && !op.hook && op.inner_ver == GDL_FULL &&
                          op.outer_ver == GDL_FULL && is_static[op.inner] && is_static[op.outer] &&
                          is_update[op.out] && !newt_read[op.out];
    }
  }
  for (const OpHost &op : L.ops) {
    if (op.kind == 0 && op.outer_ver == GDL_DELTA) p.delta_list[op.outer] = 1;
    if (op.kind != 2 && op.inner_ver == GDL_DELTA) p.delta_list[op.inner] = 1;
    if (op.kind == 2) p.acopy_src[op.inner] = 1;
    if (op.kind == 0) {
      (op.inner_ver == GDL_DELTA ? p.delta_idx : p.full_idx)[op.inner] = 1;
      if (op.inner_ver != GDL_DELTA) p.full_list[op.inner] = 1;
      if (op.outer_ver == GDL_FULL) p.full_list[op.outer] = 1;
      if (op.outer_ver == GDL_NEWT) p.newt_list[op.outer] = 1;
    } else if (op.kind == 1 && op.inner_ver == GDL_FULL) {
      p.full_list[op.inner] = 1;
    }
  }
  return p;
}

// The update step of relation r is one fused pass (pull.cuh, k_bm_update_t):
// its DELTA is read only as bitmaps (transposed by pull-form joins, as rows
// by row-gather joins) and its FULL not as a list.
bool fused_update(const Plan &p, int r) { return p.fused[r] != 0; }

// Pull-form joins (pull.cuh), decided once the LIE's dense form is known: a
// join into bitmaps over the square domain whose output is (outer column 1,
// inner column 1), without predicate, over the DELTA of an update relation
// or the NEWT of a tmp relation, or (row-gather form only) a join of two
// static FULLs, which may carry the predicate t[0] != t[1].  A NEWT read
// only by such joins needs no list.
// An update relation whose DELTA no op reads as a list and whose FULL is not
// read as a list either has the fused update step; it keeps DELTA as the
// bitmaps its readers need (transposed, rows), at least one of them, from
// which the list is written if the loop ends with a DELTA left.
void plan_pull(const gdl_engine *e, const LieHost &L, Plan &p) {
  if (!L.dense || e->instances || L.dk < kPullMinBits) return;
  const bool pull_on = e->pull_joins == 3 || (e->pull_joins == 2 && L.dk >= kPullAutoBits);
  if (!pull_on) {
    for (int r : L.update)
      if (!p.delta_list[r] && !p.full_list[r]) p.fused[r] = p.delta_n[r] = 1;
    return;
  }
  std::vector<char> is_update(e->rels.size(), 0), is_tmp(e->rels.size(), 0);
  for (int r : L.update) is_update[r] = 1;
  for (int r : L.tmps) is_tmp[r] = 1;
  std::vector<char> is_static_r(e->rels.size(), 0);
  for (int r : L.statics) is_static_r[r] = 1;
  // the row-gather form's size rule (below), for joins that have no other
  // bitmap form
  auto rows_fit = [&](const OpHost &op) {
    if (e->row_gather == 1 || L.dk < kRowsMinBits || op.hook) return false;
    const u64 bytes = e->h[op.inner].full.n * (4ull << (L.dk - 5));
    return e->row_gather == 3 || bytes <= kRowsBudget;
  };
  std::fill(p.newt_list.begin(), p.newt_list.end(), 0);
  std::fill(p.delta_list.begin(), p.delta_list.end(), 0);
  for (size_t oi = 0; oi < L.ops.size(); oi++) {
    const OpHost &op = L.ops[oi];
    if (op.kind != 0) continue;
    // (outer column 1, inner column 1), or its transpose (inner column 1,
    // outer column 1): gathered into a transposed twin of the output
    // a join of two static FULLs (same generation's first rule,
    // test/sg.cu:147-151) takes the row-gather form, and with it the
    // predicate t[0] != t[1] (the output row's diagonal bit)
    const bool statics = op.outer_ver == GDL_FULL && op.inner_ver == GDL_FULL &&
                         is_static_r[op.outer] && is_static_r[op.inner] && rows_fit(op);
    const bool diag = op.pred.kind == GDL_PRED_NE &&
                      ((op.pred.a == 0 && op.pred.b == 1) || (op.pred.a == 1 && op.pred.b == 0));
    const bool plain = !op.generic && (op.pred.kind == 0 || (statics && diag));
    const bool fwd = plain && op.sel.s0 == 3 && op.sel.s1 == 1;
    const bool rev = plain && op.sel.s0 == 1 && op.sel.s1 == 3;
    const bool outer_ok = (op.outer_ver == GDL_DELTA && is_update[op.outer]) ||
                          (op.outer_ver == GDL_NEWT && is_tmp[op.outer]) || statics;
    if ((fwd || rev) && outer_ok) {
      p.pull[oi] = 1;
      if (rev) p.pull_t[oi] = 1;
    } else if (op.outer_ver == GDL_NEWT) {
      p.newt_list[op.outer] = 1;
    } else if (op.outer_ver == GDL_DELTA) {
      p.delta_list[op.outer] = 1;
    }
    if (op.inner_ver == GDL_DELTA) p.delta_list[op.inner] = 1;
  }
  for (size_t oi = 0; oi < L.ops.size(); oi++)
    if (L.ops[oi].kind == 1 && L.ops[oi].inner_ver == GDL_DELTA) p.delta_list[L.ops[oi].inner] = 1;
  for (int r : L.update)
    if (!p.delta_list[r] && !p.full_list[r]) p.fused[r] = 1;
  // Row-gather form (pull.cuh, k_join_rows_bm) for the pull-form joins over
  // a static inner FULL small enough that reading one outer row per in-edge
  // beats expanding candidates: |inner| rows of 2^(dk-5) words within
  // kRowsBudget bytes (any size with row_gather = 3).  A DELTA outer must be
  // a relation whose update step is the fused pass (it writes DELTA's rows);
  // a static FULL outer is set as a bitmap at LIE start.
  std::vector<char> is_static(e->rels.size(), 0);
  for (int r : L.statics) is_static[r] = 1;
  for (size_t oi = 0; oi < L.ops.size(); oi++) {
    const OpHost &op = L.ops[oi];
    if (!p.pull[oi] || e->row_gather == 1 || L.dk < kRowsMinBits) continue;
    if (op.inner_ver == GDL_DELTA || !is_static[op.inner]) continue;
    const u64 bytes = e->h[op.inner].full.n * (4ull << (L.dk - 5));
    if (e->row_gather != 3 && bytes > kRowsBudget) continue;
    if (op.outer_ver == GDL_DELTA && !fused_update(p, op.outer)) continue;
    p.rows[oi] = 1;
  }
  // Which orientations of DELTA and NEWT the joins read.  A fused update
  // step keeps DELTA as rows when nothing reads it transposed (the record
  // from which the list is written if max_iteration leaves a DELTA).
  for (size_t oi = 0; oi < L.ops.size(); oi++) {
    const OpHost &op = L.ops[oi];
    if (!p.pull[oi]) continue;
    if (op.outer_ver == GDL_NEWT && !p.rows[oi]) p.newt_t[op.outer] = 1;
    if (op.outer_ver == GDL_DELTA) (p.rows[oi] ? p.delta_n : p.delta_t)[op.outer] = 1;
    p.out_twin[oi] = p.pull_t[oi] != p.rows[oi];
    if (p.out_twin[oi]) p.out_t[op.out] = 1;
  }
  for (int r : L.update)
    if (p.fused[r] && !p.delta_t[r]) p.delta_n[r] = 1;
  // A relation written only by transposed-output joins, whose NEWT no op
  // reads and whose update step is the fused pass, keeps NEWT as the
  // transposed twin: no fold after each join, the update reads it.
  for (int r : L.update) {
    if (!p.out_t[r] || !fused_update(p, r) || p.newt_list[r] || p.newt_t[r] || p.acopy_src[r])
      continue;
    bool only_t = true;
    for (size_t oi = 0; oi < L.ops.size(); oi++)
      if (L.ops[oi].out == r && !p.out_twin[oi]) only_t = false;
    p.fold_late[r] = only_t;
  }
  // A transposed twin is zero when the op that writes it starts: folded
  // (and cleared) after each writer, or read and cleared by the update step
  // when it has one writer.
  {
    std::vector<int> twin_writers(e->rels.size(), 0);
    for (size_t oi = 0; oi < L.ops.size(); oi++)
      if (p.out_twin[oi]) twin_writers[L.ops[oi].out]++;
    for (size_t oi = 0; oi < L.ops.size(); oi++) {
      const int r = L.ops[oi].out;
      p.twin_zero[oi] = p.out_twin[oi] && p.rows[oi] && (!p.fold_late[r] || twin_writers[r] == 1);
    }
  }
  // row-gather joins that write an update relation's NEWT directly and are
  // the first of the iteration's ops to write it: the update step leaves
  // NEWT zero, so the join's rows start zero
  {
    std::vector<char> written(e->rels.size(), 0);
    for (size_t oi = 0; oi < L.ops.size(); oi++) {
      const int r = L.ops[oi].out;
      if (p.rows[oi] && !p.out_twin[oi] && is_update[r] && !written[r]) p.g_zero[oi] = 1;
      written[r] = 1;
    }
  }
  // tmp relations whose first op in the iteration writes them through a
  // fold (src/lie.cu:85-87: a tmp NEWT is empty when the operators start)
  for (int r : L.tmps) {
    for (size_t oi = 0; oi < L.ops.size(); oi++) {
      const OpHost &op = L.ops[oi];
      if (op.inner != r && op.outer != r && op.out != r) continue;
      if (op.out == r && op.inner != r && op.outer != r && p.out_twin[oi] && !p.fold_late[r]) {
        p.fold_over[oi] = 1;
        p.tmp_overwritten[r] = 1;
      }
      break;
    }
  }
}

// Transposed bitmaps of the relations pull-form joins read.
gdl_status ensure_tbitmaps(gdl_engine *e, const Plan &p, int r, u64 words) {
  RelDev &h = e->h[r];
  if (p.delta_n[r] && !h.bmDN) TRY(dalloc(e, (void **)&h.bmDN, words * 4));
  if (p.delta_t[r] && !h.bmDT) TRY(dalloc(e, (void **)&h.bmDT, words * 4));
  if (p.newt_t[r] && !h.bmGT) TRY(dalloc(e, (void **)&h.bmGT, words * 4));
  if (p.out_t[r] && !h.bmOT) TRY(dalloc(e, (void **)&h.bmOT, words * 4));
  return GDL_OK;
}

// Bitmap size, in 32-bit words, of one relation version over the square
// domain of dk-bit columns, padded to whole scan tiles (the scan kernels
// work on whole tiles; padding bits are never set).
u64 dense_words(int dk) { return round_up(1ull << (2 * dk - 5), kBmTileWords); }

// One bitmap scan (dense.cuh) of relation `rel`: tile counts and their
// prefix, then (unless the caller gates it) the write pass.
void launch_scan_count(gdl_engine *e, BmScanArgs &a, int rel, Counts *kc) {
  a.tile_prefix = e->h[rel].tile_prefix;
  a.rec = &e->d_rels[rel].scan;
  a.lb = e->lb_bm;
  a.ctl = e->d_ctl;
  const u64 tiles = a.map.words / kBmTileWords;
  a.lrec = &e->recs[4];
  if (!a.idx_b) {
    // group mode: a warp per group of 4 chunks; with a dirty map (listed
    // mode) only the dirty chunks, listed first
    const u64 chunks = a.map.words / kBmChunkWords;
    const u64 groups = chunks / kGroupChunks;
    a.grouped = 1;
    if (a.skip_clean && e->h[rel].dirty) {
      a.chunk_list = reinterpret_cast<u32 *>(a.tile_prefix + groups);
      PLAUNCH(kc, kPBitmap,
              k_bm_dirty_chunks<<<grid_for(e, chunks / kDirtyUnit + 1, 1, 4), kBmBlock, 0,
                                  e->s>>>(a));
    }
    PLAUNCH(kc, kPBitmap,
            k_bm_groupcount<<<grid_for(e, groups * 32, kBmBlock, 8), kBmBlock, 0, e->s>>>(a));
    PLAUNCH(kc, kPBitmap,
            k_bm_scan<<<grid_for(e, groups / kScanChunk + 1, 1, 4), kBmBlock, 0, e->s>>>(a));
    return;
  }
  PLAUNCH(kc, kPBitmap, k_bm_tilecount<<<grid_for(e, tiles, 1, 8), kBmBlock, 0, e->s>>>(a));
  PLAUNCH(kc, kPBitmap,
          k_bm_scan<<<grid_for(e, tiles / kScanChunk + 1, 1, 4), kBmBlock, 0, e->s>>>(a));
}
void launch_scan_write(gdl_engine *e, BmScanArgs a, Counts *kc) {
  const u64 tiles = a.map.words / kBmTileWords;
  a.lrec = &e->recs[5];
  if (a.grouped) {
    const u64 groups = a.map.words / kBmChunkWords / kGroupChunks;
    PLAUNCH(kc, kPBitmap,
            k_bm_groupwrite<<<grid_for(e, groups * 32, kBmBlock, 8), kBmBlock, 0, e->s>>>(a));
    return;
  }
  PLAUNCH(kc, kPBitmap, k_bm_write<<<grid_for(e, tiles, 1, 8), kBmBlock, 0, e->s>>>(a));
}
void launch_scan(gdl_engine *e, BmScanArgs a, int rel, Counts *kc) {
  launch_scan_count(e, a, rel, kc);
  launch_scan_write(e, a, kc);
}

BmScanArgs scan_none(const DenseMap &map) {
  BmScanArgs a;
  memset(&a, 0, sizeof a);
  a.map = map;
  a.ex_a = a.ex_b = kBmNone;
  a.need_a = a.need_b = -1;
  return a;
}

// (zeroed first: argument bytes, padding included, are compared by the
// executable cache)
TransposeArgs transpose_args(const u32 *g, const u32 *f, u32 *dst, int dk, DArr *count_to,
                             u64 *count_acc, LaunchRec *lrec, Ctl *ctl) {
  TransposeArgs t;
  memset(&t, 0, sizeof t);
  t.g = g;
  t.f = f;
  t.dst = dst;
  t.dk = dk;
  t.count_to = count_to;
  t.count_acc = count_acc;
  t.lrec = lrec;
  t.ctl = ctl;
  return t;
}

void enqueue_update_step(gdl_engine *e, LieHost &L, const Plan &plan, Counts *kc,
                         bool begin_next);

// One iteration.  in_graph: the body of the graph's while-node, which the
// host opens with a k_begin before each launch and whose k_commit opens
// the next iteration; otherwise the iteration opens itself.
void launch_rows(gdl_engine *e, const RowsArgs &ra, Counts *kc) {
  // one resident wave (warps take the units round robin): 4 blocks an SM
  // at 2^12 ids, 2 at 2^13..2^15 (the row accumulators hold 2^(dk-5)
  // words a warp), 1 from 2^16
  const int g = (int)e->sms * (ra.dk >= 16 ? 1 : ra.dk >= 13 ? 2 : 4);
  switch (ra.dk) {
    case 12: PLAUNCH(kc, kPJoinMat, k_join_rows_bm<1><<<g, 256, 0, e->s>>>(ra)); break;
    case 13: PLAUNCH(kc, kPJoinMat, k_join_rows_bm<2><<<g, 256, 0, e->s>>>(ra)); break;
    case 14: PLAUNCH(kc, kPJoinMat, k_join_rows_bm<4><<<g, 256, 0, e->s>>>(ra)); break;
    case 15: PLAUNCH(kc, kPJoinMat, k_join_rows_bm<8><<<g, 256, 0, e->s>>>(ra)); break;
    default: PLAUNCH(kc, kPJoinMat, k_join_rows_bm<16><<<g, 256, 0, e->s>>>(ra)); break;
  }
}

// The sorted key list of a square-domain bitmap of `words` words (rows of
// 2^rs words) into `out` (k_bm_list_*, dense.cuh): tile counts, offsets and
// the list's size, keys.  out->n must hold the expected count.
gdl_status launch_list(gdl_engine *e, const u32 *bm, u64 words, int rs, DArr *out,
                       int check_n) {
  const u64 tiles = words / kBmTileWords;
  TRY(ensure_lb(e, e->lb_list, e->lb_list_tiles, tiles + 2));
  k_bm_list_count<<<grid_for(e, tiles, 1, 8), kBmBlock, 0, e->s>>>(bm, tiles, e->lb_list.flag,
                                                                   e->d_ctl);
  e->aux_launches += 3;  // (count, offsets, write)
  k_bm_list_offsets<<<1, kListScanBlock, 0, e->s>>>(e->lb_list.flag, tiles, e->lb_list.agg, out,
                                                    check_n, e->d_ctl);
  k_bm_list_write<<<grid_for(e, tiles, 1, 8), kBmBlock, 0, e->s>>>(
      bm, tiles, rs, e->lb_list.flag, e->lb_list.agg, out, &e->recs[8], e->d_ctl);
  CK(e, cudaGetLastError());
  return GDL_OK;
}

// dst |= transpose(src) (or := with over), src cleared: the TMA pass
// (tma.cuh) when both bitmaps have tensor maps, else the LDG/STG pass.
void launch_fold(gdl_engine *e, u32 *src, u32 *dst, u8 *dirty, int dk, int over, Counts *kc,
                 cudaStream_t s) {
  const u64 side = 1ull << (dk - kPullMinBits);
  const CUtensorMap *ms = bm_tmap(e, src, dk), *md = bm_tmap(e, dst, dk);
  if (ms && md) {
    FoldMaps m;
    m.src = *ms;
    m.dst = *md;
    const int ns = fold_tma_stages(over);
    PLAUNCH(kc, kPBitmap,
            k_bm_fold_tma<<<grid_for(e, side * side, 1, over ? 3 : 2), kTrBlock,
                            fold_tma_smem(ns, over), s>>>(m, dirty, dk, over, ns, e->d_ctl));
    return;
  }
  PLAUNCH(kc, kPBitmap, k_bm_fold_t<<<grid_for(e, side * side, 1, 8), kTrBlock, 0, s>>>(
                            src, dst, dirty, dk, over, e->d_ctl));
}

// The fused update step of relation r (k_bm_update_t): NEWT from its
// transposed twin gt or its rows, DELTA written as rows dn and/or
// transposed dt; the TMA pass when every bitmap has a tensor map.
void launch_update_t(gdl_engine *e, const BmScanArgs &a, int r, u32 *gt, u32 *dn, u32 *dt,
                     int dk, Counts *kc, cudaStream_t s) {
  const RelDev &h = e->h[r];
  const u64 side = 1ull << (dk - kPullMinBits);
  const CUtensorMap *mn = bm_tmap(e, gt ? gt : h.bmG, dk), *mf = bm_tmap(e, h.bmF, dk);
  const CUtensorMap *mdn = dn ? bm_tmap(e, dn, dk) : mf, *mdt = dt ? bm_tmap(e, dt, dk) : mf;
  if (mn && mf && mdn && mdt) {
    UpdMaps m;
    m.nsrc = *mn;
    m.f = *mf;
    m.dn = *mdn;
    m.dt = *mdt;
    const int ns = upd_tma_stages(dt != nullptr);
    PLAUNCH(kc, kPBitmap,
            k_bm_update_tma<<<grid_for(e, side * side, 1, 2), kTrBlock,
                              upd_tma_smem(ns, dt != nullptr), s>>>(
                a, m, dk, gt != nullptr, dn != nullptr, dt != nullptr, ns));
    return;
  }
  PLAUNCH(kc, kPBitmap,
          k_bm_update_t<<<grid_for(e, side * side, 1, 8), kTrBlock, 0, s>>>(a, dt, dk, gt, dn));
}

// In-edges of relation r's FULL list over 2^dk ids (k_inv_*, pull.cuh).
gdl_status build_inverse(gdl_engine *e, int r, int dk) {
  RelHost &rh = e->rels[r];
  const u64 n = e->h[r].full.n;
  const u32 ids = 1u << dk;
  if (rh.inv_ready && rh.inv_dk == dk && rh.inv_n == n) return GDL_OK;
  if (rh.inv_dk != dk || rh.inv_cap < std::max<u64>(n, 1)) {
    for (u32 **q : {&rh.inv_off, &rh.inv_cur, &rh.inv_keys, &rh.inv_ys}) {
      dfree(e, *q);
      *q = nullptr;
    }
    rh.inv_cap = std::max<u64>(n, 1);
    rh.inv_dk = dk;
    TRY(dalloc(e, (void **)&rh.inv_off, (ids + 1) * sizeof(u32)));
    TRY(dalloc(e, (void **)&rh.inv_cur, ids * sizeof(u32)));
    TRY(dalloc(e, (void **)&rh.inv_keys, rh.inv_cap * sizeof(u32)));
    TRY(dalloc(e, (void **)&rh.inv_ys, rh.inv_cap * sizeof(u32)));
  }
  CK(e, cudaMemsetAsync(rh.inv_cur, 0, ids * sizeof(u32), e->s));
  const DArr *list = &e->d_rels[r].full;
  k_inv_count<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(list, rh.inv_cur, dk, e->d_ctl);
  e->aux_launches += 3;  // (count, offsets, fill)
  // edge offsets and fill cursors, in one block
  k_inv_offsets<<<1, kInvBlock, 0, e->s>>>(rh.inv_cur, rh.inv_off, rh.inv_cur, dk);
  k_inv_fill<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(list, rh.inv_cur, rh.inv_keys, rh.inv_ys,
                                                       dk);
  rh.inv_ready = true;
  rh.inv_n = n;
  CK(e, cudaGetLastError());
  return GDL_OK;
}

static_assert(sizeof(DArr) == sizeof(gdl_dev_rows), "gdl_dev_rows mirrors DArr");
static_assert(sizeof(JoinRec) == sizeof(gdl_hook_state), "gdl_hook_state mirrors JoinRec");
static_assert(offsetof(JoinRec, written) == offsetof(gdl_hook_state, written), "JoinRec layout");
static_assert(offsetof(JoinRec, skip) == offsetof(gdl_hook_state, skip), "JoinRec layout");

// What a hooked operator's kernel reads: device addresses that stay valid
// for the launch being enqueued (the descriptors, not the arrays, whose
// pointers change when the loop swaps versions).
gdl_hook_work hook_work(gdl_engine *e, const OpHost &op, JoinRec *rec, const DArr *rows,
                        DArr *out) {
  gdl_hook_work w;
  memset(&w, 0, sizeof w);
  w.kind = op.kind;
  w.in_arity = e->rels[op.inner].arity;
  w.outer_arity = op.kind == 0 ? e->rels[op.outer].arity : 0;
  w.out_arity = e->rels[op.out].arity;
  w.k2 = e->k2;
  w.sms = e->sms;
  w.state = reinterpret_cast<gdl_hook_state *>(rec);
  w.rows = reinterpret_cast<const gdl_dev_rows *>(rows);
  w.out = reinterpret_cast<gdl_dev_rows *>(out);
  w.error = &e->d_ctl->oob;
  return w;
}

void enqueue_iteration(gdl_engine *e, LieHost &L, const Plan &plan, Counts *kc, bool in_graph) {
  cudaStream_t s = e->s;
  RelDev *R = e->d_rels;
  const bool dense = L.dense;
  const DenseMap &map = L.map;
  const u64 words = dense ? map.words : 0;
  if (!in_graph) PLAUNCH(kc, kPControl, k_begin<<<1, 32, 0, s>>>(R, L.d_lie, e->d_ctl));
  for (size_t oi = 0; oi < L.ops.size(); oi++) {
    const OpHost &op = L.ops[oi];
    if (op.kind == 0) {
      JoinArgs a;
      memset(&a, 0, sizeof a);
      const RelDev &oh = e->h[op.outer];
      if (op.outer_ver == GDL_DELTA) {
        a.outer = &R[op.outer].delta;
        a.outer_vis = &R[op.outer].w_delta_vis;
      } else if (op.outer_ver == GDL_FULL) {
        a.outer = &R[op.outer].full;
        a.outer_vis = &R[op.outer].w_full_vis;
      } else {
        a.outer = &R[op.outer].newt;
        a.outer_vis = nullptr;
        if (dense && oh.bmG && plan.pull[oi]) {
          // pull form: NEWT's bitmap transposed, its size counted (no list)
          a.outer_bm = oh.bmG;
          a.outer_bm_words = words;
        } else if (dense && oh.bmG) {
          // NEWT as a join outer: the sorted list of its bitmap (dirty
          // chunks only).
          BmScanArgs c = scan_none(map);
          c.g = oh.bmG;
          c.dirty = oh.dirty;
          c.skip_clean = oh.dirty != nullptr;
          c.ex_a = kBmUnion;
          c.list_a = &R[op.outer].newt;
          c.need_a = need_index(op.outer, kNeedNewt);
          launch_scan(e, c, op.outer, kc);
          a.outer_bm = oh.bmG;
          a.outer_bm_words = words;
        }
      }
      if (op.inner_ver == GDL_DELTA) {
        a.inner = &R[op.inner].delta;
        a.inner_vis = &R[op.inner].w_delta_vis;
        a.inner_idx = &R[op.inner].delta_idx;
      } else {  // FULL (a NEWT inner reads FULL, src/join.cu:14-19)
        a.inner = &R[op.inner].full;
        a.inner_vis = &R[op.inner].w_full_vis;
        a.inner_idx = &R[op.inner].full_idx;
      }
      a.out_newt = &R[op.out].newt;
      a.sel = op.sel;
      a.generic = op.generic;
      a.gen = op.gen;
      a.gen.k2 = e->k2;
      a.pred = op.pred;
      a.op = L.d_joinrec + oi;
      a.rec = &e->recs[0];
      a.lb_cnt = e->lb_cnt;
      a.lb_nz = e->lb_nz;
      a.crow_off = e->crow_off;
      a.crow_start = e->crow_start;
      a.crow_len = e->crow_len;
      a.crow_key = e->crow_key;
      a.crow_cap = e->crow_cap;
      a.ctl = e->d_ctl;
      a.out_rel = op.out;
      a.dense = dense;
      // Row-OR: inner FULL kept as a bitmap, output (outer column, inner
      // column 1), no predicate (dense.cuh, k_join_bm).
      a.inner_rd = &R[op.inner];
      a.row_or = dense && e->row_or_joins && op.inner_ver != GDL_DELTA &&
                 e->h[op.inner].dense && e->h[op.inner].bmF && op.pred.kind == 0 &&
                 (op.sel.s0 == 2 || op.sel.s0 == 3) && op.sel.s1 == 1;
      if (op.hook) {
        // The count pass enumerates the candidates; the caller's kernel runs
        // the hooks over them and appends what it keeps.
        a.generic = 0;
        a.pred = Pred{0, 0, 0};
        const u64 ocap = std::max({oh.delta.cap, oh.delta_next.cap, oh.full.cap,
                                   oh.full_next.cap, oh.newt.cap});
        PLAUNCH(kc, kPJoinCount,
                k_join_count<<<grid_for(e, ocap, kJoinTile, e->count_ctas_per_sm), kJoinBlock,
                               0, s>>>(a));
        PLAUNCH(kc, kPControl, k_hook_join_begin<<<1, 32, 0, s>>>(a));
        gdl_hook_work w = hook_work(e, op, L.d_joinrec + oi, a.inner, &R[op.out].newt);
        w.rec_offset = reinterpret_cast<const uint64_t *>(e->crow_off);
        w.rec_start = e->crow_start;
        w.rec_key = reinterpret_cast<const uint64_t *>(e->crow_key);
        op.hook(op.hook_ctx, &w, (void *)s);
        kc->add(kPJoinMat);
        PLAUNCH(kc, kPControl, k_hook_join_end<<<1, 32, 0, s>>>(a));
        continue;
      }
      if (plan.pull[oi] && plan.rows[oi]) {
        // gathered along the inner's in-edges from the outer's rows
        RowsArgs ra;
        memset(&ra, 0, sizeof ra);
        ra.j = a;
        ra.j.rec = &e->recs[6];
        ra.O = op.outer_ver == GDL_DELTA ? oh.bmDN : op.outer_ver == GDL_FULL ? oh.bmF : oh.bmG;
        ra.outer_clear = op.outer_ver == GDL_NEWT ? oh.bmG : nullptr;
        ra.clear_diag = op.pred.kind == GDL_PRED_NE;
        if (plan.static_once[oi]) {
          ra.j.once = &L.d_lie->jonce[oi];
          ra.j.once_pending = &L.d_lie->jonce_pending[oi];
          ra.j.produced = &L.d_lie->produced[oi];
          ra.j.phantom = &R[op.out].newt_phantom;
        }
        const RelHost &ih = e->rels[op.inner];
        ra.inv_keys = ih.inv_keys;
        ra.inv_ys = ih.inv_ys;
        ra.inv_off = ih.inv_off;
        ra.unit = (u32)e->rows_piece;
        const RelDev &out = e->h[op.out];
        ra.dst = plan.out_twin[oi] ? out.bmOT : out.bmG;
        ra.dirty = plan.out_twin[oi] ? nullptr : out.dirty;
        ra.dst_zero = plan.twin_zero[oi] || plan.g_zero[oi];
        ra.dk = L.dk;
        launch_rows(e, ra, kc);
        if (plan.out_twin[oi] && !plan.fold_late[op.out])
          launch_fold(e, out.bmOT, out.bmG, out.dirty, L.dk, plan.fold_over[oi] && !out.dirty, kc,
                      s);
        continue;
      }
      if (plan.pull[oi]) {
        const u32 *OT = oh.bmDT;
        const u64 side = 1ull << (L.dk - kPullMinBits);
        if (op.outer_ver == GDL_NEWT) {
          TransposeArgs t = transpose_args(oh.bmG, nullptr, oh.bmGT, L.dk, &R[op.outer].newt,
                                           e->d_pull_count, &e->recs[7], e->d_ctl);
          PLAUNCH(kc, kPBitmap,
                  k_bm_transpose<<<grid_for(e, side * side, 1, 8), kTrBlock, 0, s>>>(t));
          OT = oh.bmGT;
        }
        a.rec = &e->recs[6];
        // row-OR: the gathered row is the inner's column 1 in both
        // orientations
        a.row_or = e->row_or_joins && op.inner_ver != GDL_DELTA && e->h[op.inner].dense &&
                   e->h[op.inner].bmF;
        const RelDev &out = e->h[op.out];
        PLAUNCH(kc, kPJoinMat,
                k_join_pull_bm<<<(int)e->sms * 8, kPullBlock, pull_acc_words(L.dk) * 4, s>>>(
                    a, plan.pull_t[oi] ? out.bmOT : out.bmG,
                    plan.pull_t[oi] ? nullptr : out.dirty, OT, L.dk));
        if (plan.pull_t[oi] && !plan.fold_late[op.out])
          launch_fold(e, out.bmOT, out.bmG, out.dirty, L.dk, plan.fold_over[oi] && !out.dirty, kc,
                      s);
        continue;
      }
      u64 outer_cap = std::max({oh.delta.cap, oh.delta_next.cap, oh.full.cap, oh.full_next.cap,
                                oh.newt.cap});
      JoinArgs b;
      memcpy(&b, &a, sizeof b);
      b.rec = &e->recs[1];
      if (dense && e->dense_join_passes == 1) {
        const int jb = e->join_block;
        const int jg = grid_for(e, outer_cap, jb, kFuseCtasPerSm * kFuseBlock / jb);
        const int hg = (int)e->sms * 4 * kFuseBlock / jb;
        if (plan.static_once[oi]) {
          a.once = &L.d_lie->jonce[oi];
          a.once_pending = &L.d_lie->jonce_pending[oi];
          a.produced = &L.d_lie->produced[oi];
          a.phantom = &R[op.out].newt_phantom;
          b.produced = a.produced;
        }
#define GDL_PUSH(AG, B)                                                                      \
  do {                                                                                       \
    PLAUNCH(kc, kPJoinMat, k_join_bm<AG, B><<<jg, B, 0, s>>>(a, &R[op.out], map));           \
    PLAUNCH(kc, kPJoinMat, k_join_heavy_bm<AG, B><<<hg, B, 0, s>>>(b, &R[op.out], map));     \
  } while (0)
        const bool ag = e->join_aggregate == 2;
        if (jb == 128) {
          if (ag) GDL_PUSH(true, 128); else GDL_PUSH(false, 128);
        } else if (jb == 512) {
          if (ag) GDL_PUSH(true, 512); else GDL_PUSH(false, 512);
        } else {
          if (ag) GDL_PUSH(true, 256); else GDL_PUSH(false, 256);
        }
#undef GDL_PUSH
        continue;
      }
      PLAUNCH(kc, kPJoinCount,
              k_join_count<<<grid_for(e, outer_cap, kJoinTile, e->count_ctas_per_sm), kJoinBlock,
                             0, s>>>(a));
      const u64 out_cap = e->h[op.out].newt.cap;
      if (dense)
        PLAUNCH(kc, kPJoinMat,
                k_join_mat_bm<<<(int)e->sms * e->join_ctas_per_sm, kMatBlock, 0, s>>>(
                    b, &R[op.out], map));
      else if (op.pred.kind)
        PLAUNCH(kc, kPJoinMat,
                k_join_mat_pred<<<grid_for(e, outer_cap, 8 * 16, 8), kMatBlock, 0, s>>>(b));
      else
        PLAUNCH(kc, kPJoinMat,
                k_join_mat<<<grid_for(e, out_cap, kMatTile, e->join_ctas_per_sm), kMatBlock, 0,
                             s>>>(b));
    } else {
      CopyArgs c;
      memset(&c, 0, sizeof c);
      const RelDev &sh = e->h[op.inner];
      if (op.kind == 2) {
        c.src = &R[op.inner].newt;
        c.src_vis = nullptr;
      } else if (op.inner_ver == GDL_DELTA) {
        c.src = &R[op.inner].delta;
        c.src_vis = &R[op.inner].w_delta_vis;
      } else {
        c.src = &R[op.inner].full;
        c.src_vis = &R[op.inner].w_full_vis;
      }
      c.dest = &R[op.out].newt;
      c.sel = op.sel;
      c.generic = op.generic;
      c.gen = op.gen;
      c.gen.k2 = e->k2;
      bool once = op.kind == 1 && op.inner_ver == GDL_FULL;
      c.once = once ? &L.d_lie->once[oi] : nullptr;
      c.once_pending = once ? &L.d_lie->once_pending[oi] : nullptr;
      c.rec = &e->recs[3];
      c.ctl = e->d_ctl;
      c.dest_rel = op.out;
      c.replace = op.kind == 2;
      u64 cap = std::max({sh.full.cap, sh.delta.cap, sh.newt.cap, sh.delta_next.cap});
      if (op.hook) {
        JoinRec *rec = L.d_joinrec + oi;
        PLAUNCH(kc, kPControl, k_hook_copy_begin<<<1, 32, 0, s>>>(c, rec));
        gdl_hook_work w = hook_work(e, op, rec, c.src, &R[op.out].newt);
        op.hook(op.hook_ctx, &w, (void *)s);
        kc->add(kPCopy);
        PLAUNCH(kc, kPControl, k_hook_copy_end<<<1, 32, 0, s>>>(c, rec));
        continue;
      }
      if (dense && op.kind == 2) {
        // RelationalACopy: dest NEWT := sel(src NEWT), bitmap to bitmap.
        const u64 tiles = words / kBmTileWords;
        PLAUNCH(kc, kPBitmap, k_bm_clear_dirty<<<grid_for(e, tiles, 1, 8), 256, 0, s>>>(
                                  &R[op.out], map, e->d_ctl));
        if (sh.bmG)  // a source without a NEWT bitmap (static) has an empty NEWT
          PLAUNCH(kc, kPCopy, k_acopy_bm<<<grid_for(e, tiles, 1, 8), 256, 0, s>>>(
                                  &R[op.inner], op.sel, &R[op.out], map, e->d_ctl));
      } else if (dense) {
        const u64 tiles = words / kBmTileWords;
        PLAUNCH(kc, kPBitmap, k_copy_empty_clear<<<grid_for(e, tiles, 1, 8), 256, 0, s>>>(
                                  c, &R[op.out], map));
        PLAUNCH(kc, kPCopy, k_copy_bm<<<grid_for(e, cap, 256, 8), 256, 0, s>>>(
                                c, &R[op.out], map));
      } else {
        PLAUNCH(kc, kPCopy,
                k_copy<<<grid_for(e, cap / 2 + 1, kMatBlock, 8), kMatBlock, 0, s>>>(c));
      }
    }
  }
  enqueue_update_step(e, L, plan, kc, in_graph);
}

// The per-relation update step (DELTA, FULL', indexes) and the commit of
// one iteration.  After a capacity overflow in a dense scan it is enqueued
// again on its own: the NEWT bitmaps still hold the iteration's joins.
void enqueue_update_step(gdl_engine *e, LieHost &L, const Plan &plan, Counts *kc,
                         bool begin_next) {
  cudaStream_t s = e->s;
  RelDev *R = e->d_rels;
  const bool dense = L.dense;
  if (dense) {
    // DELTA = NEWT \ FULL (sorted), FULL |= NEWT in place, NEWT cleared; a
    // relation whose FULL list is read during the loop also gets FULL' and
    // its index.  All relations are counted and checked (gate) before any
    // bitmap is written.
    std::vector<BmScanArgs> scans, fused;
    for (int r : L.update) {
      BmScanArgs a = scan_none(L.map);
      a.rd = &R[r];
      a.inplace = 1;
      a.skip_clean = !plan.full_list[r] && e->h[r].dirty != nullptr;
      a.gated = 1;
      a.inst_delta = L.d_inst_delta;
      a.ex_a = kBmDelta;
      if (fused_update(plan, r) || (plan.delta_t[r] && !plan.delta_list[r])) {
        // no op reads DELTA as a list (pull-form and row-gather joins read
        // its bitmaps): only its size; the list is written from a bitmap
        // if the loop ends with a DELTA left.  (k_bm_update_t stores
        // through count_a: a fused relation always takes this branch.)
        a.count_a = &R[r].delta_next.n;
      } else {
        a.list_a = &R[r].delta_next;
        a.need_a = need_index(r, kNeedDelta);
      }
      if (plan.full_list[r]) {
        a.ex_b = kBmUnion;
        a.list_b = &R[r].full_next;
        a.need_b = need_index(r, kNeedFull);
        if (plan.full_idx[r]) a.idx_b = &R[r].full_idx_next;
      }
      a.pop_g_out = &R[r].c_newt_n;
      a.gate_rels = R;
      a.gate_update = &L.d_lie->update[0];
      a.gate_n = (int)L.update.size();
      if (fused_update(plan, r)) {
        // DELTA read only as bitmaps, FULL not as a list: one fused pass
        // (pull.cuh, k_bm_update_t) after every count pass
        a.rec = &R[r].scan;
        a.lrec = &e->recs[5];
        a.ctl = e->d_ctl;
        fused.push_back(a);
        continue;
      }
      launch_scan_count(e, a, r, kc);
      scans.push_back(a);
    }
    // the next DELTA transposed, for the pull-form joins that read it
    // (before the write passes change FULL and clear NEWT)
    for (const BmScanArgs &a : scans) {
      const int r = (int)(a.rd - R);
      if (plan.delta_t[r]) {
        const u64 side = 1ull << (L.dk - kPullMinBits);
        TransposeArgs t = transpose_args(e->h[r].bmG, e->h[r].bmF, e->h[r].bmDT, L.dk, nullptr,
                                         nullptr, &e->recs[7], e->d_ctl);
        PLAUNCH(kc, kPBitmap, k_bm_transpose<<<grid_for(e, side * side, 1, 8), kTrBlock, 0, s>>>(t));
      }
    }
    for (const BmScanArgs &a : fused) {
      const int r = (int)(a.rd - R);
      launch_update_t(e, a, r, plan.fold_late[r] ? e->h[r].bmOT : nullptr,
                      plan.delta_n[r] ? e->h[r].bmDN : nullptr,
                      plan.delta_t[r] ? e->h[r].bmDT : nullptr, L.dk, kc, s);
    }
    for (const BmScanArgs &a : scans) launch_scan_write(e, a, kc);
    // tmp relations: NEWT is cleared after the operators (src/lie.cu:85-87),
    // unless the next iteration's first op overwrites it whole
    const u64 tiles = L.map.words / kBmTileWords;
    for (int r : L.tmps)
      if (!(plan.tmp_overwritten[r] && !e->h[r].dirty))
        PLAUNCH(kc, kPBitmap, k_bm_clear_dirty<<<grid_for(e, tiles, 1, 8), 256, 0, s>>>(
                                  &R[r], L.map, e->d_ctl));
  }
  for (int r : L.update) {
    const RelDev &rh = e->h[r];
    if (!dense) {
      launch_sort(e, &R[r].newt, rh.newt.ptr, rh.newt.cap, kc);
      MergeArgs m;
      memset(&m, 0, sizeof m);
      m.newt = &R[r].newt;
      m.a = sorted_location(e, rh.newt.ptr);
      m.full = &R[r].full;
      m.full_next = &R[r].full_next;
      m.delta_next = &R[r].delta_next;
      m.c_newt_n = &R[r].c_newt_n;
      m.rec = &e->recs[2];
      m.lb = e->lb_merge;
      m.parts = e->merge_parts;
      m.parts_cap = e->lb_merge_tiles + 1;
      m.ctl = e->d_ctl;
      m.rel = r;
      u64 mcap = std::max(rh.full.cap, rh.full_next.cap) + rh.newt.cap;
      if (const u64 lm = dep_low_mask(e, e->rels[r]))
        PLAUNCH(kc, kPMerge, k_dep_mask<<<grid_for(e, rh.newt.cap, 256, 8), 256, 0, s>>>(
                                 const_cast<u64 *>(m.a), &R[r].newt, &R[r].full, lm, e->d_ctl));
      PLAUNCH(kc, kPMerge,
              k_merge_partition<<<grid_for(e, mcap / kMergeTile + 2, 256, 8), 256, 0, s>>>(m));
      PLAUNCH(kc, kPMerge,
              k_merge_diff<<<grid_for(e, mcap, kMergeTile, 4), kMergeBlock, kMergeSmemBytes, s>>>(m));
      if (plan.full_idx[r]) {
        u64 c = std::max(rh.full.cap, rh.full_next.cap);
        PLAUNCH(kc, kPIndex,
                k_index_build<<<grid_for(e, c, kIndexBlock, 8), kIndexBlock, 0, s>>>(
                    &R[r].full_next, &R[r].full_idx_next, &R[r].delta_next, e->d_ctl));
      }
    }
    if (plan.delta_idx[r]) {
      u64 c = std::max(rh.delta.cap, rh.delta_next.cap);
      PLAUNCH(kc, kPIndex,
              k_index_build<<<grid_for(e, c, kIndexBlock, 8), kIndexBlock, 0, s>>>(
                  &R[r].delta_next, &R[r].delta_idx_next, nullptr, e->d_ctl));
    }
  }
  if (L.d_inst_delta)
    PLAUNCH(kc, kPControl, k_inst_track<<<grid_for(e, L.n_inst, 256, 1), 256, 0, s>>>(
                               L.d_inst_delta, L.d_inst_last, L.n_inst, e->d_ctl));
  PLAUNCH(kc, kPControl, k_commit<<<1, 32, 0, s>>>(R, L.d_lie, e->d_ctl, begin_next ? 1 : 0));
}

// ---------------------------------------------------------------------------
// Executable cache.  Instantiating the loop's graph takes ~0.15 ms of host
// time and destroying it ~0.17 ms, during which the driver also holds off
// the caller's next CUDA calls.  A program run again after
// gdl_engine_clear (a service answering the same query shape, a benchmark)
// captures the same iteration: the same kernels with the same launch shapes
// and, because dalloc replays the previous program's blocks, the same
// argument bytes.  Such an iteration takes the cached executable, compared
// node by node (kind; kernel, grid, block, shared memory and every argument
// byte, sized by cudaFuncGetParamInfo; memset and memcpy parameters;
// edges), so a reuse is exact by construction.
// ---------------------------------------------------------------------------
constexpr size_t kGraphCacheMax = 32;

const std::vector<size_t> &param_sizes(gdl_engine *e, const void *func) {
  auto it = e->param_sizes.find(func);
  if (it != e->param_sizes.end()) return it->second;
  std::vector<size_t> v;
  for (size_t i = 0; i < 256; i++) {
    size_t off = 0, sz = 0;
    if (cudaFuncGetParamInfo(func, i, &off, &sz) != cudaSuccess) {
      cudaGetLastError();
      break;
    }
    v.push_back(sz);
  }
  return e->param_sizes.emplace(func, std::move(v)).first->second;
}

bool nodes_equal(gdl_engine *e, cudaGraphNode_t a, cudaGraphNode_t b) {
  cudaGraphNodeType ta, tb;
  if (cudaGraphNodeGetType(a, &ta) != cudaSuccess || cudaGraphNodeGetType(b, &tb) != cudaSuccess ||
      ta != tb)
    return false;
  if (ta == cudaGraphNodeTypeEmpty) return true;
  if (ta == cudaGraphNodeTypeKernel) {
    cudaKernelNodeParams pa, pb;
    if (cudaGraphKernelNodeGetParams(a, &pa) != cudaSuccess ||
        cudaGraphKernelNodeGetParams(b, &pb) != cudaSuccess)
      return false;
    if (pa.func != pb.func || pa.sharedMemBytes != pb.sharedMemBytes || pa.extra || pb.extra ||
        pa.gridDim.x != pb.gridDim.x || pa.gridDim.y != pb.gridDim.y ||
        pa.gridDim.z != pb.gridDim.z || pa.blockDim.x != pb.blockDim.x ||
        pa.blockDim.y != pb.blockDim.y || pa.blockDim.z != pb.blockDim.z)
      return false;
    // every engine kernel takes arguments: none known means none compared
    const std::vector<size_t> &sz = param_sizes(e, pa.func);
    if (sz.empty() || !pa.kernelParams || !pb.kernelParams) return false;
    for (size_t i = 0; i < sz.size(); i++)
      if (memcmp(pa.kernelParams[i], pb.kernelParams[i], sz[i]) != 0) return false;
    return true;
  }
  if (ta == cudaGraphNodeTypeMemset) {
    cudaMemsetParams ma, mb;
    if (cudaGraphMemsetNodeGetParams(a, &ma) != cudaSuccess ||
        cudaGraphMemsetNodeGetParams(b, &mb) != cudaSuccess)
      return false;
    return ma.dst == mb.dst && ma.pitch == mb.pitch && ma.value == mb.value &&
           ma.elementSize == mb.elementSize && ma.width == mb.width && ma.height == mb.height;
  }
  if (ta == cudaGraphNodeTypeMemcpy) {
    cudaMemcpy3DParms ca, cb;
    if (cudaGraphMemcpyNodeGetParams(a, &ca) != cudaSuccess ||
        cudaGraphMemcpyNodeGetParams(b, &cb) != cudaSuccess)
      return false;
    auto same_pos = [](const cudaPos &x, const cudaPos &y) {
      return x.x == y.x && x.y == y.y && x.z == y.z;
    };
    auto same_ptr = [](const cudaPitchedPtr &x, const cudaPitchedPtr &y) {
      return x.ptr == y.ptr && x.pitch == y.pitch && x.xsize == y.xsize && x.ysize == y.ysize;
    };
    return ca.srcArray == cb.srcArray && ca.dstArray == cb.dstArray && ca.kind == cb.kind &&
           same_pos(ca.srcPos, cb.srcPos) && same_pos(ca.dstPos, cb.dstPos) &&
           same_ptr(ca.srcPtr, cb.srcPtr) && same_ptr(ca.dstPtr, cb.dstPtr) &&
           ca.extent.width == cb.extent.width && ca.extent.height == cb.extent.height &&
           ca.extent.depth == cb.extent.depth;
  }
  return false;  // (the iteration records no other kind of node)
}

// A 64-bit signature of a graph's nodes (the fields nodes_equal compares)
// and its edge count: entries whose signature differs are not compared.
u64 graph_signature(gdl_engine *e, cudaGraph_t g, size_t *n_nodes) {
  size_t n = 0;
  *n_nodes = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
  std::vector<cudaGraphNode_t> x(n);
  if (n && cudaGraphGetNodes(g, x.data(), &n) != cudaSuccess) return 0;
  u64 h = mix64(n);
  auto put = [&h](u64 v) { h = mix64(h ^ v); };
  auto put_bytes = [&put](const void *p, size_t len) {
    const unsigned char *b = static_cast<const unsigned char *>(p);
    for (size_t i = 0; i < len; i += 8) {
      u64 w = 0;
      memcpy(&w, b + i, std::min<size_t>(8, len - i));
      put(w);
    }
  };
  for (cudaGraphNode_t node : x) {
    cudaGraphNodeType t;
    if (cudaGraphNodeGetType(node, &t) != cudaSuccess) return 0;
    put((u64)t);
    if (t == cudaGraphNodeTypeKernel) {
      cudaKernelNodeParams p;
      if (cudaGraphKernelNodeGetParams(node, &p) != cudaSuccess) return 0;
      put((u64)(uintptr_t)p.func);
      put(((u64)p.gridDim.x << 32) ^ ((u64)p.gridDim.y << 16) ^ p.gridDim.z);
      put(((u64)p.blockDim.x << 32) ^ ((u64)p.blockDim.y << 16) ^ p.blockDim.z);
      put(p.sharedMemBytes);
      const std::vector<size_t> &sz = param_sizes(e, p.func);
      for (size_t i = 0; i < sz.size() && p.kernelParams; i++) put_bytes(p.kernelParams[i], sz[i]);
    } else if (t == cudaGraphNodeTypeMemset) {
      cudaMemsetParams m;
      if (cudaGraphMemsetNodeGetParams(node, &m) != cudaSuccess) return 0;
      put((u64)(uintptr_t)m.dst);
      put(m.value);
      put(m.width);
    }
  }
  size_t ne = 0;
  if (cudaGraphGetEdges(g, nullptr, nullptr, &ne) != cudaSuccess) return 0;
  put(ne);
  cudaGetLastError();
  *n_nodes = n;
  return h;
}

bool graphs_equal(gdl_engine *e, cudaGraph_t a, cudaGraph_t b) {
  size_t na = 0, nb = 0;
  if (cudaGraphGetNodes(a, nullptr, &na) != cudaSuccess ||
      cudaGraphGetNodes(b, nullptr, &nb) != cudaSuccess || na != nb)
    return false;
  std::vector<cudaGraphNode_t> xa(na), xb(nb);
  if (na && (cudaGraphGetNodes(a, xa.data(), &na) != cudaSuccess ||
             cudaGraphGetNodes(b, xb.data(), &nb) != cudaSuccess))
    return false;
  for (size_t i = 0; i < na; i++)
    if (!nodes_equal(e, xa[i], xb[i])) return false;
  // the same dependencies between corresponding nodes
  size_t ea = 0, eb = 0;
  if (cudaGraphGetEdges(a, nullptr, nullptr, &ea) != cudaSuccess ||
      cudaGraphGetEdges(b, nullptr, nullptr, &eb) != cudaSuccess || ea != eb)
    return false;
  auto edges = [&](cudaGraph_t g, const std::vector<cudaGraphNode_t> &x, size_t n,
                   std::vector<std::pair<size_t, size_t>> &out) {
    std::vector<cudaGraphNode_t> from(n), to(n);
    size_t m = n;
    if (n && cudaGraphGetEdges(g, from.data(), to.data(), &m) != cudaSuccess) return false;
    std::unordered_map<cudaGraphNode_t, size_t> at;
    for (size_t i = 0; i < x.size(); i++) at[x[i]] = i;
    for (size_t i = 0; i < m; i++) out.emplace_back(at[from[i]], at[to[i]]);
    std::sort(out.begin(), out.end());
    return true;
  };
  std::vector<std::pair<size_t, size_t>> pa, pb;
  if (!edges(a, xa, ea, pa) || !edges(b, xb, eb, pb)) return false;
  cudaGetLastError();
  return pa == pb;
}

// The LIE's executable back to the cache (or, when it is not cached, to
// the engine's worker for destruction).
void release_graph(gdl_engine *e, LieHost &L) {
  if (L.gslot >= 0) {
    e->gcache[L.gslot].in_use = false;
  } else if (L.gexec) {
    e->graveyard.push_back(L.gexec);
  }
  L.gexec = nullptr;
  L.gslot = -1;
}

gdl_status build_graph(gdl_engine *e, LieHost &L, const Plan &plan) {
  release_graph(e, L);
  L.graph_reused = false;
  struct Swap {
    gdl_engine *e;
    cudaStream_t keep;
    ~Swap() { e->s = keep; }
  } swap{e, e->s};
  // captured on the capture stream (the engine stream may be running the
  // loop's first iteration)
  e->s = e->cap_s;
  // The loop: a while node whose body is one captured iteration.
  cudaGraph_t g = nullptr;
  cudaError_t r = cudaGraphCreate(&g, 0);
  cudaGraphConditionalHandle h;
  if (r == cudaSuccess) r = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
  if (r != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    return fail(e, GDL_E_CUDA, "cudaGraphConditionalHandleCreate: %s", cudaGetErrorString(r));
  }
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  r = cudaGraphAddNode(&node, g, nullptr, 0, &p);
  if (r != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(e, GDL_E_CUDA, "cudaGraphAddNode(conditional): %s", cudaGetErrorString(r));
  }
  cudaGraph_t body = p.conditional.phGraph_out[0];
  r = cudaStreamBeginCaptureToGraph(e->s, body, nullptr, nullptr, 0,
                                    cudaStreamCaptureModeThreadLocal);
  Counts kc;
  if (r == cudaSuccess) {
    enqueue_iteration(e, L, plan, &kc, true);
    cudaGraph_t captured = nullptr;
    r = cudaStreamEndCapture(e->s, &captured);
  }
  if (r != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(e, GDL_E_CUDA, "capture of the iteration failed: %s", cudaGetErrorString(r));
  }
  // An equal iteration in the cache: its executable, and this graph goes.
  // (Hooked operators launch the caller's kernels: never cached.)
  bool cacheable = getenv("GDLOG_NO_GRAPH_CACHE") == nullptr;
  for (const OpHost &op : L.ops) cacheable = cacheable && !op.hook;
  u64 sig = 0;
  size_t n_nodes = 0;
  if (cacheable) {
    sig = graph_signature(e, body, &n_nodes);
    for (size_t i = 0; i < e->gcache.size(); i++) {
      gdl_engine::CachedGraph &c = e->gcache[i];
      if (c.in_use || c.nodes != n_nodes || c.sig != sig || !graphs_equal(e, body, c.body))
        continue;
      cudaGraphDestroy(g);
      c.in_use = true;
      c.used = ++e->gcache_clock;
      L.gexec = c.exec;
      L.cond_handle = c.handle;
      L.per_iter = c.per_iter;
      L.gslot = (int)i;
      L.graph_reused = true;
      L.graph_dirty = false;
      return GDL_OK;
    }
  }
  r = cudaGraphInstantiate(&L.gexec, g, 0);
  if (r != cudaSuccess) {
    L.gexec = nullptr;
    cudaGraphDestroy(g);
    return fail(e, GDL_E_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(r));
  }
  L.cond_handle = (unsigned long long)h;
  L.per_iter = kc;
  L.graph_dirty = false;
  if (!cacheable) {
    cudaGraphDestroy(g);
    return GDL_OK;
  }
  // Into the cache (the graph kept for its body): a free slot, else the
  // least recently used idle one.
  gdl_engine::CachedGraph c;
  c.graph = g;
  c.body = body;
  c.exec = L.gexec;
  c.handle = L.cond_handle;
  c.per_iter = kc;
  c.nodes = n_nodes;
  c.sig = sig;
  c.in_use = true;
  c.used = ++e->gcache_clock;
  int slot = -1;
  if (e->gcache.size() >= kGraphCacheMax) {
    for (size_t i = 0; i < e->gcache.size(); i++)
      if (!e->gcache[i].in_use && (slot < 0 || e->gcache[i].used < e->gcache[slot].used))
        slot = (int)i;
  }
  if (slot >= 0) {
    e->graveyard.push_back(e->gcache[slot].exec);
    cudaGraphDestroy(e->gcache[slot].graph);
    e->gcache[slot] = c;
  } else {
    slot = (int)e->gcache.size();
    e->gcache.push_back(c);
  }
  L.gslot = slot;
  return GDL_OK;
}

// Grow the buffers an overflow asked for.
// Capacity after an overflow: half again the need, and at least four times
// the old capacity (within the list limit), so that a relation growing by
// orders of magnitude reruns few iterations (each rerun also rebuilds the
// graph).
u64 grown(u64 need, u64 cap) {
  return std::max<u64>(need, std::min<u64>(std::max<u64>(need + need / 2, 4 * cap), kMaxRows));
}

gdl_status grow_after_overflow(gdl_engine *e, const Ctl &c) {
  TRY(pull(e));
  for (size_t i = 0; i < e->rels.size(); i++) {
    RelDev &r = e->h[i];
    u64 nn = c.need[need_index((int)i, kNeedNewt)];
    u64 nf = c.need[need_index((int)i, kNeedFull)];
    u64 nd = c.need[need_index((int)i, kNeedDelta)];
    if (nn) {
      TRY(ensure_arr(e, r.newt, grown(nn, r.newt.cap), false));
      if (r.delta_next.cap < r.newt.cap) {
        TRY(ensure_arr(e, r.delta, r.newt.cap, true));
        TRY(ensure_arr(e, r.delta_next, r.newt.cap, false));
      }
    }
    if (nf) {
      TRY(ensure_arr(e, r.full, grown(nf, r.full.cap), true));
      TRY(ensure_arr(e, r.full_next, r.full.cap, false));
      TRY(ensure_index(e, r.full_idx, r.full.cap));
      TRY(ensure_index(e, r.full_idx_next, r.full_next.cap));
    }
    if (nd) {
      TRY(ensure_arr(e, r.delta, grown(nd, r.delta.cap), true));
      TRY(ensure_arr(e, r.delta_next, r.delta.cap, false));
      TRY(ensure_index(e, r.delta_idx, r.delta.cap));
      TRY(ensure_index(e, r.delta_idx_next, r.delta_next.cap));
    }
  }
  TRY(ensure_scratch(e));
  TRY(push(e));
  return GDL_OK;
}

gdl_status validate_rel(gdl_engine *e, int r) {
  const RelHost &h = e->rels[r];
  if ((h.arity != 2 && h.arity != 3) || h.icols != 1 || h.dep >= h.arity)
    return fail(e, GDL_E_UNSUPPORTED,
                "relation %s: only arity 2 or 3 with index_column_size 1 is supported",
                h.name.c_str());
  return GDL_OK;
}


// The lists of a dense LIE at capacity `cap` rows each (and the indexes
// some op probes on them).
gdl_status presize_lists(gdl_engine *e, LieHost &L, const Plan &plan, u64 cap) {
  for (int r : L.update) {
    RelDev &h = e->h[r];
    TRY(ensure_arr(e, h.delta, cap, true));
    TRY(ensure_arr(e, h.delta_next, cap, false));
    if (plan.newt_list[r] || plan.acopy_src[r]) TRY(ensure_arr(e, h.newt, cap, false));
    if (plan.full_list[r]) {
      TRY(ensure_arr(e, h.full, cap, true));
      TRY(ensure_arr(e, h.full_next, cap, false));
      if (plan.full_idx[r]) {
        TRY(ensure_index(e, h.full_idx, h.full.cap));
        TRY(ensure_index(e, h.full_idx_next, h.full_next.cap));
      }
    } else if (!e->instances) {
      // FULL listed once when the LIE ends: sized now, so that the listing
      // can be enqueued behind the loop without a host round trip
      TRY(ensure_arr(e, h.full, cap, true));
    }
    if (plan.delta_idx[r]) {
      TRY(ensure_index(e, h.delta_idx, h.delta.cap));
      TRY(ensure_index(e, h.delta_idx_next, h.delta_next.cap));
    }
  }
  for (int r : L.tmps) TRY(ensure_arr(e, e->h[r].newt, cap, false));
  return GDL_OK;
}

gdl_status fixpoint(gdl_engine *e, LieHost &L, uint64_t *out_iters) {
  if (e->broken) return fail(e, GDL_E_TIMEOUT, "engine is in a failed state; destroy it");
  if ((int)L.ops.size() > kMaxOps) return fail(e, GDL_E_UNSUPPORTED, "too many ops in one LIE");
  std::vector<char> is_update(e->rels.size(), 0), is_tmp(e->rels.size(), 0);
  for (int r : L.update) is_update[r] = 1;
  for (int r : L.tmps) is_tmp[r] = 1;
  for (int r : L.update) TRY(validate_rel(e, r));
  for (int r : L.statics) TRY(validate_rel(e, r));
  for (int r : L.tmps) TRY(validate_rel(e, r));
  if (e->wide && !e->k2) e->k2 = 32 - std::max(bits_for(e->max_value), 1);
  for (const OpHost &op : L.ops) {
    TRY(validate_rel(e, op.inner));
    if (op.outer >= 0) TRY(validate_rel(e, op.outer));
    TRY(validate_rel(e, op.out));
    if (!is_update[op.out] && !is_tmp[op.out])
      return fail(e, GDL_E_UNSUPPORTED,
                  "op output %s is neither an update nor a tmp relation of the LIE",
                  e->rels[op.out].name.c_str());
  }
  Plan plan = make_plan(e, L);
  // The timed span is the whole call, as the reference's drivers time the
  // whole fixpoint_loop (test/tc.cu:120-140): setup, loop and finish.
  CK(e, cudaEventRecord(e->ev0, e->s));
  const u64 aux0 = e->aux_launches;
  const auto t_setup = std::chrono::steady_clock::now();
  // GDLOG_TRACE_SETUP=1: host time of each setup phase on stderr
  static const bool trace_setup = getenv("GDLOG_TRACE_SETUP") != nullptr;
  std::vector<std::pair<const char *, double>> phases;
  auto t_phase = t_setup;
  auto mark = [&](const char *name) {
    if (!trace_setup) return;
    const auto now = std::chrono::steady_clock::now();
    phases.emplace_back(name, std::chrono::duration<double, std::milli>(now - t_phase).count());
    t_phase = now;
  };
  const u32 test_wait = e->test_wait;  // gdl_engine_test_timeout: this fixpoint only
  e->test_wait = 0;
  TRY(reset_ctl(e));
  mark("reset_ctl");
  TRY(refresh(e));
  mark("pull");
  // Setup (src/lie.cu:49-59): DELTA := the first |FULL| rows of FULL's raw
  // buffer; capacities for the loop.
  for (int r : L.update) {
    RelDev &h = e->h[r];
    RelHost &rh = e->rels[r];
    if (!h.full_vis) h.full.n = 0;  // tuple_full gets tuple_counts rows
    const u64 take = rh.raw_is_full ? h.full.n : std::min(h.full.n, rh.raw_n);
    // room to double, within the list limit (a FULL at the limit keeps it)
    const u64 base = std::max<u64>(std::min<u64>(2 * h.full.n, std::max<u64>(h.full.n, kMaxRows)),
                                   kMinCap);
    TRY(ensure_arr(e, h.full, base, true));
    TRY(ensure_arr(e, h.full_next, h.full.cap, false));
    TRY(ensure_arr(e, h.newt, std::max<u64>(h.newt.cap, base), false));
    TRY(ensure_arr(e, h.delta, std::max<u64>(take, h.newt.cap), false));
    TRY(ensure_arr(e, h.delta_next, h.delta.cap, false));
    if (take)
      CK(e, cudaMemcpyAsync(h.delta.ptr, rh.raw_is_full ? h.full.ptr : rh.raw, take * sizeof(u64),
                            cudaMemcpyDeviceToDevice, e->s));
    h.delta.n = take;
    h.delta_vis = 1;
    rh.delta_sorted = rh.raw_is_full;
    h.newt.n = 0;
    h.newt_phantom = 0;
  }
  for (int r : L.tmps) {
    RelDev &h = e->h[r];
    TRY(ensure_arr(e, h.newt, std::max<u64>(h.newt.cap, kMinCap), false));
    h.newt.n = 0;
  }
  mark("arrays");
  // Dense form (dense.cuh) when the key domain is small enough; always in
  // the batched form, whose block-diagonal bitmap is the only layout.
  for (int r : L.update)
    if (e->rels[r].full_resident)
      return fail(e, GDL_E_UNSUPPORTED,
                  "FULL of %s is kept as a bitmap only (batched form, too large for a list)",
                  e->rels[r].name.c_str());
  {
    const int dk = std::max(e->kbits, 5);
    // Bitmaps hold arity-2 tuples without dependent columns only.
    bool plain = !e->wide;
    for (auto *v : {&L.update, &L.statics, &L.tmps})
      for (int r : *v) plain = plain && e->rels[r].dep == 0;
    for (const OpHost &op : L.ops) plain = plain && !op.generic;
    L.dense = plain && (e->instances || (e->dedup_mode != 1 && 2 * dk <= e->dense_max_bits));
    L.dk = L.dense && !e->instances ? dk : 0;
    plan_pull(e, L, plan);
  }
  for (RelDev &h : e->h) {
    h.dense = h.full_lazy = 0;
    h.dirty = nullptr;
  }
  if (L.dense) {
    if (e->instances) {
      L.map = DenseMap{e->d_segs, e->d_tile_inst, (u32)e->segs.size(), e->seg_shift, e->seg_words};
      const u32 n = (u32)e->segs.size();
      if (L.n_inst != n) {
        dfree(e, L.d_inst_delta);
        dfree(e, L.d_inst_last);
        TRY(dalloc(e, (void **)&L.d_inst_delta, n * sizeof(u64)));
        TRY(dalloc(e, (void **)&L.d_inst_last, n * sizeof(u64)));
        L.n_inst = n;
      }
      CK(e, cudaMemsetAsync(L.d_inst_delta, 0, n * sizeof(u64), e->s));
      CK(e, cudaMemsetAsync(L.d_inst_last, 0, n * sizeof(u64), e->s));
    } else {
      if (!e->d_square_seg) TRY(dalloc(e, (void **)&e->d_square_seg, sizeof(SegInfo)));
      const SegInfo sq{0, (u32)(L.dk - 5), 1u << L.dk};
      CK(e, cudaMemcpyAsync(e->d_square_seg, &sq, sizeof sq, cudaMemcpyHostToDevice, e->s));
      L.map = DenseMap{e->d_square_seg, nullptr, 1, 31, dense_words(L.dk)};
    }
    const u64 words = L.map.words;
    for (int r : L.update) {
      e->rels[r].inv_ready = false;  // (its FULL changes during the LIE)
      TRY(ensure_bitmaps(e, r, words, true));
      RelDev &h = e->h[r];
      h.dense = 1;
      h.full_lazy = !plan.full_list[r];
    }
    for (int r : L.tmps) {
      TRY(ensure_bitmaps(e, r, words, false));
      e->h[r].dense = 1;
    }
    for (auto *v : {&L.update, &L.tmps})
      for (int r : *v) TRY(ensure_tbitmaps(e, plan, r, words));
    mark("bitmap_alloc");
    // A dirty map pays when a NEWT bitmap is too large to scan whole every
    // iteration; for small ones the scans read everything and the joins
    // skip the extra store.
    const bool use_dirty = words >= (1ull << e->dirty_min_log2_words);
    // (a fused update pass reads all of NEWT: no dirty map)
    for (auto *v : {&L.update, &L.tmps})
      for (int r : *v)
        e->h[r].dirty = use_dirty && !fused_update(plan, r) ? e->h[r].bmD : nullptr;
    TRY(ensure_dense_scratch(e, words));
    mark("dense_scratch");
    // Every list of the loop is bounded by the key domain: size them for
    // it up front (within a quarter of the device's memory shared among
    // the lists), so that the loop does not stop to grow buffers.  If that
    // does not fit, retry within a quarter of the memory actually free.
    u64 lists = 0;
    for (int r : L.update)
      lists += 2 + ((plan.newt_list[r] || plan.acopy_src[r]) ? 1 : 0) +
               (plan.full_list[r] ? 2 : (e->instances ? 0 : 1));
    lists += L.tmps.size();
    const u64 domain = words * 32;
    const u64 cap = std::min<u64>(
        {domain, e->total_mem / 4 / std::max<u64>(lists, 1) / 8, kMaxRows});
    gdl_status ps = presize_lists(e, L, plan, cap);
    if (ps == GDL_E_NOMEM) {
      cudaGetLastError();
      size_t free_b = 0, total_b = 0;
      CK(e, cudaMemGetInfo(&free_b, &total_b));
      ps = presize_lists(e, L, plan,
                         std::min<u64>(cap, (u64)(free_b / 4) / std::max<u64>(lists, 1) / 8));
    }
    TRY(ps);
  }
  mark("dense_alloc");
  TRY(ensure_scratch(e));
  mark("scratch");
  TRY(push(e));
  mark("push");
  if (L.dense) {
    // FULL's bitmap from its list; NEWT bitmaps empty.
    const u64 words = L.map.words;
    for (int r : L.update) {
      const RelDev &h = e->h[r];
      CK(e, cudaMemsetAsync(h.bmF, 0, words * 4, e->s));
      CK(e, cudaMemsetAsync(h.bmG, 0, words * 4, e->s));
      CK(e, cudaMemsetAsync(h.bmD, 0, words / kBmChunkWords, e->s));
      if (h.full.n) {
        k_bm_from_list<<<grid_for(e, h.full.n, 256, 8), 256, 0, e->s>>>(
            &e->d_rels[r].full, h.bmF, L.map, e->d_ctl);
        e->aux_launches++;
      }
      if (plan.delta_t[r]) {
        // the first DELTA, transposed, for the pull-form joins that read it
        CK(e, cudaMemsetAsync(h.bmDT, 0, words * 4, e->s));
        if (h.delta.n) {
          k_bm_from_list_t<<<grid_for(e, h.delta.n, 256, 8), 256, 0, e->s>>>(
              &e->d_rels[r].delta, h.bmDT, L.dk, e->d_ctl);
          e->aux_launches++;
        }
      }
      if (plan.delta_n[r]) {
        // ... and as rows, for the row-gather joins
        CK(e, cudaMemsetAsync(h.bmDN, 0, words * 4, e->s));
        if (h.delta.n) {
          k_bm_from_list<<<grid_for(e, h.delta.n, 256, 8), 256, 0, e->s>>>(
              &e->d_rels[r].delta, h.bmDN, L.map, e->d_ctl);
          e->aux_launches++;
        }
      }
      e->rels[r].bm_valid = true;
    }
    for (int r : L.tmps) {
      CK(e, cudaMemsetAsync(e->h[r].bmG, 0, words * 4, e->s));
      CK(e, cudaMemsetAsync(e->h[r].bmD, 0, words / kBmChunkWords, e->s));
    }
    for (auto *v : {&L.update, &L.tmps})
      for (int r : *v)
        if (plan.out_t[r]) CK(e, cudaMemsetAsync(e->h[r].bmOT, 0, words * 4, e->s));
    // the FULL bitmaps of the static outers of row-gather joins
    {
      std::vector<char> built_o(e->rels.size(), 0);
      for (size_t oi = 0; oi < L.ops.size(); oi++) {
        const OpHost &op = L.ops[oi];
        if (!plan.rows[oi] || op.outer_ver != GDL_FULL || built_o[op.outer]) continue;
        TRY(ensure_static_bitmap(e, op.outer, words));
        const RelDev &h = e->h[op.outer];
        CK(e, cudaMemsetAsync(h.bmF, 0, words * 4, e->s));
        if (h.full.n) {
          k_bm_from_list<<<grid_for(e, h.full.n, 256, 8), 256, 0, e->s>>>(
              &e->d_rels[op.outer].full, h.bmF, L.map, e->d_ctl);
          e->aux_launches++;
        }
        built_o[op.outer] = 1;
      }
    }
    // the in-edges of the static inners of row-gather joins
    std::vector<char> built(e->rels.size(), 0);
    for (size_t oi = 0; oi < L.ops.size(); oi++) {
      const int r = L.ops[oi].inner;
      if (!plan.rows[oi] || built[r]) continue;
      TRY(build_inverse(e, r, L.dk));
      built[r] = 1;
    }
    CK(e, cudaGetLastError());
  }
  mark("bitmaps");
  // An unsorted DELTA (raw load order) used as a join inner is sorted and
  // deduplicated first (the reference's index walk is undefined there).
  for (int r : L.update) {
    if (plan.delta_idx[r] && !e->rels[r].delta_sorted && e->h[r].delta.n) {
      RelDev &h = e->h[r];
      const u64 n = h.delta.n;
      TRY(ensure_arr(e, h.newt, n, false));
      CK(e, cudaMemcpyAsync(h.newt.ptr, h.delta.ptr, n * sizeof(u64), cudaMemcpyDeviceToDevice, e->s));
      u64 *keys = h.newt.ptr;
      h.newt.n = n;
      TRY(push(e));
      Counts kc;
      launch_sort(e, &e->d_rels[r].newt, keys, h.newt.cap, &kc);
      TRY(pull(e));
      CK(e, cudaMemcpyAsync(h.delta.ptr, sorted_location(e, keys), n * sizeof(u64),
                            cudaMemcpyDeviceToDevice, e->s));
      // unique in place on the host side is not needed: duplicates in an
      // index run only repeat outputs, which the later dedup removes.
      h.newt.n = 0;
      e->rels[r].delta_sorted = true;
      TRY(push(e));
    }
  }
  mark("delta_sort");
  // Indexes every join of this LIE probes: sized, then built with one
  // upload of the relation table (the builds take the epoch generation + 1,
  // written into the host mirror here).
  {
    bool any = false;
    const u32 epoch = (u32)(e->generation + 1);
    for (size_t r = 0; r < e->rels.size(); r++)
      for (int dv = 0; dv < 2; dv++) {
        if (!(dv ? plan.delta_idx[r] : plan.full_idx[r])) continue;
        RelDev &h = e->h[r];
        TRY(ensure_index(e, dv ? h.delta_idx : h.full_idx, dv ? h.delta.cap : h.full.cap));
        TRY(ensure_index(e, dv ? h.delta_idx_next : h.full_idx_next,
                         dv ? h.delta_next.cap : h.full_next.cap));
        (dv ? h.delta_idx : h.full_idx).epoch = epoch;
        any = true;
      }
    if (any) {
      TRY(push(e));
      for (size_t r = 0; r < e->rels.size(); r++)
        for (int dv = 0; dv < 2; dv++) {
          if (!(dv ? plan.delta_idx[r] : plan.full_idx[r])) continue;
          const RelDev &h = e->h[r];
          k_index_build<<<grid_for(e, (dv ? h.delta : h.full).n, kIndexBlock, 8), kIndexBlock, 0,
                          e->s>>>(dv ? &e->d_rels[r].delta : &e->d_rels[r].full,
                                  dv ? &e->d_rels[r].delta_idx : &e->d_rels[r].full_idx, nullptr,
                                  e->d_ctl);
          e->aux_launches++;
        }
      CK(e, cudaGetLastError());
    }
  }
  mark("indexes");
  // Device LIE description: the header and the trace buffer (the copy-once
  // flags stay as the device has them).
  LieDev &ld = L.hdr;
  ld.n_update = (int)L.update.size();
  ld.n_static = (int)L.statics.size();
  ld.n_tmp = (int)L.tmps.size();
  ld.n_ops = (int)L.ops.size();
  for (size_t i = 0; i < L.update.size(); i++) ld.update[i] = L.update[i];
  for (size_t i = 0; i < L.statics.size(); i++) ld.statics[i] = L.statics[i];
  for (size_t i = 0; i < L.tmps.size(); i++) ld.tmps[i] = L.tmps[i];
  // trace buffer: rows for one batch
  const u64 trace_rows = kTraceRows;
  if (!L.d_trace) TRY(dalloc(e, (void **)&L.d_trace, trace_rows * kMaxRels * 3 * sizeof(u64)));
  ld.trace = L.d_trace;
  CK(e, cudaMemcpyAsync(L.d_lie, &ld, offsetof(LieDev, once), cudaMemcpyHostToDevice, e->s));
  CK(e, cudaMemcpyAsync(&L.d_lie->trace, &ld.trace, sizeof(u64 *), cudaMemcpyHostToDevice, e->s));
  // Control block.
  Ctl c;
  memset(&c, 0, sizeof c);
  c.generation = ++e->generation;
  c.max_iteration = L.max_iteration < 0 ? 0 : (u64)L.max_iteration;
  c.trace_rows = trace_rows;
  c.spin_limit = e->spin_limit;
  c.test_wait = test_wait;
  L.trace.clear();
  L.retries = 0;
  L.grow_ms = L.graph_ms = 0;
  mark("lie_ctl");
  L.setup_ms = host_ms_since(t_setup);
  if (trace_setup) {
    fprintf(stderr, "gdlog setup %.3f ms:", L.setup_ms);
    for (auto &ph : phases) fprintf(stderr, " %s %.3f", ph.first, ph.second);
    fprintf(stderr, "\n");
  }
  L.graph_launches = 0;
  L.kernels = 0;
  L.graph_dirty = true;
  const bool use_graph = getenv("GDLOG_NO_GRAPH") == nullptr && !e->profile;
  u64 batch = 4;
  bool first_batch = true;
  bool tail_listed = false;
  e->mirror_fresh = false;
  // The FULL lists kept only as bitmaps during the loop are listed behind
  // every loop batch, before the host waits for it (k_ctl_resume lets the
  // listings run only once the loop ended without error), when each list
  // was sized for the whole key domain at setup; the batch's one wait then
  // also brings back the listings' checks and the relation table.
  bool spec_list = L.dense && !e->instances;
  if (spec_list) {
    const u64 domain = L.map.words * 32;
    bool any_lazy = false;
    for (int r : L.update)
      if (e->h[r].full_lazy) {
        any_lazy = true;
        if (e->h[r].full.cap < domain) spec_list = false;
      }
    spec_list = spec_list && any_lazy;
    if (spec_list) TRY(ensure_lb(e, e->lb_list, e->lb_list_tiles, L.map.words / kBmTileWords + 2));
  }
  auto enqueue_tail = [&](u64 it0, u64 stop_at) -> gdl_status {
    CK(e, cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
    if (L.trace_on) {
      const u64 rows = std::min<u64>(stop_at - it0, trace_rows) * L.update.size() * 3;
      if (rows)
        CK(e, cudaMemcpyAsync(e->h_trace, ld.trace, rows * sizeof(u64), cudaMemcpyDeviceToHost,
                              e->s));
    }
    if (!spec_list) return GDL_OK;
    k_ctl_resume<<<1, 32, 0, e->s>>>(e->d_ctl);
    e->aux_launches++;
    for (int r : L.update)
      if (e->h[r].full_lazy)
        TRY(launch_list(e, e->h[r].bmF, L.map.words, L.dk - 5, &e->d_rels[r].full, 1));
    CK(e, cudaGetLastError());
    CK(e, cudaMemcpyAsync(e->h_ctl2, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
    CK(e, cudaEventRecord(e->ev1, e->s));
    CK(e, cudaMemcpyAsync(e->h_rels_pin, e->d_rels, e->rels.size() * sizeof(RelDev),
                          cudaMemcpyDeviceToHost, e->s));
    return GDL_OK;
  };
  while (true) {
    c.pause = 0;
    c.stop_at = c.iteration + (use_graph ? std::min<u64>(trace_rows, 1u << 20) : batch);
    c.trace_base = c.iteration;
    const u64 it0 = c.iteration;
    // The loop's first iteration runs on the stream while the host captures
    // and instantiates the graph for the iterations after it; when that
    // iteration already ended the loop (and the host sees it), no graph
    // launch follows.
    const bool pre = use_graph && L.graph_dirty && first_batch;
    first_batch = false;
    Counts pre_kc;
    if (pre) {
      c.cond_set = 0;
      c.cond_handle = 0;
      CK(e, cudaMemcpyAsync(e->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, e->s));
      enqueue_iteration(e, L, plan, &pre_kc, false);
      CK(e, cudaGetLastError());
      CK(e, cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
      CK(e, cudaEventRecord(e->ev_first, e->s));
    }
    if (use_graph && L.graph_dirty) {
      const auto tg = std::chrono::steady_clock::now();
      TRY(build_graph(e, L, plan));
      L.graph_ms += host_ms_since(tg);
    }
    bool run_graph = use_graph;
    if (pre) {
      const cudaError_t q = cudaEventQuery(e->ev_first);
      if (q == cudaSuccess) {
        const Ctl &h = *e->h_ctl;
        if (h.done || h.pause || h.overflow || h.timeout || h.oob) run_graph = false;
      } else if (q != cudaErrorNotReady) {
        CK(e, q);
      }
      cudaGetLastError();
      L.kernels += pre_kc.total;
      for (int k = 0; k < kPKinds; k++) e->prof_launches[k] += pre_kc.kind[k];
    }
    u64 enqueued = 0;
    if (run_graph) {
      if (pre) {
        k_arm_graph<<<1, 32, 0, e->s>>>(e->d_ctl, L.cond_handle);
        L.kernels++;
        e->prof_launches[kPControl]++;
      } else {
        c.cond_set = 1;
        c.cond_handle = L.cond_handle;
        CK(e, cudaMemcpyAsync(e->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, e->s));
      }
      // the body's first iteration is opened here, later ones by k_commit
      k_begin<<<1, 32, 0, e->s>>>(e->d_rels, L.d_lie, e->d_ctl);
      L.kernels++;
      e->prof_launches[kPControl]++;
      CK(e, cudaGraphLaunch(L.gexec, e->s));
      L.graph_launches++;
    } else if (!use_graph) {
      c.cond_set = 0;
      c.cond_handle = 0;
      CK(e, cudaMemcpyAsync(e->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, e->s));
      // Profiling enqueues one iteration at a time, so that no launch of an
      // iteration past the fixpoint enters the per-kernel times.
      const u64 nb = e->profile ? 1 : std::min<u64>(batch, trace_rows);
      for (u64 k = 0; k < nb; k++) {
        Counts kc;
        enqueue_iteration(e, L, plan, &kc, false);
        L.per_iter = kc;
        enqueued++;
      }
      CK(e, cudaGetLastError());
    }
    TRY(enqueue_tail(it0, c.stop_at));
    CK(e, cudaStreamSynchronize(e->s));
    prof_collect(e);
    c = *e->h_ctl;
    e->generation = c.generation;
    // the listings behind the loop ran (k_ctl_resume's condition)
    tail_listed = spec_list && c.done && !c.pause && !c.overflow && !c.timeout && !c.oob;
    const u64 ran = c.iteration - it0;
    // In a graph, the body runs once per committed iteration plus once for
    // an iteration that overflowed (after a first iteration on the stream,
    // at least once); on the stream, every enqueued iteration launches
    // (those past the fixpoint return at once).
    u64 bodies = enqueued;
    if (run_graph) {
      bodies = ran + (c.overflow ? 1 : 0);
      if (pre) bodies = std::max<u64>(bodies, 2) - 1;
    } else if (use_graph) {
      bodies = 0;
    }
    L.kernels += bodies * (u64)L.per_iter.total;
    for (int k = 0; k < kPKinds; k++) e->prof_launches[k] += bodies * (u64)L.per_iter.kind[k];
    if (L.trace_on && ran) {
      // (a batch commits at most stop_at - it0 <= trace_rows iterations: all
      // their rows came back with the batch's wait)
      const u64 *rows = e->h_trace;
      for (u64 t = 0; t < ran; t++)
        for (size_t i = 0; i < L.update.size(); i++) {
          const u64 *x = &rows[(t * L.update.size() + i) * 3];
          L.trace.insert(L.trace.end(), {it0 + t, (u64)L.update[i], x[0], x[1], x[2]});
        }
    }
    if (c.oob & 32768u) {
      e->broken = true;
      return fail(e, GDL_E_UNSUPPORTED,
                  "iteration %llu generated a value too large for its column (arity-2 columns "
                  "hold values below 2^32; arity-3 keys hold column 1 below 2^%d and column 2 "
                  "below 2^%d)",
                  (unsigned long long)c.iteration, 32 - e->k2, e->k2);
    }
    if (c.timeout || c.oob) {
      e->broken = true;
      return fail(e, GDL_E_TIMEOUT,
                  "device-side check failed in iteration %llu (timeout=%u, dropped writes=%u)",
                  (unsigned long long)c.iteration, c.timeout, c.oob);
    }
    if (c.overflow) {
      const auto tg = std::chrono::steady_clock::now();
      TRY(grow_after_overflow(e, c));
      L.grow_ms += host_ms_since(tg);
      const bool resume = L.dense && c.overflow_stage == 1;
      c.overflow = 0;
      c.overflow_stage = 0;
      memset(c.need, 0, sizeof c.need);
      L.retries++;
      L.graph_dirty = true;
      if (L.dense && !resume) {
        // The iteration runs again from its start: its NEWT bitmaps must
        // be empty again (emitting relations clear them only on success).
        const u64 words = L.map.words;
        for (auto *v : {&L.update, &L.tmps})
          for (int r : *v) {
            CK(e, cudaMemsetAsync(e->h[r].bmG, 0, words * 4, e->s));
            CK(e, cudaMemsetAsync(e->h[r].bmD, 0, words / kBmChunkWords, e->s));
            // (and the transposed twins, zero between their uses)
            if (e->h[r].bmOT) CK(e, cudaMemsetAsync(e->h[r].bmOT, 0, words * 4, e->s));
          }
      }
      if (resume) {
        tail_listed = false;
        // Re-run only the update step and the commit of the iteration that
        // overflowed, launch by launch, until its lists fit.
        while (true) {
          c.pause = 0;
          c.stop_at = ~0ull;
          c.trace_base = c.iteration;
          c.cond_set = 0;
          CK(e, cudaMemcpyAsync(e->d_ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, e->s));
          const u64 it1 = c.iteration;
          Counts kc;
          enqueue_update_step(e, L, plan, &kc, false);
          CK(e, cudaGetLastError());
          CK(e, cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
          CK(e, cudaStreamSynchronize(e->s));
          prof_collect(e);
          c = *e->h_ctl;
          e->generation = c.generation;
          L.kernels += kc.total;
          for (int k = 0; k < kPKinds; k++) e->prof_launches[k] += kc.kind[k];
          if (c.timeout || c.oob) {
            e->broken = true;
            return fail(e, GDL_E_TIMEOUT,
                        "device-side check failed in iteration %llu (timeout=%u, dropped "
                        "writes=%u)",
                        (unsigned long long)c.iteration, c.timeout, c.oob);
          }
          if (c.overflow) {
            const auto tg2 = std::chrono::steady_clock::now();
            TRY(grow_after_overflow(e, c));
            L.grow_ms += host_ms_since(tg2);
            c.overflow = 0;
            c.overflow_stage = 0;
            memset(c.need, 0, sizeof c.need);
            L.retries++;
            continue;
          }
          if (L.trace_on && c.iteration > it1) {
            std::vector<u64> rows(L.update.size() * 3);
            CK(e, cudaMemcpyAsync(rows.data(), ld.trace, rows.size() * sizeof(u64),
                                  cudaMemcpyDeviceToHost, e->s));
            CK(e, cudaStreamSynchronize(e->s));
            for (size_t i = 0; i < L.update.size(); i++) {
              const u64 *x = &rows[i * 3];
              L.trace.insert(L.trace.end(), {it1, (u64)L.update[i], x[0], x[1], x[2]});
            }
          }
          break;
        }
        if (c.done) break;
      }
      continue;
    }
    if (c.done) break;
    batch = std::min<u64>(batch * 2, 64);
  }
  e->mirror_fresh = false;  // (a pull while growing buffers preceded more launches)
  bool listed = false;
  // ev1 was recorded behind the listings of the last batch, before its wait
  bool ev1_recorded = false;
  const Ctl *lc = e->h_ctl;  // the listings' device checks
  if (L.dense && tail_listed) {
    // FULL lists written behind the loop; the table came back with them
    if (e->h_ctl2->timeout || e->h_ctl2->oob) {
      e->broken = true;
      return fail(e, GDL_E_TIMEOUT, "listing FULL after the loop failed (timeout=%u oob=%u)",
                  e->h_ctl2->timeout, e->h_ctl2->oob);
    }
    memcpy(e->h.data(), e->h_rels_pin, e->rels.size() * sizeof(RelDev));
    e->mirror_fresh = true;
    for (RelHost &rh : e->rels) rh.stale = false;
    ev1_recorded = true;
    for (int r : L.update) e->h[r].full_lazy = 0;
  }
  if (L.dense) {
    // FULL lists that were not kept during the loop are written from the
    // FULL bitmaps, sorted (bit order is tuple order).
    const u64 kept_iteration = c.iteration;
    TRY(refresh(e));
    bool ctl_reset = false;
    auto resume_ctl = [&]() -> gdl_status {  // clear done/pause so that the scans below run
      if (!ctl_reset) TRY(reset_ctl(e));
      ctl_reset = true;
      return GDL_OK;
    };
    bool any = false;
    for (int r : L.update)
      if (e->h[r].full_lazy) {
        // The batched form may keep a FULL too large for a list as its
        // bitmap only (per-instance sizes, digests and exports read it).
        // So does the plain form when FULL is beyond the list limit: its
        // size and digest are then read from the bitmap.
        const u64 n = e->h[r].full.n;
        gdl_status as = GDL_E_NOMEM;
        if (n <= kMaxRows && (!e->instances || n * 8 <= e->total_mem / 4))
          as = ensure_arr(e, e->h[r].full, n, false);
        if (as == GDL_E_NOMEM && (e->instances || n > kMaxRows)) {
          cudaGetLastError();
          e->rels[r].full_resident = true;
          e->rels[r].bm_dk = L.dk;
          e->h[r].full_lazy = 0;
          continue;
        }
        TRY(as);
        any = true;
      }
    if (any) {
      TRY(resume_ctl());
      TRY(push(e));
      Counts kc;
      for (int r : L.update) {
        if (!e->h[r].full_lazy) continue;
        if (!e->instances) {
          // square domain (k_bm_list_*)
          TRY(launch_list(e, e->h[r].bmF, L.map.words, L.dk - 5, &e->d_rels[r].full, 1));
          continue;
        }
        BmScanArgs a = scan_none(L.map);
        a.f = e->h[r].bmF;
        a.ex_b = kBmUnion;
        a.list_b = &e->d_rels[r].full;
        launch_scan(e, a, r, &kc);
      }
      CK(e, cudaGetLastError());
      // The square-domain listing publishes the sizes the host already
      // holds; the batched form's scans need the table read back.
      if (e->instances) TRY(pull(e));
      listed = true;
      ev1_recorded = false;
    }
    // DELTA lists that were not kept (read only transposed by pull-form
    // joins) and are not empty (max_iteration ended the loop): transposed
    // back into the (empty) NEWT bitmap and listed from it.
    // (DELTA was only counted during the loop: a fused update step, or a
    // DELTA read only transposed)
    auto delta_unlisted = [&](int r) {
      return plan.fused[r] || (plan.delta_t[r] && !plan.delta_list[r]);
    };
    bool any_delta = false;
    for (int r : L.update)
      if (delta_unlisted(r) && e->h[r].delta.n) {
        RelDev &h = e->h[r];
        TRY(ensure_arr(e, h.delta, h.delta.n, false));
        any_delta = true;
      }
    if (any_delta) {
      TRY(resume_ctl());
      TRY(push(e));
      const u64 side = 1ull << (L.dk - kPullMinBits);
      for (int r : L.update) {
        const RelDev &h = e->h[r];
        if (!(delta_unlisted(r) && h.delta.n)) continue;
        // DELTA's rows: kept as they are, or transposed back into the
        // (empty) NEWT bitmap
        const u32 *rows = h.bmDN;
        if (!plan.delta_n[r]) {
          TransposeArgs t = transpose_args(h.bmDT, nullptr, h.bmG, L.dk, nullptr, nullptr,
                                           &e->recs[7], e->d_ctl);
          k_bm_transpose<<<grid_for(e, side * side, 1, 8), kTrBlock, 0, e->s>>>(t);
          e->aux_launches++;
          rows = h.bmG;
        }
        TRY(launch_list(e, rows, L.map.words, L.dk - 5, &e->d_rels[r].delta, 1));
        if (!plan.delta_n[r]) CK(e, cudaMemsetAsync(h.bmG, 0, L.map.words * 4, e->s));
      }
      CK(e, cudaGetLastError());
      listed = true;
      ev1_recorded = false;
    }
    // the listings' device checks, read back with the end of the fixpoint
    if (listed && !ev1_recorded)
      CK(e, cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
    else
      listed = false;  // (the listings behind the loop were checked above)
    for (RelDev &h : e->h) {
      h.dense = h.full_lazy = 0;
      h.dirty = nullptr;
    }
    TRY(push(e));
    c.iteration = kept_iteration;
  }
  if (!ev1_recorded) CK(e, cudaEventRecord(e->ev1, e->s));
  CK(e, cudaEventSynchronize(e->ev1));
  if (listed && (lc->timeout || lc->oob)) {
    e->broken = true;
    return fail(e, GDL_E_TIMEOUT, "listing FULL/DELTA after the loop failed (timeout=%u oob=%u)",
                lc->timeout, lc->oob);
  }
  float ms = 0;
  CK(e, cudaEventElapsedTime(&ms, e->ev0, e->ev1));
  L.ms = ms;
  L.iterations = c.iteration;
  L.kernels += e->aux_launches - aux0;  // (setup and listings, between ev0 and ev1)
  e->kernels_launched += L.kernels;
  for (int k = 0; k < kPKinds; k++) e->prof_bytes[k] += c.prof[k];
  // Finish (src/lie.cu:217-260).
  TRY(refresh(e));
  for (int r : L.update) {
    RelDev &h = e->h[r];
    RelHost &rh = e->rels[r];
    if (L.reload_full) {
      // FULL becomes flat, sorted and indexed; it is now its own raw buffer.
      if (rh.raw && !rh.raw_is_full) dfree(e, rh.raw);
      rh.raw = nullptr;
      rh.raw_is_full = true;
      rh.raw_n = h.full.n;
      h.full_vis = 1;
      h.delta.n = 0;
      h.delta_vis = 1;
      h.newt.n = 0;
    }
    // DELTA is now what the last iteration's update step wrote: sorted
    rh.delta_sorted = true;
  }
  TRY(push(e));
  *out_iters = c.iteration;
  return GDL_OK;
}

}  // namespace

// ===========================================================================
// C-ABI
// ===========================================================================
extern "C" {

const char *gdl_version(void) { return "gdlog-b200 0.1 (sm_100a)"; }

const char *gdl_status_string(gdl_status s) {
  switch (s) {
    case GDL_OK: return "ok";
    case GDL_E_INVALID: return "invalid argument";
    case GDL_E_CUDA: return "CUDA error";
    case GDL_E_NOMEM: return "out of device memory";
    case GDL_E_UNSUPPORTED: return "unsupported";
    case GDL_E_TIMEOUT: return "device-side wait or check failed";
    case GDL_E_CAPACITY: return "buffer too small";
  }
  return "unknown status";
}

// Message of the last failing call that has no engine (the allocation-free
// entry point below), per host thread.
static thread_local std::string g_engineless_error = "null engine";

const char *gdl_last_error(const gdl_engine *e) {
  return e ? e->err.c_str() : g_engineless_error.c_str();
}

gdl_status gdl_engine_create(int32_t device, void *stream, gdl_engine **out) {
  if (!out) return GDL_E_INVALID;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return GDL_E_CUDA;
  if (device < 0 || device >= ndev) return GDL_E_INVALID;
  if (cudaSetDevice(device) != cudaSuccess) return GDL_E_CUDA;
  gdl_engine *e = new gdl_engine;
  e->device = device;
  cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, device);
  {
    size_t f = 0, t = 0;
    if (cudaMemGetInfo(&f, &t) == cudaSuccess) e->total_mem = t;
  }
  if (stream) {
    e->s = (cudaStream_t)stream;
  } else {
    if (cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking) != cudaSuccess) {
      delete e;
      return GDL_E_CUDA;
    }
    e->own_stream = true;
  }
  auto bad = [&](cudaError_t r) {
    if (r == cudaSuccess) return false;
    e->err = cudaGetErrorString(r);
    return true;
  };
  if (const char *m = getenv("GDLOG_DEDUP")) {
    if (!strcmp(m, "sort")) e->dedup_mode = 1;
    if (!strcmp(m, "dense")) e->dedup_mode = 2;
  }
  if (const char *ro = getenv("GDLOG_ROW_OR")) e->row_or_joins = strcmp(ro, "0") != 0;
  if (const char *pj = getenv("GDLOG_PULL")) e->pull_joins = strcmp(pj, "0") != 0 ? 3 : 1;
  if (const char *b = getenv("GDLOG_DENSE_MAX_BITS"))
    e->dense_max_bits = std::min(atoi(b), kDenseMaxDomainBits);
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    u64 thr = ~0ull;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  if (bad(cudaFuncSetAttribute(k_sort_hist<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<6>())) ||
      bad(cudaFuncSetAttribute(k_sort_pass<6>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<6>())) ||
      bad(cudaFuncSetAttribute(k_sort_hist<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<8>())) ||
      bad(cudaFuncSetAttribute(k_sort_pass<8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<8>())) ||
      bad(cudaFuncSetAttribute(k_sort_hist<10>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<10>())) ||
      bad(cudaFuncSetAttribute(k_sort_pass<10>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)sort_smem_bytes<10>())) ||
      bad(cudaFuncSetAttribute(k_merge_diff, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kMergeSmemBytes)) ||
      bad(cudaFuncSetAttribute(k_join_pull_bm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(pull_acc_words(16) * 4))) ||
      bad(cudaMalloc(&e->d_rels, kMaxRels * sizeof(RelDev))) ||
      bad(cudaMalloc(&e->d_ctl, sizeof(Ctl))) || bad(cudaMallocHost(&e->h_ctl, sizeof(Ctl))) ||
      bad(cudaMallocHost(&e->h_ctl2, sizeof(Ctl))) ||
      bad(cudaMallocHost(&e->h_trace, kTraceRows * kMaxRels * 3 * sizeof(u64))) ||
      bad(cudaMallocHost(&e->h_rels_pin, kMaxRels * sizeof(RelDev))) ||
      bad(cudaMalloc(&e->recs, 16 * sizeof(LaunchRec))) ||
      bad(cudaMalloc(&e->d_tmp, 4 * sizeof(DArr))) || bad(cudaMalloc(&e->d_u64, 4 * sizeof(u64))) ||
      bad(cudaMalloc(&e->d_u32, 4 * sizeof(u32))) ||
      bad(cudaMalloc(&e->d_pull_count, sizeof(u64))) || bad(cudaEventCreate(&e->ev0)) ||
      bad(cudaEventCreate(&e->ev1)) ||
      bad(cudaEventCreateWithFlags(&e->ev_first, cudaEventDisableTiming)) ||
      bad(cudaStreamCreateWithFlags(&e->cap_s, cudaStreamNonBlocking)) ||
      bad(cudaMemsetAsync(e->d_rels, 0, kMaxRels * sizeof(RelDev), e->s)) ||
      bad(cudaMemsetAsync(e->d_ctl, 0, sizeof(Ctl), e->s)) ||
      bad(cudaMemcpyAsync(&e->d_ctl->spin_limit, &e->spin_limit, sizeof(u32),
                          cudaMemcpyHostToDevice, e->s)) ||
      bad(cudaMemsetAsync(e->recs, 0, 16 * sizeof(LaunchRec), e->s)) ||
      bad(cudaMemsetAsync(e->d_u32, 0, 4 * sizeof(u32), e->s)) ||
      bad(cudaMemsetAsync(e->d_pull_count, 0, sizeof(u64), e->s)) ||
      bad(cudaStreamSynchronize(e->s))) {
    gdl_engine_destroy(e);
    return GDL_E_CUDA;
  }
  // TMA passes: the driver's tensor-map encoder, and their shared memory
  if (!getenv("GDLOG_NO_TMA")) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess && fn &&
        cudaFuncSetAttribute(k_bm_update_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)std::max(upd_tma_smem(upd_tma_stages(0), 0),
                                           upd_tma_smem(upd_tma_stages(1), 1))) == cudaSuccess &&
        cudaFuncSetAttribute(k_bm_fold_tma, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)std::max(fold_tma_smem(fold_tma_stages(0), 0),
                                           fold_tma_smem(fold_tma_stages(1), 1))) == cudaSuccess) {
      e->tma_encode = fn;
      e->tma_ok = true;
    }
    cudaGetLastError();
  }
  *out = e;
  return GDL_OK;
}

// Free every relation and LIE of the engine (device arrays return to the
// stream-ordered pool, so a following program reuses them cheaply).
static void release_program(gdl_engine *e) {
  for (size_t i = 0; i < e->rels.size(); i++) {
    RelDev &r = e->h[i];
    for (DArr *a : {&r.full, &r.full_next, &r.delta, &r.delta_next, &r.newt})
      dfree(e, a->ptr);
    for (Index *x : {&r.full_idx, &r.full_idx_next, &r.delta_idx, &r.delta_idx_next})
      dfree(e, x->slots);
    for (u32 *bm : {r.bmF, r.bmG, r.bmDT, r.bmGT, r.bmOT, r.bmDN})
      dfree(e, bm);
    dfree(e, r.bmD);
    dfree(e, r.tile_prefix);
    const RelHost &rh = e->rels[i];
    for (u32 *q : {rh.inv_off, rh.inv_cur, rh.inv_keys, rh.inv_ys})
      dfree(e, q);
    if (!e->rels[i].raw_is_full) dfree(e, e->rels[i].raw);
  }
  for (LieHost &L : e->lies) {
    release_graph(e, L);
    // stream-ordered frees (a cudaFree would wait for the whole device)
    for (void *p : {(void *)L.d_trace, (void *)L.d_lie, (void *)L.d_joinrec})
      dfree(e, p);
    dfree(e, L.d_inst_delta);
    dfree(e, L.d_inst_last);
  }
  e->rels.clear();
  e->h.clear();
  e->lies.clear();
  e->kbits = 1;
  e->max_value = 0;
}

gdl_status gdl_engine_clear(gdl_engine *e) {
  if (!e) return GDL_E_INVALID;
  cudaSetDevice(e->device);
  // (no LIE graph may be running while its executable is destroyed)
  CK(e, cudaStreamSynchronize(e->s));
  release_program(e);
  reap_graphs(e);
  // the next program's requests take back this program's blocks
  e->replay.swap(e->alloc_log);
  e->alloc_log.clear();
  e->replay_seen.clear();
  // everything after this is stream-ordered behind the blocks released
  CK(e, cudaMemsetAsync(e->d_rels, 0, kMaxRels * sizeof(RelDev), e->s));
  if (e->broken) {
    // After a device-side check failed (a bounded wait gave up, a bounds
    // check fired) the relations are dropped above; kernels of the failed
    // launch may have stopped between counting and finishing, so the
    // launch records and every look-back flag start afresh too.
    CK(e, cudaMemsetAsync(e->recs, 0, 16 * sizeof(LaunchRec), e->s));
    for (const Lb *lb : {&e->lb_cnt, &e->lb_nz, &e->lb_merge, &e->lb_bm, &e->lb_list})
      if (lb->flag) CK(e, cudaMemsetAsync(lb->flag, 0, lb == &e->lb_cnt ? e->lb_cnt_tiles * 4
                                                     : lb == &e->lb_nz ? e->lb_nz_tiles * 4
                                                     : lb == &e->lb_merge ? e->lb_merge_tiles * 4
                                                     : lb == &e->lb_bm ? e->lb_bm_tiles * 4
                                                                        : e->lb_list_tiles * 4,
                                          e->s));
    // the sort's tile counters and digit histograms (an interrupted sort
    // leaves them part-accumulated; they return to zero only at its end)
    if (e->sort_counters)
      CK(e, cudaMemsetAsync(e->sort_counters, 0, (kMaxPasses + 1) * sizeof(u32), e->s));
    if (e->sort_offsets)
      CK(e, cudaMemsetAsync(e->sort_offsets, 0, kMaxPasses * kMaxRadix * sizeof(u32), e->s));
    CK(e, cudaMemsetAsync(e->d_u32, 0, 4 * sizeof(u32), e->s));
    CK(e, cudaMemsetAsync(e->d_pull_count, 0, sizeof(u64), e->s));
    TRY(reset_ctl(e));
    CK(e, cudaStreamSynchronize(e->s));
    e->broken = false;
  }
  return GDL_OK;
}

gdl_status gdl_engine_test_timeout(gdl_engine *e, int32_t polls) {
  if (!e || polls < 1) return GDL_E_INVALID;
  e->test_wait = (u32)polls;
  return GDL_OK;
}

gdl_status gdl_engine_destroy(gdl_engine *e) {
  if (!e) return GDL_OK;
  cudaSetDevice(e->device);
  if (e->s) cudaStreamSynchronize(e->s);
  release_program(e);
  for (auto &g : e->gcache) {
    e->graveyard.push_back(g.exec);
    cudaGraphDestroy(g.graph);
  }
  e->gcache.clear();
  for (cudaGraphExec_t x : e->graveyard) cudaGraphExecDestroy(x);
  e->graveyard.clear();
  if (e->reaper.joinable()) {
    {
      std::lock_guard<std::mutex> lock(e->reap_mu);
      e->reap_stop = true;
    }
    e->reap_cv.notify_one();
    e->reaper.join();
  }
  drop_spare(e);
  if (e->s) cudaStreamSynchronize(e->s);
  for (void *p : {(void *)e->sort_buf, (void *)e->sort_offsets, (void *)e->sort_counters,
                  (void *)e->sort_status, (void *)e->crow_off, (void *)e->crow_key,
                  (void *)e->crow_start, (void *)e->crow_len, (void *)e->lb_cnt.flag,
                  (void *)e->lb_cnt.agg, (void *)e->lb_cnt.inc, (void *)e->lb_nz.flag,
                  (void *)e->lb_nz.agg, (void *)e->lb_nz.inc, (void *)e->lb_merge.flag,
                  (void *)e->lb_merge.agg, (void *)e->lb_merge.inc, (void *)e->merge_parts,
                  (void *)e->lb_bm.flag, (void *)e->lb_bm.agg, (void *)e->lb_bm.inc,
                  (void *)e->lb_list.flag, (void *)e->lb_list.agg, (void *)e->lb_list.inc,
                  (void *)e->d_segs,
                  (void *)e->d_tile_inst, (void *)e->d_square_seg,
                  (void *)e->recs,
                  (void *)e->d_tmp, (void *)e->d_u64, (void *)e->d_u32, (void *)e->d_pull_count,
                  e->d_count, e->d_part,
                  (void *)e->d_rels,
                  (void *)e->d_ctl})
    if (p) cudaFree(p);
  if (e->h_ctl) cudaFreeHost(e->h_ctl);
  if (e->h_ctl2) cudaFreeHost(e->h_ctl2);
  if (e->h_trace) cudaFreeHost(e->h_trace);
  if (e->h_rels_pin) cudaFreeHost(e->h_rels_pin);
  if (e->ev0) cudaEventDestroy(e->ev0);
  if (e->ev1) cudaEventDestroy(e->ev1);
  if (e->ev_first) cudaEventDestroy(e->ev_first);
  if (e->cap_s) cudaStreamDestroy(e->cap_s);
  prof_collect(e);
  for (cudaEvent_t ev : e->ev_pool) cudaEventDestroy(ev);
  if (e->own_stream && e->s) cudaStreamDestroy(e->s);
  delete e;
  return GDL_OK;
}

gdl_status gdl_engine_sync(gdl_engine *e) {
  if (!e) return GDL_E_INVALID;
  CK(e, cudaStreamSynchronize(e->s));
  return GDL_OK;
}

gdl_status gdl_relation_create(gdl_engine *e, const char *name, int32_t arity, int32_t icols,
                               int32_t dep, int32_t index_flag, int32_t tmp_flag, int32_t *out) {
  if (!e || !out) return GDL_E_INVALID;
  if ((int)e->rels.size() >= kMaxRels) return fail(e, GDL_E_UNSUPPORTED, "too many relations");
  if (arity < 1 || icols < 1 || icols > arity || dep < 0 || dep >= arity)
    return fail(e, GDL_E_INVALID, "bad arity/index/dependent column sizes");
  if (arity != 2 && arity != 3)
    return fail(e, GDL_E_UNSUPPORTED, "arity %d not supported (arity 2 and 3 only)", arity);
  if (icols != 1) return fail(e, GDL_E_UNSUPPORTED, "index_column_size must be 1");
  if (arity == 3) e->wide = true;
  cudaSetDevice(e->device);
  RelHost rh;
  rh.name = name ? name : "";
  rh.arity = arity;
  rh.icols = icols;
  rh.dep = dep;
  rh.index_flag = index_flag != 0;
  rh.tmp_flag = tmp_flag != 0;
  e->rels.push_back(rh);
  RelDev d;
  memset(&d, 0, sizeof d);
  d.full_vis = d.delta_vis = d.w_full_vis = d.w_delta_vis = 1;
  e->h.push_back(d);
  *out = (int32_t)e->rels.size() - 1;
  TRY(push_rel(e, *out));  // the new entry only (loads may be in flight)
  return GDL_OK;
}

#define CHECK_REL(e, r)                                                        \
  do {                                                                          \
    if (!(e)) return GDL_E_INVALID;                                             \
    if ((r) < 0 || (r) >= (int)(e)->rels.size())                                \
      return fail((e), GDL_E_INVALID, "bad relation id %d", (int)(r));          \
    cudaSetDevice((e)->device);                                                 \
  } while (0)
#define CHECK_LIE(e, l)                                                        \
  do {                                                                          \
    if (!(e)) return GDL_E_INVALID;                                             \
    if ((l) < 0 || (l) >= (int)(e)->lies.size())                                \
      return fail((e), GDL_E_INVALID, "bad lie id %d", (int)(l));               \
    cudaSetDevice((e)->device);                                                 \
  } while (0)

static gdl_status load_common(gdl_engine *e, int32_t rel, const uint64_t *rows, uint64_t n,
                              bool on_device) {
  if (e->broken) return fail(e, GDL_E_TIMEOUT, "engine is in a failed state; destroy it");
  if (n > kMaxRows) return fail(e, GDL_E_UNSUPPORTED, "too many rows");
  if (n == 0) return load_keys(e, rel, nullptr, 0);
  if (e->rels[rel].arity == 3) {
    // arity 3: packed on the host (key_col layout), column 2 width fixed by
    // the first such load
    if (on_device) return fail(e, GDL_E_UNSUPPORTED, "arity-3 rows load from host memory");
    u64 m01 = 0, m2 = 0;
    for (u64 i = 0; i < n; i++) {
      m01 = std::max<u64>({m01, (u64)rows[3 * i], (u64)rows[3 * i + 1]});
      m2 = std::max<u64>(m2, (u64)rows[3 * i + 2]);
    }
    if (m01 >> 32) return fail(e, GDL_E_UNSUPPORTED, "column values must be below 2^32");
    if (!e->k2) e->k2 = 32 - std::max(bits_for(std::max(e->max_value, m01)), 1);
    if (bits_for(m01) > 32 - e->k2 || (m2 >> e->k2))
      return fail(e, GDL_E_UNSUPPORTED,
                  "arity-3 keys hold column 1 below 2^%d and column 2 below 2^%d",
                  32 - e->k2, e->k2);
    std::vector<u64> keys(n);
    for (u64 i = 0; i < n; i++)
      keys[i] = (rows[3 * i] << 32) | (rows[3 * i + 1] << e->k2) | rows[3 * i + 2];
    u64 *dk = nullptr;
    TRY(dalloc(e, (void **)&dk, n * sizeof(u64)));
    CK(e, cudaMemcpyAsync(dk, keys.data(), n * sizeof(u64), cudaMemcpyHostToDevice, e->s));
    e->max_value = std::max(e->max_value, m01);
    e->kbits = std::max(e->kbits, bits_for(e->max_value));
    gdl_status s = load_keys(e, rel, dk, n);
    dfree(e, dk);  // stream-ordered behind the load
    return s;
  }
  u64 *d_rows = nullptr, *d_keys = nullptr;
  u64 maxv = 0;
  u32 badv = 0;
  if (on_device) {
    d_rows = (u64 *)rows;
  } else {
    // host rows: the largest value and the range check on the host, so the
    // load needs no round trip
    u64 m = 0;
    for (u64 i = 0; i < 2 * n; i++) m = std::max<u64>(m, rows[i]);
    maxv = m;
    badv = (m >> 32) != 0;
    if (badv) return fail(e, GDL_E_UNSUPPORTED, "column values must be below 2^32");
    TRY(dalloc(e, (void **)&d_rows, n * 2 * sizeof(u64)));
    CK(e, cudaMemcpyAsync(d_rows, rows, n * 2 * sizeof(u64), cudaMemcpyHostToDevice, e->s));
  }
  TRY(dalloc(e, (void **)&d_keys, n * sizeof(u64)));
  CK(e, cudaMemsetAsync(e->d_u64, 0, sizeof(u64), e->s));
  CK(e, cudaMemsetAsync(e->d_u32, 0, sizeof(u32), e->s));
  k_pack_rows<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(d_rows, n, d_keys, e->d_u64, e->d_u32);
  CK(e, cudaGetLastError());
  if (on_device) {
    CK(e, cudaMemcpyAsync(&maxv, e->d_u64, sizeof maxv, cudaMemcpyDeviceToHost, e->s));
    CK(e, cudaMemcpyAsync(&badv, e->d_u32, sizeof badv, cudaMemcpyDeviceToHost, e->s));
    CK(e, cudaStreamSynchronize(e->s));
  }
  if (!on_device) dfree(e, d_rows);
  if (badv) {
    dfree(e, d_keys);
    return fail(e, GDL_E_UNSUPPORTED, "column values must be below 2^32");
  }
  if (e->k2 && bits_for(maxv) > 32 - e->k2) {
    dfree(e, d_keys);
    return fail(e, GDL_E_UNSUPPORTED,
                "ids must stay below 2^%d once arity-3 relations are loaded", 32 - e->k2);
  }
  e->max_value = std::max(e->max_value, maxv);
  e->kbits = std::max(e->kbits, bits_for(e->max_value));
  gdl_status s = load_keys(e, rel, d_keys, n);
  dfree(e, d_keys);
  return s;
}

gdl_status gdl_relation_load(gdl_engine *e, int32_t rel, const uint64_t *rows, uint64_t n) {
  CHECK_REL(e, rel);
  if (n && !rows) return fail(e, GDL_E_INVALID, "null rows");
  return load_common(e, rel, rows, n, false);
}

gdl_status gdl_relation_load_device(gdl_engine *e, int32_t rel, const uint64_t *rows, uint64_t n) {
  CHECK_REL(e, rel);
  if (n && !rows) return fail(e, GDL_E_INVALID, "null rows");
  return load_common(e, rel, rows, n, true);
}

static gdl_status version_view(gdl_engine *e, int rel, int ver, const u64 **ptr, u64 *n,
                               bool *sorted, bool need_rows = true) {
  TRY(refresh(e));
  const RelDev &r = e->h[rel];
  *sorted = true;
  if (ver == GDL_FULL) {
    if (e->rels[rel].full_resident && need_rows)
      return fail(e, GDL_E_UNSUPPORTED,
                  "FULL of %s is kept as a bitmap only (more than %llu tuples, or the batched "
                  "form): read its size and digest, or per instance",
                  e->rels[rel].name.c_str(), (unsigned long long)kMaxRows);
    *ptr = r.full.ptr;
    *n = r.full_vis ? r.full.n : 0;
  } else if (ver == GDL_DELTA) {
    *ptr = r.delta.ptr;
    *n = r.delta_vis ? r.delta.n : 0;
    *sorted = e->rels[rel].delta_sorted;
  } else if (ver == GDL_NEWT) {
    *ptr = r.newt.ptr;
    *n = r.newt.n;
    *sorted = false;
  } else {
    return fail(e, GDL_E_INVALID, "bad version %d", ver);
  }
  return GDL_OK;
}

static gdl_status host_rows(gdl_engine *e, int rel, int ver, std::vector<u64> &keys) {
  const u64 *p = nullptr;
  u64 n = 0;
  bool sorted;
  TRY(version_view(e, rel, ver, &p, &n, &sorted));
  keys.resize(n);
  if (n) CK(e, cudaMemcpyAsync(keys.data(), p, n * sizeof(u64), cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  if (!sorted) {
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  }
  return GDL_OK;
}

gdl_status gdl_relation_size(gdl_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  CHECK_REL(e, rel);
  if (!out) return GDL_E_INVALID;
  if (ver == GDL_NEWT) {
    std::vector<u64> k;
    TRY(host_rows(e, rel, ver, k));
    *out = k.size();
    return GDL_OK;
  }
  const u64 *p = nullptr;
  u64 n = 0;
  bool sorted;
  TRY(version_view(e, rel, ver, &p, &n, &sorted, false));
  *out = n;
  return GDL_OK;
}

gdl_status gdl_relation_export(gdl_engine *e, int32_t rel, int32_t ver, uint64_t *rows,
                               uint64_t cap, uint64_t *out_n) {
  CHECK_REL(e, rel);
  if (!out_n) return GDL_E_INVALID;
  std::vector<u64> k;
  TRY(host_rows(e, rel, ver, k));
  *out_n = k.size();
  if (k.size() > cap) return fail(e, GDL_E_CAPACITY, "export needs %zu rows", k.size());
  if (k.size() && !rows) return GDL_E_INVALID;
  const int ar = e->rels[rel].arity;
  for (size_t i = 0; i < k.size(); i++)
    for (int j = 0; j < ar; j++) rows[ar * i + j] = key_col(k[i], ar, j, e->k2);
  return GDL_OK;
}

gdl_status gdl_relation_export_device(gdl_engine *e, int32_t rel, int32_t ver, uint64_t *rows,
                                      uint64_t cap, uint64_t *out_n) {
  CHECK_REL(e, rel);
  if (!out_n) return GDL_E_INVALID;
  if (e->rels[rel].arity != 2)
    return fail(e, GDL_E_UNSUPPORTED, "device export: arity-2 relations only");
  const u64 *p = nullptr;
  u64 n = 0;
  bool sorted;
  TRY(version_view(e, rel, ver, &p, &n, &sorted));
  if (!sorted)
    return fail(e, GDL_E_UNSUPPORTED,
                "device export: this version of %s is in load order (export it to the host)",
                e->rels[rel].name.c_str());
  *out_n = n;
  if (n > cap) return fail(e, GDL_E_CAPACITY, "device export needs %llu rows",
                           (unsigned long long)n);
  if (n && !rows) return GDL_E_INVALID;
  if (n)
    k_unpack_rows<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(p, n, reinterpret_cast<u64 *>(rows));
  CK(e, cudaGetLastError());
  CK(e, cudaStreamSynchronize(e->s));
  return GDL_OK;
}

gdl_status gdl_partition_rows(gdl_engine *e, const uint64_t *rows, uint64_t n, int32_t column,
                              int32_t world, uint64_t *out_rows, uint64_t *counts) {
  if (!e) return GDL_E_INVALID;
  if (column < 0 || column > 1 || world < 1 || world > kPartMaxWorld || !counts ||
      (n && (!rows || !out_rows)))
    return fail(e, GDL_E_INVALID, "partition: column 0 or 1, 1 <= world <= %d", kPartMaxWorld);
  cudaSetDevice(e->device);
  if (!e->d_part) CK(e, cudaMalloc(&e->d_part, 2 * kPartMaxWorld * sizeof(u64)));
  u64 *cnt = reinterpret_cast<u64 *>(e->d_part), *cur = cnt + kPartMaxWorld;
  CK(e, cudaMemsetAsync(cnt, 0, world * sizeof(u64), e->s));
  if (n) {
    const int g = grid_for(e, n, 256, 8);
    const u64 *in = reinterpret_cast<const u64 *>(rows);
    k_part_count<<<g, 256, 0, e->s>>>(in, n, column, (u32)world, cnt);
    k_part_offsets<<<1, 32, 0, e->s>>>(cnt, (u32)world, cur);
    k_part_scatter<<<g, 256, 0, e->s>>>(in, n, column, (u32)world, cur,
                                        reinterpret_cast<u64 *>(out_rows));
    CK(e, cudaGetLastError());
  }
  std::vector<u64> h(world);
  CK(e, cudaMemcpyAsync(h.data(), cnt, world * sizeof(u64), cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  for (int d = 0; d < world; d++) counts[d] = h[d];
  return GDL_OK;
}

// ---------------------------------------------------------------------------
// Files (get_row_size + get_relation_from_file, test/tc.cu:17-57)
// ---------------------------------------------------------------------------
namespace {
bool tsv_space(char c) {
  return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f';
}

// Parse one "%lld" at *p (leading white space skipped); false at the end
// of the data or on a character that starts no number.
bool tsv_value(const char *&p, const char *end, u64 *v) {
  while (p < end && tsv_space(*p)) p++;
  if (p >= end) return false;
  bool neg = false;
  if (*p == '+' || *p == '-') {
    neg = *p == '-';
    p++;
  }
  if (p >= end || *p < '0' || *p > '9') return false;
  u64 x = 0;
  while (p < end && *p >= '0' && *p <= '9') x = x * 10 + (u64)(*p++ - '0');
  *v = neg ? (u64)(0 - x) : x;
  return true;
}
}  // namespace

gdl_status gdl_read_tsv(const char *path, int32_t arity, uint64_t *host_rows, uint64_t cap_rows,
                        uint64_t *out_rows) {
  auto bad = [](gdl_status s, const std::string &m) {
    g_engineless_error = m;
    return s;
  };
  if (!path || !out_rows || arity < 1) return bad(GDL_E_INVALID, "gdl_read_tsv: bad argument");
  *out_rows = 0;
  FILE *f = fopen(path, "rb");
  if (!f) return bad(GDL_E_INVALID, std::string("cannot open ") + path);
  std::string buf;
  char chunk[1 << 16];
  size_t got;
  while ((got = fread(chunk, 1, sizeof chunk, f)) > 0) buf.append(chunk, got);
  fclose(f);
  u64 rows = 0;
  for (char c : buf) rows += c == '\n';
  *out_rows = rows;
  if (rows > cap_rows || (rows && !host_rows))
    return bad(GDL_E_CAPACITY, "gdl_read_tsv: the file has " + std::to_string(rows) + " rows");
  const char *p = buf.data(), *end = buf.data() + buf.size();
  for (u64 i = 0; i < rows; i++)
    for (int j = 0; j < arity; j++) {
      u64 v = 0;
      if (!tsv_value(p, end, &v))
        return bad(GDL_E_INVALID, std::string(path) + ": no value for row " + std::to_string(i) +
                                      " column " + std::to_string(j));
      host_rows[i * arity + j] = (uint64_t)v;
      if (j != arity - 1 && p < end) p++;  // the separator character ("%lld%c")
    }
  return GDL_OK;
}

gdl_status gdl_relation_load_tsv(gdl_engine *e, int32_t rel, const char *path) {
  CHECK_REL(e, rel);
  const int arity = e->rels[rel].arity;
  uint64_t n = 0;
  gdl_status s = gdl_read_tsv(path, arity, nullptr, 0, &n);
  if (s != GDL_OK && s != GDL_E_CAPACITY) return fail(e, s, "%s", g_engineless_error.c_str());
  std::vector<uint64_t> rows(n * arity);
  s = gdl_read_tsv(path, arity, rows.data(), n, &n);
  if (s != GDL_OK) return fail(e, s, "%s", g_engineless_error.c_str());
  return gdl_relation_load(e, rel, n ? rows.data() : nullptr, n);
}

gdl_status gdl_relation_dump_tsv(gdl_engine *e, int32_t rel, int32_t ver, const char *path,
                                 uint64_t *out_rows) {
  CHECK_REL(e, rel);
  if (!path) return fail(e, GDL_E_INVALID, "null path");
  std::vector<u64> k;
  TRY(host_rows(e, rel, ver, k));
  FILE *f = fopen(path, "wb");
  if (!f) return fail(e, GDL_E_INVALID, "cannot write %s", path);
  std::string out;
  out.reserve(k.size() * 16);
  char line[48];
  const int ar = e->rels[rel].arity;
  for (u64 key : k) {
    for (int j = 0; j < ar; j++) {
      const int m = snprintf(line, sizeof line, j + 1 < ar ? "%u\t" : "%u\n",
                             key_col(key, ar, j, e->k2));
      out.append(line, (size_t)m);
    }
  }
  const bool ok = fwrite(out.data(), 1, out.size(), f) == out.size();
  fclose(f);
  if (!ok) return fail(e, GDL_E_INVALID, "short write to %s", path);
  if (out_rows) *out_rows = k.size();
  return GDL_OK;
}

static gdl_status bitmap_stats(gdl_engine *e, const u32 *bm, const DenseMap &map,
                               const std::vector<SegInfo> &segs, std::vector<u64> &size,
                               std::vector<u64> &digest);

// Device scratch of gdl_join_count: the op record and the two visibility
// words the count kernel reads (and zeroes, for an empty side) instead of
// the relations' own.
struct CountScratch {
  JoinRec rec;
  DArr newt;
  u32 outer_vis, inner_vis;
};

gdl_status gdl_join_count(gdl_engine *e, int32_t inner, int32_t inner_ver, int32_t outer,
                          int32_t outer_ver, uint64_t *out) {
  CHECK_REL(e, inner);
  CHECK_REL(e, outer);
  if (!out) return GDL_E_INVALID;
  if (e->broken) return fail(e, GDL_E_TIMEOUT, "engine is in a failed state; destroy it");
  auto ver_ok = [](int32_t v) { return v == GDL_FULL || v == GDL_DELTA; };
  if (!ver_ok(inner_ver) || !ver_ok(outer_ver))
    return fail(e, GDL_E_INVALID, "join count: versions must be GDL_FULL or GDL_DELTA");
  if (e->instances) return fail(e, GDL_E_UNSUPPORTED, "join count: not in the batched form");
  for (int r : {inner, outer})
    if (e->rels[r].full_resident)
      return fail(e, GDL_E_UNSUPPORTED, "join count: %s is kept as a bitmap only",
                  e->rels[r].name.c_str());
  TRY(refresh(e));
  RelDev &ih = e->h[inner];
  const RelDev &oh = e->h[outer];
  const DArr &ia = inner_ver == GDL_FULL ? ih.full : ih.delta;
  const DArr &oa = outer_ver == GDL_FULL ? oh.full : oh.delta;
  const u64 ni = (inner_ver == GDL_FULL ? ih.full_vis : ih.delta_vis) ? ia.n : 0;
  const u64 no = (outer_ver == GDL_FULL ? oh.full_vis : oh.delta_vis) ? oa.n : 0;
  if (ni && !e->rels[inner].index_flag)
    return fail(e, GDL_E_INVALID, "join count: %s is not indexed (index_flag)",
                e->rels[inner].name.c_str());
  if (ni && inner_ver == GDL_DELTA && !e->rels[inner].delta_sorted)
    return fail(e, GDL_E_UNSUPPORTED, "join count: DELTA of %s is in load order",
                e->rels[inner].name.c_str());
  if (ni == 0 || no == 0) {
    *out = 0;
    return GDL_OK;
  }
  TRY(ensure_scratch(e));
  // the inner version's index, built now (as a LIE builds the indexes its
  // joins probe, with a fresh epoch)
  TRY(reset_ctl(e));
  {
    Index &ixm = inner_ver == GDL_FULL ? ih.full_idx : ih.delta_idx;
    TRY(ensure_index(e, ixm, ia.cap));
    ixm.epoch = (u32)(e->generation + 1);
    TRY(push_rel(e, inner));
    k_index_build<<<grid_for(e, ni, kIndexBlock, 8), kIndexBlock, 0, e->s>>>(
        inner_ver == GDL_FULL ? &e->d_rels[inner].full : &e->d_rels[inner].delta,
        inner_ver == GDL_FULL ? &e->d_rels[inner].full_idx : &e->d_rels[inner].delta_idx,
        nullptr, e->d_ctl);
    CK(e, cudaGetLastError());
  }
  // (outside the engine's replayed allocation sequence: kept until destroy)
  if (!e->d_count) CK(e, cudaMalloc(&e->d_count, sizeof(CountScratch)));
  CountScratch cs;
  memset(&cs, 0, sizeof cs);
  cs.outer_vis = cs.inner_vis = 1;
  CK(e, cudaMemcpyAsync(e->d_count, &cs, sizeof cs, cudaMemcpyHostToDevice, e->s));
  CountScratch *d = reinterpret_cast<CountScratch *>(e->d_count);
  RelDev *R = e->d_rels;
  JoinArgs a;
  memset(&a, 0, sizeof a);
  a.outer = outer_ver == GDL_FULL ? &R[outer].full : &R[outer].delta;
  a.outer_vis = &d->outer_vis;
  a.inner = inner_ver == GDL_FULL ? &R[inner].full : &R[inner].delta;
  a.inner_vis = &d->inner_vis;
  a.inner_idx = inner_ver == GDL_FULL ? &R[inner].full_idx : &R[inner].delta_idx;
  a.out_newt = &d->newt;
  a.dense = 1;  // (no NEWT to check for room)
  a.op = &d->rec;
  a.rec = &e->recs[0];
  a.lb_cnt = e->lb_cnt;
  a.lb_nz = e->lb_nz;
  a.crow_off = e->crow_off;
  a.crow_start = e->crow_start;
  a.crow_len = e->crow_len;
  a.crow_key = e->crow_key;
  a.crow_cap = e->crow_cap;
  a.ctl = e->d_ctl;
  k_join_count<<<grid_for(e, no, kJoinTile, e->count_ctas_per_sm), kJoinBlock, 0, e->s>>>(a);
  CK(e, cudaGetLastError());
  JoinRec rec;
  CK(e, cudaMemcpyAsync(&rec, &d->rec, sizeof rec, cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaMemcpyAsync(e->h_ctl, e->d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  if (e->h_ctl->timeout || e->h_ctl->oob) {
    e->broken = true;
    return fail(e, GDL_E_TIMEOUT, "join count: device-side check failed (timeout=%u oob=%u)",
                e->h_ctl->timeout, e->h_ctl->oob);
  }
  *out = rec.total;
  return GDL_OK;
}

gdl_status gdl_relation_digest(gdl_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  CHECK_REL(e, rel);
  if (!out) return GDL_E_INVALID;
  const RelHost &rr = e->rels[rel];
  if (ver == GDL_FULL && rr.full_resident && !e->instances && rr.bm_valid && rr.bm_dk) {
    // FULL beyond the list limit, kept as its square-domain bitmap
    TRY(pull(e));
    if (!e->d_square_seg) TRY(dalloc(e, (void **)&e->d_square_seg, sizeof(SegInfo)));
    const SegInfo sq{0, (u32)(rr.bm_dk - 5), 1u << rr.bm_dk};
    CK(e, cudaMemcpyAsync(e->d_square_seg, &sq, sizeof sq, cudaMemcpyHostToDevice, e->s));
    const DenseMap map{e->d_square_seg, nullptr, 1, 31, rr.bm_words};
    std::vector<u64> size, dig;
    TRY(bitmap_stats(e, e->h[rel].bmF, map, {sq}, size, dig));
    *out = dig[0];
    return GDL_OK;
  }
  const u64 *p = nullptr;
  u64 n = 0;
  bool sorted;
  TRY(version_view(e, rel, ver, &p, &n, &sorted));
  u64 acc = 0;
  const int ar = e->rels[rel].arity;
  if (!sorted || ar != 2) {
    std::vector<u64> k;
    TRY(host_rows(e, rel, ver, k));
    for (size_t i = 0; i < k.size(); i++) {
      u64 h = mix64(i);
      for (int j = 0; j < ar; j++) h = mix64(h ^ (u64)key_col(k[i], ar, j, e->k2));
      acc += h;
    }
    *out = mix64(acc ^ (u64)k.size());
    return GDL_OK;
  }
  CK(e, cudaMemsetAsync(e->d_u64, 0, sizeof(u64), e->s));
  if (n) k_digest<<<grid_for(e, n, 256, 8), 256, 0, e->s>>>(p, n, e->d_u64);
  CK(e, cudaGetLastError());
  CK(e, cudaMemcpyAsync(&acc, e->d_u64, sizeof acc, cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  *out = mix64(acc ^ n);
  return GDL_OK;
}

gdl_status gdl_lie_create(gdl_engine *e, int32_t *out) {
  if (!e || !out) return GDL_E_INVALID;
  cudaSetDevice(e->device);
  LieHost L;
  TRY(dalloc(e, (void **)&L.d_lie, sizeof(LieDev)));
  CK(e, cudaMemsetAsync(L.d_lie, 0, sizeof(LieDev), e->s));
  TRY(dalloc(e, (void **)&L.d_joinrec, kMaxOps * sizeof(JoinRec)));
  CK(e, cudaMemsetAsync(L.d_joinrec, 0, kMaxOps * sizeof(JoinRec), e->s));
  e->lies.push_back(L);
  *out = (int32_t)e->lies.size() - 1;
  return GDL_OK;
}

gdl_status gdl_lie_add_relation(gdl_engine *e, int32_t lie, int32_t rel, int32_t static_flag) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, rel);
  LieHost &L = e->lies[lie];
  (static_flag ? L.statics : L.update).push_back(rel);
  L.graph_dirty = true;
  return GDL_OK;
}

gdl_status gdl_lie_add_tmp_relation(gdl_engine *e, int32_t lie, int32_t rel) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, rel);
  e->lies[lie].tmps.push_back(rel);
  e->lies[lie].graph_dirty = true;
  return GDL_OK;
}

// A hook given as gen entries GDL_INNER(c) / GDL_OUTER(c) / GDL_SRC(c), each
// possibly GDL_PLUS(entry, k): column moves only, between arity-2
// relations, become a Sel2; anything else (arity 3, a constant added) a
// GenSpec the kernels evaluate per tuple.
static gdl_status decode_gen(gdl_engine *e, const int32_t *gen, int32_t len, bool join, int a_in,
                             int a_outer, int a_out, OpHost *op) {
  if (!gen || len != a_out)
    return fail(e, GDL_E_INVALID, "gen must have one entry per output column (%d)", a_out);
  bool plain = a_in == 2 && a_out == 2 && (!join || a_outer == 2);
  for (int j = 0; j < len; j++) {
    const int g = gen[j] & 0xFF;
    const u32 add = (u32)gen[j] >> 8;
    const bool in_ok = g >= 0 && g < a_in;
    const bool out_ok = join && g >= 16 && g - 16 < a_outer;
    if (!in_ok && !out_ok) return fail(e, GDL_E_INVALID, "gen entry %d out of range", gen[j]);
    op->gen.src[j] = g;
    op->gen.add[j] = add;
    plain = plain && add == 0;
  }
  op->gen.out_arity = a_out;
  op->gen.in_arity = a_in;
  op->gen.outer_arity = join ? a_outer : 0;
  op->generic = !plain;
  if (plain) return GDL_OK;
  for (int j = len; j < 3; j++) op->gen.src[j] = 0, op->gen.add[j] = 0;
  return GDL_OK;
}

static gdl_status decode_sel(gdl_engine *e, const int32_t *gen, int32_t len, bool join, Sel2 *s) {
  if (!gen || len != 2) return fail(e, GDL_E_INVALID, "gen must have 2 entries (arity 2)");
  int v[2];
  for (int j = 0; j < 2; j++) {
    int g = gen[j];
    if (g == GDL_INNER(0) || g == GDL_INNER(1))
      v[j] = g;
    else if (join && (g == GDL_OUTER(0) || g == GDL_OUTER(1)))
      v[j] = 2 + (g - 16);
    else
      return fail(e, GDL_E_INVALID, "gen entry %d out of range", g);
  }
  s->s0 = v[0];
  s->s1 = v[1];
  return GDL_OK;
}

gdl_status gdl_lie_add_join(gdl_engine *e, int32_t lie, int32_t inner, int32_t inner_ver,
                            int32_t outer, int32_t outer_ver, int32_t output, const int32_t *gen,
                            int32_t gen_len, int32_t pred_kind, int32_t pa, int32_t pb) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, inner);
  CHECK_REL(e, outer);
  CHECK_REL(e, output);
  if (inner_ver < 0 || inner_ver > 2 || outer_ver < 0 || outer_ver > 2)
    return fail(e, GDL_E_INVALID, "bad version");
  if (pred_kind < GDL_PRED_NONE || pred_kind > GDL_PRED_GE)
    return fail(e, GDL_E_INVALID, "bad predicate");
  if (pred_kind && (pa < 0 || pa > 1 || pb < 0 || pb > 1))
    return fail(e, GDL_E_INVALID, "predicate column out of range");
  if ((int)e->lies[lie].ops.size() >= kMaxOps) return fail(e, GDL_E_UNSUPPORTED, "too many ops");
  OpHost op;
  op.kind = 0;
  op.inner = inner;
  op.inner_ver = inner_ver;
  op.outer = outer;
  op.outer_ver = outer_ver;
  op.out = output;
  TRY(decode_gen(e, gen, gen_len, true, e->rels[inner].arity, e->rels[outer].arity,
                 e->rels[output].arity, &op));
  if (!op.generic) TRY(decode_sel(e, gen, gen_len, true, &op.sel));
  if (op.generic && pred_kind)
    return fail(e, GDL_E_UNSUPPORTED, "predicates with arity 3 or computed columns");
  op.pred = Pred{pred_kind, pa, pb};
  e->lies[lie].ops.push_back(op);
  e->lies[lie].graph_dirty = true;
  return GDL_OK;
}

gdl_status gdl_lie_add_copy(gdl_engine *e, int32_t lie, int32_t src, int32_t src_ver, int32_t dest,
                            const int32_t *gen, int32_t gen_len) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  if (src_ver != GDL_DELTA && src_ver != GDL_FULL)
    return fail(e, GDL_E_INVALID, "copy source must be DELTA or FULL");
  if ((int)e->lies[lie].ops.size() >= kMaxOps) return fail(e, GDL_E_UNSUPPORTED, "too many ops");
  OpHost op;
  op.kind = 1;
  op.inner = src;
  op.inner_ver = src_ver;
  op.out = dest;
  TRY(decode_gen(e, gen, gen_len, false, e->rels[src].arity, 0, e->rels[dest].arity, &op));
  if (!op.generic) TRY(decode_sel(e, gen, gen_len, false, &op.sel));
  e->lies[lie].ops.push_back(op);
  e->lies[lie].graph_dirty = true;
  return GDL_OK;
}

gdl_status gdl_lie_add_acopy(gdl_engine *e, int32_t lie, int32_t src, int32_t dest,
                             const int32_t *gen, int32_t gen_len) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  if ((int)e->lies[lie].ops.size() >= kMaxOps) return fail(e, GDL_E_UNSUPPORTED, "too many ops");
  OpHost op;
  op.kind = 2;
  op.inner = src;
  op.inner_ver = GDL_NEWT;
  op.out = dest;
  TRY(decode_gen(e, gen, gen_len, false, e->rels[src].arity, 0, e->rels[dest].arity, &op));
  if (!op.generic) TRY(decode_sel(e, gen, gen_len, false, &op.sel));
  e->lies[lie].ops.push_back(op);
  e->lies[lie].graph_dirty = true;
  return GDL_OK;
}

static gdl_status add_hooked(gdl_engine *e, int32_t lie, OpHost op, gdl_hook_launch launch,
                             void *ctx) {
  if (!launch) return fail(e, GDL_E_INVALID, "null hook launcher");
  if ((int)e->lies[lie].ops.size() >= kMaxOps) return fail(e, GDL_E_UNSUPPORTED, "too many ops");
  // Tuples come from the caller's kernel: the LIE runs on sorted lists.
  op.generic = true;
  op.gen.out_arity = e->rels[op.out].arity;
  op.gen.in_arity = e->rels[op.inner].arity;
  op.gen.outer_arity = op.kind == 0 ? e->rels[op.outer].arity : 0;
  op.hook = launch;
  op.hook_ctx = ctx;
  e->lies[lie].ops.push_back(op);
  e->lies[lie].graph_dirty = true;
  return GDL_OK;
}

gdl_status gdl_lie_add_join_hooked(gdl_engine *e, int32_t lie, int32_t inner, int32_t inner_ver,
                                   int32_t outer, int32_t outer_ver, int32_t output,
                                   gdl_hook_launch launch, void *ctx) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, inner);
  CHECK_REL(e, outer);
  CHECK_REL(e, output);
  if (inner_ver < 0 || inner_ver > 2 || outer_ver < 0 || outer_ver > 2)
    return fail(e, GDL_E_INVALID, "bad version");
  OpHost op;
  op.kind = 0;
  op.inner = inner;
  op.inner_ver = inner_ver;
  op.outer = outer;
  op.outer_ver = outer_ver;
  op.out = output;
  return add_hooked(e, lie, op, launch, ctx);
}

gdl_status gdl_lie_add_copy_hooked(gdl_engine *e, int32_t lie, int32_t src, int32_t src_ver,
                                   int32_t dest, gdl_hook_launch launch, void *ctx) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  if (src_ver != GDL_DELTA && src_ver != GDL_FULL)
    return fail(e, GDL_E_INVALID, "copy source must be DELTA or FULL");
  OpHost op;
  op.kind = 1;
  op.inner = src;
  op.inner_ver = src_ver;
  op.out = dest;
  return add_hooked(e, lie, op, launch, ctx);
}

gdl_status gdl_lie_add_acopy_hooked(gdl_engine *e, int32_t lie, int32_t src, int32_t dest,
                                    gdl_hook_launch launch, void *ctx) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  OpHost op;
  op.kind = 2;
  op.inner = src;
  op.inner_ver = GDL_NEWT;
  op.out = dest;
  return add_hooked(e, lie, op, launch, ctx);
}

gdl_status gdl_lie_set_max_iteration(gdl_engine *e, int32_t lie, int64_t m) {
  CHECK_LIE(e, lie);
  e->lies[lie].max_iteration = m;
  return GDL_OK;
}

gdl_status gdl_lie_set_reload_full(gdl_engine *e, int32_t lie, int32_t flag) {
  CHECK_LIE(e, lie);
  e->lies[lie].reload_full = flag != 0;
  return GDL_OK;
}

gdl_status gdl_lie_set_trace(gdl_engine *e, int32_t lie, int32_t flag) {
  CHECK_LIE(e, lie);
  e->lies[lie].trace_on = flag != 0;
  return GDL_OK;
}

gdl_status gdl_lie_fixpoint(gdl_engine *e, int32_t lie, uint64_t *out) {
  CHECK_LIE(e, lie);
  uint64_t dummy;
  return fixpoint(e, e->lies[lie], out ? out : &dummy);
}

gdl_status gdl_lie_trace(gdl_engine *e, int32_t lie, uint64_t *rec, uint64_t cap, uint64_t *out_n) {
  CHECK_LIE(e, lie);
  const std::vector<uint64_t> &t = e->lies[lie].trace;
  uint64_t n = t.size() / 5;
  if (out_n) *out_n = n;
  if (rec) memcpy(rec, t.data(), std::min(n, cap) * 5 * sizeof(uint64_t));
  return GDL_OK;
}

static const char *const kProfNames[kPKinds] = {
    "sort_hist", "sort_pass", "merge_diff", "index_build", "join_count",
    "join_mat",  "copy",      "control",    "bitmap_scan"};

int32_t gdl_profile_kinds(void) { return kPKinds; }

const char *gdl_profile_kind_name(int32_t kind) {
  return kind >= 0 && kind < kPKinds ? kProfNames[kind] : "";
}

gdl_status gdl_engine_set_dedup(gdl_engine *e, int32_t mode, int32_t dense_max_bits) {
  if (!e || mode < GDL_DEDUP_AUTO || mode > GDL_DEDUP_DENSE) return GDL_E_INVALID;
  if (dense_max_bits < 0 || dense_max_bits > kDenseMaxDomainBits)
    return fail(e, GDL_E_INVALID, "dense_max_bits must be in [0, %d]", kDenseMaxDomainBits);
  e->dedup_mode = mode;
  if (dense_max_bits) e->dense_max_bits = dense_max_bits;
  return GDL_OK;
}

gdl_status gdl_engine_set_tuning(gdl_engine *e, const gdl_tuning *t) {
  if (!e || !t) return GDL_E_INVALID;
  if (t->dedup < 0 || t->dedup > GDL_DEDUP_DENSE || t->dense_max_bits < 0 ||
      t->dense_max_bits > kDenseMaxDomainBits || t->join_ctas_per_sm < 0 ||
      t->join_ctas_per_sm > 32 || t->count_ctas_per_sm < 0 || t->count_ctas_per_sm > 32 ||
      t->index_slots_per_key < 0 || t->index_slots_per_key > 64 ||
      (t->index_slots_per_key && (t->index_slots_per_key < 2 ||
                                  (t->index_slots_per_key & (t->index_slots_per_key - 1)))) ||
      (t->dirty_min_log2_words && (t->dirty_min_log2_words < 11 || t->dirty_min_log2_words > 40)) ||
      t->dense_join_passes < 0 || t->dense_join_passes > 2 || t->join_aggregate < 0 ||
      t->join_aggregate > 2 || t->pull_joins < 0 || t->pull_joins > 3 || t->row_gather < 0 ||
      t->row_gather > 3 || t->spin_limit_log2 < 0 || t->spin_limit_log2 > 30 ||
      (t->radix_bits && t->radix_bits != 6 && t->radix_bits != 8 && t->radix_bits != 10) ||
      (t->join_block && t->join_block != 128 && t->join_block != 256 && t->join_block != 512) ||
      (t->rows_piece && t->rows_piece != 8 && t->rows_piece != 16 && t->rows_piece != 32) ||
      t->load_dedup < 0 || t->load_dedup > 2)
    return fail(e, GDL_E_INVALID, "tuning value out of range");
  e->dedup_mode = t->dedup;
  if (t->dense_max_bits) e->dense_max_bits = t->dense_max_bits;
  if (t->join_ctas_per_sm) e->join_ctas_per_sm = t->join_ctas_per_sm;
  if (t->count_ctas_per_sm) e->count_ctas_per_sm = t->count_ctas_per_sm;
  if (t->index_slots_per_key) e->index_slots_per_key = t->index_slots_per_key;
  if (t->dirty_min_log2_words) e->dirty_min_log2_words = t->dirty_min_log2_words;
  if (t->dense_join_passes) e->dense_join_passes = t->dense_join_passes;
  if (t->join_aggregate) e->join_aggregate = t->join_aggregate;
  if (t->pull_joins) e->pull_joins = t->pull_joins;
  if (t->row_gather) e->row_gather = t->row_gather;
  if (t->spin_limit_log2) e->spin_limit = 1u << t->spin_limit_log2;
  if (t->radix_bits) e->radix_bits = t->radix_bits;
  if (t->join_block) e->join_block = t->join_block;
  if (t->rows_piece) e->rows_piece = t->rows_piece;
  if (t->load_dedup) e->load_dedup = t->load_dedup;
  for (LieHost &L : e->lies) L.graph_dirty = true;
  return GDL_OK;
}

gdl_status gdl_engine_get_tuning(gdl_engine *e, gdl_tuning *t) {
  if (!e || !t) return GDL_E_INVALID;
  t->dedup = e->dedup_mode;
  t->dense_max_bits = e->dense_max_bits;
  t->join_ctas_per_sm = e->join_ctas_per_sm;
  t->count_ctas_per_sm = e->count_ctas_per_sm;
  t->index_slots_per_key = e->index_slots_per_key;
  t->dirty_min_log2_words = e->dirty_min_log2_words;
  t->dense_join_passes = e->dense_join_passes;
  t->join_aggregate = e->join_aggregate;
  t->pull_joins = e->pull_joins;
  t->row_gather = e->row_gather;
  t->spin_limit_log2 = 0;
  while (t->spin_limit_log2 < 31 && (1u << t->spin_limit_log2) < e->spin_limit) t->spin_limit_log2++;
  t->radix_bits = e->radix_bits;
  t->join_block = e->join_block;
  t->rows_piece = e->rows_piece;
  t->load_dedup = e->load_dedup;
  return GDL_OK;
}

gdl_status gdl_engine_set_profile(gdl_engine *e, int32_t flag) {
  if (!e) return GDL_E_INVALID;
  e->profile = flag != 0;
  return GDL_OK;
}

gdl_status gdl_engine_profile(gdl_engine *e, double *out, int32_t n_out) {
  if (!e || (n_out && !out)) return GDL_E_INVALID;
  for (int k = 0; k < kPKinds; k++) {
    const double v[3] = {(double)e->prof_launches[k], e->prof_ms[k], (double)e->prof_bytes[k]};
    for (int j = 0; j < 3; j++)
      if (3 * k + j < n_out) out[3 * k + j] = v[j];
  }
  return GDL_OK;
}

gdl_status gdl_engine_profile_reset(gdl_engine *e) {
  if (!e) return GDL_E_INVALID;
  for (int k = 0; k < kPKinds; k++) {
    e->prof_ms[k] = 0;
    e->prof_launches[k] = 0;
    e->prof_bytes[k] = 0;
  }
  return GDL_OK;
}

gdl_status gdl_engine_set_instances(gdl_engine *e, const uint32_t *node_counts,
                                    int32_t n_instances) {
  if (!e || n_instances < 0 || (n_instances && !node_counts)) return GDL_E_INVALID;
  cudaSetDevice(e->device);
  CK(e, cudaStreamSynchronize(e->s));
  dfree(e, e->d_segs);
  dfree(e, e->d_tile_inst);
  e->d_segs = nullptr;
  e->d_tile_inst = nullptr;
  e->segs.clear();
  e->instances = false;
  e->seg_words = 0;
  if (n_instances == 0) return GDL_OK;
  u32 maxn = 1;
  for (int i = 0; i < n_instances; i++) {
    if (node_counts[i] < 1 || node_counts[i] > (u32)kMaxInstanceNodes)
      return fail(e, GDL_E_INVALID, "instance %d: node count must be in [1, %d]", i,
                  kMaxInstanceNodes);
    maxn = std::max(maxn, node_counts[i]);
  }
  int S = 1;
  while ((1u << S) < maxn) S++;
  if ((u64)n_instances << S > (1ull << 32))
    return fail(e, GDL_E_UNSUPPORTED, "%d instances of up to %u nodes exceed 32-bit ids",
                n_instances, maxn);
  u64 base = 0;
  std::vector<u32> tile_inst;
  for (int i = 0; i < n_instances; i++) {
    const u32 n = node_counts[i];
    u32 rs = 0;
    while ((1ull << rs) * 32 < n) rs++;
    SegInfo sg{base, rs, n};
    e->segs.push_back(sg);
    const u64 region = round_up((u64)n << rs, kBmTileWords);
    for (u64 t = 0; t < region / kBmTileWords; t++) tile_inst.push_back((u32)i);
    base += region;
  }
  e->seg_shift = S;
  e->seg_words = base;
  TRY(dalloc(e, (void **)&e->d_segs, e->segs.size() * sizeof(SegInfo)));
  TRY(dalloc(e, (void **)&e->d_tile_inst, tile_inst.size() * sizeof(u32)));
  CK(e, cudaMemcpyAsync(e->d_segs, e->segs.data(), e->segs.size() * sizeof(SegInfo),
                        cudaMemcpyHostToDevice, e->s));
  CK(e, cudaMemcpyAsync(e->d_tile_inst, tile_inst.data(), tile_inst.size() * sizeof(u32),
                        cudaMemcpyHostToDevice, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  e->instances = true;
  return GDL_OK;
}

gdl_status gdl_engine_instance_shift(gdl_engine *e, int32_t *out_shift) {
  if (!e || !out_shift) return GDL_E_INVALID;
  if (!e->instances) return fail(e, GDL_E_INVALID, "no instances declared");
  *out_shift = e->seg_shift;
  return GDL_OK;
}

gdl_status gdl_lie_instance_iterations(gdl_engine *e, int32_t lie, uint64_t *out, int32_t n) {
  CHECK_LIE(e, lie);
  const LieHost &L = e->lies[lie];
  if (!out || n < 0) return GDL_E_INVALID;
  if (!L.d_inst_last || (u32)n > L.n_inst)
    return fail(e, GDL_E_INVALID, "the LIE did not run in the batched form with %d instances", n);
  std::vector<u64> last(L.n_inst);
  CK(e, cudaMemcpyAsync(last.data(), L.d_inst_last, L.n_inst * sizeof(u64),
                        cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  // An instance's own loop would stop after the first pass without new
  // tuples: passes = last productive iteration + 2, or 1 (src/lie.cu:208-215).
  for (int i = 0; i < n; i++) out[i] = last[i] ? last[i] + 1 : 1;
  return GDL_OK;
}

// Size and digest of every instance's tuples in a FULL bitmap (local ids),
// from per-tile popcounts, their per-instance prefix, and k_inst_digest.
static gdl_status bitmap_stats(gdl_engine *e, const u32 *bm, const DenseMap &map,
                               const std::vector<SegInfo> &segs, std::vector<u64> &size,
                               std::vector<u64> &digest) {
  const u64 tiles = map.words / kBmTileWords;
  u32 *d_pop = nullptr;
  u64 *d_rank = nullptr, *d_acc = nullptr;
  TRY(dalloc(e, (void **)&d_pop, tiles * sizeof(u32)));
  TRY(dalloc(e, (void **)&d_rank, tiles * sizeof(u64)));
  TRY(dalloc(e, (void **)&d_acc, segs.size() * sizeof(u64)));
  k_inst_tile_pop<<<grid_for(e, tiles, 1, 8), 256, 0, e->s>>>(bm, map, d_pop);
  std::vector<u32> pop(tiles);
  CK(e, cudaMemcpyAsync(pop.data(), d_pop, tiles * sizeof(u32), cudaMemcpyDeviceToHost, e->s));
  CK(e, cudaStreamSynchronize(e->s));
  std::vector<u64> rank(tiles);
  size.assign(segs.size(), 0);
  for (size_t i = 0, t = 0; i < segs.size(); i++) {
    const u64 region = round_up((u64)segs[i].n << segs[i].row_shift, kBmTileWords);
    u64 run = 0;
    for (u64 k = 0; k < region / kBmTileWords; k++, t++) {
      rank[t] = run;
      run += pop[t];
    }
    size[i] = run;
  }
  CK(e, cudaMemcpyAsync(d_rank, rank.data(), tiles * sizeof(u64), cudaMemcpyHostToDevice, e->s));
  CK(e, cudaMemsetAsync(d_acc, 0, segs.size() * sizeof(u64), e->s));
  k_inst_digest<<<grid_for(e, tiles, 1, 8), 256, 0, e->s>>>(bm, map, d_rank, d_acc);
  std::vector<u64> acc(segs.size());
  CK(e, cudaMemcpyAsync(acc.data(), d_acc, acc.size() * sizeof(u64), cudaMemcpyDeviceToHost,
                        e->s));
  CK(e, cudaStreamSynchronize(e->s));
  dfree(e, d_pop);
  dfree(e, d_rank);
  dfree(e, d_acc);
  digest.resize(segs.size());
  for (size_t i = 0; i < segs.size(); i++) digest[i] = mix64(acc[i] ^ size[i]);
  return GDL_OK;
}

gdl_status gdl_relation_instance_stats(gdl_engine *e, int32_t rel, uint64_t *sizes,
                                       uint64_t *digests, int32_t n) {
  CHECK_REL(e, rel);
  if (!e->instances) return fail(e, GDL_E_INVALID, "no instances declared");
  if (n < 0 || (u32)n > e->segs.size() || (n && (!sizes || !digests))) return GDL_E_INVALID;
  const RelHost &rh = e->rels[rel];
  if (!rh.bm_valid || rh.bm_words != e->seg_words)
    return fail(e, GDL_E_INVALID, "relation %s has no FULL bitmap of the batched form",
                rh.name.c_str());
  TRY(pull(e));
  const DenseMap map{e->d_segs, e->d_tile_inst, (u32)e->segs.size(), e->seg_shift, e->seg_words};
  std::vector<u64> size, dig;
  TRY(bitmap_stats(e, e->h[rel].bmF, map, e->segs, size, dig));
  for (int i = 0; i < n; i++) {
    sizes[i] = size[i];
    digests[i] = dig[i];
  }
  return GDL_OK;
}

gdl_status gdl_lie_stats(gdl_engine *e, int32_t lie, double *out, int32_t n_out) {
  CHECK_LIE(e, lie);
  const LieHost &L = e->lies[lie];
  double v[9] = {L.ms,      (double)L.kernels,        (double)L.iterations,
                 (double)L.retries, (double)L.graph_launches, L.setup_ms,
                 L.grow_ms, L.graph_ms, L.graph_reused ? 1.0 : 0.0};
  for (int i = 0; i < n_out && i < 9; i++) out[i] = v[i];
  return GDL_OK;
}

}  // extern "C"

// ===========================================================================
// Allocation-free sort + deduplicate (gdl_sort_unique_rows_noalloc)
// ===========================================================================
// Some callers cannot allocate device memory: code running inside another
// library's memory arena, or a process that has handed all of HBM to a
// fixed-size pool before it starts.  For them this entry point sorts and
// deduplicates rows with the same kernels load_relation uses (pack, onesweep
// radix sort, merge-path dedup, unpack) but takes every byte of scratch from
// one file-scope device array of fixed size, which each GPU that loads the
// library holds until the process exits.
namespace {

constexpr u64 kNoAllocMaxRows = 1ull << 17;  // 131,072 rows per call
constexpr u64 kNoAllocSortTiles = kNoAllocMaxRows / kSortTile + 2;
constexpr u64 kNoAllocMergeTiles = (2 * kNoAllocMaxRows) / kMergeTile + 2;

// Byte layout of the scratch array.  The four key buffers come first; every
// byte after kNaCtrl is control state that must start at zero on each call.
constexpr u64 kNaKeys = 0;                                    // packed input
constexpr u64 kNaPing = kNaKeys + 8 * kNoAllocMaxRows;        // sort ping-pong
constexpr u64 kNaUniq = kNaPing + 8 * kNoAllocMaxRows;        // FULL' of the merge
constexpr u64 kNaDelta = kNaUniq + 8 * kNoAllocMaxRows;       // DELTA of the merge
constexpr u64 kNaStatus = kNaDelta + 8 * kNoAllocMaxRows;     // sort look-back words
constexpr u64 kNaCtrl = kNaStatus + 4 * kMaxPasses * kNoAllocSortTiles * kRadix;
constexpr u64 kNaOffsets = kNaCtrl;                                   // u32 [8][256]
constexpr u64 kNaCounters = kNaOffsets + 4 * kMaxPasses * kRadix;     // u32 [9] (+pad)
constexpr u64 kNaLbFlag = kNaCounters + 64;                           // u32 [tiles]
constexpr u64 kNaLbAgg = kNaLbFlag + 4 * kNoAllocMergeTiles + 256;    // u64 [tiles]
constexpr u64 kNaLbInc = kNaLbAgg + 8 * kNoAllocMergeTiles;           // u64 [tiles]
constexpr u64 kNaParts = kNaLbInc + 8 * kNoAllocMergeTiles;           // u64 [tiles + 1]
constexpr u64 kNaCtl = ((kNaParts + 8 * (kNoAllocMergeTiles + 1)) + 255) / 256 * 256;
constexpr u64 kNaRecs = kNaCtl + (sizeof(Ctl) + 255) / 256 * 256;     // LaunchRec [4]
constexpr u64 kNaDarr = kNaRecs + 256;                                // DArr [4]
constexpr u64 kNaScalars = kNaDarr + 256;                             // u64 [4]
constexpr u64 kNaBytes = kNaScalars + 256;

}  // namespace

// The scratch.  In host code this name is only a host-side stand-in for the
// device array: its device address comes from cudaGetSymbolAddress, once per
// device, and only that address is passed to kernels.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {

std::mutex g_noalloc_mutex;
void *g_noalloc_addr[64] = {nullptr};  // device address of the scratch, per device

__global__ void k_noalloc_init(unsigned char *base, u64 rows) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  DArr *d = reinterpret_cast<DArr *>(base + kNaDarr);
  d[0] = DArr{reinterpret_cast<u64 *>(base + kNaKeys), rows, kNoAllocMaxRows};   // NEWT
  d[1] = DArr{reinterpret_cast<u64 *>(base + kNaDelta), 0, 0};                   // empty FULL
  d[2] = DArr{reinterpret_cast<u64 *>(base + kNaUniq), 0, kNoAllocMaxRows};      // FULL'
  d[3] = DArr{reinterpret_cast<u64 *>(base + kNaDelta), 0, kNoAllocMaxRows};     // DELTA
  // the bounded waits' limit (the control block was zeroed)
  reinterpret_cast<Ctl *>(base + kNaCtl)->spin_limit = kSpinLimit;
}

__global__ void k_noalloc_unpack(const DArr *keys, u64 *rows) {
  const u64 n = keys->n;
  for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (u64)gridDim.x * blockDim.x) {
    const u64 k = keys->ptr[i];
    rows[2 * i] = key_c0(k);
    rows[2 * i + 1] = key_c1(k);
  }
}

gdl_status noalloc_fail(gdl_status code, const char *msg) {
  g_engineless_error = msg;
  return code;
}

#define NA_CK(call)                                                              \
  do {                                                                           \
    cudaError_t _r = (call);                                                     \
    if (_r != cudaSuccess) {                                                     \
      g_engineless_error = std::string(#call) + ": " + cudaGetErrorString(_r);   \
      return GDL_E_CUDA;                                                         \
    }                                                                            \
  } while (0)

}  // namespace

extern "C" gdl_status gdl_sort_unique_rows_noalloc(const uint64_t *device_rows, uint64_t rows,
                                                   uint64_t *device_out_rows, uint64_t *out_rows,
                                                   void *stream) {
  if (!out_rows || (rows && (!device_rows || !device_out_rows)))
    return noalloc_fail(GDL_E_INVALID, "gdl_sort_unique_rows_noalloc: null argument");
  *out_rows = 0;
  if (rows > kNoAllocMaxRows) {
    char msg[160];
    snprintf(msg, sizeof msg,
             "gdl_sort_unique_rows_noalloc: %llu rows exceed the fixed scratch limit of %llu rows",
             (unsigned long long)rows, (unsigned long long)kNoAllocMaxRows);
    return noalloc_fail(GDL_E_CAPACITY, msg);
  }
  if (rows == 0) return GDL_OK;
  int dev = 0;
  NA_CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return noalloc_fail(GDL_E_UNSUPPORTED, "device ordinal above 63");
  unsigned char *base = nullptr;
  {
    // Set-up, once per device, with that device current: the scratch
    // array's device address and the kernels' shared-memory attributes,
    // both under the lock so that two threads' first calls do not race.
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[dev]) {
      void *p = nullptr;
      NA_CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
      NA_CK(cudaFuncSetAttribute(k_sort_hist<kRadixBits>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSortSmemBytes));
      NA_CK(cudaFuncSetAttribute(k_sort_pass<kRadixBits>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSortSmemBytes));
      NA_CK(cudaFuncSetAttribute(k_merge_diff, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kMergeSmemBytes));
      g_noalloc_addr[dev] = p;
    }
    base = static_cast<unsigned char *>(g_noalloc_addr[dev]);
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int sms = 148;
  NA_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  // The array keeps the previous call's contents: zero the control state.
  NA_CK(cudaMemsetAsync(base + kNaCtrl, 0, kNaBytes - kNaCtrl, s));
  k_noalloc_init<<<1, 32, 0, s>>>(base, rows);
  u64 *keys = reinterpret_cast<u64 *>(base + kNaKeys);
  u64 *scal = reinterpret_cast<u64 *>(base + kNaScalars);  // [0] max value, [1] bad flag
  auto blocks = [&](u64 work, u64 per, int per_sm) {
    u64 g = (work + per - 1) / per, lim = (u64)sms * per_sm;
    return (int)std::max<u64>(1, std::min(g, lim));
  };
  k_pack_rows<<<blocks(rows, 256, 8), 256, 0, s>>>(reinterpret_cast<const u64 *>(device_rows),
                                                    rows, keys, scal,
                                                    reinterpret_cast<u32 *>(scal + 1));
  NA_CK(cudaGetLastError());
  u64 host_scal[2] = {0, 0};
  NA_CK(cudaMemcpyAsync(host_scal, scal, sizeof host_scal, cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  if (host_scal[1])
    return noalloc_fail(GDL_E_UNSUPPORTED, "gdl_sort_unique_rows_noalloc: values must be below 2^32");
  int kbits = 1;
  while (kbits < 64 && (host_scal[0] >> kbits)) kbits++;
  Ctl *ctl = reinterpret_cast<Ctl *>(base + kNaCtl);
  DArr *d = reinterpret_cast<DArr *>(base + kNaDarr);
  LaunchRec *recs = reinterpret_cast<LaunchRec *>(base + kNaRecs);
  SortArgs a;
  memset(&a, 0, sizeof a);
  a.keys = &d[0];
  a.buf0 = keys;
  a.buf1 = reinterpret_cast<u64 *>(base + kNaPing);
  a.cap = kNoAllocMaxRows;
  a.kbits = kbits;
  a.passes = std::max(1, (2 * kbits + 7) / 8);
  a.offsets = reinterpret_cast<u32 *>(base + kNaOffsets);
  a.status = reinterpret_cast<u32 *>(base + kNaStatus);
  a.max_tiles = kNoAllocSortTiles;
  a.counters = reinterpret_cast<u32 *>(base + kNaCounters);
  a.ctl = ctl;
  k_sort_hist<kRadixBits><<<blocks(rows, (u64)kSortTile * 4, 2), kSortBlock, kSortSmemBytes, s>>>(a);
  for (int p = 0; p < a.passes; p++)
    k_sort_pass<kRadixBits><<<blocks(rows, kSortTile, 4), kSortBlock, kSortSmemBytes, s>>>(a, p);
  MergeArgs m;
  memset(&m, 0, sizeof m);
  m.newt = &d[0];
  m.a = (a.passes & 1) ? a.buf1 : a.buf0;
  m.full = &d[1];
  m.full_next = &d[2];
  m.delta_next = &d[3];
  m.c_newt_n = scal + 2;
  m.rec = &recs[0];
  m.lb = Lb{reinterpret_cast<u32 *>(base + kNaLbFlag), reinterpret_cast<u64 *>(base + kNaLbAgg),
            reinterpret_cast<u64 *>(base + kNaLbInc)};
  m.parts = reinterpret_cast<u64 *>(base + kNaParts);
  m.parts_cap = kNoAllocMergeTiles + 1;
  m.ctl = ctl;
  m.rel = 0;
  k_merge_partition<<<blocks(rows / kMergeTile + 2, 256, 8), 256, 0, s>>>(m);
  k_merge_diff<<<blocks(rows, kMergeTile, 4), kMergeBlock, kMergeSmemBytes, s>>>(m);
  k_noalloc_unpack<<<blocks(rows, 256, 8), 256, 0, s>>>(&d[2],
                                                         reinterpret_cast<u64 *>(device_out_rows));
  NA_CK(cudaGetLastError());
  DArr uniq;
  Ctl c;
  NA_CK(cudaMemcpyAsync(&uniq, &d[2], sizeof uniq, cudaMemcpyDeviceToHost, s));
  NA_CK(cudaMemcpyAsync(&c, ctl, sizeof c, cudaMemcpyDeviceToHost, s));
  NA_CK(cudaStreamSynchronize(s));
  if (c.timeout || c.oob || c.overflow)
    return noalloc_fail(GDL_E_TIMEOUT, "gdl_sort_unique_rows_noalloc: device-side check failed");
  *out_rows = uniq.n;
  return GDL_OK;
}
