// oracle_bitset.cpp — second CPU oracle for the semi-naive fixpoint path,
// over bit matrices.  TEST INFRASTRUCTURE ONLY: tests and fixture scripts
// use it to check the CUDA engine; the product never links or calls it.
//
// The list oracle (oracle.cpp) materialises every candidate tuple of a join
// and sorts it, which cannot finish the 20,000-variable points-to analysis
// (about 13.7 T candidates for 0.56 G distinct tuples).  This oracle keeps
// each relation version as a D x D bit matrix over the id domain (bit
// (c0, c1) = tuple (c0, c1)) and evaluates a join as a boolean matrix
// product, so its cost follows the distinct rows touched, not the
// candidates.  It restates the same container-level semantics of the
// reference's LIE loop (src/lie.cu:26-274) as oracle.cpp, independently of
// it and of the CUDA engine:
//   * inputs are deduplicated at load (src/relation.cu:570-593);
//   * at loop start DELTA := the first |FULL| rows of FULL's raw load-order
//     buffer (src/lie.cu:49-59, copy_relation_container,
//     src/relation.cu:764-795);
//   * a FULL-source Copy runs once per LIE (src/lie.cu:69-75); Copy and ACopy
//     ignore the predicate (src/relation.cu:390-403);
//   * a join whose outer is empty does nothing; a join whose inner is empty
//     zeroes the OUTER's count (src/join.cu:38-45); a Copy from an empty
//     source zeroes the destination NEWT (src/copy.cu:24-27); an ACopy from an
//     empty source clears it (src/acopy.cu:14-18);
//   * join outputs are unioned into NEWT (src/join.cu:130-261); tmp
//     relations concatenate without dedup there (src/join.cu:226-254), which
//     is the same set — a tmp NEWT is read only as a set of outer rows;
//   * tmp NEWTs are cleared after the operators (src/lie.cu:85-87);
//   * the update step is set_difference(NEWT, FULL) -> DELTA and
//     flush_delta's merge (src/lie.cu:93-198, src/relation.cu:405-521);
//   * the iteration count includes the final empty pass and the loop stops
//     when iteration > max_iteration (src/lie.cu:208-215).
// Scope: arity 2, one index column, no dependent column, hooks that select
// columns (no constants), ids below 2^15.  Anything else is refused with
// GDL_E_UNSUPPORTED.  The entry points mirror oracle.h with the prefix orb_.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace {

constexpr int32_t OK = 0, E_INVALID = 1, E_UNSUPPORTED = 4, E_CAPACITY = 6;
constexpr int DELTA = 0, FULL = 1, NEWT = 2;
constexpr int PRED_NONE = 0, PRED_NE = 1, PRED_EQ = 2, PRED_LT = 3, PRED_LE = 4,
              PRED_GT = 5, PRED_GE = 6;
constexpr uint64_t kMaxDomain = 1ull << 15;

inline uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014); the digest the engines
  // share is defined with it.
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

// 64 x 64 bit-matrix transpose in place: bit c of a[r] moves to bit r of
// a[c].  Recursive block exchange (Warren, Hacker's Delight, 2nd ed., 7-3):
// swap the two off-diagonal 32x32 blocks, then the 16x16 blocks inside each
// quadrant, and so on down to single bits.
inline void transpose64(uint64_t a[64]) {
  uint64_t m = 0x00000000FFFFFFFFull;
  for (int j = 32; j != 0; j >>= 1, m ^= (m << j)) {
    for (int k = 0; k < 64; k = ((k | j) + 1) & ~j) {
      const uint64_t t = ((a[k] >> j) ^ a[k | j]) & m;
      a[k] ^= t << j;
      a[k | j] ^= t;
    }
  }
}

// A square bit matrix of R = 64 * W rows of W words.  Bit (r, c) is bit
// c % 64 of word c / 64 of row r, so reading rows in order and bits from the
// least significant up lists the tuples in the reference's order.
struct Bits {
  std::vector<uint64_t> w;  // empty: all zero
  uint64_t n = 0;           // number of set bits (kept current)
};

struct Op {
  int kind;  // 0 join, 1 copy, 2 acopy
  int inner = -1, inner_ver = FULL, outer = -1, outer_ver = DELTA, out = -1;
  int g0 = 0, g1 = 0;  // output column selections (INNER c = c, OUTER c = 16 + c)
  int pred = PRED_NONE, pa = 0, pb = 0;
  bool copied = false;  // RelationalCopy::copied (relational_algebra.cuh:72)
};

struct Lie {
  std::vector<int> update, statics, tmps;
  std::vector<Op> ops;
  int64_t max_iteration = INT32_MAX;  // include/lie.cuh:30
  bool reload_full = true;            // include/lie.cuh:29
  std::vector<uint64_t> trace;
  double seconds = 0;
};

struct Rel {
  std::string name;
  bool index_flag = true, tmp_flag = false;
  Bits full, delta, newt;
  // The FULL container's count was zeroed by an empty-inner join
  // (src/join.cu:42-45) while tuple_full, which `full` also holds, keeps
  // the rows; the next non-empty flush or the end-of-loop reload restores it.
  bool full_zeroed = false;
  // FULL's raw buffer in load order (packed c0 << 32 | c1), or, after a
  // reload at the end of a loop, the sorted FULL of that moment (raw_full).
  std::vector<uint64_t> raw;
  bool raw_is_full = false;
  Bits raw_full;
};

struct Engine {
  std::string err;
  int threads = 1;
  uint32_t W = 1;  // words per row; the domain is R = 64 W ids
  std::vector<Rel> rels;
  std::vector<Lie> lies;

  int32_t fail(int32_t code, const std::string &m) {
    err = m;
    return code;
  }
  uint64_t R() const { return 64ull * W; }
  size_t words() const { return (size_t)R() * W; }

  // -- bit matrix helpers ----------------------------------------------------
  void alloc(Bits &b) {
    if (b.w.empty()) {
      b.w.assign(words(), 0);
      b.n = 0;
    }
  }
  void clear(Bits &b) {
    if (b.w.empty()) return;
    uint64_t *p = b.w.data();
    const int64_t nw = (int64_t)b.w.size();
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t i = 0; i < nw; i++) p[i] = 0;
    b.n = 0;
  }
  void recount(Bits &b) {
    if (b.w.empty()) {
      b.n = 0;
      return;
    }
    const uint64_t *p = b.w.data();
    const int64_t nw = (int64_t)b.w.size();
    uint64_t s = 0;
#pragma omp parallel for reduction(+ : s) schedule(static) num_threads(threads)
    for (int64_t i = 0; i < nw; i++) s += (uint64_t)__builtin_popcountll(p[i]);
    b.n = s;
  }
  // dst |= src
  void or_into(Bits &dst, const Bits &src) {
    if (src.w.empty() || src.n == 0) return;
    alloc(dst);
    uint64_t *d = dst.w.data();
    const uint64_t *s = src.w.data();
    const int64_t nw = (int64_t)src.w.size();
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t i = 0; i < nw; i++) d[i] |= s[i];
    recount(dst);
  }
  // dst = transpose(src); dst is overwritten.
  void transpose(const Bits &src, Bits &dst) {
    alloc(dst);
    const uint32_t w = W;
    const uint64_t *s = src.w.data();
    uint64_t *d = dst.w.data();
#pragma omp parallel for collapse(2) schedule(static) num_threads(threads)
    for (int64_t bi = 0; bi < (int64_t)w; bi++) {
      for (int64_t bj = 0; bj < (int64_t)w; bj++) {
        uint64_t a[64];
        for (int r = 0; r < 64; r++) a[r] = s[(size_t)(bi * 64 + r) * w + bj];
        transpose64(a);
        for (int r = 0; r < 64; r++) d[(size_t)(bj * 64 + r) * w + bi] = a[r];
      }
    }
    dst.n = src.n;
  }
  void set_bit(Bits &b, uint64_t r, uint64_t c) { b.w[r * W + (c >> 6)] |= 1ull << (c & 63); }
  static void set_bit_atomic(uint64_t *row, uint64_t c) {
    __atomic_fetch_or(row + (c >> 6), 1ull << (c & 63), __ATOMIC_RELAXED);
  }

  // Re-lay every matrix out for a wider domain.
  void grow(uint32_t newW) {
    if (newW <= W) return;
    const uint32_t oldW = W;
    auto relayout = [&](Bits &b) {
      if (b.w.empty()) return;
      std::vector<uint64_t> nw((size_t)64 * newW * newW, 0);
      for (uint64_t r = 0; r < 64ull * oldW; r++)
        std::memcpy(&nw[r * newW], &b.w[r * oldW], oldW * sizeof(uint64_t));
      b.w.swap(nw);
    };
    for (Rel &r : rels) {
      relayout(r.full);
      relayout(r.delta);
      relayout(r.newt);
      relayout(r.raw_full);
    }
    W = newW;
  }

  // Per-row counts and, for sparse rows, their set columns.
  struct RowInfo {
    std::vector<uint32_t> cnt;
    std::vector<uint64_t> off;  // sparse-position offsets (rows with cnt <= kSparse)
    std::vector<uint32_t> pos;
  };
  static constexpr uint32_t kSparse = 8;
  void row_info(const Bits &b, RowInfo &ri) {
    const uint64_t rows = R();
    ri.cnt.assign(rows, 0);
    const uint64_t *p = b.w.data();
    const uint32_t w = W;
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t r = 0; r < (int64_t)rows; r++) {
      uint32_t c = 0;
      for (uint32_t j = 0; j < w; j++) c += (uint32_t)__builtin_popcountll(p[r * w + j]);
      ri.cnt[r] = c;
    }
    ri.off.assign(rows + 1, 0);
    for (uint64_t r = 0; r < rows; r++)
      ri.off[r + 1] = ri.off[r] + (ri.cnt[r] <= kSparse ? ri.cnt[r] : 0);
    ri.pos.assign(ri.off[rows], 0);
#pragma omp parallel for schedule(static) num_threads(threads)
    for (int64_t r = 0; r < (int64_t)rows; r++) {
      if (ri.cnt[r] == 0 || ri.cnt[r] > kSparse) continue;
      uint64_t o = ri.off[r];
      for (uint32_t j = 0; j < w; j++) {
        uint64_t x = p[r * w + j];
        while (x) {
          ri.pos[o++] = j * 64 + (uint32_t)__builtin_ctzll(x);
          x &= x - 1;
        }
      }
    }
  }
  // dst_row |= row k of src (through its sparse positions when it has few).
  inline void or_row(uint64_t *dst, const Bits &src, const RowInfo &ri, uint64_t k) const {
    const uint32_t c = ri.cnt[k];
    if (c <= kSparse) {
      for (uint64_t i = ri.off[k]; i < ri.off[k + 1]; i++) {
        const uint32_t v = ri.pos[i];
        dst[v >> 6] |= 1ull << (v & 63);
      }
      return;
    }
    const uint64_t *s = src.w.data() + k * W;
    for (uint32_t j = 0; j < W; j++) dst[j] |= s[j];
  }

  // T = { (a, b) : inner(k, a) and outer(k, b) } (or its transpose when
  // `swap`), T zero on entry.  Every key k is charged to one of two
  // gathers: by rows a of innerᵀ (T[a] |= outer[k]) or by rows b of outerᵀ
  // (Tᵀ[b] |= inner[k]), whichever touches fewer words for that key.  Each
  // gather writes its own destination rows, so the rows run in parallel.
  void product(const Bits &inner, const Bits &outer, Bits &T, bool swap) {
    RowInfo ri, ro;
    row_info(inner, ri);
    row_info(outer, ro);
    const uint64_t rows = R();
    auto cost = [&](uint32_t c) { return (uint64_t)std::min<uint32_t>(c, W); };
    std::vector<uint64_t> maskA(W, 0), maskB(W, 0);
    bool anyA = false, anyB = false;
    for (uint64_t k = 0; k < rows; k++) {
      if (!ri.cnt[k] || !ro.cnt[k]) continue;
      const uint64_t a = (uint64_t)ri.cnt[k] * cost(ro.cnt[k]);
      const uint64_t b = (uint64_t)ro.cnt[k] * cost(ri.cnt[k]);
      if (a <= b) {
        maskA[k >> 6] |= 1ull << (k & 63);
        anyA = true;
      } else {
        maskB[k >> 6] |= 1ull << (k & 63);
        anyB = true;
      }
    }
    Bits X, Tt;
    alloc(T);
    auto gather = [&](const Bits &side, const std::vector<uint64_t> &mask, const Bits &src,
                      const RowInfo &rs, Bits &dst) {
      Bits sideT;
      transpose(side, sideT);
      const uint32_t w = W;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
      for (int64_t x = 0; x < (int64_t)rows; x++) {
        const uint64_t *st = sideT.w.data() + (uint64_t)x * w;
        uint64_t *d = dst.w.data() + (uint64_t)x * w;
        for (uint32_t j = 0; j < w; j++) {
          uint64_t m = st[j] & mask[j];
          while (m) {
            const uint64_t k = (uint64_t)j * 64 + (uint64_t)__builtin_ctzll(m);
            m &= m - 1;
            or_row(d, src, rs, k);
          }
        }
      }
    };
    // A keys: rows a of innerᵀ gather outer rows -> (a, b) entries.
    // B keys: rows b of outerᵀ gather inner rows -> (b, a) entries.
    Bits *dstA = &T, *dstB = &Tt;
    if (swap) std::swap(dstA, dstB);
    alloc(Tt);
    if (anyA) gather(inner, maskA, outer, ro, *dstA);
    if (anyB) gather(outer, maskB, inner, ri, *dstB);
    // fold the transposed partial into T
    recount(Tt);
    if (Tt.n) {
      transpose(Tt, X);
      uint64_t *d = T.w.data();
      const uint64_t *s = X.w.data();
      const int64_t nw = (int64_t)T.w.size();
#pragma omp parallel for schedule(static) num_threads(threads)
      for (int64_t i = 0; i < nw; i++) d[i] |= s[i];
    }
    recount(T);
  }

  static inline uint64_t sel(int g, uint64_t k, uint64_t a, uint64_t b) {
    // INNER(0) = OUTER(0) = the join key, INNER(1) = a, OUTER(1) = b.
    if (g == 0 || g == 16) return k;
    return g == 1 ? a : b;
  }
  static inline bool pred_ok(int kind, uint64_t x, uint64_t y) {
    switch (kind) {
      case PRED_NE: return x != y;
      case PRED_EQ: return x == y;
      case PRED_LT: return x < y;
      case PRED_LE: return x <= y;
      case PRED_GT: return x > y;
      case PRED_GE: return x >= y;
    }
    return true;
  }

  // Any other column selection or predicate: every candidate enumerated.
  void product_generic(const Bits &inner, const Bits &outer, Bits &T, const Op &op) {
    alloc(T);
    const uint64_t rows = R();
    const uint32_t w = W;
    uint64_t *t = T.w.data();
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads)
    for (int64_t k = 0; k < (int64_t)rows; k++) {
      const uint64_t *ir = inner.w.data() + (uint64_t)k * w;
      const uint64_t *orow = outer.w.data() + (uint64_t)k * w;
      bool any_o = false;
      for (uint32_t j = 0; j < w && !any_o; j++) any_o = orow[j] != 0;
      if (!any_o) continue;
      for (uint32_t ja = 0; ja < w; ja++) {
        for (uint64_t xa = ir[ja]; xa; xa &= xa - 1) {
          const uint64_t a = (uint64_t)ja * 64 + (uint64_t)__builtin_ctzll(xa);
          for (uint32_t jb = 0; jb < w; jb++) {
            for (uint64_t xb = orow[jb]; xb; xb &= xb - 1) {
              const uint64_t b = (uint64_t)jb * 64 + (uint64_t)__builtin_ctzll(xb);
              const uint64_t o[2] = {sel(op.g0, k, a, b), sel(op.g1, k, a, b)};
              if (op.pred != PRED_NONE && !pred_ok(op.pred, o[op.pa], o[op.pb])) continue;
              set_bit_atomic(t + o[0] * w, o[1]);
            }
          }
        }
      }
    }
    recount(T);
  }

  // Projection of a version through a copy hook (src/relation.cu:390-403).
  void project(const Bits &src, int g0, int g1, Bits &T) {
    if (g0 == 0 && g1 == 1) {
      alloc(T);
      std::memcpy(T.w.data(), src.w.data(), src.w.size() * sizeof(uint64_t));
      T.n = src.n;
      return;
    }
    if (g0 == 1 && g1 == 0) {
      transpose(src, T);
      return;
    }
    alloc(T);
    const uint64_t rows = R();
    const uint32_t w = W;
    uint64_t *t = T.w.data();
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t k = 0; k < (int64_t)rows; k++) {
      const uint64_t *s = src.w.data() + (uint64_t)k * w;
      for (uint32_t j = 0; j < w; j++) {
        for (uint64_t x = s[j]; x; x &= x - 1) {
          const uint64_t v = (uint64_t)j * 64 + (uint64_t)__builtin_ctzll(x);
          const uint64_t o0 = g0 == 0 ? (uint64_t)k : v, o1 = g1 == 0 ? (uint64_t)k : v;
          set_bit_atomic(t + o0 * w, o1);
        }
      }
    }
    recount(T);
  }

  // -- relations -------------------------------------------------------------
  uint64_t full_size(const Rel &r) const { return r.full_zeroed ? 0 : r.full.n; }
  Bits *version(Rel &r, int ver) { return ver == DELTA ? &r.delta : ver == FULL ? &r.full : &r.newt; }
  bool empty_version(Rel &r, int ver) { return ver == FULL ? full_size(r) == 0 : version(r, ver)->n == 0; }
  void zero_version(Rel &r, int ver) {
    if (ver == FULL)
      r.full_zeroed = true;
    else
      clear(*version(r, ver));
  }

  int32_t rel_create(const char *name, int arity, int icols, int dep, int index_flag,
                     int tmp_flag, int32_t *out) {
    if (arity != 2) return fail(E_UNSUPPORTED, "bitset oracle: arity 2 only");
    if (icols != 1) return fail(E_UNSUPPORTED, "bitset oracle: one index column only");
    if (dep != 0) return fail(E_UNSUPPORTED, "bitset oracle: no dependent column");
    Rel r;
    r.name = name ? name : "";
    r.index_flag = index_flag != 0;
    r.tmp_flag = tmp_flag != 0;
    rels.push_back(std::move(r));
    *out = (int32_t)rels.size() - 1;
    return OK;
  }

  // load_relation (src/relation.cu:815-838): FULL = the set of the rows,
  // DELTA and NEWT fresh and empty; the rows are kept in load order.
  int32_t rel_load(int id, const uint64_t *rows, uint64_t n) {
    uint64_t mx = 0;
    for (uint64_t i = 0; i < 2 * n; i++) mx = std::max(mx, rows[i]);
    if (n && mx >= kMaxDomain) return fail(E_UNSUPPORTED, "bitset oracle: ids must be below 2^15");
    if (n) grow((uint32_t)((mx + 64) / 64));
    Rel &r = rels[id];
    clear(r.full);
    clear(r.delta);
    clear(r.newt);
    r.full_zeroed = false;
    r.raw.resize(n);
    r.raw_is_full = false;
    r.raw_full = Bits();
    if (n) alloc(r.full);
    for (uint64_t i = 0; i < n; i++) {
      r.raw[i] = rows[2 * i] << 32 | rows[2 * i + 1];
      set_bit(r.full, rows[2 * i], rows[2 * i + 1]);
    }
    recount(r.full);
    return OK;
  }

  // Rows of a version in the reference's order, or just their count.
  template <class F>
  void for_each_row_ranked(const Bits &b, F f) {
    const uint64_t rows = R();
    const uint32_t w = W;
    std::vector<uint64_t> start(rows + 1, 0);
    for (uint64_t r = 0; r < rows; r++) {
      uint64_t c = 0;
      for (uint32_t j = 0; j < w; j++) c += (uint64_t)__builtin_popcountll(b.w[r * w + j]);
      start[r + 1] = start[r] + c;
    }
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads)
    for (int64_t r = 0; r < (int64_t)rows; r++) {
      uint64_t i = start[r];
      for (uint32_t j = 0; j < w; j++)
        for (uint64_t x = b.w[(uint64_t)r * w + j]; x; x &= x - 1)
          f(i++, (uint64_t)r, (uint64_t)j * 64 + (uint64_t)__builtin_ctzll(x));
    }
  }

  int32_t rel_size(int id, int ver, uint64_t *out) {
    Rel &r = rels[id];
    *out = ver == FULL ? full_size(r) : version(r, ver)->n;
    return OK;
  }

  int32_t rel_export(int id, int ver, uint64_t *out, uint64_t cap, uint64_t *out_n) {
    Rel &r = rels[id];
    uint64_t n = 0;
    rel_size(id, ver, &n);
    *out_n = n;
    if (n > cap) return fail(E_CAPACITY, "export buffer too small");
    if (n == 0) return OK;
    for_each_row_ranked(*version(r, ver), [&](uint64_t i, uint64_t c0, uint64_t c1) {
      out[2 * i] = c0;
      out[2 * i + 1] = c1;
    });
    return OK;
  }

  // Same digest as the other engines: sum over sorted rows of a hash of
  // (position, columns), finished with the row count.
  int32_t rel_digest(int id, int ver, uint64_t *out) {
    Rel &r = rels[id];
    uint64_t n = 0;
    rel_size(id, ver, &n);
    if (n) {
      std::atomic<uint64_t> s{0};
      for_each_row_ranked(*version(r, ver), [&](uint64_t i, uint64_t c0, uint64_t c1) {
        uint64_t h = mix64(i);
        h = mix64(h ^ c0);
        h = mix64(h ^ c1);
        s.fetch_add(h, std::memory_order_relaxed);
      });
      *out = mix64(s.load() ^ n);
    } else {
      *out = mix64(0);
    }
    return OK;
  }

  // -- operators ---------------------------------------------------------------
  // RelationalJoin::operator() (src/join.cu:12-270).
  void run_join(Op &op) {
    Rel &I = rels[op.inner];
    Rel &O = rels[op.outer];
    const int iv = op.inner_ver == DELTA ? DELTA : FULL;  // join.cu:14-19
    if (empty_version(O, op.outer_ver)) return;           // join.cu:38-41
    if (empty_version(I, iv)) {                           // join.cu:42-45
      zero_version(O, op.outer_ver);
      return;
    }
    const Bits &inner = *version(I, iv);
    const Bits &outer = *version(O, op.outer_ver);
    Bits T;
    const bool ab = op.g0 == 1 && op.g1 == 17, ba = op.g0 == 17 && op.g1 == 1;
    const bool ne01 = op.pred == PRED_NE && ((op.pa == 0 && op.pb == 1) || (op.pa == 1 && op.pb == 0));
    if ((ab || ba) && (op.pred == PRED_NONE || ne01)) {
      product(inner, outer, T, ba);
      if (ne01) {  // drop the candidates (v, v)
        for (uint64_t v = 0; v < R(); v++) T.w[v * W + (v >> 6)] &= ~(1ull << (v & 63));
        recount(T);
      }
    } else {
      product_generic(inner, outer, T, op);
    }
    or_into(rels[op.out].newt, T);  // join.cu:130-261 (union into NEWT)
  }

  // RelationalCopy::operator() (src/copy.cu:12-95).
  void run_copy(Op &op) {
    Rel &S = rels[op.inner];
    Rel &D = rels[op.out];
    const int sv = op.inner_ver == DELTA ? DELTA : FULL;
    if (empty_version(S, sv)) {  // copy.cu:24-27
      clear(D.newt);
      return;
    }
    Bits T;
    project(*version(S, sv), op.g0, op.g1, T);
    or_into(D.newt, T);
  }

  // RelationalACopy::operator() (src/acopy.cu:12-50): NEWT(dest) replaced by
  // the projection of NEWT(src).
  void run_acopy(Op &op) {
    Rel &S = rels[op.inner];
    Rel &D = rels[op.out];
    if (S.newt.n == 0) {
      clear(D.newt);
      return;
    }
    Bits T;
    project(S.newt, op.g0, op.g1, T);
    clear(D.newt);
    or_into(D.newt, T);
  }

  // LIE::fixpoint_loop (src/lie.cu:26-274).
  int32_t fixpoint(Lie &L, uint64_t *out_iters) {
    auto t0 = std::chrono::steady_clock::now();
    L.trace.clear();
    for (int id : L.update) {  // lie.cu:49-59
      Rel &r = rels[id];
      if (r.full_zeroed) {  // tuple_full := the zero rows FULL shows
        clear(r.full);
        r.full_zeroed = false;
      }
      clear(r.delta);
      if (r.full.n == 0) continue;
      if (r.raw_is_full) {
        // The first |FULL| rows of the sorted snapshot: FULL only grows
        // between a reload and the next loop, so that is all of it.
        if (r.full.n < r.raw_full.n) {
          err = "bitset oracle: FULL shrank below its reloaded rows";
          return E_UNSUPPORTED;
        }
        or_into(r.delta, r.raw_full);
        continue;
      }
      alloc(r.delta);
      const uint64_t take = std::min<uint64_t>(r.full.n, r.raw.size());
      for (uint64_t i = 0; i < take; i++) set_bit(r.delta, r.raw[i] >> 32, r.raw[i] & 0xFFFFFFFFull);
      recount(r.delta);
    }
    int64_t it = 0;
    while (true) {
      for (Op &op : L.ops) {  // lie.cu:62-82
        if (op.kind == 0) {
          run_join(op);
        } else if (op.kind == 2) {
          run_acopy(op);
        } else if (op.inner_ver == FULL) {
          if (!op.copied) {
            run_copy(op);
            op.copied = true;
          }
        } else {
          run_copy(op);
        }
      }
      for (int id : L.tmps) clear(rels[id].newt);  // lie.cu:85-87
      bool fixpoint_flag = true;
      for (int id : L.update) {  // lie.cu:93-198
        Rel &r = rels[id];
        if (r.newt.n == 0) {  // lie.cu:114-121
          clear(r.delta);
          L.trace.insert(L.trace.end(), {(uint64_t)it, (uint64_t)id, UINT64_MAX, 0, r.full.n});
          continue;
        }
        // DELTA = NEWT \ tuple_full (lie.cu:131-138); FULL |= DELTA
        // (flush_delta, src/relation.cu:405-521).
        alloc(r.delta);
        alloc(r.full);
        {
          uint64_t *d = r.delta.w.data(), *f = r.full.w.data();
          const uint64_t *g = r.newt.w.data();
          const int64_t nw = (int64_t)words();
#pragma omp parallel for schedule(static) num_threads(threads)
          for (int64_t i = 0; i < nw; i++) {
            const uint64_t x = g[i] & ~f[i];
            d[i] = x;
            f[i] |= x;
          }
        }
        recount(r.delta);
        clear(r.newt);
        if (r.delta.n != 0) {
          fixpoint_flag = false;
          recount(r.full);
          r.full_zeroed = false;  // full->tuples = tuple_full
        }
        L.trace.insert(L.trace.end(),
                       {(uint64_t)it, (uint64_t)id, r.delta.n, r.delta.n, r.full.n});
      }
      it++;
      if (fixpoint_flag || it > L.max_iteration) break;  // lie.cu:208-215
    }
    if (L.reload_full) {  // lie.cu:219-254
      for (int id : L.update) {
        Rel &r = rels[id];
        r.full_zeroed = false;
        r.raw.clear();
        r.raw_is_full = true;
        clear(r.raw_full);
        or_into(r.raw_full, r.full);
        clear(r.delta);
        clear(r.newt);
      }
    }
    *out_iters = (uint64_t)it;
    L.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return OK;
  }
};

}  // namespace

struct orb_engine {
  Engine e;
};

extern "C" {

int32_t orb_engine_create(int32_t max_arity, int32_t threads, orb_engine **out) {
  if (!out) return E_INVALID;
  if (max_arity < 1 || max_arity > 2) return E_UNSUPPORTED;
  auto *e = new orb_engine;
  e->e.threads = threads > 0 ? threads : omp_get_max_threads();
  *out = e;
  return OK;
}

int32_t orb_engine_clear(orb_engine *e) {
  if (!e) return E_INVALID;
  const int t = e->e.threads;
  e->e = Engine();
  e->e.threads = t;
  return OK;
}

int32_t orb_engine_destroy(orb_engine *e) {
  delete e;
  return OK;
}

const char *orb_last_error(const orb_engine *e) { return e ? e->e.err.c_str() : "null engine"; }
int32_t orb_threads(const orb_engine *e) { return e ? e->e.threads : 0; }

#define ORB_REL(e, r)                                                          \
  do {                                                                          \
    if (!(e) || (r) < 0 || (r) >= (int)(e)->e.rels.size())                      \
      return (e) ? (e)->e.fail(E_INVALID, "bad relation id") : E_INVALID;       \
  } while (0)
#define ORB_LIE(e, l)                                                          \
  do {                                                                          \
    if (!(e) || (l) < 0 || (l) >= (int)(e)->e.lies.size())                      \
      return (e) ? (e)->e.fail(E_INVALID, "bad lie id") : E_INVALID;            \
  } while (0)

int32_t orb_relation_create(orb_engine *e, const char *name, int32_t arity, int32_t icols,
                            int32_t dep, int32_t index_flag, int32_t tmp_flag, int32_t *out) {
  if (!e || !out) return E_INVALID;
  return e->e.rel_create(name, arity, icols, dep, index_flag, tmp_flag, out);
}

int32_t orb_relation_load(orb_engine *e, int32_t rel, const uint64_t *rows, uint64_t n) {
  ORB_REL(e, rel);
  if (n && !rows) return e->e.fail(E_INVALID, "null rows");
  return e->e.rel_load(rel, rows, n);
}

int32_t orb_relation_size(orb_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  ORB_REL(e, rel);
  if (ver < 0 || ver > 2 || !out) return e->e.fail(E_INVALID, "bad version");
  return e->e.rel_size(rel, ver, out);
}

int32_t orb_relation_export(orb_engine *e, int32_t rel, int32_t ver, uint64_t *rows,
                            uint64_t cap, uint64_t *out_n) {
  ORB_REL(e, rel);
  if (ver < 0 || ver > 2 || !out_n) return e->e.fail(E_INVALID, "bad version");
  return e->e.rel_export(rel, ver, rows, cap, out_n);
}

int32_t orb_relation_digest(orb_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  ORB_REL(e, rel);
  if (ver < 0 || ver > 2 || !out) return e->e.fail(E_INVALID, "bad version");
  return e->e.rel_digest(rel, ver, out);
}

int32_t orb_lie_create(orb_engine *e, int32_t *out) {
  if (!e || !out) return E_INVALID;
  e->e.lies.emplace_back();
  *out = (int32_t)e->e.lies.size() - 1;
  return OK;
}

int32_t orb_lie_add_relation(orb_engine *e, int32_t lie, int32_t rel, int32_t static_flag) {
  ORB_LIE(e, lie);
  ORB_REL(e, rel);
  (static_flag ? e->e.lies[lie].statics : e->e.lies[lie].update).push_back(rel);
  return OK;
}

int32_t orb_lie_add_tmp_relation(orb_engine *e, int32_t lie, int32_t rel) {
  ORB_LIE(e, lie);
  ORB_REL(e, rel);
  e->e.lies[lie].tmps.push_back(rel);
  return OK;
}

// Hook encoding as in oracle.h / gdlog_b200.h: INNER(c) = c, OUTER(c) = 16 + c,
// SRC(c) = c, a constant in bits 8.. (GDL_PLUS), which this oracle refuses.
static int32_t orb_gen(orb_engine *e, const int32_t *gen, int32_t n, bool join, int *g0, int *g1) {
  if (!gen || n != 2) return e->e.fail(E_INVALID, "gen length != output arity");
  for (int j = 0; j < 2; j++) {
    if (gen[j] >> 8) return e->e.fail(E_UNSUPPORTED, "bitset oracle: no constants in hooks");
    const int g = gen[j];
    const bool ok = join ? (g == 0 || g == 1 || g == 16 || g == 17) : (g == 0 || g == 1);
    if (!ok) return e->e.fail(E_INVALID, "gen column out of range");
  }
  *g0 = gen[0];
  *g1 = gen[1];
  return OK;
}

int32_t orb_lie_add_join(orb_engine *e, int32_t lie, int32_t inner, int32_t inner_ver,
                         int32_t outer, int32_t outer_ver, int32_t output, const int32_t *gen,
                         int32_t gen_len, int32_t pred, int32_t pa, int32_t pb) {
  ORB_LIE(e, lie);
  ORB_REL(e, inner);
  ORB_REL(e, outer);
  ORB_REL(e, output);
  Op op;
  int32_t s = orb_gen(e, gen, gen_len, true, &op.g0, &op.g1);
  if (s) return s;
  if (pred < 0 || pred > PRED_GE) return e->e.fail(E_INVALID, "bad predicate");
  if (pred && (pa < 0 || pb < 0 || pa >= 2 || pb >= 2))
    return e->e.fail(E_INVALID, "predicate column out of range");
  op.kind = 0;
  op.inner = inner;
  op.inner_ver = inner_ver;
  op.outer = outer;
  op.outer_ver = outer_ver;
  op.out = output;
  op.pred = pred;
  op.pa = pa;
  op.pb = pb;
  e->e.lies[lie].ops.push_back(op);
  return OK;
}

int32_t orb_lie_add_copy(orb_engine *e, int32_t lie, int32_t src, int32_t src_ver, int32_t dest,
                         const int32_t *gen, int32_t gen_len) {
  ORB_LIE(e, lie);
  ORB_REL(e, src);
  ORB_REL(e, dest);
  Op op;
  int32_t s = orb_gen(e, gen, gen_len, false, &op.g0, &op.g1);
  if (s) return s;
  op.kind = 1;
  op.inner = src;
  op.inner_ver = src_ver;
  op.out = dest;
  e->e.lies[lie].ops.push_back(op);
  return OK;
}

int32_t orb_lie_add_acopy(orb_engine *e, int32_t lie, int32_t src, int32_t dest,
                          const int32_t *gen, int32_t gen_len) {
  ORB_LIE(e, lie);
  ORB_REL(e, src);
  ORB_REL(e, dest);
  Op op;
  int32_t s = orb_gen(e, gen, gen_len, false, &op.g0, &op.g1);
  if (s) return s;
  op.kind = 2;
  op.inner = src;
  op.inner_ver = NEWT;
  op.out = dest;
  e->e.lies[lie].ops.push_back(op);
  return OK;
}

int32_t orb_lie_set_max_iteration(orb_engine *e, int32_t lie, int64_t m) {
  ORB_LIE(e, lie);
  e->e.lies[lie].max_iteration = m;
  return OK;
}

int32_t orb_lie_set_reload_full(orb_engine *e, int32_t lie, int32_t flag) {
  ORB_LIE(e, lie);
  e->e.lies[lie].reload_full = flag != 0;
  return OK;
}

int32_t orb_lie_fixpoint(orb_engine *e, int32_t lie, uint64_t *out) {
  ORB_LIE(e, lie);
  uint64_t dummy;
  return e->e.fixpoint(e->e.lies[lie], out ? out : &dummy);
}

int32_t orb_lie_trace(orb_engine *e, int32_t lie, uint64_t *rec, uint64_t cap, uint64_t *out_n) {
  ORB_LIE(e, lie);
  const std::vector<uint64_t> &t = e->e.lies[lie].trace;
  const uint64_t n = t.size() / 5;
  if (out_n) *out_n = n;
  if (rec) std::memcpy(rec, t.data(), std::min(n, cap) * 5 * sizeof(uint64_t));
  return OK;
}

int32_t orb_lie_seconds(orb_engine *e, int32_t lie, double *out) {
  ORB_LIE(e, lie);
  *out = e->e.lies[lie].seconds;
  return OK;
}

}  // extern "C"
