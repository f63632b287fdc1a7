// oracle.cpp — CPU oracle for the semi-naive fixpoint path.
//
// TEST INFRASTRUCTURE ONLY: the tests, the smoke check and the CPU-baseline
// leg of the benchmark use it to check (and to time against) the CUDA
// engine.  The product never links or calls it.
//
// It restates, on the CPU, the container-level semantics of the slog GPU
// backend's semi-naive engine.  Each function cites the reference code it
// follows (paths relative to the reference project root).  Relations hold
// rows of up to W unsigned 64-bit columns; the order is the reference's
// unsigned lexicographic order over all columns (include/tuple.cuh:106-126).
// Rows narrower than W are zero-padded, which leaves that order unchanged.
//
// The quirks of the reference that decide result sets, sizes and iteration
// counts are kept on purpose:
//   * inputs are sorted and deduplicated at load (src/relation.cu:570-593);
//   * at loop start DELTA := the first |FULL| rows of FULL's raw buffer, in
//     raw (load) order (src/lie.cu:49-59 via copy_relation_container,
//     src/relation.cu:764-795, which reloads with sorted_flag=true);
//   * a FULL-source Copy runs once per LIE (src/lie.cu:69-75), Copy/ACopy
//     ignore the predicate (src/relation.cu:390-403);
//   * a join with an empty inner zeroes the OUTER's tuple count
//     (src/join.cu:38-45); a Copy with an empty source zeroes dest NEWT
//     (src/copy.cu:24-27); an ACopy with an empty source clears dest NEWT
//     (src/acopy.cu:14-18);
//   * outputs into a tmp_flag relation are concatenated without sort or
//     dedup (src/join.cu:145-150,226-254);
//   * set difference compares arity - dependent_column_size columns
//     (src/lie.cu:131-138);
//   * the iteration count includes the final empty pass and the loop stops
//     when iteration_counter > max_iteration (src/lie.cu:208-215).
#include "oracle.h"

#include <omp.h>
#include <parallel/algorithm>

#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

namespace {

constexpr int32_t OK = 0, E_INVALID = 1, E_UNSUPPORTED = 4, E_CAPACITY = 6;
constexpr int DELTA = 0, FULL = 1, NEWT = 2;
constexpr int PRED_NONE = 0, PRED_NE = 1, PRED_EQ = 2, PRED_LT = 3,
              PRED_LE = 4, PRED_GT = 5, PRED_GE = 6;

inline uint64_t mix64(uint64_t x) {
  // splitmix64 finaliser (Steele, Lea, Flood 2014).
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

struct Op {
  int kind;  // 0 join, 1 copy, 2 acopy
  int inner = -1, inner_ver = FULL, outer = -1, outer_ver = DELTA, out = -1;
  std::vector<int32_t> gen;
  int pred = PRED_NONE, pa = 0, pb = 0;
  bool copied = false;  // RelationalCopy::copied (relational_algebra.cuh:72)
};

struct Lie {
  std::vector<int> update, statics, tmps;
  std::vector<Op> ops;
  int64_t max_iteration = INT32_MAX;  // include/lie.cuh:30 (INT_MAX)
  bool reload_full = true;            // include/lie.cuh:29
  std::vector<uint64_t> trace;
  double seconds = 0;
};

struct EngineBase {
  std::string err;
  int threads = 1;
  virtual ~EngineBase() = default;
  virtual int32_t rel_create(const char *, int, int, int, int, int, int32_t *) = 0;
  virtual int32_t rel_load(int, const uint64_t *, uint64_t) = 0;
  virtual int32_t rel_size(int, int, uint64_t *) = 0;
  virtual int32_t rel_export(int, int, uint64_t *, uint64_t, uint64_t *) = 0;
  virtual int32_t rel_digest(int, int, uint64_t *) = 0;
  virtual int32_t fixpoint(Lie &, uint64_t *) = 0;
  virtual int nrels() const = 0;
  virtual int arity(int r) const = 0;
  std::vector<Lie> lies;
  int32_t fail(int32_t code, const std::string &m) {
    err = m;
    return code;
  }
};

template <int W>
struct Engine final : EngineBase {
  using Row = std::array<uint64_t, W>;

  // GHashRelContainer (include/relation.cuh:43-73) reduced to what decides
  // results: the rows in "tuples" order and tuple_counts.  A container is
  // empty when tuple_counts == 0 (the reference also tests tuples ==
  // nullptr, which coincides with a zero count everywhere it is read).
  struct Container {
    std::vector<Row> rows;
    uint64_t n = 0;
    bool sorted = true;  // false only for DELTA taken from raw load order
    void clear() {
      rows.clear();
      rows.shrink_to_fit();
      n = 0;
      sorted = true;
    }
  };

  // Relation (include/relation.cuh:257-300).
  struct Rel {
    std::string name;
    int arity = 2, icols = 1, dep = 0;
    bool index_flag = true, tmp_flag = false;
    Container full, delta, newt;
    // FULL's data_raw: the raw rows FULL was loaded from, in load order.
    // copy_relation_container copies the first tuple_counts rows of it.
    std::vector<Row> raw;
    std::vector<Row> tuple_full;  // Relation::tuple_full
    uint64_t current_full_size = 0;
  };
  std::vector<Rel> rels;

  int nrels() const override { return (int)rels.size(); }
  int arity(int r) const override { return rels[r].arity; }

  static bool less_full(const Row &a, const Row &b) {
    for (int i = 0; i < W; i++) {
      if (a[i] < b[i]) return true;
      if (a[i] > b[i]) return false;
    }
    return false;
  }
  struct PrefixLess {
    int k;
    bool operator()(const Row &a, const Row &b) const {
      for (int i = 0; i < k; i++) {
        if (a[i] < b[i]) return true;
        if (a[i] > b[i]) return false;
      }
      return false;
    }
  };

  // sort + unique, as load_relation_container does when sorted_flag is
  // false (src/relation.cu:570-593).
  void sort_unique(std::vector<Row> &v) {
    __gnu_parallel::sort(v.begin(), v.end(), less_full);
    v.erase(std::unique(v.begin(), v.end()), v.end());
  }

  int32_t rel_create(const char *name, int arity, int icols, int dep, int index_flag,
                     int tmp_flag, int32_t *out) override {
    if (arity < 1 || arity > W) return fail(E_UNSUPPORTED, "arity out of range");
    if (icols < 1 || icols > arity) return fail(E_INVALID, "bad index_column_size");
    if (dep < 0 || dep >= arity) return fail(E_INVALID, "bad dependent_column_size");
    Rel r;
    r.name = name ? name : "";
    r.arity = arity;
    r.icols = icols;
    r.dep = dep;
    r.index_flag = index_flag != 0;
    r.tmp_flag = tmp_flag != 0;
    rels.push_back(std::move(r));
    *out = (int32_t)rels.size() - 1;
    return OK;
  }

  // load_relation (src/relation.cu:815-838): FULL = sort+unique of the rows,
  // DELTA and NEWT fresh and empty.
  int32_t rel_load(int id, const uint64_t *rows, uint64_t n) override {
    Rel &r = rels[id];
    r.full.clear();
    r.delta.clear();
    r.newt.clear();
    r.raw.assign(n, Row{});
    for (uint64_t i = 0; i < n; i++)
      for (int c = 0; c < r.arity; c++) r.raw[i][c] = rows[i * r.arity + c];
    r.full.rows = r.raw;
    sort_unique(r.full.rows);
    r.full.n = r.full.rows.size();
    r.tuple_full.clear();
    r.current_full_size = 0;
    return OK;
  }

  const Container *version(const Rel &r, int ver) const {
    return ver == DELTA ? &r.delta : ver == FULL ? &r.full : &r.newt;
  }

  int32_t rel_size(int id, int ver, uint64_t *out) override {
    *out = version(rels[id], ver)->n;
    return OK;
  }

  std::vector<Row> sorted_rows(int id, int ver) {
    const Container *c = version(rels[id], ver);
    std::vector<Row> v(c->rows.begin(), c->rows.begin() + std::min<uint64_t>(c->n, c->rows.size()));
    __gnu_parallel::sort(v.begin(), v.end(), less_full);
    return v;
  }

  int32_t rel_export(int id, int ver, uint64_t *out, uint64_t cap, uint64_t *out_n) override {
    std::vector<Row> v = sorted_rows(id, ver);
    *out_n = v.size();
    if (v.size() > cap) return fail(E_CAPACITY, "export buffer too small");
    int a = rels[id].arity;
    for (size_t i = 0; i < v.size(); i++)
      for (int c = 0; c < a; c++) out[i * a + c] = v[i][c];
    return OK;
  }

  // Digest of the sorted rows: sum over rows of a hash of (position, row),
  // finished with the row count.  The CUDA engine computes the same value.
  int32_t rel_digest(int id, int ver, uint64_t *out) override {
    std::vector<Row> v = sorted_rows(id, ver);
    int a = rels[id].arity;
    uint64_t s = 0;
#pragma omp parallel for reduction(+ : s) num_threads(threads)
    for (int64_t i = 0; i < (int64_t)v.size(); i++) {
      uint64_t h = mix64((uint64_t)i);
      for (int c = 0; c < a; c++) h = mix64(h ^ v[i][c]);
      s += h;
    }
    *out = mix64(s ^ (uint64_t)v.size());
    return OK;
  }

  // tuple_generator_hook / tuple_copy_hook restated as a column selection.
  static inline Row gen_join(const std::vector<int32_t> &g, const Row &in, const Row &outr) {
    Row t{};
    for (size_t j = 0; j < g.size(); j++) {
      const int s = g[j] & 0xFF;  // GDL_PLUS: constant in bits 8..
      t[j] = (s < 16 ? in[s] : outr[s - 16]) + (uint64_t)((uint32_t)g[j] >> 8);
    }
    return t;
  }
  static inline Row gen_copy(const std::vector<int32_t> &g, const Row &s) {
    Row t{};
    for (size_t j = 0; j < g.size(); j++) t[j] = s[g[j] & 0xFF] + (uint64_t)((uint32_t)g[j] >> 8);
    return t;
  }
  static inline bool pred_ok(int kind, int a, int b, const Row &t) {
    switch (kind) {
      case PRED_NONE: return true;
      case PRED_NE: return t[a] != t[b];
      case PRED_EQ: return t[a] == t[b];
      case PRED_LT: return t[a] < t[b];
      case PRED_LE: return t[a] <= t[b];
      case PRED_GT: return t[a] > t[b];
      case PRED_GE: return t[a] >= t[b];
    }
    return true;
  }

  // Put freshly generated rows R into NEWT of relation `o`, the way
  // RelationalJoin and RelationalCopy do (src/join.cu:130-261,
  // src/copy.cu:42-93): a tmp_flag output takes the rows as they are (first
  // time) or appended (after), anything else keeps NEWT sorted and unique.
  void newt_accept(Rel &o, std::vector<Row> &&R, bool concat_if_tmp) {
    if (concat_if_tmp && o.tmp_flag) {
      if (o.newt.n == 0) {
        o.newt.rows = std::move(R);
      } else {
        o.newt.rows.resize(o.newt.n);
        o.newt.rows.insert(o.newt.rows.end(), R.begin(), R.end());
      }
      o.newt.n = o.newt.rows.size();
      return;
    }
    sort_unique(R);
    if (o.newt.n == 0) {
      o.newt.rows = std::move(R);
    } else {
      std::vector<Row> m(R.size() + o.newt.n);
      __gnu_parallel::merge(R.begin(), R.end(), o.newt.rows.begin(),
                            o.newt.rows.begin() + o.newt.n, m.begin(), less_full);
      m.erase(std::unique(m.begin(), m.end()), m.end());
      o.newt.rows = std::move(m);
    }
    o.newt.n = o.newt.rows.size();
  }

  // RelationalJoin::operator() (src/join.cu:12-270).  For every outer row,
  // the inner rows whose first join_column_counts (= outer's
  // index_column_size) columns equal the outer row's are enumerated; the
  // reference finds the first of them through its hash index and walks
  // forward, which is the same range because the inner is sorted.
  void run_join(Op &op) {
    Rel &I = rels[op.inner];
    Rel &O = rels[op.outer];
    Rel &Out = rels[op.out];
    Container &inner = op.inner_ver == DELTA ? I.delta : I.full;  // join.cu:14-19
    Container &outer = op.outer_ver == DELTA ? O.delta : op.outer_ver == FULL ? O.full : O.newt;
    if (outer.n == 0) {  // join.cu:38-41
      outer.n = 0;
      return;
    }
    if (inner.n == 0) {  // join.cu:42-45: zeroes the OUTER's count
      outer.n = 0;
      return;
    }
    const int k = O.icols;
    PrefixLess pl{k};
    // An inner DELTA taken from raw load order is unsorted; the reference's
    // index walk is undefined there.  The oracle (and the CUDA engine) use
    // its sorted, unique form instead.
    std::vector<Row> sorted_inner;
    const Row *ib = inner.rows.data();
    const Row *ie = ib + inner.n;
    if (!inner.sorted) {
      sorted_inner.assign(ib, ie);
      sort_unique(sorted_inner);
      ib = sorted_inner.data();
      ie = ib + sorted_inner.size();
    }
    const int64_t no = (int64_t)outer.n;
    std::vector<std::vector<Row>> parts(threads);
#pragma omp parallel num_threads(threads)
    {
      std::vector<Row> &mine = parts[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 1024)
      for (int64_t i = 0; i < no; i++) {
        const Row &orow = outer.rows[i];
        auto rng = std::equal_range(ib, ie, orow, pl);
        for (const Row *p = rng.first; p != rng.second; ++p) {
          Row t = gen_join(op.gen, *p, orow);
          if (pred_ok(op.pred, op.pa, op.pb, t)) mine.push_back(t);
        }
      }
    }
    size_t total = 0;
    for (auto &p : parts) total += p.size();
    std::vector<Row> R;
    R.reserve(total);
    for (auto &p : parts) R.insert(R.end(), p.begin(), p.end());
    newt_accept(Out, std::move(R), true);
  }

  // RelationalCopy::operator() (src/copy.cu:12-95).
  void run_copy(Op &op) {
    Rel &S = rels[op.inner];
    Rel &D = rels[op.out];
    Container &src = op.inner_ver == DELTA ? S.delta : S.full;
    if (src.n == 0) {  // copy.cu:24-27
      D.newt.n = 0;
      return;
    }
    std::vector<Row> R(src.n);
#pragma omp parallel for num_threads(threads)
    for (int64_t i = 0; i < (int64_t)src.n; i++) R[i] = gen_copy(op.gen, src.rows[i]);
    newt_accept(D, std::move(R), false);
  }

  // RelationalACopy::operator() (src/acopy.cu:12-50): dest NEWT is replaced
  // by the sorted, unique projection of src NEWT.
  void run_acopy(Op &op) {
    Rel &S = rels[op.inner];
    Rel &D = rels[op.out];
    if (S.newt.n == 0) {
      D.newt.clear();
      return;
    }
    std::vector<Row> R(S.newt.n);
#pragma omp parallel for num_threads(threads)
    for (int64_t i = 0; i < (int64_t)S.newt.n; i++) R[i] = gen_copy(op.gen, S.newt.rows[i]);
    sort_unique(R);
    D.newt.rows = std::move(R);
    D.newt.n = D.newt.rows.size();
  }

  // LIE::fixpoint_loop (src/lie.cu:26-274).
  int32_t fixpoint(Lie &L, uint64_t *out_iters) override {
    auto t0 = std::chrono::steady_clock::now();
    L.trace.clear();
    // Setup (lie.cu:49-59): tuple_full := FULL's tuples; DELTA := copy of
    // FULL, i.e. the first |FULL| rows of FULL's raw buffer in raw order.
    for (int id : L.update) {
      Rel &r = rels[id];
      r.tuple_full.assign(r.full.rows.begin(), r.full.rows.begin() + r.full.n);
      r.current_full_size = r.full.n;
      uint64_t take = std::min<uint64_t>(r.full.n, r.raw.size());
      r.delta.rows.assign(r.raw.begin(), r.raw.begin() + take);
      r.delta.n = take;
      r.delta.sorted = false;
    }
    int64_t it = 0;
    while (true) {
      for (Op &op : L.ops) {  // lie.cu:62-82
        if (op.kind == 0) {
          run_join(op);
        } else if (op.kind == 2) {
          run_acopy(op);
        } else {
          if (op.inner_ver == FULL) {
            if (!op.copied) {
              run_copy(op);
              op.copied = true;
            }
          } else {
            run_copy(op);
          }
        }
      }
      for (int id : L.tmps) rels[id].newt.clear();  // lie.cu:85-87
      bool fixpoint_flag = true;
      for (int id : L.update) {  // lie.cu:93-198
        Rel &r = rels[id];
        if (r.newt.n == 0) {  // lie.cu:114-121
          r.delta.clear();
          L.trace.insert(L.trace.end(), {(uint64_t)it, (uint64_t)id, UINT64_MAX, 0,
                                         r.current_full_size});
          continue;
        }
        // set_difference(newt, tuple_full) over arity - dep columns
        // (lie.cu:131-138); NEWT and tuple_full are sorted.
        std::vector<Row> d(r.newt.n);
        PrefixLess pl{r.arity - r.dep};
        auto end = __gnu_parallel::set_difference(
            r.newt.rows.begin(), r.newt.rows.begin() + r.newt.n, r.tuple_full.begin(),
            r.tuple_full.begin() + r.current_full_size, d.begin(), pl);
        d.erase(end, d.end());
        if (!d.empty()) fixpoint_flag = false;
        uint64_t dedup = d.size();
        r.newt.clear();
        r.delta.rows = std::move(d);  // lie.cu:167-174 (sorted, indexed)
        r.delta.n = r.delta.rows.size();
        r.delta.sorted = true;
        // flush_delta (src/relation.cu:405-521).
        if (r.delta.n != 0) {
          std::vector<Row> m(r.current_full_size + r.delta.n);
          __gnu_parallel::merge(r.tuple_full.begin(), r.tuple_full.begin() + r.current_full_size,
                                r.delta.rows.begin(), r.delta.rows.end(), m.begin(), less_full);
          r.tuple_full = std::move(m);
          r.current_full_size = r.tuple_full.size();
          r.full.rows = r.tuple_full;  // full->tuples = tuple_full
          r.full.n = r.current_full_size;
        }
        L.trace.insert(L.trace.end(), {(uint64_t)it, (uint64_t)id, dedup, r.delta.n,
                                       r.current_full_size});
      }
      it++;
      if (fixpoint_flag || it > L.max_iteration) break;  // lie.cu:208-215
    }
    // lie.cu:219-254: flatten tuple_full into a fresh sorted FULL.
    if (L.reload_full) {
      for (int id : L.update) {
        Rel &r = rels[id];
        r.full.rows.assign(r.tuple_full.begin(), r.tuple_full.begin() + r.current_full_size);
        r.full.n = r.current_full_size;
        r.raw = r.full.rows;  // data_raw is now the flattened, sorted FULL
        r.delta.clear();
        r.newt.clear();
      }
    }
    *out_iters = (uint64_t)it;
    L.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return OK;
  }
};

}  // namespace

struct orc_engine {
  std::unique_ptr<EngineBase> impl;
  int32_t max_arity = 2;
};

static EngineBase *make_impl(int32_t max_arity) {
  switch (max_arity) {
    case 1:
    case 2: return new Engine<2>;
    case 3: return new Engine<3>;
    case 4: return new Engine<4>;
    default: return nullptr;
  }
}

extern "C" {

int32_t orc_engine_create(int32_t max_arity, int32_t threads, orc_engine **out) {
  if (!out) return E_INVALID;
  EngineBase *impl = make_impl(max_arity);
  if (!impl) return E_UNSUPPORTED;
  auto *e = new orc_engine;
  e->impl.reset(impl);
  e->max_arity = max_arity;
  e->impl->threads = threads > 0 ? threads : omp_get_max_threads();
  *out = e;
  return OK;
}

int32_t orc_engine_clear(orc_engine *e) {
  if (!e) return E_INVALID;
  const int32_t threads = e->impl->threads;
  e->impl.reset(make_impl(e->max_arity));
  e->impl->threads = threads;
  return OK;
}

int32_t orc_engine_destroy(orc_engine *e) {
  delete e;
  return OK;
}

const char *orc_last_error(const orc_engine *e) { return e ? e->impl->err.c_str() : "null engine"; }
int32_t orc_threads(const orc_engine *e) { return e ? e->impl->threads : 0; }

#define CHECK_REL(e, r)                                                       \
  do {                                                                         \
    if (!(e) || (r) < 0 || (r) >= (e)->impl->nrels())                          \
      return (e) ? (e)->impl->fail(E_INVALID, "bad relation id") : E_INVALID;  \
  } while (0)
#define CHECK_LIE(e, l)                                                       \
  do {                                                                         \
    if (!(e) || (l) < 0 || (l) >= (int)(e)->impl->lies.size())                 \
      return (e) ? (e)->impl->fail(E_INVALID, "bad lie id") : E_INVALID;       \
  } while (0)

int32_t orc_relation_create(orc_engine *e, const char *name, int32_t arity, int32_t icols,
                            int32_t dep, int32_t index_flag, int32_t tmp_flag, int32_t *out) {
  if (!e || !out) return E_INVALID;
  return e->impl->rel_create(name, arity, icols, dep, index_flag, tmp_flag, out);
}

int32_t orc_relation_load(orc_engine *e, int32_t rel, const uint64_t *rows, uint64_t n) {
  CHECK_REL(e, rel);
  if (n && !rows) return e->impl->fail(E_INVALID, "null rows");
  return e->impl->rel_load(rel, rows, n);
}

int32_t orc_relation_size(orc_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  CHECK_REL(e, rel);
  if (ver < 0 || ver > 2 || !out) return e->impl->fail(E_INVALID, "bad version");
  return e->impl->rel_size(rel, ver, out);
}

int32_t orc_relation_export(orc_engine *e, int32_t rel, int32_t ver, uint64_t *rows,
                            uint64_t cap, uint64_t *out_n) {
  CHECK_REL(e, rel);
  if (ver < 0 || ver > 2 || !out_n) return e->impl->fail(E_INVALID, "bad version");
  return e->impl->rel_export(rel, ver, rows, cap, out_n);
}

int32_t orc_relation_digest(orc_engine *e, int32_t rel, int32_t ver, uint64_t *out) {
  CHECK_REL(e, rel);
  if (ver < 0 || ver > 2 || !out) return e->impl->fail(E_INVALID, "bad version");
  return e->impl->rel_digest(rel, ver, out);
}

// get_join_result_size (src/relation.cu:221-288: per outer row, the length
// of the inner run its column 0 selects) summed as RelationalJoin::operator()
// does (src/join.cu:77-102).  Restated over the exported sorted rows.
int32_t orc_join_count(orc_engine *e, int32_t inner, int32_t inner_ver, int32_t outer,
                       int32_t outer_ver, uint64_t *out) {
  CHECK_REL(e, inner);
  CHECK_REL(e, outer);
  auto ver_ok = [](int32_t v) { return v == FULL || v == DELTA; };
  if (!out || !ver_ok(inner_ver) || !ver_ok(outer_ver))
    return e->impl->fail(E_INVALID, "join_count: versions must be FULL or DELTA");
  auto rows = [&](int32_t r, int32_t v, std::vector<uint64_t> &dst) -> int32_t {
    uint64_t n = 0;
    int32_t st = e->impl->rel_size(r, v, &n);
    if (st != OK) return st;
    dst.resize(n * (uint64_t)e->impl->arity(r) + 1);
    uint64_t got = 0;
    return e->impl->rel_export(r, v, dst.data(), n, &got);
  };
  std::vector<uint64_t> in, ou;
  int32_t st = rows(inner, inner_ver, in);
  if (st != OK) return st;
  st = rows(outer, outer_ver, ou);
  if (st != OK) return st;
  const int ai = e->impl->arity(inner), ao = e->impl->arity(outer);
  std::unordered_map<uint64_t, uint64_t> run;  // column 0 -> inner rows with it
  for (size_t i = 0; i + ai <= in.size() - 1; i += ai) run[in[i]]++;
  uint64_t total = 0;
  for (size_t i = 0; i + ao <= ou.size() - 1; i += ao) {
    auto it = run.find(ou[i]);
    if (it != run.end()) total += it->second;
  }
  *out = total;
  return OK;
}

int32_t orc_lie_create(orc_engine *e, int32_t *out) {
  if (!e || !out) return E_INVALID;
  e->impl->lies.emplace_back();
  *out = (int32_t)e->impl->lies.size() - 1;
  return OK;
}

int32_t orc_lie_add_relation(orc_engine *e, int32_t lie, int32_t rel, int32_t static_flag) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, rel);
  (static_flag ? e->impl->lies[lie].statics : e->impl->lies[lie].update).push_back(rel);
  return OK;
}

int32_t orc_lie_add_tmp_relation(orc_engine *e, int32_t lie, int32_t rel) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, rel);
  e->impl->lies[lie].tmps.push_back(rel);
  return OK;
}

static int32_t check_gen(orc_engine *e, const int32_t *gen, int32_t n, int out_arity, bool join,
                         int a_in, int a_out) {
  if (!gen || n != out_arity) return e->impl->fail(E_INVALID, "gen length != output arity");
  for (int j = 0; j < n; j++) {
    int g = gen[j] & 0xFF;
    if (join) {
      if (!((g >= 0 && g < a_in) || (g >= 16 && g - 16 < a_out)))
        return e->impl->fail(E_INVALID, "gen column out of range");
    } else if (g < 0 || g >= a_in) {
      return e->impl->fail(E_INVALID, "gen column out of range");
    }
  }
  return OK;
}

int32_t orc_lie_add_join(orc_engine *e, int32_t lie, int32_t inner, int32_t inner_ver,
                         int32_t outer, int32_t outer_ver, int32_t output, const int32_t *gen,
                         int32_t gen_len, int32_t pred, int32_t pa, int32_t pb) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, inner);
  CHECK_REL(e, outer);
  CHECK_REL(e, output);
  int32_t s = check_gen(e, gen, gen_len, e->impl->arity(output), true, e->impl->arity(inner),
                        e->impl->arity(outer));
  if (s) return s;
  if (pred < 0 || pred > PRED_GE) return e->impl->fail(E_INVALID, "bad predicate");
  if (pred && (pa < 0 || pb < 0 || pa >= gen_len || pb >= gen_len))
    return e->impl->fail(E_INVALID, "predicate column out of range");
  Op op;
  op.kind = 0;
  op.inner = inner;
  op.inner_ver = inner_ver;
  op.outer = outer;
  op.outer_ver = outer_ver;
  op.out = output;
  op.gen.assign(gen, gen + gen_len);
  op.pred = pred;
  op.pa = pa;
  op.pb = pb;
  e->impl->lies[lie].ops.push_back(op);
  return OK;
}

int32_t orc_lie_add_copy(orc_engine *e, int32_t lie, int32_t src, int32_t src_ver, int32_t dest,
                         const int32_t *gen, int32_t gen_len) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  int32_t s = check_gen(e, gen, gen_len, e->impl->arity(dest), false, e->impl->arity(src), 0);
  if (s) return s;
  Op op;
  op.kind = 1;
  op.inner = src;
  op.inner_ver = src_ver;
  op.out = dest;
  op.gen.assign(gen, gen + gen_len);
  e->impl->lies[lie].ops.push_back(op);
  return OK;
}

int32_t orc_lie_add_acopy(orc_engine *e, int32_t lie, int32_t src, int32_t dest,
                          const int32_t *gen, int32_t gen_len) {
  CHECK_LIE(e, lie);
  CHECK_REL(e, src);
  CHECK_REL(e, dest);
  int32_t s = check_gen(e, gen, gen_len, e->impl->arity(dest), false, e->impl->arity(src), 0);
  if (s) return s;
  Op op;
  op.kind = 2;
  op.inner = src;
  op.inner_ver = NEWT;
  op.out = dest;
  op.gen.assign(gen, gen + gen_len);
  e->impl->lies[lie].ops.push_back(op);
  return OK;
}

int32_t orc_lie_set_max_iteration(orc_engine *e, int32_t lie, int64_t m) {
  CHECK_LIE(e, lie);
  e->impl->lies[lie].max_iteration = m;
  return OK;
}

int32_t orc_lie_set_reload_full(orc_engine *e, int32_t lie, int32_t flag) {
  CHECK_LIE(e, lie);
  e->impl->lies[lie].reload_full = flag != 0;
  return OK;
}

int32_t orc_lie_fixpoint(orc_engine *e, int32_t lie, uint64_t *out) {
  CHECK_LIE(e, lie);
  uint64_t dummy;
  return e->impl->fixpoint(e->impl->lies[lie], out ? out : &dummy);
}

int32_t orc_lie_trace(orc_engine *e, int32_t lie, uint64_t *rec, uint64_t cap, uint64_t *out_n) {
  CHECK_LIE(e, lie);
  const std::vector<uint64_t> &t = e->impl->lies[lie].trace;
  uint64_t n = t.size() / 5;
  if (out_n) *out_n = n;
  if (rec) std::memcpy(rec, t.data(), std::min(n, cap) * 5 * sizeof(uint64_t));
  return OK;
}

int32_t orc_lie_seconds(orc_engine *e, int32_t lie, double *out) {
  CHECK_LIE(e, lie);
  *out = e->impl->lies[lie].seconds;
  return OK;
}

}  // extern "C"
