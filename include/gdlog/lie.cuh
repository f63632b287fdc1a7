// gdlog/lie.cuh — LIE (logical inference engine) of the drop-in C++ API.
//
// Same members as the reference (include/lie.cuh:11-65).  fixpoint_loop
// hands the SCC to the engine (gdl_lie_*), which runs the semi-naive loop on
// the device, then refreshes the tuple counts of every relation involved.
#pragma once

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <type_traits>
#include <vector>

#include "relational_algebra.cuh"

struct LIE {
  std::vector<ra_op> ra_ops;
  std::vector<Relation *> update_relations;
  std::vector<Relation *> static_relations;
  std::vector<Relation *> tmp_relations;
  int grid_size;
  int block_size;
  bool reload_full_flag = true;
  int max_iteration = INT_MAX;
  // Loop passes of the last fixpoint_loop, including the final empty one
  // (the reference's iteration_counter, src/lie.cu:208-215).
  unsigned long long iteration_counter = 0;

  LIE(int grid_size, int block_size) : grid_size(grid_size), block_size(block_size) {}

  void add_relations(Relation *rel, bool static_flag) {
    (static_flag ? static_relations : update_relations).push_back(rel);
  }
  void add_tmp_relation(Relation *rel) { tmp_relations.push_back(rel); }
  void add_ra(ra_op op) { ra_ops.push_back(op); }

  void fixpoint_loop() {
    using namespace gdlog_compat;
    gdl_engine *e = engine();
    const bool profile = getenv("GDLOG_PROFILE") != nullptr;
    if (profile) {
      check(gdl_engine_set_profile(e, 1), "gdl_engine_set_profile");
      check(gdl_engine_profile_reset(e), "gdl_engine_profile_reset");
    }
    int32_t lie = -1;
    check(gdl_lie_create(e, &lie), "gdl_lie_create");
    for (Relation *r : static_relations) check(gdl_lie_add_relation(e, lie, r->id, 1), "add_relations");
    for (Relation *r : update_relations) check(gdl_lie_add_relation(e, lie, r->id, 0), "add_relations");
    for (Relation *r : tmp_relations) check(gdl_lie_add_tmp_relation(e, lie, r->id), "add_tmp_relation");
    for (ra_op &op : ra_ops) std::visit([&](auto &o) { add_op(e, lie, o); }, op);
    check(gdl_lie_set_max_iteration(e, lie, max_iteration), "set_max_iteration");
    check(gdl_lie_set_reload_full(e, lie, reload_full_flag ? 1 : 0), "set_reload_full");
    uint64_t it = 0;
    check(gdl_lie_fixpoint(e, lie, &it), "gdl_lie_fixpoint");
    iteration_counter = it;
    for (auto *v : {&update_relations, &static_relations, &tmp_relations})
      for (Relation *r : *v) r->refresh();
    if (!getenv("GDLOG_QUIET")) print_log(e, lie);
    if (profile) {
      double p[3 * 8] = {0};
      check(gdl_engine_profile(e, p, 3 * 8), "gdl_engine_profile");
      for (ra_op &op : ra_ops)
        if (auto *j = std::get_if<RelationalJoin>(&op))
          if (j->detail_time) {
            // families: 0 sort_hist 1 sort_pass 2 merge 3 index 4 count 5 mat
            j->detail_time[0] = (float)(p[3 * 4 + 1] / 1e3);
            j->detail_time[2] = (float)(p[3 * 5 + 1] / 1e3);
            j->detail_time[3] = (float)((p[3 * 0 + 1] + p[3 * 1 + 1]) / 1e3);
            j->detail_time[5] = (float)(p[3 * 3 + 1] / 1e3);
            j->detail_time[6] = (float)(p[3 * 2 + 1] / 1e3);
          }
      check(gdl_engine_set_profile(e, 0), "gdl_engine_set_profile");
    }
  }

 private:
  // The per-iteration lines the reference prints inside its loop
  // (src/lie.cu:114-121, 193-200), written once the device loop is done;
  // GDLOG_QUIET=1 leaves them out.
  void print_log(gdl_engine *e, int32_t lie) {
    using namespace gdlog_compat;
    uint64_t n = 0;
    check(gdl_lie_trace(e, lie, nullptr, 0, &n), "gdl_lie_trace");
    std::vector<uint64_t> rec(5 * n);
    check(gdl_lie_trace(e, lie, rec.data(), n, &n), "gdl_lie_trace");
    auto name = [&](uint64_t id) -> const char * {
      for (Relation *r : update_relations)
        if ((uint64_t)r->id == id) return r->name.c_str();
      return "?";
    };
    for (uint64_t i = 0; i < n; i++) {
      const uint64_t *x = &rec[5 * i];
      if (x[2] == UINT64_MAX)
        printf("iteration %llu relation %s no new tuple added\n", (unsigned long long)x[0],
               name(x[1]));
      else
        printf("iteration %llu relation %s finish dedup new tuples : %llu delta tuple size: %llu "
               "full counts %llu\n",
               (unsigned long long)x[0], name(x[1]), (unsigned long long)x[2],
               (unsigned long long)x[3], (unsigned long long)x[4]);
      if (i + 1 == n || rec[5 * (i + 1)] != x[0])
        printf("Iteration %llu finish populating\n", (unsigned long long)x[0]);
    }
    fflush(stdout);
  }

  static void add_op(gdl_engine *e, int32_t lie, RelationalJoin &j) {
    using namespace gdlog_compat;
    int32_t gen[3];
    const int out_arity = j.output_rel->arity;
    if (!j.tuple_generator ||
        !decode_generator(j.tuple_generator, j.inner_rel->arity, j.outer_rel->arity, out_arity, gen))
      check(GDL_E_UNSUPPORTED,
            "RelationalJoin: the generator hook must move columns (plus constants) only");
    int32_t kind = GDL_PRED_NONE;
    if (j.tuple_pred && !decode_predicate(j.tuple_pred, &kind))
      check(GDL_E_UNSUPPORTED, "RelationalJoin: the predicate must compare t[0] with t[1]");
    check(gdl_lie_add_join(e, lie, j.inner_rel->id, (int32_t)j.inner_ver, j.outer_rel->id,
                           (int32_t)j.outer_ver, j.output_rel->id, gen, out_arity, kind, 0, 1),
          "gdl_lie_add_join");
  }
  static void add_op(gdl_engine *e, int32_t lie, RelationalCopy &c) {
    using namespace gdlog_compat;
    int32_t gen[2];
    if (!c.tuple_generator || !decode_copy(c.tuple_generator, gen))
      check(GDL_E_UNSUPPORTED, "RelationalCopy: the copy hook must move columns only");
    check(gdl_lie_add_copy(e, lie, c.src_rel->id, (int32_t)c.src_ver, c.dest_rel->id, gen, 2),
          "gdl_lie_add_copy");
  }
  static void add_op(gdl_engine *e, int32_t lie, RelationalACopy &c) {
    using namespace gdlog_compat;
    int32_t gen[2];
    if (!c.tuple_generator || !decode_copy(c.tuple_generator, gen))
      check(GDL_E_UNSUPPORTED, "RelationalACopy: the copy hook must move columns only");
    check(gdl_lie_add_acopy(e, lie, c.src_rel->id, c.dest_rel->id, gen, 2), "gdl_lie_add_acopy");
  }
};
