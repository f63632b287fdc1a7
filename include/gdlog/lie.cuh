// gdlog/lie.cuh — LIE (logical inference engine) of the drop-in C++ API.
//
// Same members as the reference (include/lie.cuh:11-65).  fixpoint_loop
// hands the SCC to the engine (gdl_lie_*), which runs the semi-naive loop on
// the device, then refreshes the tuple counts of every relation involved.
#pragma once

#include <climits>
#include <cstdio>
#include <cstdlib>
#include <deque>
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
    join_hooks_.clear();
    copy_hooks_.clear();
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

  // Hook state the engine's launchers read while this LIE runs (a deque
  // keeps element addresses fixed as it grows).
  std::deque<gdlog_compat::JoinHooks> join_hooks_;
  std::deque<tuple_copy_hook> copy_hooks_;

  void add_op(gdl_engine *e, int32_t lie, RelationalJoin &j) {
    using namespace gdlog_compat;
    if (!j.tuple_generator)  // the reference calls it unconditionally (src/relation.cu:348-358)
      check(GDL_E_INVALID, "RelationalJoin: null tuple_generator_hook");
    const int out_arity = j.output_rel->arity;
    int32_t gen[4], kind = GDL_PRED_NONE, pa = 0, pb = 1;
    bool sel = !exact_hooks() &&
               decode_generator(j.tuple_generator, j.inner_rel->arity, j.outer_rel->arity,
                                out_arity, gen);
    if (sel && j.tuple_pred) {
      // The engine's own predicate compares columns 0 and 1 of a plain
      // arity-2 tuple; anything else runs through the hooks.
      bool plain = out_arity == 2;
      for (int c = 0; c < out_arity; c++) plain = plain && (gen[c] >> 8) == 0;
      sel = plain && decode_predicate(j.tuple_pred, out_arity, &kind, &pa, &pb) && pa < 2 &&
            pb < 2;
    }
    if (sel) {
      log_hook("RelationalJoin", "column selection");
      check(gdl_lie_add_join(e, lie, j.inner_rel->id, (int32_t)j.inner_ver, j.outer_rel->id,
                             (int32_t)j.outer_ver, j.output_rel->id, gen, out_arity, kind, pa, pb),
            "gdl_lie_add_join");
      return;
    }
    log_hook("RelationalJoin", "device function pointers");
    join_hooks_.push_back(JoinHooks{j.tuple_generator, j.tuple_pred});
    check(gdl_lie_add_join_hooked(e, lie, j.inner_rel->id, (int32_t)j.inner_ver, j.outer_rel->id,
                                  (int32_t)j.outer_ver, j.output_rel->id, launch_join_hooks,
                                  &join_hooks_.back()),
          "gdl_lie_add_join_hooked");
  }
  void add_op(gdl_engine *e, int32_t lie, RelationalCopy &c) {
    using namespace gdlog_compat;
    if (!c.tuple_generator) check(GDL_E_INVALID, "RelationalCopy: null tuple_copy_hook");
    int32_t gen[4];
    const int out_arity = c.dest_rel->arity;
    if (!exact_hooks() && decode_copy(c.tuple_generator, c.src_rel->arity, out_arity, gen)) {
      log_hook("RelationalCopy", "column selection");
      check(gdl_lie_add_copy(e, lie, c.src_rel->id, (int32_t)c.src_ver, c.dest_rel->id, gen,
                             out_arity),
            "gdl_lie_add_copy");
      return;
    }
    log_hook("RelationalCopy", "device function pointers");
    copy_hooks_.push_back(c.tuple_generator);
    check(gdl_lie_add_copy_hooked(e, lie, c.src_rel->id, (int32_t)c.src_ver, c.dest_rel->id,
                                  launch_copy_hook, &copy_hooks_.back()),
          "gdl_lie_add_copy_hooked");
  }
  void add_op(gdl_engine *e, int32_t lie, RelationalACopy &c) {
    using namespace gdlog_compat;
    if (!c.tuple_generator) check(GDL_E_INVALID, "RelationalACopy: null tuple_copy_hook");
    int32_t gen[4];
    const int out_arity = c.dest_rel->arity;
    if (!exact_hooks() && decode_copy(c.tuple_generator, c.src_rel->arity, out_arity, gen)) {
      log_hook("RelationalACopy", "column selection");
      check(gdl_lie_add_acopy(e, lie, c.src_rel->id, c.dest_rel->id, gen, out_arity),
            "gdl_lie_add_acopy");
      return;
    }
    log_hook("RelationalACopy", "device function pointers");
    copy_hooks_.push_back(c.tuple_generator);
    check(gdl_lie_add_acopy_hooked(e, lie, c.src_rel->id, c.dest_rel->id, launch_copy_hook,
                                   &copy_hooks_.back()),
          "gdl_lie_add_acopy_hooked");
  }
};
