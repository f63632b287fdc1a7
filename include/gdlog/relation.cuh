// gdlog/relation.cuh — Relation and load_relation of the drop-in C++ API.
//
// Field names follow the reference's Relation / GHashRelContainer
// (include/relation.cuh:43-73, 257-300) so a program that sets index_flag
// before loading (test/tc.cu:108) and reads full->tuple_counts after a
// fixpoint (test/tc.cu:138) works unchanged.  The tuples themselves live in
// the engine, packed and indexed on the device; tuple_counts is refreshed
// after each load and each LIE::fixpoint_loop.
#pragma once

#include <climits>

#include <string>
#include <vector>

#include "engine.cuh"
#include "tuple.cuh"

enum RelationVersion { DELTA, FULL, NEWT };  // include/relation.cuh:13
enum JoinDirection { LEFT, RIGHT };          // include/relation.cuh:75 (unused)

// The reference's empty-slot marker of its hash index (include/relation.cuh:
// 27); drivers print it.  This engine's index slots carry a build epoch
// instead, so the value marks nothing here.
#ifndef EMPTY_HASH_ENTRY
#define EMPTY_HASH_ENTRY ULONG_MAX
#endif

struct GHashRelContainer {
  tuple_size_t index_column_size = 1;
  int dependent_column_size = 0;
  tuple_size_t tuple_counts = 0;
  int arity = 2;
  bool tmp_flag = false;
  // which engine relation and version this container stands for (set by
  // load_relation; used by the printers of print.cuh)
  int32_t rel_id = -1;
  int32_t version = -1;
  GHashRelContainer(int arity, int indexed_column_size, int dependent_column_size,
                    bool tmp_flag = false)
      : index_column_size(indexed_column_size), dependent_column_size(dependent_column_size),
        arity(arity), tmp_flag(tmp_flag) {}
};

struct Relation {
  int arity = 2;
  int index_column_size = 1;
  std::string name;
  int dependent_column_size = 0;
  bool index_flag = true;
  bool tmp_flag = false;
  GHashRelContainer *delta = nullptr;
  GHashRelContainer *newt = nullptr;
  GHashRelContainer *full = nullptr;
  tuple_size_t current_full_size = 0;
  int32_t id = -1;  // the engine's relation id

  // Re-read the three tuple counts from the engine.
  void refresh() {
    if (id < 0) return;
    gdl_engine *e = gdlog_compat::engine();
    uint64_t n = 0;
    gdlog_compat::check(gdl_relation_size(e, id, GDL_FULL, &n), "gdl_relation_size");
    full->tuple_counts = n;
    current_full_size = n;
    gdlog_compat::check(gdl_relation_size(e, id, GDL_DELTA, &n), "gdl_relation_size");
    delta->tuple_counts = n;
    gdlog_compat::check(gdl_relation_size(e, id, GDL_NEWT, &n), "gdl_relation_size");
    newt->tuple_counts = n;
  }

  // The sorted tuples of one version, row-major (arity columns per row).
  std::vector<column_type> rows(RelationVersion v = FULL) const {
    gdl_engine *e = gdlog_compat::engine();
    uint64_t n = 0;
    gdlog_compat::check(gdl_relation_size(e, id, (int32_t)v, &n), "gdl_relation_size");
    std::vector<column_type> out(n * arity);
    uint64_t got = 0;
    gdlog_compat::check(gdl_relation_export(e, id, (int32_t)v, (uint64_t *)out.data(), n, &got),
                        "gdl_relation_export");
    out.resize(got * arity);
    return out;
  }

  uint64_t digest(RelationVersion v = FULL) const {
    uint64_t d = 0;
    gdlog_compat::check(gdl_relation_digest(gdlog_compat::engine(), id, (int32_t)v, &d),
                        "gdl_relation_digest");
    return d;
  }
};

// load_relation (src/relation.cu:815-838): create the relation in the engine
// and load `data_row_size` host rows into FULL (sorted, deduplicated,
// indexed).  data == nullptr with 0 rows gives an empty relation
// (test/sg.cu:126-127).  grid_size / block_size are accepted for source
// compatibility; the engine sizes its own launches.
inline void load_relation(Relation *target, std::string name, int arity, column_type *data,
                          tuple_size_t data_row_size, tuple_size_t index_column_size,
                          int dependent_column_size, int grid_size, int block_size,
                          bool tmp_flag = false) {
  (void)grid_size;
  (void)block_size;
  gdl_engine *e = gdlog_compat::engine();
  target->name = name;
  target->arity = arity;
  target->index_column_size = (int)index_column_size;
  target->dependent_column_size = dependent_column_size;
  target->tmp_flag = tmp_flag;
  if (!target->full) {
    target->full = new GHashRelContainer(arity, (int)index_column_size, dependent_column_size);
    target->delta = new GHashRelContainer(arity, (int)index_column_size, dependent_column_size);
    target->newt = new GHashRelContainer(arity, (int)index_column_size, dependent_column_size);
  }
  if (target->id < 0)
    gdlog_compat::check(gdl_relation_create(e, name.c_str(), arity, (int32_t)index_column_size,
                                            dependent_column_size, target->index_flag ? 1 : 0,
                                            tmp_flag ? 1 : 0, &target->id),
                        "gdl_relation_create");
  target->full->rel_id = target->delta->rel_id = target->newt->rel_id = target->id;
  target->full->version = GDL_FULL;
  target->delta->version = GDL_DELTA;
  target->newt->version = GDL_NEWT;
  gdlog_compat::check(
      gdl_relation_load(e, target->id, (const uint64_t *)data, data ? data_row_size : 0),
      "gdl_relation_load");
  target->refresh();
}
