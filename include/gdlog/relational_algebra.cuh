// gdlog/relational_algebra.cuh — RA operators of the drop-in C++ API.
//
// Same constructors as the reference (include/relational_algebra.cuh:46-106)
// and the same std::variant.  The operators are descriptions: LIE::add_ra
// copies them and LIE::fixpoint_loop hands them to the engine, which runs
// them on the device.  Hooks are probed once, when the LIE is first run.
#pragma once

#include <variant>

#include "relation.cuh"

struct RelationalJoin {
  Relation *inner_rel;
  RelationVersion inner_ver;
  Relation *outer_rel;
  RelationVersion outer_ver;
  Relation *output_rel;
  tuple_generator_hook tuple_generator;
  tuple_predicate tuple_pred;
  JoinDirection direction;
  int grid_size;
  int block_size;
  bool disable_load = false;
  // Per-phase milliseconds (the reference's detail_time[0..7],
  // src/join.cu:74-215), filled after each fixpoint while the engine runs
  // with profiling on (GDLOG_PROFILE=1): [0] count pass, [2] materialise,
  // [3] sort, [5] index build, [6] merge / set difference.
  float *detail_time;

  RelationalJoin(Relation *inner_rel, RelationVersion inner_ver, Relation *outer_rel,
                 RelationVersion outer_ver, Relation *output_rel, tuple_generator_hook tp_gen,
                 tuple_predicate tp_pred, JoinDirection direction, int grid_size, int block_size,
                 float *detail_time)
      : inner_rel(inner_rel), inner_ver(inner_ver), outer_rel(outer_rel), outer_ver(outer_ver),
        output_rel(output_rel), tuple_generator(tp_gen), tuple_pred(tp_pred),
        direction(direction), grid_size(grid_size), block_size(block_size),
        detail_time(detail_time) {}

  // The reference runs an operator standalone with operator()(); here the
  // operators run inside LIE::fixpoint_loop only.
  void operator()() {
    gdlog_compat::check(GDL_E_UNSUPPORTED, "RelationalJoin::operator() outside a LIE");
  }
};

struct RelationalCopy {
  Relation *src_rel;
  RelationVersion src_ver;
  Relation *dest_rel;
  tuple_copy_hook tuple_generator;
  tuple_predicate tuple_pred;  // accepted, not applied (src/relation.cu:390-403)
  int grid_size;
  int block_size;
  bool copied = false;

  RelationalCopy(Relation *src, RelationVersion src_ver, Relation *dest,
                 tuple_copy_hook tuple_generator, tuple_predicate tuple_pred, int grid_size,
                 int block_size)
      : src_rel(src), src_ver(src_ver), dest_rel(dest), tuple_generator(tuple_generator),
        tuple_pred(tuple_pred), grid_size(grid_size), block_size(block_size) {}

  void operator()() {
    gdlog_compat::check(GDL_E_UNSUPPORTED, "RelationalCopy::operator() outside a LIE");
  }
};

struct RelationalACopy {
  Relation *src_rel;
  Relation *dest_rel;
  tuple_copy_hook tuple_generator;
  tuple_predicate tuple_pred;  // accepted, not applied (src/acopy.cu:12-50)
  int grid_size;
  int block_size;

  RelationalACopy(Relation *src, Relation *dest, tuple_copy_hook tuple_generator,
                  tuple_predicate tuple_pred, int grid_size, int block_size)
      : src_rel(src), dest_rel(dest), tuple_generator(tuple_generator), tuple_pred(tuple_pred),
        grid_size(grid_size), block_size(block_size) {}

  void operator()() {
    gdlog_compat::check(GDL_E_UNSUPPORTED, "RelationalACopy::operator() outside a LIE");
  }
};

using ra_op = std::variant<RelationalJoin, RelationalCopy, RelationalACopy>;

enum RAtypes { JOIN, COPY, ACOPY };
