// print.cuh — the reference's test printers (include/print.cuh, src/print.cu)
// for drivers written against this drop-in API.  Debug output only; the
// layouts they print differ from the reference's where its internals do not
// exist here (row-pointer arrays, the (hash, first row) index table).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <vector>

#include "relation.cuh"
#include "tuple.cuh"

// The index is one device slot per join key (start, length of its run); the
// reference's per-row hash table has no counterpart.  Prints the sizes.
inline void print_hashes(GHashRelContainer *target, const char *rel_name) {
  printf("%s: %llu tuples, indexed on %llu column(s) (one device slot per join key)\n", rel_name,
         (unsigned long long)target->tuple_counts, (unsigned long long)target->index_column_size);
}

// The container's tuples, sorted, one row per line (src/print.cu prints
// the same rows from the device).
inline void print_tuple_rows(GHashRelContainer *target, const char *rel_name) {
  printf("Relation %s, %llu tuples:\n", rel_name, (unsigned long long)target->tuple_counts);
  if (target->rel_id < 0) return;
  gdl_engine *e = gdlog_compat::engine();
  uint64_t n = 0;
  gdlog_compat::check(gdl_relation_size(e, target->rel_id, target->version, &n),
                      "gdl_relation_size");
  std::vector<uint64_t> rows(n * (uint64_t)target->arity);
  uint64_t got = 0;
  gdlog_compat::check(gdl_relation_export(e, target->rel_id, target->version, rows.data(), n, &got),
                      "gdl_relation_export");
  for (uint64_t i = 0; i < got; i++) {
    for (int c = 0; c < target->arity; c++)
      printf("%llu%s", (unsigned long long)rows[i * target->arity + c],
             c + 1 < target->arity ? "\t" : "\n");
  }
}

// Rows are kept as packed keys, never as a raw row-major buffer apart from
// the sorted export: prints the same as print_tuple_rows.
inline void print_tuple_raw_data(GHashRelContainer *target, const char *rel_name) {
  print_tuple_rows(target, rel_name);
}

inline tuple_size_t get_free_memory() {
  size_t f = 0, t = 0;
  cudaMemGetInfo(&f, &t);
  return (tuple_size_t)f;
}

inline tuple_size_t get_total_memory() {
  size_t f = 0, t = 0;
  cudaMemGetInfo(&f, &t);
  return (tuple_size_t)t;
}

inline void print_memory_usage() {
  const double mb = 1024.0 * 1024.0;
  const tuple_size_t f = get_free_memory(), t = get_total_memory();
  printf("GPU memory: %.1f MB used of %.1f MB\n", (double)(t - f) / mb, (double)t / mb);
}

// `rows` tuples given as host row pointers of `arity` columns each.
inline void print_tuple_list(tuple_type *tuples, tuple_size_t rows, tuple_size_t arity) {
  for (tuple_size_t i = 0; i < rows; i++)
    for (tuple_size_t c = 0; c < arity; c++)
      printf("%llu%s", (unsigned long long)tuples[i][c], c + 1 < arity ? "\t" : "\n");
}
