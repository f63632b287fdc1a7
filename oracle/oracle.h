/*
 * oracle.h — CPU oracle for the semi-naive fixpoint path (TEST
 * INFRASTRUCTURE ONLY).
 *
 * A CPU restatement, in C++/OpenMP, of the slog GPU backend's fixpoint
 * semantics: LIE::fixpoint_loop (src/lie.cu:26-274) driving RelationalJoin
 * (src/join.cu:12-270), RelationalCopy (src/copy.cu:12-95) and
 * RelationalACopy (src/acopy.cu:12-50) over FULL/DELTA/NEWT relation
 * containers (include/relation.cuh:257-300).  It is the checker the tests,
 * the smoke check and the bench's CPU-baseline leg compare the CUDA engine
 * against; nothing in the product links or calls it.
 *
 * The entry points mirror include/gdlog_b200.h one for one (orc_ instead of
 * gdl_, same arguments and hook encoding), so one program builder can drive
 * both.  Status codes are the GDL_* codes.
 */
#ifndef GDLOG_ORACLE_H
#define GDLOG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_engine orc_engine;

/* max_arity: widest relation the engine will hold (1..4).  threads: OpenMP
 * threads to use (<= 0: all available). */
int32_t orc_engine_create(int32_t max_arity, int32_t threads, orc_engine **out);
int32_t orc_engine_destroy(orc_engine *e);
/* Drop every relation and LIE (mirrors gdl_engine_clear). */
int32_t orc_engine_clear(orc_engine *e);
const char *orc_last_error(const orc_engine *e);
int32_t orc_threads(const orc_engine *e);

int32_t orc_relation_create(orc_engine *e, const char *name, int32_t arity,
                            int32_t index_column_size,
                            int32_t dependent_column_size, int32_t index_flag,
                            int32_t tmp_flag, int32_t *out_rel);
int32_t orc_relation_load(orc_engine *e, int32_t rel, const uint64_t *rows,
                          uint64_t n);
int32_t orc_relation_size(orc_engine *e, int32_t rel, int32_t version,
                          uint64_t *out);
int32_t orc_relation_export(orc_engine *e, int32_t rel, int32_t version,
                            uint64_t *rows, uint64_t cap, uint64_t *out_n);
int32_t orc_relation_digest(orc_engine *e, int32_t rel, int32_t version,
                            uint64_t *out_digest);

/* gdl_join_count: (outer row, inner row) pairs agreeing on column 0. */
int32_t orc_join_count(orc_engine *e, int32_t inner, int32_t inner_version, int32_t outer,
                       int32_t outer_version, uint64_t *out_candidates);

int32_t orc_lie_create(orc_engine *e, int32_t *out_lie);
int32_t orc_lie_add_relation(orc_engine *e, int32_t lie, int32_t rel,
                             int32_t static_flag);
int32_t orc_lie_add_tmp_relation(orc_engine *e, int32_t lie, int32_t rel);
int32_t orc_lie_add_join(orc_engine *e, int32_t lie, int32_t inner,
                         int32_t inner_version, int32_t outer,
                         int32_t outer_version, int32_t output,
                         const int32_t *gen, int32_t gen_len,
                         int32_t pred_kind, int32_t pred_a, int32_t pred_b);
int32_t orc_lie_add_copy(orc_engine *e, int32_t lie, int32_t src,
                         int32_t src_version, int32_t dest, const int32_t *gen,
                         int32_t gen_len);
int32_t orc_lie_add_acopy(orc_engine *e, int32_t lie, int32_t src,
                          int32_t dest, const int32_t *gen, int32_t gen_len);
int32_t orc_lie_set_max_iteration(orc_engine *e, int32_t lie, int64_t m);
int32_t orc_lie_set_reload_full(orc_engine *e, int32_t lie, int32_t flag);
int32_t orc_lie_fixpoint(orc_engine *e, int32_t lie, uint64_t *out_iterations);
int32_t orc_lie_trace(orc_engine *e, int32_t lie, uint64_t *records,
                      uint64_t cap_records, uint64_t *out_records);
/* Wall seconds of the last fixpoint. */
int32_t orc_lie_seconds(orc_engine *e, int32_t lie, double *out);

/* Second oracle over bit matrices (oracle_bitset.cpp): the same entry
 * points with the prefix orb_, for arity-2 programs over ids below 2^15
 * whose hooks select columns.  Its joins are boolean matrix products, so it
 * finishes programs whose joins have far more candidates than results. */
typedef struct orb_engine orb_engine;
int32_t orb_engine_create(int32_t max_arity, int32_t threads, orb_engine **out);
int32_t orb_engine_destroy(orb_engine *e);
int32_t orb_engine_clear(orb_engine *e);
const char *orb_last_error(const orb_engine *e);
int32_t orb_threads(const orb_engine *e);
int32_t orb_relation_create(orb_engine *e, const char *name, int32_t arity,
                            int32_t index_column_size,
                            int32_t dependent_column_size, int32_t index_flag,
                            int32_t tmp_flag, int32_t *out_rel);
int32_t orb_relation_load(orb_engine *e, int32_t rel, const uint64_t *rows,
                          uint64_t n);
int32_t orb_relation_size(orb_engine *e, int32_t rel, int32_t version,
                          uint64_t *out);
int32_t orb_relation_export(orb_engine *e, int32_t rel, int32_t version,
                            uint64_t *rows, uint64_t cap, uint64_t *out_n);
int32_t orb_relation_digest(orb_engine *e, int32_t rel, int32_t version,
                            uint64_t *out_digest);
int32_t orb_lie_create(orb_engine *e, int32_t *out_lie);
int32_t orb_lie_add_relation(orb_engine *e, int32_t lie, int32_t rel,
                             int32_t static_flag);
int32_t orb_lie_add_tmp_relation(orb_engine *e, int32_t lie, int32_t rel);
int32_t orb_lie_add_join(orb_engine *e, int32_t lie, int32_t inner,
                         int32_t inner_version, int32_t outer,
                         int32_t outer_version, int32_t output,
                         const int32_t *gen, int32_t gen_len,
                         int32_t pred_kind, int32_t pred_a, int32_t pred_b);
int32_t orb_lie_add_copy(orb_engine *e, int32_t lie, int32_t src,
                         int32_t src_version, int32_t dest, const int32_t *gen,
                         int32_t gen_len);
int32_t orb_lie_add_acopy(orb_engine *e, int32_t lie, int32_t src,
                          int32_t dest, const int32_t *gen, int32_t gen_len);
int32_t orb_lie_set_max_iteration(orb_engine *e, int32_t lie, int64_t m);
int32_t orb_lie_set_reload_full(orb_engine *e, int32_t lie, int32_t flag);
int32_t orb_lie_fixpoint(orb_engine *e, int32_t lie, uint64_t *out_iterations);
int32_t orb_lie_trace(orb_engine *e, int32_t lie, uint64_t *records,
                      uint64_t cap_records, uint64_t *out_records);
int32_t orb_lie_seconds(orb_engine *e, int32_t lie, double *out);

#ifdef __cplusplus
}
#endif

#endif
