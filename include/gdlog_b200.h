/*
 * gdlog_b200.h — C-ABI of the B200-native Datalog fixpoint engine.
 *
 * This is the drop-in boundary for the semi-naive fixpoint path of the
 * slog GPU backend (harp-lab/gdlog-multinode).  Every entry point below
 * replaces one piece of that project's C++ operator API; the citation on
 * each names the reference interface (file:line, paths relative to the
 * reference project root).  The C++ drop-in headers in include/gdlog/
 * (Relation, load_relation, LIE, RelationalJoin/Copy/ACopy) are written on
 * top of these calls.
 *
 * Conventions
 *  - Plain C types only: pointers, sizes, int32 ids.  No CUDA, no torch.
 *  - Every call returns gdl_status; GDL_OK == 0.  The reference aborts the
 *    process on any CUDA error (include/exception.cuh:9-18); here the
 *    failure is returned and gdl_last_error() holds a one-line message.
 *  - Tuples are rows of `arity` unsigned 64-bit columns (the reference's
 *    column_type, include/tuple.cuh:5-10), row-major, on the host unless a
 *    function says "device".  The engine stores arity-2 relations packed as
 *    one 64-bit key (c0 << 32 | c1), which is order-preserving for column
 *    values below 2^32; larger values are rejected with GDL_E_UNSUPPORTED.
 *    Arity 3 (with dependent_column_size 0 or 1, as test/path_length.cu
 *    uses it) packs c0 << 32 | c1 << k2 | c2, k2 fixed by the first arity-3
 *    load to 32 minus the bits of the ids loaded so far: ids then stay below
 *    2^(32-k2) and column 2 below 2^k2.  Relations of arity 3, dependent
 *    columns and computed hooks run on the sorted-list path.
 *  - Hooks.  The reference passes __device__ function pointers
 *    (tuple_generator_hook / tuple_copy_hook / tuple_predicate,
 *    include/tuple.cuh:23-25).  Across a C-ABI they are described instead
 *    as column selections: gen[j] names the source of output column j,
 *    GDL_INNER(c) or GDL_OUTER(c) for a join, GDL_SRC(c) for a copy,
 *    optionally plus a constant (GDL_PLUS).
 *    A predicate compares two columns of the generated tuple.
 *  - One engine owns one CUDA stream; calls on one engine are not
 *    thread-safe.  Device memory is owned by the engine.
 */
#ifndef GDLOG_B200_H
#define GDLOG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t gdl_status;
#define GDL_OK 0
#define GDL_E_INVALID 1     /* bad argument, id or state                 */
#define GDL_E_CUDA 2        /* a CUDA runtime call failed                */
#define GDL_E_NOMEM 3       /* device allocation failed                  */
#define GDL_E_UNSUPPORTED 4 /* arity/values/hook shape not supported     */
#define GDL_E_TIMEOUT 5     /* a bounded device-side wait gave up        */
#define GDL_E_CAPACITY 6    /* a caller-provided buffer is too small     */

/* RelationVersion (include/relation.cuh:13): same numeric order. */
#define GDL_DELTA 0
#define GDL_FULL 1
#define GDL_NEWT 2

/* Column-selection encoding of a hook's output column. */
#define GDL_INNER(c) (c)
#define GDL_OUTER(c) (16 + (c))
#define GDL_SRC(c) (c)
/* A hook column plus a constant k (0 <= k < 2^23), e.g. path_length's
 * outer[2] + 1 (test/path_length.cu:52-57): GDL_PLUS(GDL_OUTER(2), 1). */
#define GDL_PLUS(sel, k) ((sel) | ((k) << 8))

/* Predicate on the generated tuple t: t[a] <op> t[b]. */
#define GDL_PRED_NONE 0
#define GDL_PRED_NE 1
#define GDL_PRED_EQ 2
#define GDL_PRED_LT 3
#define GDL_PRED_LE 4
#define GDL_PRED_GT 5
#define GDL_PRED_GE 6

typedef struct gdl_engine gdl_engine;

/* Library identification (no reference counterpart). */
const char *gdl_version(void);
const char *gdl_status_string(gdl_status s);
/* Message of the last failing call on `e` (never NULL). */
const char *gdl_last_error(const gdl_engine *e);

/* Create an engine on CUDA device `device`.  `stream` is a cudaStream_t or
 * NULL (the engine then creates its own non-blocking stream).  Replaces the
 * implicit device/legacy-stream state that every reference call assumes
 * (src/relation.cu, src/lie.cu: legacy stream + cudaDeviceSynchronize). */
gdl_status gdl_engine_create(int32_t device, void *stream, gdl_engine **out);
gdl_status gdl_engine_destroy(gdl_engine *e);

/* Drop every relation and LIE of the engine, keeping its stream, scratch
 * buffers and memory pool, so the next program starts without device
 * allocation cost.  Relation and LIE ids restart at 0.  The reference has
 * no counterpart (its drivers leak relations at exit, test/tc.cu:80-149).
 * A program that repeats the previous one (the same relations, loads and
 * LIEs in the same order, as a service answering one query shape does)
 * gets the same device blocks back, and its loops reuse the executable
 * graphs of the previous program's (compared node by node) instead of
 * instantiating new ones.
 * After a call failed with GDL_E_TIMEOUT (a device-side check: a bounded
 * wait gave up or a bounds check fired), every call but this one and
 * gdl_engine_destroy is refused; this one also resets the engine's device
 * bookkeeping, after which the engine runs programs again. */
gdl_status gdl_engine_clear(gdl_engine *e);

/* Testing failure handling (no reference counterpart): the next fixpoint's
 * first control kernel waits on a device flag that nothing sets, giving up
 * after `polls` polls, so that fixpoint returns GDL_E_TIMEOUT without any
 * GPU fault; gdl_engine_clear then recovers the engine. */
gdl_status gdl_engine_test_timeout(gdl_engine *e, int32_t polls);

/* How a fixpoint deduplicates NEWT and merges it into FULL.  SORT: radix
 * sort of NEWT, then one merge-path pass giving NEWT \ FULL and FULL ∪ NEWT
 * (the reference's sort/unique/set_difference/merge, src/lie.cu:122-185).
 * DENSE: when 2 * bits(largest column value) <= dense_max_bits (at most 32,
 * the default), relations are kept as bitmaps over the key domain during the
 * loop and NEWT is deduplicated by setting bits.  AUTO (default): DENSE
 * where the domain allows, else SORT.  Results are identical in all modes.
 * dense_max_bits == 0 keeps the current bound.  The environment variables
 * GDLOG_DEDUP=auto|sort|dense and GDLOG_DENSE_MAX_BITS set the defaults.
 * No reference counterpart. */
#define GDL_DEDUP_AUTO 0
#define GDL_DEDUP_SORT 1
#define GDL_DEDUP_DENSE 2
gdl_status gdl_engine_set_dedup(gdl_engine *e, int32_t mode, int32_t dense_max_bits);

/* Launch and layout parameters an autotuner may set (no reference
 * counterpart; the reference takes grid/block sizes per call, e.g.
 * LIE(grid, block), include/lie.cuh:26-34, and fixes the index load factor
 * at 0.8, src/relation.cu:836).  A zero field keeps the engine's default. */
typedef struct gdl_tuning {
  int32_t dedup;               /* GDL_DEDUP_* */
  int32_t dense_max_bits;      /* largest 2*bits domain kept as bitmaps (<= 32) */
  int32_t join_ctas_per_sm;    /* materialisation grid, CTAs per SM (default 8) */
  int32_t count_ctas_per_sm;   /* count-pass grid, CTAs per SM (default 4) */
  int32_t index_slots_per_key; /* hashed index: slots per distinct key, power of two >= 2 (default 2) */
  int32_t dirty_min_log2_words;/* keep a dirty map for NEWT bitmaps of at least 2^this
                                  words (default 24 = 64 MB; 11..40) */
  int32_t dense_join_passes;   /* joins into bitmaps: 1 = probe and expand in one
                                  pass (default), 2 = count pass, then a pass
                                  balanced by output position */
  int32_t join_aggregate;      /* one-pass joins into bitmaps: 1 = one reduction
                                  per candidate (default), 2 = lanes of a warp
                                  that hit the same word combine their bits */
  int32_t pull_joins;          /* joins into bitmaps whose output is (outer
                                  column 1, inner column 1) over a DELTA or
                                  tmp NEWT outer: 1 = push form (outer in key
                                  order), 2 = pull form (gathered by output
                                  row from the transposed outer) when ids
                                  reach 2^10 (default), 3 = pull form from
                                  2^8 ids */
  int32_t row_gather;          /* those joins over a static inner when ids reach
                                  2^12: 1 = off, 2 = gather the outer's bitmap
                                  rows along the inner's in-edges when the
                                  inner is small enough (|inner| x row bytes
                                  <= 256 MB; default), 3 = whenever possible */
  int32_t spin_limit_log2;     /* a bounded device-side wait (look-back of a scan)
                                  gives up after 2^this polls and the call
                                  returns GDL_E_TIMEOUT (default 22; 1..30) */
  int32_t radix_bits;          /* digit width of the radix sort: 6, 8 (default) or
                                  10 bits (64 / 256 / 1024 buckets a pass); a
                                  width that would need more than 8 passes
                                  falls back to 8 */
  int32_t join_block;          /* threads per block of the one-pass join into
                                  bitmaps: 128, 256 (default) or 512 */
  int32_t rows_piece;          /* row-gather joins: at most this many consecutive
                                  in-edges (grouped by output row) per unit of
                                  work, 8, 16 or 32 (default); every warp takes
                                  the same number of units */
  int32_t load_dedup;          /* load_relation's sort + unique: 1 = radix sort
                                  and merge; 2 = set the rows' bits in a bitmap
                                  over the key domain and list it, when the ids
                                  are below 2^15, the load has more than 4096
                                  rows, and the bitmap is at most 32 MB or 1 KB
                                  a row (default; same result) */
} gdl_tuning;
gdl_status gdl_engine_set_tuning(gdl_engine *e, const gdl_tuning *t);
gdl_status gdl_engine_get_tuning(gdl_engine *e, gdl_tuning *t);

/* Declare a relation.  Replaces `new Relation()` plus the field writes the
 * drivers make before loading (include/relation.cuh:257-300; index_flag as
 * set at test/tc.cu:108, tmp_flag as in load_relation's last argument,
 * src/relation.cu:815-824). */
gdl_status gdl_relation_create(gdl_engine *e, const char *name, int32_t arity,
                               int32_t index_column_size,
                               int32_t dependent_column_size,
                               int32_t index_flag, int32_t tmp_flag,
                               int32_t *out_rel);

/* load_relation (src/relation.cu:815-838): copy `rows` host rows into FULL,
 * sort, deduplicate, index.  rows == 0 (host_rows may be NULL) gives an
 * empty relation, as at test/sg.cu:126-127.  Reloading replaces FULL and
 * clears DELTA and NEWT. */
gdl_status gdl_relation_load(gdl_engine *e, int32_t rel,
                             const uint64_t *host_rows, uint64_t rows);

/* Same as gdl_relation_load with the rows already in device memory
 * (load_relation_container with gpu_data_flag, src/relation.cu:547-548). */
gdl_status gdl_relation_load_device(gdl_engine *e, int32_t rel,
                                    const uint64_t *device_rows, uint64_t rows);

/* Container->tuple_counts of one version (GHashRelContainer::tuple_counts,
 * include/relation.cuh:60); the drivers read full->tuple_counts after the
 * fixpoint (test/tc.cu:138). */
gdl_status gdl_relation_size(gdl_engine *e, int32_t rel, int32_t version,
                             uint64_t *out_rows);

/* Copy one version's tuples to the host, sorted lexicographically over all
 * columns (the order of include/tuple.cuh:106-126).  Fails with
 * GDL_E_CAPACITY (and sets *out_rows) if cap_rows is too small.  The
 * reference has no export; its printers (src/print.cu) are debug only. */
gdl_status gdl_relation_export(gdl_engine *e, int32_t rel, int32_t version,
                               uint64_t *host_rows, uint64_t cap_rows,
                               uint64_t *out_rows);

/* Device-side gdl_relation_export: one version's tuples, sorted, as rows
 * of two uint64 columns into `device_rows` (device memory, room for
 * cap_rows rows); *out_rows receives the count (GDL_E_CAPACITY when it
 * exceeds cap_rows).  Arity 2; a DELTA still in load order is refused (the
 * host export sorts it).  With gdl_partition_rows and
 * gdl_relation_load_device it keeps a partitioned fixpoint's exchange on
 * the device; no reference counterpart (the reference is one GPU). */
gdl_status gdl_relation_export_device(gdl_engine *e, int32_t rel, int32_t version,
                                      uint64_t *device_rows, uint64_t cap_rows,
                                      uint64_t *out_rows);

/* Group `rows` rows of two uint64 columns (device memory) by owning rank,
 * owner = rows[i][column] % world (column 0 or 1, world <= 1024): rank d's
 * rows go, in no particular order, to out_rows[off_d .. off_d + counts[d])
 * with off_d the sum of the counts before d (device memory, room for `rows`
 * rows); counts[0 .. world) is written to host memory.  Returns after the
 * engine's stream has finished.  No reference counterpart. */
gdl_status gdl_partition_rows(gdl_engine *e, const uint64_t *device_rows, uint64_t rows,
                              int32_t column, int32_t world, uint64_t *device_out_rows,
                              uint64_t *counts);

/* Size of a join's output before any deduplication: the number of (outer
 * row, inner row) pairs that agree on column 0, as the count pass of a
 * join computes it on the device (k_join_count: one index probe per outer
 * row, the run lengths summed).  Replaces get_join_result_size
 * (src/relation.cu:221-288) followed by the reduce in
 * RelationalJoin::operator() (src/join.cu:77-102).  The inner version must
 * be indexed (index_flag at load for FULL); versions are GDL_FULL or
 * GDL_DELTA.  Nothing is materialised; the relations are not changed.
 * Serving admission sizes a query's first join with it. */
gdl_status gdl_join_count(gdl_engine *e, int32_t inner, int32_t inner_version, int32_t outer,
                          int32_t outer_version, uint64_t *out_candidates);

/* Order-sensitive 64-bit digest of one version's sorted tuples, computed on
 * the device (no reference counterpart; used for bit-exact parity of large
 * results without copying them to the host). */
gdl_status gdl_relation_digest(gdl_engine *e, int32_t rel, int32_t version,
                               uint64_t *out_digest);

/* Input and output files.
 *
 * gdl_read_tsv replaces the drivers' get_row_size + get_relation_from_file
 * (test/tc.cu:17-57) with the same reading rules: the row count is the
 * number of '\n' characters in the file (a last line without one is not
 * read), each value is a signed decimal integer read after any white space
 * (fscanf "%lld"), and after every column but the last exactly one
 * character (the separator) is consumed.  Values are stored as uint64_t
 * (a negative value wraps, as the reference's stores do).  Host only: no
 * engine and no GPU needed.  Writes at most cap_rows rows of `arity`
 * columns to host_rows and the file's row count to *out_rows; with too
 * small a cap_rows (or host_rows NULL) it returns GDL_E_CAPACITY after
 * setting *out_rows, so a first call can size the buffer.  GDL_E_INVALID
 * if the file cannot be read or runs out of values. */
gdl_status gdl_read_tsv(const char *path, int32_t arity, uint64_t *host_rows, uint64_t cap_rows,
                        uint64_t *out_rows);

/* gdl_read_tsv + gdl_relation_load: the driver's file read followed by
 * load_relation (test/tc.cu:101-111). */
gdl_status gdl_relation_load_tsv(gdl_engine *e, int32_t rel, const char *path);

/* Write one version's tuples, sorted (gdl_relation_export), one row per
 * line, columns separated by a tab, in decimal: the layout of Souffle's
 * .output files, for diffs against them (no reference counterpart; the
 * reference only prints, src/print.cu).  *out_rows (may be NULL) receives
 * the rows written. */
gdl_status gdl_relation_dump_tsv(gdl_engine *e, int32_t rel, int32_t version, const char *path,
                                 uint64_t *out_rows);

/* LIE(grid, block) (include/lie.cuh:11-65, src/lie.cu:13-24). */
gdl_status gdl_lie_create(gdl_engine *e, int32_t *out_lie);
/* LIE::add_relations (src/lie.cu:15-22). */
gdl_status gdl_lie_add_relation(gdl_engine *e, int32_t lie, int32_t rel,
                                int32_t static_flag);
/* LIE::add_tmp_relation (src/lie.cu:24). */
gdl_status gdl_lie_add_tmp_relation(gdl_engine *e, int32_t lie, int32_t rel);

/* LIE::add_ra(RelationalJoin(...)) (include/relational_algebra.cuh:18-57,
 * src/join.cu:12-270).  gen has gen_len == arity(output) entries. */
gdl_status gdl_lie_add_join(gdl_engine *e, int32_t lie, int32_t inner,
                            int32_t inner_version, int32_t outer,
                            int32_t outer_version, int32_t output,
                            const int32_t *gen, int32_t gen_len,
                            int32_t pred_kind, int32_t pred_a, int32_t pred_b);

/* LIE::add_ra(RelationalCopy(...)) (include/relational_algebra.cuh:63-82,
 * src/copy.cu:12-95).  As in the reference the predicate is not applied
 * (src/relation.cu:390-403), so none is taken. */
gdl_status gdl_lie_add_copy(gdl_engine *e, int32_t lie, int32_t src,
                            int32_t src_version, int32_t dest,
                            const int32_t *gen, int32_t gen_len);

/* LIE::add_ra(RelationalACopy(...)) (include/relational_algebra.cuh:90-109,
 * src/acopy.cu:12-50). */
gdl_status gdl_lie_add_acopy(gdl_engine *e, int32_t lie, int32_t src,
                             int32_t dest, const int32_t *gen, int32_t gen_len);

/* Operators whose per-tuple work is the caller's own code.
 *
 * The reference calls a program's __device__ hooks through device function
 * pointers, once per candidate tuple (get_join_result, src/relation.cu:
 * 290-373, with tp_gen and tp_pred at :348-358; get_copy_result,
 * src/relation.cu:390-403).  A hook that is not a column selection (plus a
 * constant) cannot be given to gdl_lie_add_join as `gen`; these entry points
 * take it as a launcher instead.  In every iteration the engine does what
 * surrounds the hook (the count pass over the inner index, the reference's
 * empty-operand rules, the once-per-LIE FULL copy, NEWT capacity), then
 * calls `launch(ctx, &work, stream)`, which must only enqueue kernels on
 * `stream` (it is also called while the engine captures its loop into a CUDA
 * graph, and again whenever it re-captures).  The kernels read the work
 * from device memory through `work`, call the hook on every candidate, and
 * append the packed keys of the tuples they keep to `out` (see
 * gdl_hook_work).  The drop-in C++ API (include/gdlog/engine.cuh) supplies
 * such launchers for a program's hooks.  A LIE with one of these operators
 * runs on sorted tuple lists (no bitmaps). */
typedef struct gdl_dev_rows {
  uint64_t *ptr; /* packed keys: c0 << 32 | c1, or c0 << 32 | c1 << k2 | c2 */
  uint64_t n;    /* rows present */
  uint64_t cap;  /* rows allocated */
} gdl_dev_rows;

typedef struct gdl_hook_state {
  uint64_t total;    /* join: candidates; copy: source rows */
  uint64_t records;  /* join: candidate records (see rec_offset) */
  uint64_t base;     /* first position in out->ptr this operator writes */
  uint64_t overflow; /* engine-internal */
  uint64_t written;  /* rows appended so far: reserve with atomicAdd */
  uint64_t skip;     /* nonzero: the operator does nothing this iteration */
} gdl_hook_state;

typedef struct gdl_hook_work {
  int32_t kind;        /* 0 join, 1 copy, 2 acopy */
  int32_t in_arity;    /* inner (join) or source (copy) arity */
  int32_t outer_arity; /* join only */
  int32_t out_arity;
  int32_t k2;          /* bits of column 2 in arity-3 keys */
  int32_t sms;         /* multiprocessors of the device, for grid sizing */
  gdl_hook_state *state;     /* device */
  const gdl_dev_rows *rows;  /* device: join inner version / copy source */
  /* Join candidates, device: record k (k < state->records) covers candidate
   * positions [rec_offset[k], rec_offset[k+1]); candidate p pairs inner row
   * rows->ptr[rec_start[k] + p - rec_offset[k]] with outer row rec_key[k].
   * Copy: candidate p is source row rows->ptr[p], p < state->total. */
  const uint64_t *rec_offset;
  const uint32_t *rec_start;
  const uint64_t *rec_key;
  gdl_dev_rows *out;  /* device: NEWT of the output; write out->ptr[state->base + i] */
  uint32_t *error;    /* device: OR 32768 when a generated value does not fit its column */
} gdl_hook_work;

typedef void (*gdl_hook_launch)(void *ctx, const gdl_hook_work *work, void *stream);

/* RelationalJoin with its generator and predicate run by `launch`. */
gdl_status gdl_lie_add_join_hooked(gdl_engine *e, int32_t lie, int32_t inner,
                                   int32_t inner_version, int32_t outer,
                                   int32_t outer_version, int32_t output,
                                   gdl_hook_launch launch, void *ctx);
/* RelationalCopy / RelationalACopy with the copy hook run by `launch`. */
gdl_status gdl_lie_add_copy_hooked(gdl_engine *e, int32_t lie, int32_t src,
                                   int32_t src_version, int32_t dest,
                                   gdl_hook_launch launch, void *ctx);
gdl_status gdl_lie_add_acopy_hooked(gdl_engine *e, int32_t lie, int32_t src,
                                    int32_t dest, gdl_hook_launch launch, void *ctx);

/* LIE::max_iteration / LIE::reload_full_flag (include/lie.cuh:29-30). */
gdl_status gdl_lie_set_max_iteration(gdl_engine *e, int32_t lie,
                                     int64_t max_iteration);
gdl_status gdl_lie_set_reload_full(gdl_engine *e, int32_t lie, int32_t flag);

/* LIE::fixpoint_loop (src/lie.cu:26-274).  *out_iterations receives the
 * loop-pass count, including the final empty pass (the reference's
 * iteration_counter after the loop). */
gdl_status gdl_lie_fixpoint(gdl_engine *e, int32_t lie,
                            uint64_t *out_iterations);

/* Per-iteration log of the last fixpoint: one record per (iteration,
 * update relation) with the three numbers the reference prints at
 * src/lie.cu:193-197 (dedup new tuples, delta size, full count); dedup is
 * UINT64_MAX for the "no new tuple added" branch (src/lie.cu:114-121).
 * Records are 5 uint64: iteration, relation id, dedup, delta, full.
 * Returns the number of records in *out_records (always), copies at most
 * cap_records. */
gdl_status gdl_lie_trace(gdl_engine *e, int32_t lie, uint64_t *records,
                         uint64_t cap_records, uint64_t *out_records);

/* Enable/disable the per-iteration trace (it costs one small device->host
 * copy per iteration at the end of the fixpoint, not per iteration). */
gdl_status gdl_lie_set_trace(gdl_engine *e, int32_t lie, int32_t flag);

/* Timing and launch accounting of the last fixpoint on this engine:
 * out[0] = fixpoint device milliseconds, out[1] = kernels launched,
 * out[2] = iterations, out[3] = capacity retries, out[4] = graph launches,
 * out[5] = host setup ms, out[6] = host ms growing buffers after capacity
 * overflows, out[7] = host ms capturing and instantiating graphs,
 * out[8] = 1 if the loop's executable graph was taken from the engine's
 * cache (an equal iteration of an earlier program, see gdl_engine_clear).
 * n_out is the number of doubles the caller provides. */
gdl_status gdl_lie_stats(gdl_engine *e, int32_t lie, double *out,
                         int32_t n_out);

/* Block until all work queued on the engine's stream has finished. */
gdl_status gdl_engine_sync(gdl_engine *e);

/* Per-kernel accounting of the fixpoint loops run on this engine (the
 * reference threads a float detail_time[] through RelationalJoin and
 * accumulates phase times in LIE::fixpoint_loop, include/
 * relational_algebra.cuh:43-44, src/lie.cu:28-45; this replaces it).
 * Kernels are grouped in gdl_profile_kinds() families named by
 * gdl_profile_kind_name().  gdl_engine_profile writes, per family k,
 * out[3k] = launches, out[3k+1] = device milliseconds (measured only while
 * profiling is on: loops then run launch by launch with a CUDA event pair
 * around each kernel instead of from the captured graph), out[3k+2] =
 * algorithmic bytes (what the operation must read and write; counted by
 * the kernels themselves, always on).  Totals accumulate until
 * gdl_engine_profile_reset. */
int32_t gdl_profile_kinds(void);
const char *gdl_profile_kind_name(int32_t kind);
gdl_status gdl_engine_set_profile(gdl_engine *e, int32_t flag);
gdl_status gdl_engine_profile(gdl_engine *e, double *out, int32_t n_out);
gdl_status gdl_engine_profile_reset(gdl_engine *e);

/* Batched form: many independent instances of one program in one LIE.  No
 * reference counterpart (the reference runs one fixpoint at a time).
 * Declare node_counts[i] local node ids for instance i before loading; the
 * instance's tuples then use the global ids (i << S) | local, where S is
 * given by gdl_engine_instance_shift, and both columns of every tuple must
 * belong to the same instance.  The fixpoint over the disjoint union equals
 * the union of the per-instance fixpoints (every rule joins on shared
 * values); the engine keeps the relations as one block-diagonal bitmap, so
 * all instances advance together in the same kernels and an instance that
 * has converged costs nothing but its scan.  Passing 0 instances returns to
 * the plain form.  Node counts are limited to 65,536 per instance. */
gdl_status gdl_engine_set_instances(gdl_engine *e, const uint32_t *node_counts,
                                    int32_t n_instances);
gdl_status gdl_engine_instance_shift(gdl_engine *e, int32_t *out_shift);

/* Loop passes each instance would have taken alone (the reference's
 * iteration_counter for that instance, src/lie.cu:208-215), for the last
 * fixpoint of `lie` in the batched form. */
gdl_status gdl_lie_instance_iterations(gdl_engine *e, int32_t lie, uint64_t *out,
                                       int32_t n_instances);

/* Per-instance size and digest of FULL of a relation updated by a batched
 * fixpoint, in the instance's local ids: the values gdl_relation_size and
 * gdl_relation_digest give when the instance runs alone.  Works also when
 * FULL is too large for a list and is kept only as its bitmap. */
gdl_status gdl_relation_instance_stats(gdl_engine *e, int32_t rel, uint64_t *sizes,
                                       uint64_t *digests, int32_t n_instances);

/* Allocation-free sort + deduplicate.  No counterpart in the reference; it
 * is an extra entry point for callers that cannot allocate device memory
 * (code running inside another library's memory arena, or a process that
 * gave all of HBM to a fixed pool before starting): it makes no cudaMalloc
 * or cudaFree call and no call into any allocating library.
 *
 * Sorts `rows` rows of two uint64 columns (device memory, row-major, values
 * below 2^32) lexicographically, removes duplicates, writes the unique rows
 * to `device_out_rows` (caller-provided, room for `rows` rows) and their
 * count to *out_rows (host).  Same result as gdl_relation_load_device
 * followed by gdl_relation_export of FULL.  At most 131,072 rows per call;
 * larger inputs are refused with GDL_E_CAPACITY.  Runs on `stream` (a
 * cudaStream_t, NULL for the legacy default stream) on the current device
 * and returns after that stream has finished the work.
 *
 * Scratch is one fixed array of about 4.3 MB inside the library, present on
 * every GPU that loads the library until the process exits.  The first call
 * on a device looks up that array's device address (cudaGetSymbolAddress).
 * Every call waits for its stream and copies results to host memory, so it
 * must not be called while its stream (or the legacy stream) is being
 * captured into a CUDA graph.  All calls on a device
 * share the array: calls that can overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller.  On failure,
 * gdl_last_error(NULL) holds the message. */
gdl_status gdl_sort_unique_rows_noalloc(const uint64_t *device_rows, uint64_t rows,
                                        uint64_t *device_out_rows, uint64_t *out_rows,
                                        void *stream);

#ifdef __cplusplus
}
#endif

#endif /* GDLOG_B200_H */
