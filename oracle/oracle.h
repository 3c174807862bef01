/*
 * oracle.h — CPU restatement of QumirDB's hot-path algorithms.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker of the device
 * kernels (tests/, __graft_entry__.smoke(), bench.py's cpu_baseline and
 * reference arm); nothing in the product links, loads or calls it.
 *
 * Each function restates the reference algorithm it names (file:line within
 * the reference project).  The reference cannot be compiled in this build
 * environment (its kernels are oz-lang, compiled by the absent Qumir/LLVM
 * toolchain), so parity is pinned by the reference's own regression goldens
 * (tests/golden/) and by the known-answer invariants of its unit tests.
 */
#ifndef QDB_ORACLE_H
#define QDB_ORACLE_H

#include "../include/qdb_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* A result table: columns of 16-byte cells (i128 or f64 bits in the low    */
/* word) plus a validity byte per cell.  Owned by the oracle.               */
typedef struct oracle_table {
    int64_t rows;
    int32_t cols;
    int32_t* types;      /* qdb_type per column                             */
    int32_t* scales;
    int64_t* cells;      /* rows * cols * 2 words, row-major                */
    uint8_t* valid;      /* rows * cols                                     */
} oracle_table;

void oracle_table_free(oracle_table* t);

/* Fused filter -> project -> hash aggregate over `n_batches` row sets, in  */
/* the reference's dense first-seen group order (single lane), or with     */
/* `lanes` > 1 the threaded plan: per-lane partial tables, hash % lanes     */
/* repartition and a final combine.  Returns 0, or -1 with `err` filled.    */
int oracle_aggregate(const qdb_aggregate_spec* spec, const qdb_rowset* batches,
                     int32_t n_batches, int32_t lanes, oracle_table* out,
                     char* err, size_t err_len);

/* Filter: writes selection[i] in {0,1} (qdb/kernel/gen.cpp:911-1095).      */
int oracle_filter(int32_t n_columns, const qdb_column_type* columns,
                  int32_t n_nodes, const qdb_expr* nodes, int32_t predicate,
                  const qdb_rowset* batch, uint8_t* selection,
                  char* err, size_t err_len);

/* Project: out_buffers[k][i] = expr_k(row i) in its storage width.          */
int oracle_project(int32_t n_columns, const qdb_column_type* columns,
                   int32_t n_nodes, const qdb_expr* nodes, int32_t n_exprs,
                   const int32_t* exprs, const qdb_rowset* batch,
                   void** out_buffers, uint8_t** out_valid,
                   char* err, size_t err_len);

/* rh_hash of the key columns for every row (qdb/kernel/gen.cpp:233-379).   */
int oracle_hash(int32_t n_columns, const qdb_column_type* columns,
                int32_t n_keys, const int32_t* key_columns,
                const qdb_rowset* batch, uint64_t* hashes,
                char* err, size_t err_len);

/* Row join build + probe in the reference's pair emission order            */
/* (qdb/kernel/join/join_rows.oz:70-197, qdb/kernel/row_table.oz:140-295).   */
/* pairs[2*i] = probe row, pairs[2*i+1] = build row (append order index).   */
/* Returns the pair count (pairs may be NULL to count), or -1.              */
int64_t oracle_row_join(const qdb_row_join_spec* spec,
                        const qdb_rowset* build, int32_t n_build,
                        const qdb_rowset* probe, int64_t* pairs,
                        int64_t pair_cap, char* err, size_t err_len);

/* Join then aggregate over (probe columns ++ build payload columns).        */
/* Row join of any served join type over probe batches: pairs of
   (probe batch << 32 | probe row, or -1 for an emitted build row;
   build row as an index over the concatenated build batches, or -1 for a
   padded probe row), in the order the engine emits them. */
int64_t oracle_row_join_typed(const qdb_row_join_spec* spec, const qdb_rowset* build, int32_t n_build,
                              const qdb_rowset* probe, int32_t n_probe, int64_t* pairs, int64_t pair_cap,
                              char* err, size_t err_len);

int oracle_join_aggregate(const qdb_row_join_spec* join,
                          const qdb_aggregate_spec* agg,
                          const qdb_rowset* build, int32_t n_build,
                          const qdb_rowset* probe, int32_t n_probe,
                          int32_t lanes, oracle_table* out,
                          char* err, size_t err_len);

/* Stable LSD radix sort of packed row ids over `store`                     */
/* (qdb/kernel/sort/sort_rowids.oz:63-228, compiler.cpp:595-599).           */
int oracle_sort(const qdb_sort_spec* spec, const qdb_rowset* store,
                int64_t* row_ids, int64_t n, const bool* descs,
                const bool* nulls_firsts, char* err, size_t err_len);

/* Heap top-K (qdb/kernel/sort/heap.oz:156-188): first `limit` row ids of    */
/* the order with the packed row id as tie break; returns the kept count.    */
int64_t oracle_top_k(const qdb_sort_spec* spec, const qdb_rowset* store,
                     int64_t* row_ids, int64_t size, int64_t limit,
                     const bool* descs, const bool* nulls_firsts);

/* One TTopSortProcessor::Add step (qdb/exec/sort_exec.cpp:627-760) through  */
/* qdb_top_sort_update (qdb/kernel/compiler.cpp:881-975): sorts the batch's  */
/* row ids in place when sort_input, then merges them with the `state` rows  */
/* (already in order), a state row first on equal keys; writes the picks     */
/* (0 = state row pick_idx, 1 = batch row pick_idx) and returns their count. */
int64_t oracle_top_sort_update(const qdb_sort_spec* spec, const qdb_rowset* state,
                               const qdb_rowset* batch, int64_t* row_ids, int64_t n,
                               bool sort_input, uint8_t* pick_src, uint32_t* pick_idx,
                               int64_t limit, char* err, size_t err_len);

/* Threaded baselines (timed on the host; the reference's plan shapes).      */
/* Each returns elapsed seconds of the operator only, or < 0 on error.       */
double oracle_bench_aggregate(const qdb_aggregate_spec* spec,
                              const qdb_rowset* batch, int32_t threads,
                              int64_t* groups_out);
double oracle_bench_join_sum(const int64_t* b_key, const int64_t* b_payload,
                             const int32_t* b_attr, int64_t build_rows,
                             int32_t attr_lt, const int64_t* p_fk,
                             const int64_t* p_value, int64_t probe_rows,
                             int32_t threads, int64_t* sum_out,
                             int64_t* count_out);
double oracle_bench_sort(const int64_t* k1, const int32_t* k2, int64_t rows,
                         int32_t threads, int64_t* rowids_out);

/* Runtime join filter (qdb/kernel/join/runtime_filter.oz) on host memory:
   the same state structs as the device entries (qdb_gpu.h). */
int64_t oracle_rf_build(qdb_rf_build_state* st, const uint64_t* hashes, const uint8_t* sel, int64_t count);
int64_t oracle_rf_publish(qdb_rf_publish_state* st, const qdb_rf_partial* partials, int64_t n);
int64_t oracle_rf_probe(const qdb_rf_data* data, const uint64_t* hashes, const uint8_t* sel, uint8_t* out,
                        int64_t count);
void oracle_rf_merge(uint64_t* target, const uint64_t* source, int64_t count);
void oracle_mt19937_64(uint64_t seed, int64_t n, uint64_t* out);

/* THashShuffleTask's routing of a batch: dest[r] = output of selected row r
   (-1 unselected); -1 when a row's partition is routed nowhere. */
int64_t oracle_route(const uint64_t* hashes, const uint8_t* sel, int64_t n, const int64_t* routes,
                     int64_t n_routes, int64_t n_outputs, int64_t* dest);

/* qdb_string_hash_bytes (qdb/modules/qumirdb_runtime.cpp:270-300) of one
   string, and the 136-byte XXH3 secret it hashes strings above 16 bytes with. */
uint64_t oracle_string_hash(const uint8_t* data, int64_t size);
const uint8_t* oracle_string_secret(void);

#ifdef __cplusplus
}
#endif

#endif
