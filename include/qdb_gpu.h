/*
 * qdb_gpu.h — C ABI of the B200 (sm_100a) execution hot path of QumirDB.
 *
 * The engine's physical task graph calls its operator kernels through plain
 * function pointers whose arguments are pointers, integers of at most 64 bits
 * and bool (qdb/kernel/generated.h:28-51, TKernelSlot::Call).  Each entry
 * point below takes a compiled program handle as its first argument and then
 * exactly the arguments of the reference entry it replaces, so the engine's
 * binding is a closure `[prog](args...) { return qdb_gpu_X(prog, args...); }`
 * stored in the existing std::function dispatch members
 * (qdb/kernel/compiler.h:207-242, :363-405, :486-596).
 *
 * Programs are built from plain-data descriptors that a lowering fills from
 * TOperatorKernelSpec (qdb/kernel/spec.h:65-90) instead of from a Qumir AST.
 * Expression evaluation selects hand-written device functors; there is no JIT.
 *
 * Row sets may point at host memory or at device memory (HBM).  Host columns
 * are staged to the device on each call; device columns are used in place.
 * Outputs are written where the program's `flags` say (QDB_OUT_DEVICE).
 *
 * Every entry point is re-entrant across host threads.  Device work of one
 * table/arena state runs on the stream that was current when it was
 * initialised (qdb_gpu_set_stream), so concurrent task states overlap.
 *
 * Errors: compile functions return NULL and fill `err`; dispatch entries use
 * the reference's error conventions (documented per entry) and record a
 * message retrievable with qdb_gpu_last_error() on the calling thread.
 * Nothing here falls back to the CPU: a program the device kernels cannot
 * serve is rejected at compile time.
 */
#ifndef QDB_GPU_H
#define QDB_GPU_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Data ABI — layout-identical to TColumn / TRowSet (qdb/io/io.h:17-39).     */
/* ------------------------------------------------------------------------ */

typedef struct qdb_column {
    char* Data;
    int32_t DataBitOffset;   /* bit offset of bitmap-backed (bool) columns  */
    const uint8_t* Mask;     /* Arrow validity bitmap; NULL = all valid     */
    int32_t MaskBitOffset;
    void* Offsets;           /* string offsets; NULL for fixed width        */
    uint8_t OffsetWidth;     /* 4 (STRING), 8 (LARGE_STRING), 0 otherwise  */
} qdb_column;

typedef struct qdb_rowset {
    qdb_column* Columns;
    int64_t ColumnCount;
    int64_t RowCount;
    uint8_t* Selection;      /* NULL = every row; Selection[i]==0 skips i   */
    uint64_t* Hash;          /* precomputed shuffle hashes, or NULL         */
    void (*Destroy)(struct qdb_rowset*);
    void* Private;
    int64_t RefCount;
} qdb_rowset;

/* Value types of columns and expression results. */
typedef enum qdb_type {
    QDB_TYPE_INVALID = 0,
    QDB_TYPE_BOOL = 1,        /* input: bitmap at DataBitOffset (io.h:18);
                                 project output: one byte 0/1 per row        */
    QDB_TYPE_I8 = 2,
    QDB_TYPE_I16 = 3,
    QDB_TYPE_I32 = 4,
    QDB_TYPE_I64 = 5,
    QDB_TYPE_U8 = 6,
    QDB_TYPE_U16 = 7,
    QDB_TYPE_U32 = 8,
    QDB_TYPE_U64 = 9,
    QDB_TYPE_F32 = 10,
    QDB_TYPE_F64 = 11,
    QDB_TYPE_DATE32 = 12,     /* i32 days since 1970-01-01 (qdb/plan/types/date.h:14-29) */
    QDB_TYPE_DECIMAL64 = 13,  /* unscaled i64, precision <= 18 (qdb/plan/types/decimal.h:80-99) */
    QDB_TYPE_DECIMAL128 = 14, /* unscaled i128 "BinInt", precision 19..38     */
    QDB_TYPE_CHAR1 = 15,      /* a string column whose values are one byte,
                                 staged as one code byte per row             */
    QDB_TYPE_STRING = 16      /* a string column as Arrow lays it out: row r's
                                 bytes are Data[Offsets[r] .. Offsets[r+1]),
                                 Offsets of OffsetWidth 4 (utf8) or 8
                                 (large_utf8) bytes each.  Served as a key
                                 column of hash programs (qdb_gpu_hash and
                                 the runtime-filter probe of a row set).     */
} qdb_type;

typedef struct qdb_column_type {
    int32_t type;       /* qdb_type                                          */
    int32_t precision;  /* decimals only                                     */
    int32_t scale;      /* decimals only                                     */
    int32_t nullable;   /* non-zero: the column may carry a validity mask    */
} qdb_column_type;

/* ------------------------------------------------------------------------ */
/* Expressions: a flat array of nodes, operands before their users.          */
/* Types are the lowering's annotated result types (AnnotateExprType,        */
/* qdb/kernel/annotate_type.cpp:725-945); arithmetic follows them exactly:   */
/*   integer ops wrap in the result width; DECIMAL +/- rescale operands to   */
/*   the result scale; DECIMAL * multiplies unscaled values (scales add);    */
/*   DECIMAL / integer truncates toward zero keeping the dividend's scale    */
/*   (qdb/modules/qumirdb_runtime.cpp:703-705); comparisons align scales.   */
/* ------------------------------------------------------------------------ */

typedef enum qdb_expr_op {
    QDB_EXPR_COLUMN = 1,      /* input column `column`                      */
    QDB_EXPR_CONST = 2,       /* imm_lo/imm_hi (f64 bits in imm_lo)          */
    QDB_EXPR_NULL = 3,
    QDB_EXPR_ADD = 4,
    QDB_EXPR_SUB = 5,
    QDB_EXPR_MUL = 6,
    QDB_EXPR_DIV = 7,
    QDB_EXPR_NEG = 8,
    QDB_EXPR_CAST = 9,        /* args[0] converted to `type`/`scale`         */
    QDB_EXPR_EQ = 10,
    QDB_EXPR_NE = 11,
    QDB_EXPR_LT = 12,
    QDB_EXPR_LE = 13,
    QDB_EXPR_GT = 14,
    QDB_EXPR_GE = 15,
    QDB_EXPR_AND = 16,
    QDB_EXPR_OR = 17,
    QDB_EXPR_NOT = 18,
    QDB_EXPR_BETWEEN = 19,    /* args[1] <= args[0] <= args[2]               */
    QDB_EXPR_IN_LIST = 20,    /* args[0] IN list[0..list_len)                */
    QDB_EXPR_CASE = 21,       /* CASE WHEN args[0] THEN args[1] ELSE args[2] */
    QDB_EXPR_IS_NULL = 22,
    QDB_EXPR_IS_NOT_NULL = 23,
    QDB_EXPR_MOD = 24         /* remainder, sign of the dividend (truncating) */
} qdb_expr_op;

typedef struct qdb_expr {
    int32_t op;         /* qdb_expr_op                                       */
    int32_t type;       /* qdb_type of the result                            */
    int32_t scale;      /* decimal scale of the result                       */
    int32_t column;     /* QDB_EXPR_COLUMN: input column index               */
    int32_t args[3];    /* operand node indices, each below this node's      */
    int32_t list_len;   /* QDB_EXPR_IN_LIST                                  */
    int64_t imm_lo;     /* QDB_EXPR_CONST low word                           */
    int64_t imm_hi;     /* QDB_EXPR_CONST high word (DECIMAL128)             */
    const int64_t* list;/* IN-list constants, in args[0]'s type and scale    */
} qdb_expr;

/* Program flags. */
#define QDB_OUT_DEVICE 1u   /* outputs stay in device memory                 */

/* ------------------------------------------------------------------------ */
/* Aggregate: fused filter -> project -> hash aggregate.                    */
/* ------------------------------------------------------------------------ */

/* Reducers of qdb/kernel/gen.cpp:3301-3593; AVG is lowered by the planner  */
/* into SUM and COUNT (qdb/plan/sql_lowering.cpp:799-814).                  */
typedef enum qdb_agg_func {
    QDB_AGG_COUNT_STAR = 1,
    QDB_AGG_COUNT = 2,
    QDB_AGG_SUM = 3,
    QDB_AGG_MIN = 4,
    QDB_AGG_MAX = 5
} qdb_agg_func;

typedef struct qdb_agg_item {
    int32_t func;       /* qdb_agg_func                                      */
    int32_t arg;        /* expression node, -1 for COUNT(*)                  */
} qdb_agg_item;

typedef struct qdb_aggregate_spec {
    int32_t n_columns;
    const qdb_column_type* columns;   /* input batch schema                 */
    int32_t n_nodes;
    const qdb_expr* nodes;
    int32_t filter;                   /* predicate node, -1 for none        */
    int32_t n_keys;
    const int32_t* keys;              /* GROUP BY key expression nodes      */
    int32_t n_aggs;
    const qdb_agg_item* aggs;
    /* Optional projection over the aggregate row (keys ++ aggregate        */
    /* results, in that order): output column k is output_nodes[outputs[k]] */
    /* whose COLUMN leaves index that row.  n_outputs == 0 emits the row.    */
    int32_t n_outputs;
    const int32_t* outputs;
    int32_t n_output_nodes;
    const qdb_expr* output_nodes;
    uint32_t flags;                   /* QDB_OUT_DEVICE                     */
    int64_t expected_groups;          /* sizing hint, 0 = unknown           */
} qdb_aggregate_spec;

/* agg_dispatch op codes (EAggregateKernelOp, qdb/kernel/compiler.h:217-230). */
#define QDB_AGG_OP_INIT 0
#define QDB_AGG_OP_UPDATE 1
#define QDB_AGG_OP_INIT_ROWS 3
#define QDB_AGG_OP_SWITCH_TO_ROWS_AT 4
#define QDB_AGG_OP_EXPECT_ROW_GROUPS 5

/* Size of the caller-owned, zero-initialised table state (HashTableSize,   */
/* qdb/kernel/compiler.h:603).  The int64 at byte offset 72 is the group    */
/* count (HashTable.Size), kept current after every call, as the processor   */
/* reads it (qdb/exec/aggregate_exec.cpp:18-38, :128).                       */
#define QDB_HASH_TABLE_SIZE 304

/* ------------------------------------------------------------------------ */
/* Row join (equi-join, build side fixed).                                  */
/* ------------------------------------------------------------------------ */

/* EJoinType (qdb/plan/ops/join_type.h:5-18), in its order.  Served, as by   */
/* TKernelCompiler::CompileRowJoin (qdb/kernel/compiler.cpp:3127-3148):      */
/*   INNER;                                                                  */
/*   LEFT with the right side built and RIGHT with the left side built: the  */
/*     preserved side streams through Probe, and a probe row that matches    */
/*     nothing (a NULL key included) is paired with a NULL build row;        */
/*   LEFT_SEMI / LEFT_ANTI with the left side built: Probe marks the build   */
/*     rows it matches and emits nothing; once the probe side has ended,     */
/*     EMIT_BY_MARK pairs the marked (SEMI) or unmarked (ANTI) build rows,   */
/*     in build order, and materialize writes build columns only.  An ANTI   */
/*     join keeps its NULL-key build rows in a second arena (APPEND_NULL_KEYS */
/*     with that arena), whose EMIT_BY_MARK pairs every row.                  */
/* The others are rejected at compile time.                                  */
typedef enum qdb_join_type {
    QDB_JOIN_INNER = 0,
    QDB_JOIN_LEFT = 1,
    QDB_JOIN_RIGHT = 2,
    QDB_JOIN_FULL = 3,
    QDB_JOIN_LEFT_SEMI = 4,
    QDB_JOIN_RIGHT_SEMI = 5,
    QDB_JOIN_LEFT_ANTI = 6,
    QDB_JOIN_RIGHT_ANTI = 7
} qdb_join_type;

typedef struct qdb_row_join_spec {
    int32_t join_type;                 /* qdb_join_type                      */
    int32_t build_is_left;             /* pair/output order (left, right)    */
    int32_t n_build_columns;
    const qdb_column_type* build_columns;
    int32_t n_probe_columns;
    const qdb_column_type* probe_columns;
    int32_t n_keys;
    const int32_t* build_keys;         /* build column per key               */
    const int32_t* probe_keys;         /* probe column per key               */
    int32_t n_payload;
    const int32_t* build_payload;      /* build columns kept in the rows     */
    /* Materialize output: column k is probe column out_column[k] when       */
    /* out_side[k] == 0, else build payload out_column[k].                   */
    int32_t n_out;
    const int32_t* out_side;
    const int32_t* out_column;
    /* Optional build-side predicate fused into Append (-1 = none); its      */
    /* COLUMN leaves index the build schema.                                 */
    int32_t n_build_nodes;
    const qdb_expr* build_nodes;
    int32_t build_filter;
    uint32_t flags;                    /* QDB_OUT_DEVICE                     */
} qdb_row_join_spec;

/* jr_dispatch op codes (ERowJoinKernelOp, qdb/kernel/compiler.h:363-388). */
#define QDB_JR_OP_INIT 0
#define QDB_JR_OP_APPEND 1
#define QDB_JR_OP_BUILD 2
#define QDB_JR_OP_PROBE 3
#define QDB_JR_OP_APPEND_NULL_KEYS 5   /* LEFT_ANTI: NULL-key rows, into the second arena */
#define QDB_JR_OP_EMIT_BY_MARK 6       /* LEFT_SEMI / LEFT_ANTI: appends (NULL, build row) pairs */

/* Caller-owned zeroed state sizes (qdb/kernel/compiler.h:599-621).  The    */
/* pair buffer's int64 at offset 0 is its pair count, read by               */
/* TRowJoinProcessor::ProbeBatch (qdb/exec/row_join_exec.cpp:176).           */
#define QDB_ROW_ARENA_SIZE 56
#define QDB_ROW_TABLE_SIZE 48
#define QDB_ROW_SCRATCH_SIZE 64
#define QDB_PAIR_BUFFER_SIZE 24

/* ------------------------------------------------------------------------ */
/* Sort (ORDER BY over packed row ids) and top-K.                           */
/* ------------------------------------------------------------------------ */

typedef struct qdb_sort_key {
    int32_t column;      /* key column of the store's row sets               */
    int32_t desc;        /* default direction; the run's descs[] overrides   */
    int32_t nulls_first; /* default; the run's nulls_firsts[] overrides      */
    int32_t pad;
} qdb_sort_key;

typedef struct qdb_sort_spec {
    int32_t n_columns;
    const qdb_column_type* columns;    /* schema of every stored row set     */
    int32_t n_keys;
    const qdb_sort_key* keys;          /* most significant first             */
    int32_t n_out;
    const int32_t* out_columns;        /* materialized columns               */
    uint32_t flags;                    /* QDB_OUT_DEVICE                     */
} qdb_sort_spec;

/* ------------------------------------------------------------------------ */
/* Programs.                                                                */
/* ------------------------------------------------------------------------ */

typedef struct qdb_gpu_program qdb_gpu_program;

/* TKernelCompiler::CompileAggregate (qdb/kernel/compiler.h:659-663).       */
qdb_gpu_program* qdb_gpu_compile_aggregate(
    const qdb_aggregate_spec* spec, char* err, size_t err_len);

/* TKernelCompiler::CompileFilter (qdb/kernel/compiler.h:632-633).          */
qdb_gpu_program* qdb_gpu_compile_filter(
    int32_t n_columns, const qdb_column_type* columns,
    int32_t n_nodes, const qdb_expr* nodes, int32_t predicate,
    char* err, size_t err_len);

/* TKernelCompiler::CompileProject (qdb/kernel/compiler.h:640-642): output   */
/* k is node exprs[k], written as its qdb_type's storage width.              */
qdb_gpu_program* qdb_gpu_compile_project(
    int32_t n_columns, const qdb_column_type* columns,
    int32_t n_nodes, const qdb_expr* nodes,
    int32_t n_exprs, const int32_t* exprs,
    char* err, size_t err_len);

/* TKernelCompiler::CompileAggregateHash / CompileJoinHash                  */
/* (qdb/kernel/compiler.h:691-697): rh_hash of the key columns.              */
qdb_gpu_program* qdb_gpu_compile_hash(
    int32_t n_columns, const qdb_column_type* columns,
    int32_t n_keys, const int32_t* key_columns,
    char* err, size_t err_len);

/* TKernelCompiler::CompileRowJoin (qdb/kernel/compiler.h:677-679).         */
qdb_gpu_program* qdb_gpu_compile_row_join(
    const qdb_row_join_spec* spec, char* err, size_t err_len);

/* Join fused with the aggregate downstream of it: `agg`'s input schema is   */
/* the probe columns followed by the build payload columns.  No reference    */
/* counterpart: it replaces the row join -> project -> aggregate chain       */
/* (qdb/exec/row_join_exec.cpp:166-188 feeding aggregate_exec.cpp:104-117).  */
qdb_gpu_program* qdb_gpu_compile_join_aggregate(
    const qdb_row_join_spec* join, const qdb_aggregate_spec* agg,
    char* err, size_t err_len);

/* TKernelCompiler::CompileRadixSortComposite / CompileHeapTopK             */
/* (qdb/kernel/compiler.h:644-653).                                          */
qdb_gpu_program* qdb_gpu_compile_sort(
    const qdb_sort_spec* spec, char* err, size_t err_len);

void qdb_gpu_program_destroy(qdb_gpu_program* program);

/* ------------------------------------------------------------------------ */
/* Reference-shaped entry points.                                           */
/* ------------------------------------------------------------------------ */

/* agg_dispatch(ht, batch, arg, op) (qdb/kernel/compiler.h:207-230).         */
/* Init/InitRows return 0 on failure; Update returns < 0 on failure; an op   */
/* the kernel does not serve returns 0 and changes nothing.                  */
int64_t qdb_gpu_agg_dispatch(const qdb_gpu_program* program, void* ht,
                             qdb_rowset* batch, int64_t arg, int64_t op);

/* agg_finish_rowset(ht, out) (qdb/kernel/compiler.h:232-242): writes every  */
/* group into `out`, returns the group count (< 0 on failure) and destroys   */
/* the table.  `out->Destroy` frees the output buffers.                      */
int64_t qdb_gpu_agg_finish_rowset(const qdb_gpu_program* program, void* ht,
                                  qdb_rowset* out);

/* TFilterDispatch (qdb/kernel/compiler.h:488-495): writes rs->Selection     */
/* (allocated by the caller, RowCount bytes) for the rows input_selection    */
/* selects (NULL = all); NULL predicates reject.                             */
void qdb_gpu_filter(const qdb_gpu_program* program, qdb_rowset* rs,
                    const uint8_t* input_selection);

/* TProjectDispatch (qdb/kernel/compiler.h:502-510).  `arena` is unused.     */
void qdb_gpu_project(const qdb_gpu_program* program, qdb_rowset* in,
                     void** out_buffers, void* arena,
                     const uint8_t* input_selection);

/* Hash dispatch (qdb/kernel/compiler.h:426-438, :513-520): one uint64 per   */
/* selected row, equal to the engine's rh_hash of the key (gen.cpp:233-379), */
/* so hash % P routes rows as THashShuffleTask does                          */
/* (qdb/scheduler/tasks/runtime_adapter.cpp:1001-1003).                      */
bool qdb_gpu_hash(const qdb_gpu_program* program, qdb_rowset* batch,
                  uint64_t* hashes);

/* jr_dispatch(arena, table, scratch, pairs, batch, op)                      */
/* (qdb/kernel/compiler.h:390-395); returns false on failure, and for an op  */
/* the program's join type does not use.  Probe replaces the pair buffer's   */
/* pairs; EMIT_BY_MARK appends to them (TRowJoinProcessor::Finish calls it   */
/* for the arena, then for the NULL-key arena, qdb/exec/row_join_exec.cpp).   */
bool qdb_gpu_jr_dispatch(const qdb_gpu_program* program, void* arena,
                         void* table, void* scratch, void* pairs,
                         qdb_rowset* batch, int64_t op);

/* jr_materialize(pairs, stream, start, limit, out)                          */
/* (qdb/kernel/compiler.h:397-405): returns the rows written (<= limit).     */
int64_t qdb_gpu_jr_materialize(const qdb_gpu_program* program, void* pairs,
                               qdb_rowset* stream, int64_t start,
                               int64_t limit, qdb_rowset* out);

/* Release of device state behind caller-owned state buffers.  The engine    */
/* keeps these states in its task heap and drops them with the task          */
/* (qdb/exec/row_join_exec.cpp:35-46 frees only row sets); a device library  */
/* has no such heap, so a binding calls these where the processor is         */
/* destroyed.  No reference counterpart.  Each pointer may be NULL; the      */
/* buffers are zeroed and may be initialised again.  Frees are ordered on    */
/* the library stream.                                                       */
void qdb_gpu_agg_release(void* ht);
void qdb_gpu_jr_release(void* arena, void* table, void* scratch, void* pairs);

/* Probe of a fused join-aggregate program: probes `batch` against the built */
/* arena/table and folds the joined rows into the aggregate state `ht`.      */
/* Returns the matched pair count, < 0 on failure.                           */
int64_t qdb_gpu_join_aggregate_probe(const qdb_gpu_program* program,
                                     void* arena, void* table, void* ht,
                                     qdb_rowset* batch);

/* Many joins of one program at once (the per-partition row tables of a     */
/* partitioned join, qdb/exec/row_join_exec.cpp:93-220, or the joins of many  */
/* queries of one template).  No reference counterpart as entries.           */
/* jr_build_batch: Build (jr_dispatch op 2) for n appended arenas in one     */
/* launch that clears every table and one that inserts every arena's rows;   */
/* these tables carry no Bloom filter or direct index (a table larger than   */
/* L2 still gets its own partitioned build).  Returns false on failure.      */
bool qdb_gpu_jr_build_batch(const qdb_gpu_program* program, void* const* arenas, void* const* tables, int64_t n);
/* jr_append_batch: Append (jr_dispatch op 1) of batches[i] to arenas[i] for  */
/* every i, waiting on the device once for all of them.  false on failure.   */
bool qdb_gpu_jr_append_batch(const qdb_gpu_program* program, void* const* arenas, qdb_rowset* const* batches,
                             int64_t n);
/* join_aggregate_probe_batch: qdb_gpu_join_aggregate_probe of batches[i]    */
/* into hts[i] for every i, in one persistent launch when the program has   */
/* the keyless join-sum shape (COUNT / SUM of products of the build payload */
/* and one probe column) and no batch has a selection; one by one otherwise. */
/* Returns the total matched pairs, < 0 on failure.                          */
int64_t qdb_gpu_join_aggregate_probe_batch(const qdb_gpu_program* program, void* const* arenas,
                                           void* const* tables, void* const* hts, qdb_rowset* const* batches,
                                           int64_t n);

/* qdb_sort_run (qdb/kernel/compiler.h:522-541, compiler.cpp:1165-1218).     */
/* With do_sort, sorts the n packed row ids (batch << 32 | row) in place by  */
/* the keys, stable in input order; then materializes [start, start+limit)   */
/* into `out` and returns its row count (0 at the end).  `work`/`counts`     */
/* may be NULL: the device path keeps its own scratch.                       */
int64_t qdb_gpu_sort_run(const qdb_gpu_program* program, qdb_rowset* store,
                         int64_t* row_ids, int64_t* work, uint32_t* counts,
                         int64_t n, bool* descs, bool* nulls_firsts,
                         bool do_sort, int64_t start, int64_t limit,
                         qdb_rowset* out);

/* qdb_top_k_select (THeapTopKDispatch, qdb/kernel/compiler.h:585-596):      */
/* keeps the first `limit` row ids of the stable order in row_ids[0..k)      */
/* and returns k.                                                            */
int64_t qdb_gpu_top_k_select(const qdb_gpu_program* program, qdb_rowset* store,
                             int64_t* row_ids, int64_t size, int64_t limit);

/* qdb_top_sort_update (TTopSortDispatch, qdb/kernel/compiler.h:570-583;    */
/* the update built by BuildTopSortUpdateAst, compiler.cpp:881-975), the     */
/* step of TTopSortProcessor::Add (qdb/exec/sort_exec.cpp:627-760) for a     */
/* LIMIT the heap rule turns away (K > 1024 or K > rows / 4).  `state` holds  */
/* the rows kept so far, in order (zeroed before the first call: no rows);    */
/* `batch` the new rows, named by row_ids[0, n) = (0 << 32) | row in         */
/* ascending order.  With sort_input the batch's rows are ordered here        */
/* (stable: equal keys keep row-id order); without it row_ids already lists  */
/* them in order (qdb_gpu_top_k_select's output).  They are merged with the  */
/* state, a state row first on equal keys, and the first `limit` rows are    */
/* materialized into `out` (every column: the program's out_columns must be  */
/* all columns in order, so `out` can be the next call's state).  Writes     */
/* pick_src[i] (0 = state, 1 = batch), pick_idx[i] (row in it) and           */
/* row_ids[i] = pick_src << 32 | pick_idx for the kept rows (host or device   */
/* arrays), and returns their count (0 when limit <= 0), < 0 on failure.     */
/* `work`/`counts` may be NULL: the device path keeps its own scratch.        */
/* Two NULL keys compare equal here (the earlier row first).                  */
int64_t qdb_gpu_top_sort_update(const qdb_gpu_program* program, qdb_rowset* state, qdb_rowset* batch,
                                int64_t* row_ids, int64_t* work, uint32_t* counts, int64_t n,
                                bool sort_input, uint8_t* pick_src, uint32_t* pick_idx, int64_t limit,
                                qdb_rowset* out);

/* ------------------------------------------------------------------------ */
/* Batched aggregation: many aggregate states of one program per launch.    */
/* ------------------------------------------------------------------------ */

/* Replaces a loop of agg_dispatch(ht, batch, 0, Update) over independent    */
/* aggregate tasks of one program (the partitions of a partitioned GROUP BY, */
/* qdb/exec/aggregate_exec.cpp:104-117 per task; or small aggregations of    */
/* many queries of one template): states[i] is updated with batches[i] as    */
/* one call of qdb_gpu_agg_dispatch would, all in one persistent launch.  A  */
/* zeroed state buffer is initialised first (as Init with no hint), its table */
/* taken from a device arena shared by the batch.  Block shape and work item */
/* size come from an autotuner (set QDB_AUTOTUNE=0 to keep the defaults); the */
/* launch sequence is replayed as a CUDA graph while the batch keeps its     */
/* structure.  High-cardinality programs run a shared tier in front of each  */
/* aggregate's table; keyless ones and ones whose hint is <= 64 groups fold  */
/* into lane-private accumulators per work item.  States whose program shape */
/* has no batched kernel (or whose columns are not on a four-value boundary, */
/* for the latter) are updated one by one.  Returns n, or < 0 on failure.    */
int64_t qdb_gpu_agg_dispatch_batch(const qdb_gpu_program* program, void* const* states,
                                   qdb_rowset* const* batches, int64_t n);

/* agg_finish_rowset (qdb/kernel/compiler.h:232-242) for n states in one      */
/* batched finalize: outs[i] receives state i's groups and the states are     */
/* destroyed and zeroed.  The outputs are slices of shared buffers, freed     */
/* when the last of them is destroyed.  Returns the total group count.       */
int64_t qdb_gpu_agg_finish_batch(const qdb_gpu_program* program, void* const* states, int64_t n,
                                 qdb_rowset* outs);

/* Calls Destroy on each of n row sets (the outputs of a batched finish):    */
/* one call instead of n for a binding that pays per foreign call.  No       */
/* reference counterpart.                                                    */
void qdb_gpu_release_rowsets(qdb_rowset* rowsets, int64_t n);

/* The autotuner's state as JSON (searches, timed trials, reuses, graph      */
/* replays, chosen configurations); returns the JSON length.  No reference   */
/* counterpart.                                                              */
int64_t qdb_gpu_autotune_info(char* buf, int64_t cap);
void qdb_gpu_autotune_reset(void);

/* ------------------------------------------------------------------------ */
/* Runtime join filter (qdb/kernel/join/runtime_filter.oz, driven by         */
/* qdb/exec/runtime_filter.cpp): a join's build side publishes its key       */
/* hashes as an exact set (at most MaxKeys distinct) or a blocked Bloom      */
/* filter, and the probe side's scan drops rows whose hash it rejects.       */
/* The four entries take the kernel's state structs (mirrored below, field   */
/* for field) with every array they point at in DEVICE memory; hashes,       */
/* selections and outputs passed to them are device arrays too.  Results     */
/* are the reference's, bit for bit: the build's mode, key count, key order  */
/* and Bloom words; the published kind, exact key count, table size, Bloom   */
/* words and set bits; the probe's output bytes (1 kept, 0 rejected).        */
/* ------------------------------------------------------------------------ */

/* RuntimeFilterBuild (runtime_filter.oz:29-41; TRuntimeFilterBuildState).   */
/* Mode 0 collecting, 1 deduplicating, 2 overflowing, 3 Bloom; Want 1 asks   */
/* for SortOrder / SortKeys / the set, 2 for Bloom storage (BloomWords >= 0). */
/* Keys has room for KeyCount + the batch's rows; SetSlots for SetCapacity   */
/* words (the device keeps its own set layout there; SetCtrl is unused);     */
/* SortOrder holds 2 * KeyCount + 256 words and SortKeys KeyCount.           */
typedef struct qdb_rf_build_state {
    int64_t MaxKeys;
    int64_t Mode;
    int64_t Want;
    uint64_t* Keys;
    int64_t KeyCount;
    uint8_t* SetCtrl;
    uint64_t* SetSlots;
    int64_t SetCapacity;
    uint32_t* SortOrder;
    uint64_t* SortKeys;
    uint64_t* Bloom;
    int64_t BloomWords;
} qdb_rf_build_state;

/* RuntimeFilterPartial (runtime_filter.oz:44-48).                           */
typedef struct qdb_rf_partial {
    const uint64_t* Keys;
    int64_t KeyCount;
    const uint64_t* Bloom;
    int64_t BloomWords;
} qdb_rf_partial;

/* RuntimeFilterPublish (runtime_filter.oz:56-69; TPublishState).  Kind: 0   */
/* cannot answer, 1 exact, 2 Bloom.  Table is zeroed and sized for           */
/* min(keys, MaxKeys) keys; Bloom is zeroed, or holds one fragment when      */
/* BloomSeeded.                                                              */
typedef struct qdb_rf_publish_state {
    int64_t MaxKeys;
    uint64_t* Keys;
    uint8_t* SetCtrl;
    uint64_t* SetSlots;
    int64_t SetCapacity;
    uint64_t* Table;
    uint64_t* Bloom;
    int64_t BloomWords;
    int64_t BloomSeeded;
    int64_t Kind;
    int64_t ExactKeys;
    int64_t TableSize;
    int64_t BloomSetBits;
} qdb_rf_publish_state;

/* RuntimeFilterData (runtime_filter.oz:72-75): Words is the exact table     */
/* (Kind 1) or the Bloom words (Kind 2).                                     */
typedef struct qdb_rf_data {
    int64_t Kind;
    const uint64_t* Words;
    int64_t WordCount;
} qdb_rf_data;

/* rf_build (runtime_filter.oz:419-499): adds the selected hashes to a        */
/* producer's contribution; returns the rows consumed (all of them unless    */
/* state->Want asks for storage), < 0 on failure.                            */
int64_t qdb_gpu_rf_build(qdb_rf_build_state* state, const uint64_t* hashes, const uint8_t* selection,
                         int64_t count);
/* rf_publish (runtime_filter.oz:502-556): merges the producers'             */
/* contributions into the published filter.  Returns 0, < 0 on failure.     */
int64_t qdb_gpu_rf_publish(qdb_rf_publish_state* state, const qdb_rf_partial* partials,
                           int64_t partial_count);
/* rf_probe (runtime_filter.oz:561-577): output[i] = 1 when selected row i's  */
/* hash may be in the filter, else 0; returns the kept count (< 0 on         */
/* failure).  `vectorized` and the two scratch arrays serve the CPU's vector */
/* probe and are ignored.                                                    */
int64_t qdb_gpu_rf_probe(const qdb_rf_data* data, const uint64_t* hashes, const uint8_t* selection,
                         uint8_t* output, int64_t count, int64_t vectorized, uint64_t* selected_hashes,
                         uint8_t* selected_output);
/* rf_merge (runtime_filter.oz:580-584): ORs Bloom fragment `source` into    */
/* `target` (count words).  Returns 0, < 0 on failure.                       */
int64_t qdb_gpu_rf_merge(uint64_t* target, const uint64_t* source, int64_t count);

/* The probe-side scan fused with the filter: for a hash program (the join   */
/* key's rh_hash, qdb_gpu_compile_hash), output[i] = 1 when batch row i is    */
/* selected and its key hash may be in the filter, without writing the       */
/* hashes.  Equals qdb_gpu_hash followed by qdb_gpu_rf_probe.  No reference  */
/* counterpart (the engine hashes, then probes).  `output` and the filter's  */
/* words are device memory; the batch may be host or device.  Returns the    */
/* kept count, < 0 on failure.                                               */
int64_t qdb_gpu_rf_probe_rowset(const qdb_gpu_program* hash_program, const qdb_rf_data* data,
                                qdb_rowset* batch, uint8_t* output);

/* ------------------------------------------------------------------------ */
/* Hash shuffle (THashShuffleTask, qdb/scheduler/tasks/runtime_adapter.h:444; */
/* its scatter of one batch, runtime_adapter.cpp:998-1112).                  */
/* ------------------------------------------------------------------------ */

/* Routes every selected row of `batch` to output routes[hash % n_routes],   */
/* or hash % n_outputs when n_routes is 0; the hash is batch->Hash when set, */
/* else the hash program's rh_hash of its key columns (qdb_gpu_hash), so a    */
/* row lands where the engine's shuffle sends it.  outs[0, n_outputs)         */
/* receive each output's rows in input order with every column of the        */
/* program's schema (fixed-width types and one-byte strings; bit-packed BOOL */
/* is rejected) and Hash pointing at their hashes.  Outputs are device-      */
/* resident slices of shared buffers (validity as MaskBitOffset into a shared */
/* bitmap), freed when the last is destroyed (qdb_gpu_release_rowsets).      */
/* Returns the rows routed, < 0 on failure — a row whose route is outside    */
/* [0, n_outputs) included, which the engine reports as a partition routed   */
/* nowhere.  No reference counterpart as an entry: the engine's task does    */
/* this on the host.                                                          */
int64_t qdb_gpu_shuffle(const qdb_gpu_program* hash_program, qdb_rowset* batch, const int64_t* routes,
                        int64_t n_routes, int64_t n_outputs, qdb_rowset* outs);

/* ------------------------------------------------------------------------ */
/* Device column cache: host scan batches (TParquetSource::Next,             */
/* qdb/io/parquet/source.h:89, 2^18-row batches, source.cpp:333) staged into  */
/* HBM through pinned buffers and kept resident across queries.  No         */
/* reference counterpart: the engine's kernels read host batches.           */
/* ------------------------------------------------------------------------ */

typedef struct qdb_gpu_column_cache qdb_gpu_column_cache;

typedef struct qdb_gpu_cache_stats {
    int64_t hits;             /* columns served from HBM                     */
    int64_t misses;           /* columns copied in                           */
    int64_t evictions;        /* columns dropped to stay within the budget   */
    int64_t resident_bytes;   /* bytes of cached columns in HBM              */
    int64_t pinned_bytes;     /* bytes of entries held by live row sets      */
    int64_t h2d_bytes;        /* bytes copied host -> device so far          */
    int64_t entries;          /* cached columns                              */
} qdb_gpu_cache_stats;

/* A cache holding at most budget_bytes of columns in HBM, staging copies   */
/* from pageable host memory through two pinned buffers of staging_bytes    */
/* each (0 picks 8 MiB), so that filling one overlaps the copy of the other. */
/* Copies run on the stream current at creation.  NULL on failure.          */
qdb_gpu_column_cache* qdb_gpu_cache_create(size_t budget_bytes, size_t staging_bytes);
/* Frees every cached column; row sets it handed out must be destroyed first. */
void qdb_gpu_cache_destroy(qdb_gpu_column_cache* cache);
/* A device row set of batch `batch_index` of source `source_id`: columns    */
/* columns[0, n) of `host` (typed by types[]) in that order.  A column       */
/* already resident under (source, batch, column) is used in place; the     */
/* others are copied in (data, and the validity bitmap when the host column  */
/* has one) and kept, the least recently used unpinned columns evicted to    */
/* stay within the budget.  The host batch's Selection is copied per call    */
/* and not cached.  The entries stay pinned until out->Destroy(out).         */
/* Returns 0, < 0 on failure (a batch larger than the budget included).      */
/* Re-entrant across host threads.                                          */
int64_t qdb_gpu_cache_get(qdb_gpu_column_cache* cache, uint64_t source_id, int64_t batch_index,
                          const qdb_rowset* host, const qdb_column_type* types, const int32_t* columns,
                          int32_t n, qdb_rowset* out);
/* Drops the unpinned columns of one source (its file changed); returns how */
/* many were dropped.                                                       */
int64_t qdb_gpu_cache_invalidate(qdb_gpu_column_cache* cache, uint64_t source_id);
void qdb_gpu_cache_get_stats(qdb_gpu_column_cache* cache, qdb_gpu_cache_stats* stats);

/* ------------------------------------------------------------------------ */
/* Aggregation without device allocation.                                   */
/* ------------------------------------------------------------------------ */

/* No counterpart in the reference: an addition for embedders that cannot     */
/* allocate device memory while a query runs — an engine that hands the GPU   */
/* a fixed memory budget up front and must not exceed it mid-query, or a      */
/* process whose device allocator belongs to another runtime (a host that     */
/* owns all of the device's memory through its own pool).                     */
/*                                                                           */
/* Runs one whole aggregate of an aggregate program (table set-up, the fused  */
/* filter -> project -> aggregate over `batch`, finalize) and writes the      */
/* groups into the caller's output columns.  Every column, mask and the       */
/* selection of `batch` must already be in device memory (nothing is copied), */
/* and out_columns[k] describes caller-owned device buffers for output        */
/* column k: Data holds out_capacity values (aligned to the value width);    */
/* Mask, when set, is (out_capacity + 31) / 32 uint32 words, 4-byte aligned   */
/* (all are cleared, then bit i set for a valid row i; bits past the group    */
/* count inside the last word written are unspecified); Offsets,             */
/* when set on a one-byte string column, out_capacity + 1 int32.             */
/* Returns the group count, or -1 (see qdb_gpu_last_error) when an input is   */
/* not in device memory, a buffer is misaligned, the groups exceed            */
/* out_capacity or the scratch table.  The call returns after the device     */
/* work has finished (it reads the group count back).                        */
/*                                                                           */
/* Table, counters and finalize scratch live in one file-scope device array   */
/* of QDB_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds      */
/* until the process exits.  It serves one-word group keys; the table holds  */
/* at most 2^18 groups with one state word, and fewer for wider states        */
/* (2^17 for 2 to 5 state words, e.g. COUNT, SUM, MIN, MAX and an f64 SUM);   */
/* the error message states the limit of the program at hand.  The first      */
/* call on a device looks up that array's device address, so make the first  */
/* call before any stream capture.  Calls share the array and each clears    */
/* what it uses: calls whose work overlaps on the GPU (other streams, other   */
/* host threads) race on it and must be serialised by the caller.  It runs on */
/* the stream set by qdb_gpu_set_stream.                                      */
#define QDB_NOALLOC_SCRATCH_BYTES (16u << 20)
int64_t qdb_gpu_agg_run_noalloc(const qdb_gpu_program* program, const qdb_rowset* batch,
                                qdb_column* out_columns, int64_t out_capacity);

/* ------------------------------------------------------------------------ */
/* Runtime.                                                                  */
/* ------------------------------------------------------------------------ */

/* Binds the calling thread to `device` (call once per thread). 0 = ok.      */
int qdb_gpu_init(int device);
/* Last error message of the calling thread ("" if none).                    */
const char* qdb_gpu_last_error(void);
/* cudaStream_t used by states initialised after this call on this thread;   */
/* NULL selects the library's own stream.                                    */
void qdb_gpu_set_stream(void* stream);
void* qdb_gpu_get_stream(void);
int qdb_gpu_synchronize(void);

/* Device and pinned host memory for column staging (the column cache).      */
void* qdb_gpu_alloc(size_t bytes);
void qdb_gpu_free(void* ptr);
void* qdb_gpu_host_alloc(size_t bytes);
void qdb_gpu_host_free(void* ptr);
int qdb_gpu_memcpy(void* dst, const void* src, size_t bytes);   /* async on the current stream */
int qdb_gpu_memset(void* dst, int value, size_t bytes);

/* Kernel timing: when enabled, every kernel launch of this library is       */
/* bracketed by CUDA events on its stream.  `read` copies up to `cap`        */
/* records (name, milliseconds) and clears the log; returns the count.       */
typedef struct qdb_gpu_kernel_time {
    char name[48];
    double ms;
    int64_t units;       /* rows (or items) the launch processed            */
} qdb_gpu_kernel_time;
void qdb_gpu_profile_enable(int on);
int64_t qdb_gpu_profile_read(qdb_gpu_kernel_time* out, int64_t cap);
/* Kernel launches of this library since the counter was last reset.         */
int64_t qdb_gpu_launch_count(int reset);

/* Seeded synthetic generators for the benchmark configurations (host, all   */
/* cores).  Every generator is deterministic in (seed, row).                 */
void qdb_gen_lineitem(uint64_t seed, int64_t rows, int64_t* qty, int64_t* price,
                      int64_t* disc, int64_t* tax, uint8_t* flag, uint8_t* status,
                      int32_t* shipdate);
void qdb_gen_join(uint64_t seed, int64_t build_rows, int64_t probe_rows,
                  int64_t fk_domain, int64_t* b_key, int64_t* b_payload,
                  int32_t* b_attr, int64_t* p_fk, int64_t* p_value);
void qdb_gen_zipf(uint64_t seed, int64_t rows, int64_t distinct, double s,
                  int64_t* key, int64_t* a, double* x);
void qdb_gen_sort(uint64_t seed, int64_t rows, int64_t* k1, int32_t* k2,
                  int64_t* rowid);

#ifdef __cplusplus
}
#endif

#endif /* QDB_GPU_H */
