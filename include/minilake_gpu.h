/*
 * minilake_gpu.h — C ABI of the B200 (sm_100a) execution core for MiniLake's
 * data-parallel hot path: filter/projection expressions over selection vectors
 * and dictionary codes, hash aggregation, hash-join build/probe and top-N.
 *
 * The entry points mirror MiniLake's pipeline contract
 * (crates/minilake-exec/src/pipeline.rs:32-79):
 *   Operator  { execute(&self, Batch) }            -> ml_gpu_filter / ml_gpu_project /
 *                                                    ml_gpu_join_probe
 *   Sink      { create_local, finalize }           -> ml_gpu_{hashagg,join_build,topn}_create /
 *                                                    *_finalize
 *   LocalSink { sink(&mut self, Batch), combine }  -> ml_gpu_*_local_create / *_sink /
 *                                                    *_combine
 * A sink may be given a "prologue": the streaming operators (Filter,
 * Projection, HashJoinProbe) that sit between the pipeline's source and the
 * sink. The sink's kernel then runs the whole pipeline for one morsel in one
 * pass over HBM, without materializing selection vectors or join pairs.
 *
 * Conventions
 *  - Every function returns an int status (ML_OK == 0). On failure the message
 *    is available from ml_gpu_last_error() (thread-local). Nothing aborts and
 *    no kernel traps: device-side failures (hash-table overflow, bounded waits
 *    that ran out) are reported through a device error word that the host reads.
 *  - Column buffers are BORROWED for the duration of the call
 *    (crates/minilake-exec/src/pipeline.rs:109-161 hands each batch to the
 *    operator by value; the FFI takes (ptr, len) views).  A column may live in
 *    host memory (it is staged through pinned memory and copied with
 *    cudaMemcpyAsync) or in device memory (used in place).
 *  - Handles are owned by the caller and released with the matching *_destroy.
 *  - All calls are thread-safe.  Each local-sink handle owns a CUDA stream, so
 *    morsels pushed from different threads run concurrently on the device.
 */
#ifndef MINILAKE_GPU_H
#define MINILAKE_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes: crates/minilake-core/src/error.rs:8-48 ------------------ */
enum {
    ML_OK = 0,
    ML_ERR_INVALID = 1,     /* MiniLakeError::Internal / Execution (bad arguments, type errors) */
    ML_ERR_BUDGET = 2,      /* MiniLakeError::ResourcesExhausted (memory.rs:114-128) */
    ML_ERR_CUDA = 3,        /* a CUDA runtime call failed */
    ML_ERR_TIMEOUT = 4,     /* a bounded device-side wait ran out */
    ML_ERR_UNSUPPORTED = 5, /* MiniLakeError::Unsupported */
    ML_ERR_INTERNAL = 6,
    ML_ERR_STALE_PLAN = 7   /* a prepared query's data no longer fits its plan: prepare it again */
};

/* ---- data types: crates/minilake-core/src/types.rs:15-28 -------------------- */
enum {
    ML_TYPE_BOOL = 0,    /* one byte per value (Vec<bool>) */
    ML_TYPE_INT32 = 1,
    ML_TYPE_INT64 = 2,
    ML_TYPE_FLOAT64 = 3,
    ML_TYPE_DATE = 4,    /* i32 days since 1970-01-01 */
    ML_TYPE_UTF8 = 5,
    ML_TYPE_NULL = 6     /* untyped NULL literal only */
};

/* ---- string encodings: crates/minilake-core/src/column.rs:126-150 ----------- */
enum {
    ML_ENC_PLAIN = 0, /* values (or offsets+bytes for UTF8) */
    ML_ENC_DICT = 1   /* u32 codes + dictionary (offsets+bytes), ColumnData::Dict */
};

enum { ML_LOC_HOST = 0, ML_LOC_DEVICE = 1 };

/*
 * A borrowed column view.  Layout follows minilake-core:
 *  - fixed width: `data` holds `len` values (bool: u8 0/1, i32, i64, f64, date i32)
 *  - UTF8 plain: `offsets` has len+1 u32 entries into `data` (bytes), column.rs:14-22
 *  - UTF8 dict:  `data` holds len u32 codes; the dictionary is `dict_offsets`
 *    (dict_len+1 u32) + `dict_data` (bytes), column.rs:126-131.  Dictionaries are
 *    always host memory (they are small: <= 65,536 entries, parquet_reader.rs:173).
 *  - validity: optional u64 words, bit i = row i is valid, LSB first (bitmap.rs:1-12)
 */
typedef struct ml_column {
    int32_t dtype;
    int32_t encoding;
    int32_t location;
    int32_t _pad;
    int64_t len;
    const void* data;
    const uint32_t* offsets;
    const uint64_t* validity;
    int64_t dict_len;
    const uint32_t* dict_offsets;
    const uint8_t* dict_data;
} ml_column;

/* ---- expressions: crates/minilake-exec/src/expr/mod.rs:18-173 --------------- */
enum { /* BinaryOp, expr/mod.rs:20-47 */
    ML_BIN_ADD = 0, ML_BIN_SUB, ML_BIN_MUL, ML_BIN_DIV, ML_BIN_MOD,
    ML_BIN_EQ, ML_BIN_NOTEQ, ML_BIN_LT, ML_BIN_LTEQ, ML_BIN_GT, ML_BIN_GTEQ,
    ML_BIN_AND, ML_BIN_OR
};

enum { /* PhysicalExpr variants, expr/mod.rs:109-173 */
    ML_EXPR_COLUMN = 0,  /* i64 = column index in the input batch */
    ML_EXPR_LITERAL = 1, /* dtype + i64 / f64 / str */
    ML_EXPR_BINARY = 2,  /* op = ML_BIN_*, 2 children */
    ML_EXPR_NOT = 3,     /* 1 child */
    ML_EXPR_NEGATE = 4,  /* 1 child */
    ML_EXPR_IS_NULL = 5, /* flag = negated (IS NOT NULL), 1 child */
    ML_EXPR_LIKE = 6,    /* flag = negated, str = pattern, 1 child */
    ML_EXPR_IN_LIST = 7, /* flag = negated, child 0 = operand, children 1.. = literals */
    ML_EXPR_CASE = 8,    /* flag = has ELSE; children: cond0, val0, cond1, val1, ..., [else];
                            dtype = result type */
    ML_EXPR_CAST = 9     /* dtype = target type, 1 child */
};

/*
 * One node of an expression tree, serialized in prefix order: a node is
 * followed by its `nchild` subtrees.
 */
typedef struct ml_expr_node {
    int32_t kind;
    int32_t op;     /* BINARY: ML_BIN_* */
    int32_t dtype;  /* LITERAL: value type; CAST: target; CASE: result type */
    int32_t nchild;
    int32_t flag;   /* negated / has_else */
    int32_t _pad;
    int64_t i64;    /* COLUMN: index; LITERAL int/bool/date value */
    double f64;     /* LITERAL float value */
    const char* str;/* LITERAL utf8 value / LIKE pattern (not NUL-terminated) */
    int64_t str_len;
} ml_expr_node;

/* One expression = pointer to its first node + node count. */
typedef struct ml_expr {
    const ml_expr_node* nodes;
    int32_t nnodes;
    int32_t dtype; /* the planner's output type for this expression (evaluate_to_column's dt) */
} ml_expr;

/* ---- aggregates: operators/aggregate/accumulator.rs:25-38 ------------------- */
enum { ML_AGG_COUNT_STAR = 0, ML_AGG_COUNT, ML_AGG_SUM, ML_AGG_AVG, ML_AGG_MIN, ML_AGG_MAX };

typedef struct ml_agg_spec {  /* AggregateExpr, operators/aggregate/mod.rs:22-31 */
    int32_t func;
    int32_t arg_type;   /* type of the argument expression; ignored for COUNT(*) */
    ml_expr arg;        /* nnodes == 0 for COUNT(*) */
} ml_agg_spec;

typedef struct ml_sort_key {  /* SortKey, operators/sort.rs:25-32 */
    ml_expr expr;
    int32_t asc;
    int32_t nulls_first;
} ml_sort_key;

/* ---- streaming operators (the prologue of a fused sink) --------------------- */
enum { ML_PIPE_FILTER = 0, ML_PIPE_PROJECT = 1, ML_PIPE_PROBE = 2 };

typedef struct ml_join_table ml_join_table; /* finalized JoinBuildSink (JoinTableRef, join.rs:58) */

typedef struct ml_pipe_op {
    int32_t kind;
    int32_t nexprs;
    const ml_expr* exprs;  /* FILTER: 1 predicate; PROJECT: output exprs; PROBE: probe key exprs */
    ml_join_table* join;   /* PROBE only */
    int32_t build_is_left; /* PROBE only: output = build columns ++ probe columns (join.rs:252-253) */
    int32_t _pad;
} ml_pipe_op;

/* ---- opaque handles ---------------------------------------------------------- */
typedef struct ml_ctx ml_ctx;
typedef struct ml_batch ml_batch;          /* device-resident columns (an HBM table or a sink's output) */
typedef struct ml_hashagg ml_hashagg;      /* HashAggregateSink */
typedef struct ml_hashagg_local ml_hashagg_local; /* HashAggLocal */
typedef struct ml_join_build ml_join_build;
typedef struct ml_join_build_local ml_join_build_local;
typedef struct ml_topn ml_topn;
typedef struct ml_topn_local ml_topn_local;

/* ---- context, memory pool, errors -------------------------------------------- */
/* flags: ML_CTX_PROFILE times the library's main kernels with CUDA events recorded on the
 * stream each kernel is launched on (read back with ml_gpu_profile_read).
 * ML_CTX_INTERPRET runs every fused pipeline through the ahead-of-time interpreter kernels;
 * by default the filter, aggregate, join-build and cardinality pipelines are specialized at run
 * time (NVRTC, compiled once per pipeline shape and cached for the process).  Both give the same
 * results.  Floating-point SUM/AVG accumulate with atomics, so they agree with a sequential sum
 * within rounding, not bit for bit from run to run.  ML_CTX_SPILL lets a hash aggregate outgrow the
 * HBM budget (ExecConfig::spill_dir, context.rs:14-34): when the budget refuses a table resize,
 * every group's partial state moves to host memory, split into 16 partitions by key hash, and
 * finalize merges one partition at a time (aggregate/hash.rs:189-281, 330-425).  Any other flag
 * bit is rejected. */
enum { ML_CTX_PROFILE = 2, ML_CTX_INTERPRET = 4, ML_CTX_SPILL = 8 };

/* ExecConfig (context.rs:14-34) for one device: hbm_budget_bytes is the query-wide
 * MemoryPool limit (memory.rs:22-26) applied to device bytes; 0 = unlimited. */
int ml_gpu_ctx_create(int device, uint64_t hbm_budget_bytes, uint32_t flags, ml_ctx** out);
int ml_gpu_ctx_destroy(ml_ctx* ctx);
/* MemoryPool::used / peak / limit (memory.rs:39-53). */
int ml_gpu_pool_stats(ml_ctx* ctx, uint64_t* used, uint64_t* peak, uint64_t* limit);
/* Details of the last ML_ERR_BUDGET on this thread: ResourcesExhausted{operator, requested,
 * used, limit} (error.rs).  `op` receives a NUL-terminated operator name. */
int ml_gpu_last_budget_error(char* op, size_t op_cap, uint64_t* requested, uint64_t* used,
                             uint64_t* limit);
const char* ml_gpu_last_error(void);
/* Wait for all work issued on the context (every stream). */
int ml_gpu_ctx_synchronize(ml_ctx* ctx);

/* ---- device-resident batches ------------------------------------------------- */
/* Copy columns into HBM (pinned staging + cudaMemcpyAsync); the batch is reserved
 * against the pool like a join build side (join.rs:122-157). */
int ml_gpu_batch_upload(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows,
                        ml_batch** out);
int ml_gpu_batch_num_rows(const ml_batch* b, int64_t* nrows);
int ml_gpu_batch_num_columns(const ml_batch* b, int32_t* ncols);
/* Device views of the columns (location = ML_LOC_DEVICE), for feeding another operator. */
int ml_gpu_batch_columns(const ml_batch* b, ml_column* out, int32_t ncols);
/* dtype and, for UTF8 columns, the number of string bytes (to size fetch buffers). */
int ml_gpu_batch_column_info(const ml_batch* b, int32_t col, int32_t* dtype, int64_t* str_bytes,
                             int32_t* has_validity);
/* Copy one column to caller-allocated host buffers.  `values`: len values (UTF8: str_bytes
 * bytes); `offsets`: len+1 (UTF8 only); `validity`: ceil(len/64) words or NULL. */
int ml_gpu_batch_fetch(const ml_batch* b, int32_t col, void* values, uint32_t* offsets,
                       uint64_t* validity);
int ml_gpu_batch_destroy(ml_batch* b);

/* ---- Operator: FilterOperator (operators/filter.rs:19-25, expr/eval.rs:167-196) --- */
/* Rows of the selection (or of 0..n when sel_in is NULL) where `pred` is TRUE, in increasing
 * order.  sel_out must have room for n (or nsel_in) entries; sel_in/sel_out are host or
 * device memory as `location` says.  The call's device temporaries (flag words, counts, the
 * selection) are charged to the context's HBM budget: ML_ERR_BUDGET when it has no room. */
int ml_gpu_filter(ml_ctx* ctx, const ml_expr* pred, const ml_column* cols, int32_t ncols,
                  int64_t nrows, const uint32_t* sel_in, int64_t nsel_in, int32_t location,
                  uint32_t* sel_out, int64_t* nsel_out);

/* ---- FilterOperator without allocation (no counterpart in the reference) ----------- */
/* ml_gpu_filter for callers that cannot allocate device memory: a query whose HBM budget
 * is spent (ml_gpu_filter, like every new reservation, would fail with ML_ERR_BUDGET) but
 * that still has to filter, and latency-critical callers for which cudaMalloc / cudaFree are
 * off limits because they can synchronize the whole device.  Same predicate semantics, inputs and
 * result as ml_gpu_filter (ordered selection, count on the host), with these limits:
 *  - every column is device resident (ML_LOC_DEVICE); sel_in (optional) and sel_out are
 *    device pointers; sel_out has room for nsel_in (or nrows) entries;
 *  - at most 16,777,216 rows per call (selected rows when sel_in is given), 2048 program
 *    instructions, 64 KiB of literals and 512 KiB of dictionary tables; a larger call fails
 *    with ML_ERR_INVALID and a message that names the limit;
 *  - its temporaries live in one static device array of 2,953,472 bytes per device, whose
 *    address the first call on a device looks up (cudaGetSymbolAddress, with that device
 *    current): make that first call before any stream capture.  Nothing in the array has
 *    to start at zero (each call clears its own error word);
 *  - calls on the same device share the array, so overlapping calls would race on it: each
 *    call holds a per-device lock until its work on the device has finished (a call that
 *    fails part-way drains its stream before it releases the lock).
 * It allocates no device memory and no pinned host memory; the predicate is compiled on the
 * host heap. */
int ml_gpu_filter_static(ml_ctx* ctx, const ml_expr* pred, const ml_column* cols, int32_t ncols,
                         int64_t nrows, const uint32_t* sel_in, int64_t nsel_in, uint32_t* sel_out,
                         int64_t* nsel_out);

/* ---- Operator: ProjectionOperator (operators/projection.rs:21-32) -------------- */
/* Evaluate `expr` over ALL physical rows into a new device column (batch of 1 column). */
int ml_gpu_project(ml_ctx* ctx, const ml_expr* expr, const ml_column* cols, int32_t ncols,
                   int64_t nrows, ml_batch** out);

/* ---- kernels/hash.rs:16-23: one hash per active row over the key columns -------- */
int ml_gpu_hash_columns(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows,
                        const uint32_t* sel, int64_t nsel, int32_t location, uint64_t* out);

/* ---- exchange step of the multi-GPU plan (minilake-dist/src/split.rs:54-127) ----- */
/* Reorder a batch's rows by partition: partition = hash_columns of the key columns
 * (kernels/hash.rs:16-23) modulo nparts (1..64).  *out holds the rows grouped by partition,
 * partition 0 first, each partition's rows in input order; counts[p] receives partition p's row
 * count (nparts entries).  MiniLake's distributed mode merges every worker's partial aggregate
 * on its coordinator; the multi-GPU plan sends each partial group to the rank that owns its key
 * hash instead, so every rank merges 1/nparts of the groups.  Columns may be host or device
 * memory; the output is device resident. */
int ml_gpu_partition(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows, const int32_t* key_cols,
                     int32_t nkeys, int32_t nparts, ml_batch** out, int64_t* counts);

/* ---- Sink: HashAggregateSink (operators/aggregate/hash.rs:285-484) ------------- */
/* `input_types` describes the pipeline source's columns (the prologue's first input).
 * `size_hint` presizes the device table (expected number of groups; 0 = start small and
 * grow on overflow, swiss.rs:287-301). */
int ml_gpu_hashagg_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue,
                          const int32_t* input_types, int32_t ninput, const ml_expr* group_exprs,
                          int32_t ngroup, const ml_agg_spec* aggs, int32_t nagg,
                          int64_t size_hint, ml_hashagg** out);
int ml_gpu_hashagg_local_create(ml_hashagg* sink, ml_hashagg_local** out);
/* LocalSink::sink: run the prologue and the aggregation over one morsel.  `sel` (optional)
 * is the batch's selection vector (batch.rs:8-14). */
int ml_gpu_hashagg_sink(ml_hashagg_local* local, const ml_column* cols, int32_t ncols,
                        int64_t nrows, const uint32_t* sel, int64_t nsel);
/* LocalSink::combine: merge into the global state (device-side partial-state merge). */
int ml_gpu_hashagg_combine(ml_hashagg_local* local);
/* Sink::finalize: final values (AVG = sum/count, seen-flags -> NULL), one row per group:
 * key columns then one column per aggregate (hash.rs:307-314). */
int ml_gpu_hashagg_finalize(ml_hashagg* sink, ml_batch** out);
/* Number of groups, table capacity and number of resize-on-overflow events so far. */
int ml_gpu_hashagg_stats(ml_hashagg* sink, int64_t* groups, int64_t* capacity, int64_t* resizes);
/* With ML_CTX_SPILL: how often the groups moved to host memory and how many group states moved
 * in all (the spill files and bytes of OperatorMetrics, aggregate/hash.rs:270-279). */
int ml_gpu_hashagg_spill_stats(ml_hashagg* sink, int64_t* spills, int64_t* spilled_groups);
int ml_gpu_hashagg_destroy(ml_hashagg* sink);

/* ---- resident hash aggregates for a serving loop (no counterpart in the reference) ---- */
/* Re-point a sink at new constants: the arguments are those of ml_gpu_hashagg_create (minus
 * the size hint) and must compile to the same pipeline shape, differing only in literal
 * values, LIKE patterns of the same length, and the join tables probed.  ML_ERR_INVALID
 * otherwise.  The sink's device state is kept. */
int ml_gpu_hashagg_rebind(ml_hashagg* sink, const ml_pipe_op* prologue, int32_t nprologue,
                          const int32_t* input_types, int32_t ninput, const ml_expr* group_exprs,
                          int32_t ngroup, const ml_agg_spec* aggs, int32_t nagg);
/* Empty the sink's groups and accumulators, keeping its tables allocated (size included). */
int ml_gpu_hashagg_reset(ml_hashagg* sink);
/* Sink one batch of device-resident columns from the calling thread (one call at a time per
 * sink), as a CUDA graph: with `reset` the graph first empties the group state, then runs the
 * fused pipeline kernel and reads back its overflow count and error word.  The graph is
 * captured on the second call with a given set of launch parameters (columns, the constants'
 * buffers, join tables, table size; the first such call runs the same steps without a graph)
 * and replayed by later calls; a table that overflows grows and the rows that did not fit are
 * aggregated again outside the graph.  Finalize as usual. */
int ml_gpu_hashagg_run_resident(ml_hashagg* sink, const ml_column* cols, int32_t ncols, int64_t nrows,
                                int32_t reset);
/* Graphs captured and graph launches replayed by ml_gpu_hashagg_run_resident. */
int ml_gpu_hashagg_graph_stats(ml_hashagg* sink, uint64_t* built, uint64_t* replayed);

/* ---- Sink: JoinBuildSink (operators/join.rs:72-242) --------------------------- */
/* `build_input_types`: columns of the batches pushed into the build side (after the
 * prologue, these become the build batch whose columns HashJoinProbe gathers). */
int ml_gpu_join_build_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue,
                             const int32_t* input_types, int32_t ninput, const ml_expr* key_exprs,
                             int32_t nkeys, ml_join_build** out);
int ml_gpu_join_build_local_create(ml_join_build* sink, ml_join_build_local** out);
int ml_gpu_join_build_sink(ml_join_build_local* local, const ml_column* cols, int32_t ncols,
                           int64_t nrows, const uint32_t* sel, int64_t nsel);
int ml_gpu_join_build_combine(ml_join_build_local* local);
/* Sink::finalize -> build_table (join.rs:160-203).  The table stays owned by the sink.
 * A single integer key (int32/date/int64 build column) whose value range spans at most
 * 4 entries per build row (+1024), or at most 2^20 entries, is indexed directly by value;
 * other keys use the hash table.  Both give the same matches. */
int ml_gpu_join_build_finalize(ml_join_build* sink, ml_join_table** table);
/* capacity: hash-table slots, or the value range of a direct (dense) index. */
int ml_gpu_join_table_stats(const ml_join_table* t, int64_t* build_rows, int64_t* distinct_keys,
                            int64_t* capacity);
int ml_gpu_join_build_destroy(ml_join_build* sink);

/* ---- Operator: HashJoinProbe (operators/join.rs:244-337) ----------------------- */
/* All (probe_row, build_row) pairs of the active rows.  Pairs are ordered by probe row.
 * out arrays need `cap` entries; *npairs receives the count (if it exceeds cap, nothing is
 * written and ML_ERR_INVALID is returned with *npairs set, so the caller can retry). */
int ml_gpu_join_probe(ml_ctx* ctx, ml_join_table* table, const ml_expr* key_exprs, int32_t nkeys,
                      const ml_column* cols, int32_t ncols, int64_t nrows, const uint32_t* sel,
                      int64_t nsel, int32_t location, uint32_t* probe_idx, uint32_t* build_idx,
                      int64_t cap, int64_t* npairs);

/* ---- Sink: SortSink (ORDER BY [LIMIT]; operators/sort.rs:85-132, 186-267) ------- */
/* Output = the input columns (after the prologue) of the best `limit` rows, sorted; limit < 0
 * is ORDER BY without a limit (every row).  Limits up to 2048 keep each morsel's best rows with
 * the per-warp top-N kernels; no limit, a larger one, or a dictionary-coded sort key sorts every
 * row with a stable radix sort (equal keys keep their input order). */
int ml_gpu_topn_create(ml_ctx* ctx, const ml_pipe_op* prologue, int32_t nprologue,
                       const int32_t* input_types, int32_t ninput, const ml_sort_key* keys,
                       int32_t nkeys, int64_t limit, ml_topn** out);
int ml_gpu_topn_local_create(ml_topn* sink, ml_topn_local** out);
int ml_gpu_topn_sink(ml_topn_local* local, const ml_column* cols, int32_t ncols, int64_t nrows,
                     const uint32_t* sel, int64_t nsel);
int ml_gpu_topn_combine(ml_topn_local* local);
int ml_gpu_topn_finalize(ml_topn* sink, ml_batch** out);
int ml_gpu_topn_destroy(ml_topn* sink);

/* ---- Parquet column-chunk decode (parquet_reader.rs:215-294 read_column_chunk,
 *      :176-212 encode_strings) ------------------------------------------------------ */
/* Parquet physical types (parquet.thrift Type) and compression codecs (CompressionCodec). */
enum { ML_PQ_BOOLEAN = 0, ML_PQ_INT32 = 1, ML_PQ_INT64 = 2, ML_PQ_FLOAT = 4, ML_PQ_DOUBLE = 5,
       ML_PQ_BYTE_ARRAY = 6, ML_PQ_FIXED_LEN_BYTE_ARRAY = 7 };
enum { ML_PQ_CODEC_UNCOMPRESSED = 0, ML_PQ_CODEC_SNAPPY = 1 };
/* Conversion (parquet_reader.rs:31-56): how the leaf column becomes a MiniLake column. */
enum { ML_PQ_CONV_BOOL = 0, ML_PQ_CONV_INT32, ML_PQ_CONV_DATE, ML_PQ_CONV_INT64, ML_PQ_CONV_FLOAT,
       ML_PQ_CONV_DOUBLE, ML_PQ_CONV_UTF8, ML_PQ_CONV_DECIMAL_I32, ML_PQ_CONV_DECIMAL_I64,
       ML_PQ_CONV_DECIMAL_BYTES };
/* Decode one column chunk of a row group: `chunk` holds its pages as stored in the file (the
 * dictionary page, when there is one, then the data pages, each after its Thrift page header),
 * in host memory; `num_rows` is the row group's row count and `max_def` the column's maximum
 * definition level (0: required).  Pages may be PLAIN, RLE_DICTIONARY / PLAIN_DICTIONARY or
 * (booleans) RLE encoded, DATA_PAGE or DATA_PAGE_V2, uncompressed or Snappy.  The one-column
 * batch holds what read_column_chunk returns: one slot per row (NULL rows hold 0), a validity
 * bitmap only when some value is NULL, FLOAT and DECIMAL(scale) as f64 (x / 10^scale), and
 * strings dictionary-encoded in order of first occurrence when there are at most
 * clamp(num_rows / 8, 1, 65536) distinct values (NULL rows count as ""), else plain.
 * Decompression, level and index decoding, value conversion and the string dictionary run on
 * the device; the host reads the page headers.  ML_ERR_INVALID for a malformed chunk,
 * ML_ERR_UNSUPPORTED for other codecs, encodings or repeated columns. */
int ml_gpu_parquet_decode(ml_ctx* ctx, const uint8_t* chunk, int64_t chunk_bytes, int32_t physical_type,
                          int32_t type_length, int32_t conversion, int32_t scale, int32_t codec,
                          int64_t num_rows, int32_t max_def, ml_batch** out);

/* ---- Prepared query: a plan's pipelines as one CUDA graph (executor.rs:270-288) ---- */
/* The pipelines of one physical plan over device-resident batches, in dependency order: join
 * builds, then one hash aggregate whose prologue probes their tables, then (optionally) a top-N
 * of the aggregate's output.  The first ml_gpu_query_run runs them through the sink calls above
 * and records what depends on the data: each dense join index's key range (or hash capacity),
 * whether build keys repeat, the group table's capacity and the result's row count.  Every later
 * run replays all of it as one CUDA graph launch over the same buffers -- the build columns are
 * copied in and the join indexes rebuilt, the group table reset and the fused kernel run, the
 * groups' final values written, the top-N taken -- so it recomputes the result from the current
 * contents of the batches.  Kernels in the graph check each recorded choice against the data;
 * a failed check returns ML_ERR_STALE_PLAN (no result; the sinks hold partial state) and every
 * later run does too: create the sinks and the query again.  A plan the graph cannot replay
 * (a build pipeline with filters or computed columns, string build columns or group keys,
 * sort keys that are not output columns, a limit above 32, a spilled aggregate, an empty
 * result) runs once; later runs return ML_ERR_UNSUPPORTED,
 * and ml_gpu_query_stats gives the reason.  The sinks and batches must outlive the query, and
 * nothing else may use the sinks meanwhile. */
typedef struct ml_query ml_query;
int ml_gpu_query_create(ml_ctx* ctx, ml_query** out);
/* Runs the build pipeline over the device-resident batch now and returns its table, for the
 * Probe operators of the aggregate's prologue. */
int ml_gpu_query_add_build(ml_query* q, ml_join_build* sink, const ml_column* cols, int32_t ncols,
                           int64_t nrows, ml_join_table** table);
int ml_gpu_query_set_aggregate(ml_query* q, ml_hashagg* sink, const ml_column* cols,
                               int32_t ncols, int64_t nrows);
/* ORDER BY keys[] LIMIT limit (limit > 0) over the aggregate's output columns. */
int ml_gpu_query_set_topn(ml_query* q, const ml_sort_key* keys, int32_t nkeys, int64_t limit);
int ml_gpu_query_run(ml_query* q, ml_batch** out);
/* A replay of a planned top-N query whose result goes to host memory inside the graph (no
 * device batch): *nrows result rows, read with ml_gpu_query_result.  ML_ERR_UNSUPPORTED before
 * the planning run (ml_gpu_query_run) or for a plan that is not replayed. */
int ml_gpu_query_run_host(ml_query* q, int64_t* nrows);
/* Column `col` of the last ml_gpu_query_run_host result: nrows values (fixed width) and, when
 * the column has one, its validity words ((nrows + 63) / 64 u64). */
int ml_gpu_query_result(const ml_query* q, int32_t col, void* values, uint64_t* validity,
                        int32_t* has_validity);
/* runs, graph replays, kernels per replay, and why the plan is not replayed ("" if it is). */
int ml_gpu_query_stats(const ml_query* q, int64_t* runs, int64_t* replays, int32_t* kernels,
                       char* why, int32_t why_cap);
int ml_gpu_query_destroy(ml_query* q);

/* ---- learned cardinality estimator (no counterpart in the reference) ------------- */
/* Predicts log2 of the number of distinct keys (GROUP BY groups, join-build keys; a NULL key
 * counts as one group) from scan statistics, to presize hash tables.  Sizing never changes a
 * result: an underestimate falls back to resize-on-overflow. */
enum { ML_CARD_FEATURES = 72, ML_CARD_PARAMS = 13057 };

/* One pass over the key expressions of the active rows: a HyperLogLog sketch (2^14 registers
 * of the engine's key hash) and scan statistics, as the estimator's 72 FP32 features:
 *   [0, 64)  fraction of registers holding each value 0..63;
 *   64 log2(rows + 1) / 32;   65 log2(max - min + 1) / 64 of the first normalized key word
 *   over non-NULL rows;  66 NULL-key fraction;  67 log2(HLL estimate + 1) / 32;
 *   68 key expressions / 4;  69 normalized key bits / 128;
 *   70 log2(min(rows, max - min + 1) + 1) / 32;  71 1 if any key is NULL, else 0.
 * hll_estimate (optional) receives the HyperLogLog estimate (linear counting when small). */
int ml_gpu_card_features(ml_ctx* ctx, const ml_column* cols, int32_t ncols, int64_t nrows,
                         const uint32_t* sel, int64_t nsel, int32_t location, const ml_expr* keys,
                         int32_t nkeys, float* features, double* hll_estimate);

typedef struct ml_card_model ml_card_model;
/* FP32 MLP 72 -> 64 -> 64 -> 64 -> 1 (ReLU); the prediction of log2(distinct) is the MLP's
 * output plus 32 * feature 67 (= log2(HLL estimate + 1)), so the network learns the sketch's
 * correction.  Parameters are laid out
 * [W1 (64x72, row-major [out][in]), b1, W2 (64x64), b2, W3 (64x64), b3, W4 (1x64), b4];
 * the hidden layers start U(-1/sqrt(fan_in), 1/sqrt(fan_in)) from `seed`, W4 and b4 at zero
 * (an untrained model predicts the sketch's estimate). */
int ml_gpu_card_model_create(ml_ctx* ctx, uint64_t seed, ml_card_model** out);
/* Copy the ML_CARD_PARAMS parameters out (get != NULL) and/or in (set != NULL, also resets Adam). */
int ml_gpu_card_model_params(ml_card_model* m, float* get, const float* set);
/* One Adam step (lr, betas 0.9/0.999, eps 1e-8) on a batch of `batch` host rows (x: batch x 72,
 * y: log2 targets) under mean squared error; *loss = the batch loss before the step. */
int ml_gpu_card_model_step(ml_card_model* m, const float* x, const float* y, int32_t batch, float lr, float* loss);
/* `epochs` passes over n host rows in batches, shuffled per epoch from `seed`;
 * *final_loss = mean batch loss of the last epoch. */
int ml_gpu_card_model_train(ml_card_model* m, const float* x, const float* y, int64_t n, int32_t epochs,
                            int32_t batch, float lr, uint64_t seed, float* final_loss);
/* out[i] = predicted log2(distinct) of host row x[i]. */
int ml_gpu_card_model_predict(ml_card_model* m, const float* x, int64_t n, float* out);
int ml_gpu_card_model_destroy(ml_card_model* m);

/* ---- profiling ------------------------------------------------------------------ */
/* Number of kernels this library has launched since the context was created. */
int ml_gpu_kernel_launches(ml_ctx* ctx, uint64_t* count);
/* With ML_CTX_PROFILE: launches and summed device time (ms, CUDA events) of one kernel
 * family: "pipeline_aggregate" (fused filter/probe/aggregate), "join_insert", "topn",
 * "select" (filter flags and counts), "select_write" (filter compaction), "card_hll"
 * (cardinality features scan).  Always recorded: "jit_compile" (runtime compilations and
 * their host time), "jit_launch" (launches of runtime-specialized kernels; time 0),
 * "device_alloc" / "pinned_alloc" (cudaMalloc / cudaHostAlloc calls the context made and
 * their host time) and "graph_capture" (CUDA graphs captured and instantiated).
 * `reset` clears the counters after reading. */
int ml_gpu_profile_read(ml_ctx* ctx, const char* kernel, uint64_t* launches, double* total_ms, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif /* MINILAKE_GPU_H */
