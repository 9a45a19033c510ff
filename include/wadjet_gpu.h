/*
 * wadjet_gpu.h — C ABI of libwadjetgpu.so, the B200 (sm_100a) filter → hash-join →
 * hash-aggregate pipeline that drops in under Wadjet's operator contract
 * (internal/engine/exec/operators.go:10-108).
 *
 * Every entry point is plain C: opaque handles, raw pointers and sizes, an int
 * status. A Go cgo wrapper implements exec.UnaryOperator / exec.Sink /
 * exec.MergeableSink on top of these calls. The reference interface each
 * function replaces is cited beside it as path:line within the Wadjet source
 * tree.
 *
 * Conventions
 *  - Status: 0 = WG_OK; WG_E_NOMEM maps to memory.ErrMemoryExceeded
 *    (internal/engine/memory/tracker.go:15). wg_last_error() returns a
 *    thread-local message for the most recent failing call on this thread.
 *  - Host pointers passed in are read only during the call (the cgo rule that C
 *    must not retain Go pointers). Device memory belongs to the handle and is
 *    released by the matching *_destroy.
 *  - A handle is not re-entrant; callers serialise calls per handle (the Go
 *    wrapper holds a mutex the way HashAggregate.Consume does,
 *    exec/aggregate.go:1076). The context is thread-safe.
 *  - "_device" variants take descriptors whose data/valid/sel pointers are
 *    device addresses on the context's GPU; the others take host memory and
 *    stage it through the context's pinned buffers.
 */
#ifndef WADJET_GPU_H
#define WADJET_GPU_H

#include <stdint.h>

#if defined(__GNUC__)
#define WG_API __attribute__((visibility("default")))
#else
#define WG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
typedef int32_t wg_status;
#define WG_OK             0
#define WG_E_NOMEM        1  /* HBM ledger refused a reservation (memory.ErrMemoryExceeded) */
#define WG_E_INVALID      2  /* bad argument / schema mismatch                              */
#define WG_E_TIMEOUT      3  /* a bounded device-side wait ran out                           */
#define WG_E_CUDA         4  /* a CUDA runtime call failed                                   */
#define WG_E_UNSUPPORTED  5  /* shape the GPU path does not cover (e.g. string keys)          */
#define WG_E_STATE        6  /* call out of order (consume after finalize, ...)               */
#define WG_E_CANCELLED    7  /* a queued serving request was cancelled (context.Canceled)      */

/* ---- type ids: values of parquet.TypeID (internal/storage/parquet/schema.go:13-34) ---- */
#define WG_TYPE_BOOL       0
#define WG_TYPE_INT32      1
#define WG_TYPE_INT64      2
#define WG_TYPE_FLOAT32    3
#define WG_TYPE_FLOAT64    4
#define WG_TYPE_STRING     5
#define WG_TYPE_BYTES      6
#define WG_TYPE_TIMESTAMP  7
#define WG_TYPE_IPV4       8   /* stored in Int64Data (kernel/compare.go:158) */
#define WG_TYPE_IPV6       9
#define WG_TYPE_CIDR      10
#define WG_TYPE_MAC       11
#define WG_TYPE_PORT      12
#define WG_TYPE_PROTOCOL  13
#define WG_TYPE_DURATION  14
#define WG_TYPE_UUID      15
#define WG_TYPE_DATE      16
#define WG_TYPE_DECIMAL   17   /* element = wg_int128 */

/* ---- compare ops: kernel.CompareOp (internal/engine/exec/kernel/compare.go:16-23) ---- */
#define WG_OP_EQ 0
#define WG_OP_NE 1
#define WG_OP_LT 2
#define WG_OP_LE 3
#define WG_OP_GT 4
#define WG_OP_GE 5

/* kind of a filter constant (the Go `any` value handed to ResolveFilterKernel,
 * kernel/compare.go:145). It is converted to the column's type exactly as
 * toInt64 / toFloat64 do (kernel/compare.go:580-640). */
#define WG_CONST_INT   0
#define WG_CONST_FLOAT 1

/* ---- aggregate functions: exec.AggFunc (internal/engine/exec/aggregate.go:27-31) ---- */
#define WG_AGG_SUM   0
#define WG_AGG_COUNT 1   /* input_col = -1 is COUNT(*) */
#define WG_AGG_MIN   2
#define WG_AGG_MAX   3
#define WG_AGG_AVG   4

/* ---- join types: exec.JoinType (internal/engine/exec/join.go:20-30) ---- */
#define WG_JOIN_INNER 0
#define WG_JOIN_LEFT  1   /* unmatched probe rows once, build columns NULL */
#define WG_JOIN_SEMI  5   /* probe rows with a match, once each; no build columns */
#define WG_JOIN_ANTI  6   /* probe rows without a match (NULL keys included); no build columns */

/* Int128 DECIMAL element. Field order is Go's batch.Int128{Hi int64; Lo uint64}
 * (internal/engine/batch/decimal.go:11), i.e. the opposite of a little-endian
 * __int128. */
typedef struct wg_int128 {
  int64_t  hi;
  uint64_t lo;
} wg_int128;

/* One column vector (batch.Vector, internal/engine/batch/vector.go:302).
 * valid_words: NULL = no nulls; otherwise bit i of word i/64 is 1 when row i is
 * valid, LSB first (batch.Bitmap, internal/engine/batch/bitmap.go:7,84). */
typedef struct wg_column {
  int32_t         type_id;
  int32_t         scale;       /* DECIMAL scale, else 0 */
  const void*     data;
  const uint64_t* valid_words;
  int64_t         len;
} wg_column;

/* A STRING or BYTES column (batch.BytesColumn, internal/engine/batch/vector.go:92):
 * its wg_column.data points to this descriptor, in host memory; offsets
 * (len + 1 entries: row i is bytes[offsets[i], offsets[i + 1])) and bytes lie in
 * the batch's memory (host or device). On the GPU path a string column can be
 * an aggregate's single GROUP BY key (consumeBatchStrGroup,
 * exec/aggregate.go:3038); see wg_agg_key_strings. */
typedef struct wg_bytes {
  const uint32_t* offsets;
  const uint8_t*  bytes;
} wg_bytes;

/* One record batch (batch.RecordBatch, internal/engine/batch/batch.go:9).
 * sel: NULL = all rows active, else sel_len ascending row indices (batch.go:13). */
typedef struct wg_batch_desc {
  int32_t          ncols;
  int32_t          _pad;
  const wg_column* cols;
  int64_t          len;
  const uint32_t*  sel;
  int64_t          sel_len;
} wg_batch_desc;

/* One aggregate (exec.AggColumn, internal/engine/exec/aggregate.go:73).
 * out_type: WG_TYPE_FLOAT64 / WG_TYPE_INT64 as the planner declares it
 * (planner/physical/plan.go:9954); 0 picks the planner default: COUNT → INT64,
 * SUM/AVG → FLOAT64, MIN/MAX → their input's class (exec/aggregate.go:4611). */
typedef struct wg_agg_spec {
  int32_t func;
  int32_t input_col;
  int32_t out_type;
  int32_t _pad;
} wg_agg_spec;

/* One filter predicate `col OP const` (exec.KernelFilter, exec/filter.go:347). */
typedef struct wg_predicate {
  int32_t col;
  int32_t op;
  int32_t const_kind;
  int32_t _pad;
  int64_t const_i64;
  double  const_f64;
} wg_predicate;

/* A projection expression in postfix form (exec.Project over expr.BinOpNumeric,
 * internal/engine/expr/binop_numeric.go). Integer arithmetic wraps like Go
 * int64; float arithmetic is IEEE binary64 with no contraction; a DECIMAL input
 * read as float goes through Int128.ToFloat64 (expr/expr.go:225,257). */
#define WG_EXPR_COL      0   /* push column `arg` */
#define WG_EXPR_CONST_I  1   /* push imm_i64 */
#define WG_EXPR_CONST_F  2   /* push imm_f64 */
#define WG_EXPR_ADD      3
#define WG_EXPR_SUB      4
#define WG_EXPR_MUL      5
#define WG_EXPR_DIV      6   /* float only */
#define WG_EXPR_SHR      7   /* int only: arithmetic shift right by imm_i64 (top of stack) */
#define WG_EXPR_AND      8   /* int only */
#define WG_EXPR_MAX_OPS 12
typedef struct wg_expr_op {
  int32_t opcode;
  int32_t arg;
  int64_t imm_i64;
  double  imm_f64;
} wg_expr_op;
typedef struct wg_expr {
  int32_t    result_type;      /* WG_TYPE_INT64 or WG_TYPE_FLOAT64 */
  int32_t    n_ops;
  wg_expr_op ops[WG_EXPR_MAX_OPS];
} wg_expr;

/* Raw per-group aggregate state, the SoA accumulators of exec.flatAccumArrays
 * (internal/engine/exec/agg_scatter.go:16). Arrays are caller-allocated with
 * n_groups entries per key column / aggregate, laid out [k * n_groups + g].
 * Any pointer may be NULL to skip that field. */
typedef struct wg_group_export {
  int64_t*   keys;       /* group key widened to int64 (packed keys unpacked per column) */
  uint8_t*   key_valid;  /* 0 = the NULL group for that key column */
  int64_t*   count;      /* non-null input rows per aggregate (COUNT(*) = all rows) */
  int64_t*   i64;        /* sumI64 / minI64 / maxI64 */
  double*    f64;        /* sumF64 / minF64 / maxF64 */
  wg_int128* dec;        /* sumDec / minDec / maxDec */
  uint8_t*   has;        /* hasMin / hasMax; for SUM/COUNT/AVG: count > 0 */
} wg_group_export;

typedef struct wg_ctx    wg_ctx;
typedef struct wg_filter wg_filter;
typedef struct wg_join   wg_join;
typedef struct wg_agg    wg_agg;

/* ======================================================================== */
/* Context, HBM ledger                                                       */
/* ======================================================================== */

/* Thread-local message of the last failing call on this thread ("" if none). */
WG_API const char* wg_last_error(void);

/* Library version string. */
WG_API const char* wg_version(void);

/* Create a context on `device`: one CUDA stream, a pinned staging area and an
 * HBM ledger with `hbm_budget_bytes` (0 = free device memory at creation)
 * (memory.NewTracker, internal/engine/memory/tracker.go:36). pinned_spill_bytes
 * caps the pinned host memory used for aggregate spill partitions. */
WG_API wg_status wg_ctx_create(int32_t device, int64_t hbm_budget_bytes,
                        int64_t pinned_spill_bytes, wg_ctx** out);
/* A context on the parent's device with its own streams and a child ledger
 * that shares the parent's budget (Tracker.Child, memory/tracker.go:44):
 * concurrent queries each get one, and every reservation also counts against
 * the parent. The parent must outlive its children. */
WG_API wg_status wg_ctx_create_child(wg_ctx* parent, wg_ctx** out);
WG_API wg_status wg_ctx_destroy(wg_ctx* ctx);
/* Wait until all work queued on the context's stream is done. */
WG_API wg_status wg_ctx_synchronize(wg_ctx* ctx);
/* Ledger counters (Tracker.Used / Peak / Budget, tracker.go:129,151,134). */
WG_API wg_status wg_ledger_stats(wg_ctx* ctx, int64_t* used, int64_t* peak, int64_t* budget);
/* Explicit reservations against the ledger (Tracker.Reserve/Release,
 * tracker.go:53,73); WG_E_NOMEM when over budget, nothing reserved then. */
WG_API wg_status wg_ledger_reserve(wg_ctx* ctx, int64_t bytes);
WG_API wg_status wg_ledger_release(wg_ctx* ctx, int64_t bytes);
/* The CUDA stream (cudaStream_t) the context launches on, for callers that
 * order their own work against it. */
WG_API void*     wg_ctx_stream(wg_ctx* ctx);
/* Number of kernels this context has launched since creation. */
WG_API int64_t   wg_ctx_launch_count(wg_ctx* ctx);

/* ======================================================================== */
/* Batches on the device: the scan's hand-off to the pipeline                */
/* (internal/planner/physical/plan.go:11096-11115)                          */
/* ======================================================================== */
typedef struct wg_batch wg_batch;

/* Upload a decoded host batch: device copies of every column (data, validity)
 * and of the selection vector, charged to the context's ledger
 * (memory.Tracker, tracker.go:53); WG_E_NOMEM when they do not fit. */
WG_API wg_status wg_batch_upload(wg_ctx* ctx, const wg_batch_desc* host, wg_batch** out);
/* The batch's device descriptor, for the "_device" entry points; its pointers
 * stay valid until wg_batch_destroy. cols must have room for the batch's
 * columns (*out->ncols on return). */
WG_API wg_status wg_batch_device_desc(wg_batch* b, wg_batch_desc* out, wg_column* cols, int32_t max_cols);
WG_API wg_status wg_batch_destroy(wg_batch* b);

/* ---- Parquet pages decoded on the device -------------------------------- */
/* Encodings of a page's values section (parquet.Encoding values,
 * internal/storage/parquet/page_reader.go:610-640). */
#define WG_ENC_PLAIN             0
#define WG_ENC_PLAIN_DICTIONARY  2
#define WG_ENC_RLE_DICTIONARY    8

/* One data page of a flat column, after decompression (the reader's Decompress
 * step stays on the host). def_levels: the RLE / bit-packed hybrid definition
 * levels (bit width 1) of an optional column, NULL for a required one; a row is
 * NULL where its level is 0. data: the values section, i.e. PLAIN values of the
 * page's non-NULL rows (physical width: 4 bytes for INT32-class and FLOAT, 8
 * for INT64-class, DOUBLE and DECIMAL's INT64), or for a dictionary encoding
 * one bit-width byte followed by the hybrid-encoded indices (rle.go). */
typedef struct wg_page {
  int32_t        encoding;
  int32_t        _pad;
  int64_t        num_values;   /* rows of the page, NULLs included */
  const uint8_t* def_levels;
  int64_t        def_len;
  const uint8_t* data;
  int64_t        data_len;
} wg_page;

/* A column chunk: its pages in order and its dictionary page's values (PLAIN,
 * physical width, dict_len entries; NULL without one). type_id is the
 * column's logical type; a DECIMAL chunk holds INT64 physical values that
 * decode to Int128 as Int128From does (scan/columnar_native.go:619-625). */
typedef struct wg_column_chunk {
  int32_t        type_id;
  int32_t        scale;
  int32_t        n_pages;
  int32_t        _pad;
  const wg_page* pages;
  const void*    dict;
  int64_t        dict_len;
} wg_column_chunk;

/* Decode column chunks into a device batch, one column per chunk, every chunk
 * with the same row count: the native scan's page decode and copy into a
 * batch.Vector (ColumnPageReader.decodeValues, page_reader.go:607; dictionary
 * gather with its index bounds check, columnar_native.go:470-520;
 * copyNativeDataDirect, :612) on the GPU. Page and dictionary bytes are host
 * memory; only these encoded bytes cross to the device. A malformed page
 * (levels or indices that end early, an index past the dictionary, PLAIN data
 * shorter than its values) fails with WG_E_INVALID. */
WG_API wg_status wg_batch_decode(wg_ctx* ctx, const wg_column_chunk* chunks, int32_t n_chunks, wg_batch** out);

/* ======================================================================== */
/* Filter: exec.KernelFilter (internal/engine/exec/filter.go:347-425) with    */
/* kernel.ResolveFilterKernel / compareFilterImpl (kernel/compare.go:47,145)  */
/* ======================================================================== */

/* Bind a predicate on column `col_idx`; the typed kernel is resolved on the
 * first execute from that column's type (KernelFilter.Execute, filter.go:373). */
WG_API wg_status wg_filter_create(wg_ctx* ctx, int32_t col_idx, int32_t op,
                           int32_t const_kind, int64_t const_i64, double const_f64,
                           wg_filter** out);
/* Host batch in, ascending selection out (out_sel must hold in->sel_len rows if
 * in->sel, else in->len). *out_n = 0 means "fully filtered": the Go wrapper
 * returns a nil batch (filter.go:420). Nulls never match (compare.go:53-60). */
WG_API wg_status wg_filter_execute(wg_filter* f, const wg_batch_desc* in,
                            uint32_t* out_sel, int64_t* out_n);
/* Device batch in, device selection out; *out_n is read back to the host. */
WG_API wg_status wg_filter_execute_device(wg_filter* f, const wg_batch_desc* in,
                                   uint32_t* out_sel_dev, int64_t* out_n);
WG_API wg_status wg_filter_destroy(wg_filter* f);

/* The filter for callers that cannot allocate device memory. No counterpart in
 * the reference. Some callers must not call cudaMalloc: a Go operator whose
 * device memory was reserved up front from the engine's memory budget (the
 * ledger would not see a private allocation), a thread that issues work while
 * another thread captures a CUDA graph in global mode (a cudaMalloc there
 * invalidates the capture), or a latency-critical serving thread (cudaMalloc
 * and cudaFree can synchronise the whole device). This entry point allocates
 * nothing: the compaction's tile-status scratch lives in a fixed static device
 * array of WG_NOALLOC_SCRATCH_BYTES, held by every GPU that loads the library
 * until the process exits. It takes a CUDA stream instead of a context, a
 * device column and optional device selection vector (n_items = selection
 * length, else column length), writes the ascending selection to out_sel (device,
 * n_items entries of room) and the count to *out_n (host). It refuses inputs
 * of more than WG_NOALLOC_MAX_ITEMS rows with WG_E_INVALID.
 * - The first call on a device looks up the array's device address (set-up);
 *   make that first call before any stream capture.
 * - Every call uses the same array and leaves its contents behind (each call
 *   clears what must start at zero); calls whose work overlaps on the GPU race
 *   on it, so callers serialise them (one stream, or their own lock). */
#define WG_NOALLOC_MAX_ITEMS (1LL << 26)
#define WG_NOALLOC_SCRATCH_BYTES (65536 * 8 + 256)
WG_API wg_status wg_filter_execute_device_noalloc(void* stream, const wg_column* col, const uint32_t* sel,
                                                  int64_t n_items, int32_t op, int32_t const_kind,
                                                  int64_t const_i64, double const_f64, uint32_t* out_sel,
                                                  int64_t* out_n);

/* ======================================================================== */
/* Hash join: exec.HashJoin / HashJoinProbe (internal/engine/exec/join.go)   */
/* ======================================================================== */

/* Equi-join on one integer-class key column (tryEnableIntKey, join.go:520).
 * join_type: WG_JOIN_INNER, WG_JOIN_LEFT, WG_JOIN_SEMI or WG_JOIN_ANTI
 * (semi and anti carry no payload columns, as executeSemiAntiJoin returns only
 * probe rows, join.go:3247). build_key_col indexes the build batches;
 * probe_key_col the probe batches; payload_cols are build columns carried to
 * the output. build_row_hint pre-sizes the build buffers (HashJoin.BuildRowHint). */
WG_API wg_status wg_join_create(wg_ctx* ctx, int32_t join_type, int32_t build_key_col,
                         int32_t probe_key_col, int32_t n_payload,
                         const int32_t* payload_cols, int64_t build_row_hint,
                         wg_join** out);
/* Append one build batch (the per-batch arenaAppendInt loop, join.go:551). */
WG_API wg_status wg_join_build_append(wg_join* j, const wg_batch_desc* build);
WG_API wg_status wg_join_build_append_device(wg_join* j, const wg_batch_desc* build);
/* Build the device hash index over everything appended (end of
 * HashJoin.Build, join.go:771). Null keys never join.
 * When the context's HBM budget refuses the build's columns (at append) or its
 * index (here), the build becomes partitioned (HashJoin.buildPartitioned,
 * join_partition_arrival.go:48): its rows move to host memory in 64 key-hash
 * partitions, and the pipeline entry points probe it in passes over groups of
 * partitions that fit; wg_join_probe and wg_join_gather then return
 * WG_E_UNSUPPORTED. */
WG_API wg_status wg_join_build_finish(wg_join* j);
/* BloomFilterOp.Execute (exec/bloom_filter_op.go:39) for the join's probe key:
 * the rows of `probe` (or its selection entries) whose non-NULL key the build
 * side's bloom filter (HashJoin.buildBloom, join.go:1441: about 10 bits per
 * distinct key, two bits per key from bloomHashInt) may contain, ascending, in
 * out_sel (host memory with room for every row or selection entry); *n_out
 * their count. The fused pipeline's hash probe checks the same bloom first
 * when the hash index is larger than half of L2 (WG_JOIN_BLOOM=0/1 forces). */
WG_API wg_status wg_join_bloom_filter(wg_join* j, const wg_batch_desc* probe, uint32_t* out_sel, int64_t* n_out);
/* Number of build rows stored and number of distinct keys indexed (-1 for a
 * partitioned build: keys are not counted across partitions). */
WG_API wg_status wg_join_build_stats(wg_join* j, int64_t* build_rows, int64_t* distinct_keys);
/* HashJoinProbe.Execute → inlineIntProbe (join.go:2306,2670), bounded output
 * (BoundedOutputOperator, operators.go:86): emits at most `cap` output pairs
 * (probe_row, build_row) ordered by probe position, starting at output pair
 * *cursor (0 on the first call). On return *cursor is the next pair to resume
 * from and *out_n the number of pairs written. build_row is -1 where the output
 * has no build row: an unmatched LEFT row (matchPair{matched: false},
 * join.go:3180) and every SEMI / ANTI row. */
WG_API wg_status wg_join_probe(wg_join* j, const wg_batch_desc* probe,
                        uint32_t* out_probe_rows, int64_t* out_build_rows,
                        int64_t cap, int64_t* cursor, int64_t* out_n);
/* Gather build payload column `payload_idx` for `n` build rows
 * (gatherVector, exec/sort.go:611). out/out_valid are host buffers
 * (out_valid may be NULL; it receives one byte per row, 1 = valid); a build
 * row of -1 (an unmatched LEFT row) gathers NULL. */
WG_API wg_status wg_join_gather(wg_join* j, int32_t payload_idx, const int64_t* build_rows,
                         int64_t n, void* out, uint8_t* out_valid);
/* Forget the build side so the handle can build again (a fresh HashJoin for the
 * next query over the same plan); device buffers are kept for reuse. */
WG_API wg_status wg_join_reset(wg_join* j);
WG_API wg_status wg_join_destroy(wg_join* j);

/* ======================================================================== */
/* Hash aggregate: exec.HashAggregate (internal/engine/exec/aggregate.go)     */
/* ======================================================================== */

/* GROUP BY key_cols with aggs (NewHashAggregate, aggregate.go:1023). One
 * integer-class key column takes the int-key path (aggregate.go:1544); 2-4
 * integer-class columns of at most 16 bytes take the packed path
 * (aggregate.go:1596, packed_hash.go:386). group_ndv_hint pre-sizes the device
 * table (HashAggregate.GroupNDVHint); 0 = grow on demand. */
WG_API wg_status wg_agg_create(wg_ctx* ctx, int32_t n_keys, const int32_t* key_cols,
                        int32_t n_aggs, const wg_agg_spec* aggs,
                        int64_t group_ndv_hint, wg_agg** out);
/* HashAggregate.Consume (aggregate.go:1075) of a host / device batch. */
WG_API wg_status wg_agg_consume(wg_agg* a, const wg_batch_desc* in);
WG_API wg_status wg_agg_consume_device(wg_agg* a, const wg_batch_desc* in);
/* CloneSink / MergeSink (aggregate.go:4646,4682): a fresh handle of the same
 * shape, and folding src's groups into dst (src is left untouched). */
WG_API wg_status wg_agg_clone(wg_agg* a, wg_agg** out);
WG_API wg_status wg_agg_merge(wg_agg* dst, wg_agg* src);
/* Finalize (aggregate.go:3855): no more input; *n_groups = output rows. */
WG_API wg_status wg_agg_finalize(wg_agg* a, int64_t* n_groups);
/* Next (aggregate.go:4202): finalized rows [start, start+max_rows) into host
 * columns out_cols[0..n_keys+n_aggs) — keys in their input types, then one
 * column per aggregate in its output type. out_cols[i].data / valid_words
 * point at caller buffers (valid_words may be NULL when the caller does not
 * want null bits; bit layout as batch.Bitmap). *n_out = rows written. */
WG_API wg_status wg_agg_emit(wg_agg* a, int64_t start, int64_t max_rows,
                      wg_column* out_cols, int64_t* n_out);
/* Raw accumulator state of every group, for bit-exact checks. */
WG_API wg_status wg_agg_export(wg_agg* a, const wg_group_export* out);
/* An aggregate grouped by one STRING / BYTES column keys its groups by dense
 * ids (its exports' and emits' key column holds the id; the NULL-key group is
 * the NULL key as for any column): the strings of n ids, as offsets (n + 1
 * entries, from 0) and bytes, into host buffers. *need_bytes receives the
 * bytes the strings take; nothing is written to out_bytes when that is more
 * than bytes_cap (call again with room). */
WG_API wg_status wg_agg_key_strings(wg_agg* a, const int64_t* ids, int64_t n, uint32_t* out_offsets,
                                    uint8_t* out_bytes, int64_t bytes_cap, int64_t* need_bytes);
/* Forget all groups and input (the state after wg_agg_create). */
WG_API wg_status wg_agg_reset(wg_agg* a);
/* ---- exchange of partial state between ranks (one process per GPU) ----
 * The multi-GPU GROUP BY pre-aggregates each rank's shard, then hash-partitions
 * the partial groups by owner rank and exchanges them (an NCCL all-to-all into
 * each rank's HBM) so every rank finishes a disjoint key range: the device form
 * of partitionFor (internal/engine/exec/partitioned_agg.go:221) and the
 * distributed shuffle (internal/worker/partitioned_shuffle_sink.go:1039).
 * A state row is (1 + slot_words) uint64 words: a flag (0 a regular key, 1 the
 * key equal to the table's empty pattern, 2 the NULL key) and the group's slot. */
typedef struct wg_state_layout {
  int32_t key_words, slot_words, n_keys, n_aggs;
  int32_t key_type[4];                        /* parquet.TypeID of each group column */
  int32_t key_i32[4], key_word[4], key_shift[4];  /* packed-key placement (buildPackedLayout) */
  int32_t null_word, null_shift;              /* packed keys: 4-bit NULL field (-1: none) */
  int32_t agg_kind[8], agg_off[8], agg_null_off[8];
  int32_t agg_in_cls[8], agg_in_scale[8], agg_out_type[8], agg_nullable[8];
} wg_state_layout;
/* The row layout of a's state (a must have consumed or merged something). */
WG_API wg_status wg_agg_state_layout(wg_agg* a, wg_state_layout* out);
/* After finalize: every group's state row into rows_dev (device, rows_cap rows of
 * 1 + slot_words words), grouped by owner = hi64(route_hash * n_parts) where
 * route_hash is fibHash(key) / packedHash(lo, hi) / routeNullHash as partitionFor's
 * router computes it (partitioned_agg.go:508-535); part_rows[p] (host) = rows of owner p,
 * stored from row sum(part_rows[0..p)) on. */
WG_API wg_status wg_agg_partition_state(wg_agg* a, int32_t n_parts, void* rows_dev, int64_t rows_cap,
                                        int64_t* part_rows);
/* MergeSink (aggregate.go:4682) of n_rows state rows (device) laid out as *src into a,
 * which must not be finalized; an aggregate that has consumed nothing adopts the
 * source's schema. */
WG_API wg_status wg_agg_merge_state(wg_agg* a, const wg_state_layout* src, const void* rows_dev, int64_t n_rows);
/* Diagnostic, no counterpart in the reference: the compiled query shape the
 * last fused launch into `a` ran on (1..6: a kernel built for exactly that
 * query shape; 0: the generic kernel; -1: no fused launch yet). Results never
 * depend on it. */
WG_API int32_t wg_agg_kernel_shape(const wg_agg* a);
WG_API wg_status wg_agg_destroy(wg_agg* a);

/* ======================================================================== */
/* Fused pipeline: Pipeline.Run (exec/pipeline.go:81) over                    */
/* KernelFilter* → HashJoinProbe → Project → HashAggregate in one kernel      */
/* ======================================================================== */

/* Virtual schema seen by the aggregate: input columns [0, ncols), then the
 * join's payload columns, then one column per expression. Filters apply to
 * input columns before the probe (the planner's pushdown order, plan.go:5750). */
typedef struct wg_pipeline_desc {
  const wg_batch_desc* input;
  int32_t              n_filters;
  int32_t              n_exprs;
  const wg_predicate*  filters;
  wg_join*             join;       /* NULL = no join; probe key = join's probe_key_col */
  const wg_expr*       exprs;
  wg_agg*              agg;        /* sink; must not be finalized */
} wg_pipeline_desc;

/* Run one pass of the pipeline over a host-resident input (staged to HBM in
 * chunks that overlap copies with the kernel) or a device-resident input. */
WG_API wg_status wg_pipeline_run(wg_ctx* ctx, const wg_pipeline_desc* p);
WG_API wg_status wg_pipeline_run_device(wg_ctx* ctx, const wg_pipeline_desc* p);

/* ======================================================================== */
/* Batched mode: many small, independent filter + GROUP BY queries in one    */
/* persistent launch, replayed from a CUDA graph. No counterpart in the      */
/* reference, which runs each query's Pipeline.Run separately                */
/* (exec/pipeline.go:81); every query keeps that operator contract's result. */
/* ======================================================================== */
typedef struct wg_batched wg_batched;

typedef struct wg_batched_query {
  const wg_batch_desc* input;    /* device-resident columns, no selection vector */
  int32_t              n_filters;
  int32_t              n_aggs;
  const wg_predicate*  filters;  /* AND chain on input columns */
  const int32_t*       key_cols; /* n_keys group columns (of the virtual schema, as wg_pipeline_desc) */
  int32_t              n_keys;
  int32_t              n_exprs;  /* projections appended to the virtual schema (0..2) */
  const wg_agg_spec*   aggs;
  int64_t              ndv_hint; /* expected groups; sizes the query's table */
  wg_join*             join;     /* NULL = no join; else a finished build, probed per row (a fused
                                    filter + probe + aggregate); it must outlive the batched handle */
  const wg_expr*       exprs;
} wg_batched_query;

/* Launch shape and table sizing (picked per workload by the autotuner,
 * wadjet_b200/autotune.py); a zero field takes the built-in default. */
typedef struct wg_tune_params {
  int32_t tile_rows;        /* rows per work item */
  int32_t block;            /* threads per CTA */
  int32_t ctas_per_sm;
  int32_t smem_max_groups;  /* queries expecting at most this many groups pre-combine each
                               work item in a shared-memory table */
  double  max_load;         /* table load the hint is sized for */
} wg_tune_params;

WG_API wg_status wg_batched_create(wg_ctx* ctx, int32_t n_queries, const wg_batched_query* queries,
                                   const wg_tune_params* params, wg_batched** out);
/* Run every query once (one graph launch) and wait; n_groups[q] receives each
 * query's group count (may be NULL). Queries whose table overflowed its hint are
 * re-run on a grown table before returning. */
WG_API wg_status wg_batched_run(wg_batched* b, int64_t* n_groups);
/* Raw state of query q's groups (as wg_agg_export) after a run. */
WG_API wg_status wg_batched_export(wg_batched* b, int32_t q, const wg_group_export* out);
WG_API wg_status wg_batched_destroy(wg_batched* b);

/* ======================================================================== */
/* Serving: a continuous-batching request loop. Requests are admitted into   */
/* free slots (each with its own child context and stream) as slots and HBM  */
/* (the shared ledger) free up, so requests that arrive while others run     */
/* overlap on the device. Tables and join indexes stay resident across       */
/* requests. No counterpart in the reference (its server runs each query's   */
/* Pipeline.Run on goroutines, internal/server/grpc.go:120).                  */
/* ======================================================================== */
typedef struct wg_server wg_server;

typedef struct wg_serve_request {
  const wg_pipeline_desc* plan;  /* device-resident input; plan->agg is ignored */
  const int32_t*          key_cols;
  const wg_agg_spec*      aggs;
  int32_t                 n_keys;
  int32_t                 n_aggs;
  int64_t                 ndv_hint;
  int64_t                 est_bytes;  /* HBM held for admission; 0 = estimated from the hint */
} wg_serve_request;

typedef struct wg_serve_stats {
  int64_t submitted, completed, failed, in_flight, queued, cancelled;
  double  p50_s, p99_s, mean_s, max_s;   /* latency = completion - submission */
  double  qps;                           /* completed / (last completion - first submission) */
  double  mean_queue_s;                  /* mean time from submission to a slot starting the request */
  double  mean_service_s;                /* mean time a slot spent on a request (run + finalize) */
} wg_serve_stats;

WG_API wg_status wg_server_create(wg_ctx* ctx, int32_t n_slots, wg_server** out);
/* Queue a request (copied); thread-safe. */
WG_API wg_status wg_server_submit(wg_server* s, const wg_serve_request* r, int64_t* ticket);
/* Wait for a request (timeout_s < 0: forever); its status is returned. */
WG_API wg_status wg_server_wait(wg_server* s, int64_t ticket, double timeout_s, int64_t* n_groups, double* latency_s);
WG_API wg_status wg_server_export(wg_server* s, int64_t ticket, const wg_group_export* out);
/* Free a finished request's result and its HBM. */
WG_API wg_status wg_server_release(wg_server* s, int64_t ticket);
/* Cancel a request that is still queued (the caller's context was cancelled,
 * as a gRPC handler sees ctx.Done(), internal/server/grpc.go:120): it leaves the
 * queue without touching the device and its wait returns WG_E_CANCELLED.
 * A request a slot has already started runs to completion (WG_E_STATE); the
 * caller then releases it as usual. The ticket stays valid until released. */
WG_API wg_status wg_server_cancel(wg_server* s, int64_t ticket);
WG_API wg_status wg_server_stats(wg_server* s, wg_serve_stats* out);
/* Forget latency statistics (e.g. after a warm-up). */
WG_API wg_status wg_server_reset_stats(wg_server* s);
WG_API wg_status wg_server_destroy(wg_server* s);

/* ======================================================================== */
/* Synthetic benchmark tables, generated in HBM (include/wadjet_synth.h).    */
/* No counterpart in the reference, whose benchmarks fill batches with       */
/* SetValue loops (internal/engine/exec/bench_test.go). Rows [row0, row0+n)  */
/* of each column are written to device pointers; NULL skips a column.       */
/* ======================================================================== */
WG_API wg_status wg_synth_starjoin_fact(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int32_t* fk,
                                        int32_t* qty, wg_int128* price, double* disc);
WG_API wg_status wg_synth_starjoin_dim(wg_ctx* ctx, uint64_t seed, int64_t n, int32_t* key, int32_t* grp);
WG_API wg_status wg_synth_groupby(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int64_t ngroups,
                                  int64_t* k, int64_t* v, double* f, int32_t* flag);
WG_API wg_status wg_synth_highcard(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int32_t* a, int64_t* b,
                                   wg_int128* amt, double* x);
/* Batched workload, query q: its row count, key cardinality and filter
 * threshold (host), and its columns (device; vi for even q, vf for odd q). */
WG_API wg_status wg_synth_batched_params(uint64_t seed, int32_t q, int64_t* rows, int64_t* card, int32_t* threshold);
WG_API wg_status wg_synth_batched(wg_ctx* ctx, uint64_t seed, int32_t q, int64_t n, int64_t card, int64_t* key,
                                  int64_t* vi, double* vf, int32_t* filt);

#ifdef __cplusplus
}
#endif
#endif /* WADJET_GPU_H */
