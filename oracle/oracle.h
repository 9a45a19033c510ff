/*
 * oracle.h — TEST INFRASTRUCTURE ONLY. The CPU restatement of Wadjet's
 * filter → hash-join → hash-aggregate semantics that the GPU library is checked
 * against, and the CPU baseline that bench.py times beside it. Nothing in the
 * product (wadjet_b200/, include/) includes, links or loads this.
 *
 * Parity is pinned by the reference's own known-answer tests restated as golden
 * fixtures under tests/golden/ (see tests/golden/make_golden.py); the Go
 * reference itself cannot be built or run in this environment (no Go toolchain).
 *
 * Each function cites the reference file:line (paths inside the Wadjet tree)
 * whose algorithm it follows.
 */
#ifndef WADJET_ORACLE_H
#define WADJET_ORACLE_H

#include <stdint.h>
#include "../include/wadjet_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

const char* or_last_error(void);

/* KernelFilter.Execute + compareFilterImpl (exec/filter.go:373-425,
 * exec/kernel/compare.go:47-90,145-182). Returns the number of selected rows
 * written to out_sel (ascending), or -1 on an unsupported column type. */
int64_t or_join_bloom_filter(void* join, const wg_column* key, int64_t len, const uint32_t* sel, int64_t sel_len,
                             uint32_t* out_sel, int64_t* n_words);
int64_t or_filter(const wg_column* col, int64_t len, const uint32_t* sel, int64_t sel_len,
                  const wg_predicate* p, uint32_t* out_sel);

/* HashJoin int-key build (exec/join.go:520-575,771-840) and inlineIntProbe
 * (exec/join.go:2670-2820). */
void*   or_join_new(int64_t build_row_hint);
int     or_join_append(void* j, const wg_column* key, int64_t base_row);
int64_t or_join_rows(void* j);
int64_t or_join_distinct(void* j);
/* Emits (probe_row, build_row) pairs in probe order, chain order inside a
 * probe row (most recently built first, as arenaNext links); build_row is -1
 * where the output has none (unmatched LEFT rows, SEMI and ANTI rows).
 * Returns the total number of pairs; only the first `cap` are written. */
int64_t or_join_probe(void* j, const wg_column* key, int64_t len, const uint32_t* sel,
                      int64_t sel_len, uint32_t* out_probe, int64_t* out_build, int64_t cap);
/* exec.JoinType of the probe: WG_JOIN_INNER (default), _LEFT, _SEMI, _ANTI. */
void    or_join_set_type(void* j, int32_t type);
void    or_join_free(void* j);

/* HashAggregate (exec/aggregate.go:1296-2613, agg_scatter.go, kernel/types.go). */
void*   or_agg_new(int32_t n_keys, const int32_t* key_cols, int32_t n_aggs, const wg_agg_spec* aggs);
int     or_agg_consume(void* a, const wg_batch_desc* b);
int64_t or_agg_groups(void* a);
int     or_agg_export(void* a, const wg_group_export* out);
/* Finalized output of every group (nextOwn/writeAccToColumn,
 * exec/aggregate.go:4226, aggregate_partial_spill.go:1855), n_keys+n_aggs
 * host columns with room for or_agg_groups() rows; valid_words may be NULL. */
int     or_agg_emit(void* a, wg_column* out_cols);
int     or_agg_merge(void* dst, void* src);
void*   or_agg_clone(void* a);
void    or_agg_free(void* a);

/* Pipeline.Run over 2048-row batches (exec/pipeline.go:81,351): KernelFilter
 * chain → HashJoinProbe (+ gather of the build payload) → Project → the
 * aggregate. `threads` workers each consume into a CloneSink; the clones are
 * merged into `agg` in worker order (MergeSink, aggregate.go:4682). */
int     or_pipeline_run(const wg_batch_desc* input, int32_t n_filters, const wg_predicate* filters,
                        void* join, int32_t probe_key_col, const wg_batch_desc* build,
                        int32_t n_payload, const int32_t* payload_cols,
                        int32_t n_exprs, const wg_expr* exprs, void* agg, int32_t threads);

/* Host generators over include/wadjet_synth.h (rows [row0, row0+n)). */
void    or_gen_starjoin_fact(uint64_t seed, int64_t row0, int64_t n, int32_t* fk, int32_t* qty,
                             wg_int128* price, double* disc, int32_t threads);
void    or_gen_starjoin_dim(uint64_t seed, int64_t n, int32_t* key, int32_t* grp);
void    or_gen_groupby(uint64_t seed, int64_t row0, int64_t n, int64_t ngroups, int64_t* k,
                       int64_t* v, double* f, int32_t* flag, int32_t threads);
void    or_gen_highcard(uint64_t seed, int64_t row0, int64_t n, int32_t* a, int64_t* b,
                        wg_int128* amt, double* x, int32_t threads);

/* The Parquet RLE / bit-packed hybrid (rle.go DecodeRLEInt32Into): values
 * decoded into out (fewer than count when the stream ends), -1 on a malformed
 * stream. */
int64_t or_rle_decode(const uint8_t* data, int64_t len, int32_t bit_width, int64_t count, int32_t* out);
/* A column chunk's pages decoded into a host column and validity words (the
 * native scan's page decode, page_reader.go:607, columnar_native.go:470-640);
 * 0, or -1 on a malformed page. */
int     or_page_decode(const wg_column_chunk* chunk, void* out, uint64_t* valid_words);

/* String GROUP BY keys as consumeBatchStrGroup numbers them
 * (exec/aggregate.go:3038-3110): each distinct string takes the next group
 * index at its first appearance, in row (selection) order across batches; a
 * NULL string is the NULL-key group (ids[row] = 0, its validity kept). map
 * writes ids[row] for the batch's rows (offsets len + 1 entries) and returns
 * the distinct strings so far; get copies string `id` into out (at most cap
 * bytes) and returns its length. */
void*   or_strindex_new(void);
int64_t or_strindex_map(void* h, const uint32_t* offsets, const uint8_t* bytes, const uint64_t* valid_words,
                        int64_t len, const uint32_t* sel, int64_t sel_len, int32_t* ids);
int64_t or_strindex_get(void* h, int64_t id, uint8_t* out, int64_t cap);
void    or_strindex_free(void* h);

/* Int128.ToFloat64 (batch/decimal.go:39) for fixture checks. */
double  or_i128_to_f64(int64_t hi, uint64_t lo, int32_t scale);

#ifdef __cplusplus
}
#endif
#endif
