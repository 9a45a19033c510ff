// wg_agg.cuh — device structures of the hash aggregate and the fused pipeline.
//
// The aggregate restates exec.HashAggregate's state (internal/engine/exec/
// aggregate.go:1296-2613, agg_scatter.go) as one open-addressing table in HBM
// whose slots hold the key and every accumulator inline (array-of-structs, so a
// row touches one or two 32-byte sectors):
//
//   slot = [key words (0 scalar | 1 int key | 2 packed key)] [rows]
//          [per aggregate: state words (0..2)] [per nullable aggregate: nulls]
//
// The per-aggregate non-NULL count is `rows - nulls`, so COUNT needs no state
// and columns without NULLs cost no count traffic. Two extra slots follow the
// table: [cap] holds the group whose key equals the empty sentinel, [cap+1]
// the NULL key (single-key path, processRow's NULL group, aggregate.go:3422).
#pragma once

#include "wg_join.cuh"
#include "wg_pred.cuh"

#define WG_MAX_KEYS 4
#define WG_MAX_AGGS 8
#define WG_MAX_IN 8
#define WG_MAX_EXPRS 2
#define WG_MAX_FILTERS 4
#define WG_MAX_SLOT_WORDS 32
#define WG_EXPR_OPS 12

#define WG_EMPTY_KEY 0x8000000000000001ULL   // -0x7FFFFFFFFFFFFFFF, intHashEmpty (int_hash.go:42)

namespace wgd {

enum Kind : int32_t {
  K_COUNT = 0,
  K_SUM_I64, K_SUM_F64, K_SUM_DEC,
  K_MIN_I64, K_MAX_I64, K_MIN_F64, K_MAX_F64, K_MIN_DEC, K_MAX_DEC
};

__host__ __device__ __forceinline__ int kind_words(int k) {
  return (k == K_COUNT) ? 0 : (k == K_SUM_DEC || k == K_MIN_DEC || k == K_MAX_DEC) ? 2 : 1;
}

struct AggD {
  int32_t kind;
  int32_t off;        // first state word, -1 when none
  int32_t null_off;   // null-count word, -1 when the input has no NULLs
  int32_t vcol;       // virtual input column, -1 = COUNT(*)
};

struct Layout {
  int32_t key_words;
  int32_t slot_words;
  int32_t n_keys;
  int32_t n_aggs;
  int32_t key_vcol[WG_MAX_KEYS];
  int32_t key_i32[WG_MAX_KEYS];    // packed field is 4 bytes wide
  int32_t key_word[WG_MAX_KEYS];
  int32_t key_shift[WG_MAX_KEYS];
  // Packed keys with NULLs: bit k of the 4-bit field at (null_word, null_shift)
  // marks key column k NULL (its value bits are then 0). The field lies in a
  // 32-bit half the packing leaves unused, so a key without NULLs keeps its
  // plain packing; null_word = -1 when every bit is taken (NULLs refused).
  int32_t null_word;
  int32_t null_shift;
  AggD agg[WG_MAX_AGGS];
  unsigned long long init[WG_MAX_SLOT_WORDS];   // empty-slot pattern
};

struct Table {
  unsigned long long* slots;     // (cap + 2) * slot_words words
  unsigned long long* n_groups;  // regular slots taken (reservations)
  int32_t* overflow;             // set when an insert was refused at the limit
  int32_t shift;
  int32_t credit_chunk;          // group reservations a thread takes from n_groups at a time (1 = one per insert)
  uint64_t mask;                 // cap - 1
  unsigned long long limit;      // max regular groups before inserts are refused
};

struct ExprD {
  int32_t n_ops;
  int32_t result_cls;            // WG_CLS_I64 or WG_CLS_F64
  int32_t opc[WG_EXPR_OPS];
  int32_t arg[WG_EXPR_OPS];
  long long imm[WG_EXPR_OPS];    // int immediate, or the bits of a float immediate
};

struct Plan {
  int64_t n_items;
  const uint32_t* sel;           // nullptr = rows [0, n_items)
  int32_t n_in, n_filters, has_join, n_exprs;
  int32_t probe_col;
  int32_t smem_slots;            // >0: CTA-private shared-memory table of this many slots
  int32_t shape;                 // compiled query shape (wg_shapes.cuh), 0 = generic
  int32_t prefetch;              // grid-stride iterations of input prefetched into L2 ahead (0 = off)
  int32_t smem_sw;               // words per shared-table slot (0 = the layout's slot_words)
  int32_t smem_rep;              // copies of each float SUM in a shared slot (0 or 1 = one)
  int32_t smem_combine;          // 1: lanes of a warp combine rows of one group before the shared atomics
  int32_t gdense;                // 1: the shared table is indexed by key - gmin (keys known to lie in
                                 //    [gmin, gmin + smem_slots)), no hashing and no key words
  long long gmin;
  int32_t minmax_test;           // 1: HBM MIN/MAX read the slot first and skip an atomic that cannot win
  int32_t stage_off;             // self-staged vector kernel: byte offset of the warps' staging buffers
                                 // in dynamic shared memory (after the shared table)
  int32_t smem_hash_shift;       // shared-table slot from the key hash's bits below the top
                                 // smem_hash_shift (the bits that picked the rows' bucket)
  int32_t smem_list;             // >0: word offset in shared memory of a list of the bucketed
                                 // table's used slots, entry i written by its i-th insert
  int32_t vec_rows;              // batched work items: 2 rows per lane with vector loads (compiled
                                 // shape, 16-byte aligned columns, no join or the direct one, no selection)
  DCol in[WG_MAX_IN];
  Pred filt[WG_MAX_FILTERS];
  JoinView join;
  ExprD expr[WG_MAX_EXPRS];
  int32_t vcls[WG_MAX_IN + WG_MAX_PAYLOAD + WG_MAX_EXPRS];
  int32_t vscale[WG_MAX_IN + WG_MAX_PAYLOAD + WG_MAX_EXPRS];
  // DECIMAL columns: pow10_divisor_host(vscale) — the divisor and its rounded
  // reciprocal of the conversion to float64, so rows need no table lookups
  double vdiv_b[WG_MAX_IN + WG_MAX_PAYLOAD + WG_MAX_EXPRS];
  double vdiv_y[WG_MAX_IN + WG_MAX_PAYLOAD + WG_MAX_EXPRS];
  Layout L;
  Table T;
  int32_t* err;
};

}  // namespace wgd
