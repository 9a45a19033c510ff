// wg_shapes.cuh — query shapes compiled as constants into the fused kernel.
//
// A shape fixes everything about a query except its data: the storage class of
// each referenced input column, the filter columns and operators, the join
// flavour, the projection program, the group-key packing and the slot layout
// with its aggregate kinds. The filter constants, the projection immediates,
// the column pointers and the tables stay run-time values.
//
// A plan runs on a StatShape<C> instantiation only when shape_matches<C> finds
// every one of these facts equal to the plan's (the plan's compact column
// numbering is part of the shape) and no input or payload column carries a
// validity bitmap, so a specialised launch computes exactly what the generic
// DynShape launch computes for the same plan, with every NULL test compiled out.
//
// Shapes (ids are what wg_agg_kernel_shape reports; 0 = generic):
//  1 star join    WHERE qty > c, fk → dim (direct payload), GROUP BY grp,
//                 SUM(price*(1-disc)) f64, SUM(price) Int128
//  2 group-by     WHERE flag < c GROUP BY k int64: SUM(v int64), COUNT(*),
//                 MIN(f), MAX(f) f64
//  3 high-card    GROUP BY (a int32, b int64) packed: SUM(amount) Int128,
//                 COUNT(*), MIN(x), MAX(x) f64
//  4 filtered int64 group-by: WHERE filt < c GROUP BY key: SUM/COUNT/MIN/MAX(v int64)
//  5 the same over a float64 value
//  6 IPv4 /24     GROUP BY addr >> 8: SUM(bytes), COUNT(*)
#pragma once

#include "wg_agg_kernels.cuh"

#define WG_SHAPE_LIST(name, ...)                                                    \
  __host__ __device__ static constexpr int name(int i) {                           \
    constexpr int v[] = {__VA_ARGS__};                                              \
    return i >= 0 && i < (int)(sizeof(v) / sizeof(v[0])) ? v[i] : 0;               \
  }
#define WG_SHAPE_PROG(name, ...)                                                    \
  __host__ __device__ static constexpr int name(int e, int i) {                    \
    constexpr int v[] = {__VA_ARGS__};                                              \
    return e == 0 && i >= 0 && i < (int)(sizeof(v) / sizeof(v[0])) ? v[i] : 0;     \
  }

namespace wgd {

enum : int32_t { SHAPE_GENERIC = 0, SHAPE_STARJOIN, SHAPE_GROUPBY, SHAPE_HIGHCARD, SHAPE_BATCH_I64, SHAPE_BATCH_F64,
                 SHAPE_IPV4 };

// Fields every shape without a join or projection shares.
struct ShapeNoJoin {
  static constexpr int has_join = 0, direct = 0, probe_col = 0, n_pay = 0, n_exprs = 0;
  WG_SHAPE_LIST(pay_cls, 0)
  WG_SHAPE_PROG(expr_nops, 0)
  WG_SHAPE_PROG(expr_opc, 0)
  WG_SHAPE_PROG(expr_arg, 0)
  WG_SHAPE_LIST(expr_cls, 0)
};
struct ShapeNoFilter {
  static constexpr int n_filters = 0;
  WG_SHAPE_LIST(filt_col, 0)
  WG_SHAPE_LIST(filt_cls, 0)
  WG_SHAPE_LIST(filt_op, 0)
};
struct ShapeOneKey {
  static constexpr int key_words = 1, n_keys = 1;
  WG_SHAPE_LIST(key_i32, 0)
  WG_SHAPE_LIST(key_word, 0)
  WG_SHAPE_LIST(key_shift, 0)
};

// fact (fk int32, qty int32, price DECIMAL, disc float64) ⋈ dim (key int32, grp int32)
struct ShapeStarJoin : ShapeOneKey {
  static constexpr int id = SHAPE_STARJOIN;
  static constexpr bool smem_ok = true;
  static constexpr int n_in = 4;
  WG_SHAPE_LIST(in_cls, WG_CLS_I32, WG_CLS_I32, WG_CLS_DEC, WG_CLS_F64)   // qty, fk, price, disc
  static constexpr int n_filters = 1;
  WG_SHAPE_LIST(filt_col, 0)
  WG_SHAPE_LIST(filt_cls, WG_CLS_I32)
  WG_SHAPE_LIST(filt_op, WG_OP_GT)
  static constexpr int has_join = 1, direct = 1, probe_col = 1, n_pay = 1;
  WG_SHAPE_LIST(pay_cls, WG_CLS_I32)
  static constexpr int n_exprs = 1;
  WG_SHAPE_PROG(expr_nops, 5)
  WG_SHAPE_PROG(expr_opc, WG_EXPR_COL, WG_EXPR_CONST_F, WG_EXPR_COL, WG_EXPR_SUB, WG_EXPR_MUL)
  WG_SHAPE_PROG(expr_arg, 2, 0, 3, 0, 0)
  WG_SHAPE_LIST(expr_cls, WG_CLS_F64)
  WG_SHAPE_LIST(vcls, WG_CLS_I32, WG_CLS_I32, WG_CLS_DEC, WG_CLS_F64, WG_CLS_I32, WG_CLS_F64)
  static constexpr int n_vcols = 6;
  WG_SHAPE_LIST(key_vcol, 4)
  static constexpr int slot_words = 5, n_aggs = 2;
  WG_SHAPE_LIST(agg_kind, K_SUM_F64, K_SUM_DEC)
  WG_SHAPE_LIST(agg_off, 2, 3)
  WG_SHAPE_LIST(agg_null_off, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 5, 2)
};

// (flag int32, k int64, v int64, f float64)
struct ShapeGroupBy : ShapeNoJoin, ShapeOneKey {
  static constexpr int id = SHAPE_GROUPBY;
  static constexpr bool smem_ok = true;
  static constexpr int n_in = 4;
  WG_SHAPE_LIST(in_cls, WG_CLS_I32, WG_CLS_I64, WG_CLS_I64, WG_CLS_F64)
  static constexpr int n_filters = 1;
  WG_SHAPE_LIST(filt_col, 0)
  WG_SHAPE_LIST(filt_cls, WG_CLS_I32)
  WG_SHAPE_LIST(filt_op, WG_OP_LT)
  WG_SHAPE_LIST(vcls, WG_CLS_I32, WG_CLS_I64, WG_CLS_I64, WG_CLS_F64)
  static constexpr int n_vcols = 4;
  WG_SHAPE_LIST(key_vcol, 1)
  static constexpr int slot_words = 5, n_aggs = 4;
  WG_SHAPE_LIST(agg_kind, K_SUM_I64, K_COUNT, K_MIN_F64, K_MAX_F64)
  WG_SHAPE_LIST(agg_off, 2, -1, 3, 4)
  WG_SHAPE_LIST(agg_null_off, -1, -1, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 2, -1, 3, 3)
};

// (a int32, b int64, amount DECIMAL, x float64); key packed as word0 = b,
// word1 low half = a (buildPackedLayout's widest-first order)
struct ShapeHighCard : ShapeNoJoin, ShapeNoFilter {
  static constexpr int id = SHAPE_HIGHCARD;
  static constexpr bool smem_ok = false;
  static constexpr int n_in = 4;
  WG_SHAPE_LIST(in_cls, WG_CLS_I32, WG_CLS_I64, WG_CLS_DEC, WG_CLS_F64)
  WG_SHAPE_LIST(vcls, WG_CLS_I32, WG_CLS_I64, WG_CLS_DEC, WG_CLS_F64)
  static constexpr int n_vcols = 4;
  static constexpr int key_words = 2, n_keys = 2;
  WG_SHAPE_LIST(key_vcol, 0, 1)
  WG_SHAPE_LIST(key_i32, 1, 0)
  WG_SHAPE_LIST(key_word, 1, 0)
  WG_SHAPE_LIST(key_shift, 0, 0)
  static constexpr int slot_words = 8, n_aggs = 4;
  WG_SHAPE_LIST(agg_kind, K_SUM_DEC, K_COUNT, K_MIN_F64, K_MAX_F64)
  WG_SHAPE_LIST(agg_off, 3, -1, 5, 6)
  WG_SHAPE_LIST(agg_null_off, -1, -1, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 2, -1, 3, 3)
};

// (filt int32, key int64, val int64)
struct ShapeBatchI64 : ShapeNoJoin, ShapeOneKey {
  static constexpr int id = SHAPE_BATCH_I64;
  static constexpr bool smem_ok = true;
  static constexpr int n_in = 3;
  WG_SHAPE_LIST(in_cls, WG_CLS_I32, WG_CLS_I64, WG_CLS_I64)
  static constexpr int n_filters = 1;
  WG_SHAPE_LIST(filt_col, 0)
  WG_SHAPE_LIST(filt_cls, WG_CLS_I32)
  WG_SHAPE_LIST(filt_op, WG_OP_LT)
  WG_SHAPE_LIST(vcls, WG_CLS_I32, WG_CLS_I64, WG_CLS_I64)
  static constexpr int n_vcols = 3;
  WG_SHAPE_LIST(key_vcol, 1)
  static constexpr int slot_words = 5, n_aggs = 4;
  WG_SHAPE_LIST(agg_kind, K_SUM_I64, K_COUNT, K_MIN_I64, K_MAX_I64)
  WG_SHAPE_LIST(agg_off, 2, -1, 3, 4)
  WG_SHAPE_LIST(agg_null_off, -1, -1, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 2, -1, 2, 2)
};

// (filt int32, key int64, val float64)
struct ShapeBatchF64 : ShapeNoJoin, ShapeOneKey {
  static constexpr int id = SHAPE_BATCH_F64;
  static constexpr bool smem_ok = true;
  static constexpr int n_in = 3;
  WG_SHAPE_LIST(in_cls, WG_CLS_I32, WG_CLS_I64, WG_CLS_F64)
  static constexpr int n_filters = 1;
  WG_SHAPE_LIST(filt_col, 0)
  WG_SHAPE_LIST(filt_cls, WG_CLS_I32)
  WG_SHAPE_LIST(filt_op, WG_OP_LT)
  WG_SHAPE_LIST(vcls, WG_CLS_I32, WG_CLS_I64, WG_CLS_F64)
  static constexpr int n_vcols = 3;
  WG_SHAPE_LIST(key_vcol, 1)
  static constexpr int slot_words = 5, n_aggs = 4;
  WG_SHAPE_LIST(agg_kind, K_SUM_F64, K_COUNT, K_MIN_F64, K_MAX_F64)
  WG_SHAPE_LIST(agg_off, 2, -1, 3, 4)
  WG_SHAPE_LIST(agg_null_off, -1, -1, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 2, -1, 2, 2)
};

// (addr int64, bytes int64), key = addr >> 8
struct ShapeIPv4 : ShapeNoFilter, ShapeOneKey {
  static constexpr int id = SHAPE_IPV4;
  static constexpr bool smem_ok = true;
  static constexpr int n_in = 2;
  WG_SHAPE_LIST(in_cls, WG_CLS_I64, WG_CLS_I64)
  static constexpr int has_join = 0, direct = 0, probe_col = 0, n_pay = 0;
  WG_SHAPE_LIST(pay_cls, 0)
  static constexpr int n_exprs = 1;
  WG_SHAPE_PROG(expr_nops, 3)
  WG_SHAPE_PROG(expr_opc, WG_EXPR_COL, WG_EXPR_CONST_I, WG_EXPR_SHR)
  WG_SHAPE_PROG(expr_arg, 0, 0, 0)
  WG_SHAPE_LIST(expr_cls, WG_CLS_I64)
  WG_SHAPE_LIST(vcls, WG_CLS_I64, WG_CLS_I64, WG_CLS_I64)
  static constexpr int n_vcols = 3;
  WG_SHAPE_LIST(key_vcol, 2)
  static constexpr int slot_words = 3, n_aggs = 2;
  WG_SHAPE_LIST(agg_kind, K_SUM_I64, K_COUNT)
  WG_SHAPE_LIST(agg_off, 2, -1)
  WG_SHAPE_LIST(agg_null_off, -1, -1)
  WG_SHAPE_LIST(agg_vcol, 1, -1)
};

// Host side: is every shape fact of P equal to C's?
template <class C>
inline bool shape_matches(const Plan& P) {
  if (P.n_in != C::n_in || P.n_filters != C::n_filters || P.has_join != C::has_join || P.n_exprs != C::n_exprs)
    return false;
  for (int j = 0; j < C::n_in; ++j)
    if (P.in[j].cls != C::in_cls(j) || P.in[j].valid != nullptr) return false;
  for (int f = 0; f < C::n_filters; ++f)
    if (P.filt[f].col != C::filt_col(f) || P.filt[f].cls != C::filt_cls(f) || P.filt[f].op != C::filt_op(f))
      return false;
  if (C::has_join) {
    if (P.join.direct != C::direct || P.probe_col != C::probe_col || P.join.n_pay != C::n_pay ||
        P.join.jtype != WG_JOIN_INNER)
      return false;
    for (int p = 0; p < C::n_pay; ++p)
      if (P.join.pay[p].cls != C::pay_cls(p) || P.join.pay[p].valid != nullptr) return false;
  }
  for (int e = 0; e < C::n_exprs; ++e) {
    if (P.expr[e].n_ops != C::expr_nops(e, 0) || P.expr[e].result_cls != C::expr_cls(e)) return false;
    for (int k = 0; k < P.expr[e].n_ops; ++k)
      if (P.expr[e].opc[k] != C::expr_opc(e, k) || P.expr[e].arg[k] != C::expr_arg(e, k)) return false;
  }
  const int nv = P.n_in + (P.has_join ? P.join.n_pay : 0) + P.n_exprs;
  if (nv != C::n_vcols) return false;
  for (int j = 0; j < nv; ++j)
    if (P.vcls[j] != C::vcls(j)) return false;
  const Layout& L = P.L;
  if (L.key_words != C::key_words || L.slot_words != C::slot_words || L.n_keys != C::n_keys || L.n_aggs != C::n_aggs)
    return false;
  for (int k = 0; k < C::n_keys; ++k) {
    if (L.key_vcol[k] != C::key_vcol(k)) return false;
    if (C::key_words == 2 && (L.key_i32[k] != C::key_i32(k) || L.key_word[k] != C::key_word(k) ||
                              L.key_shift[k] != C::key_shift(k)))
      return false;
  }
  for (int a = 0; a < C::n_aggs; ++a)
    if (L.agg[a].kind != C::agg_kind(a) || L.agg[a].off != C::agg_off(a) || L.agg[a].null_off != C::agg_null_off(a) ||
        L.agg[a].vcol != C::agg_vcol(a))
      return false;
  return true;
}

// The compiled shape of a plan, SHAPE_GENERIC when none matches.
inline int32_t shape_of(const Plan& P) {
  if (shape_matches<ShapeStarJoin>(P)) return SHAPE_STARJOIN;
  if (shape_matches<ShapeGroupBy>(P)) return SHAPE_GROUPBY;
  if (shape_matches<ShapeHighCard>(P)) return SHAPE_HIGHCARD;
  if (shape_matches<ShapeBatchI64>(P)) return SHAPE_BATCH_I64;
  if (shape_matches<ShapeBatchF64>(P)) return SHAPE_BATCH_F64;
  if (shape_matches<ShapeIPv4>(P)) return SHAPE_IPV4;
  return SHAPE_GENERIC;
}

}  // namespace wgd
