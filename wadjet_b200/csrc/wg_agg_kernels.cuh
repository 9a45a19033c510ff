// wg_agg_kernels.cuh — device code of the hash aggregate and the fused
// filter → probe → project → aggregate kernel.
//
// Every decision about the query's shape (column types, filter operators, the
// projection program, the slot layout, the aggregate kinds) goes through a
// shape accessor. DynShape reads those facts from the launch plan at run time,
// so one kernel serves any plan. StatShape<C> answers from the compile-time
// constants of C: after unrolling, every switch on a type or kind folds away
// and the kernel is straight-line code for that query shape. The host launches
// a StatShape instantiation when the plan matches one exactly (shape_matches,
// wg_shapes.cuh) and the DynShape one otherwise; results are identical.
#pragma once

#include "wg_agg.cuh"
#include "wg_tma.cuh"

namespace wgd {

struct Val {
  unsigned long long lo, hi;
  bool null;
};

__device__ __forceinline__ double as_f(unsigned long long w) { return __longlong_as_double((long long)w); }
__device__ __forceinline__ unsigned long long as_w(double d) { return (unsigned long long)__double_as_longlong(d); }

// One value of storage class `cls` at element i of `data` (read-only path).
__device__ __forceinline__ Val load_typed(const void* data, int cls, int64_t i) {
  Val v;
  v.hi = 0;
  v.null = false;
  switch (cls) {
    case WG_CLS_I32: v.lo = (unsigned long long)(long long)__ldg((const int32_t*)data + i); break;
    case WG_CLS_I64: v.lo = (unsigned long long)__ldg((const long long*)data + i); break;
    case WG_CLS_F32: v.lo = as_w((double)__ldg((const float*)data + i)); break;
    case WG_CLS_F64: v.lo = (unsigned long long)__ldg((const long long*)data + i); break;
    case WG_CLS_DEC: {
      const longlong2 d = __ldg((const longlong2*)data + i);  // .x = hi, .y = lo
      v.lo = (unsigned long long)d.y;
      v.hi = (unsigned long long)d.x;
      break;
    }
    default: v.lo = 0;
  }
  return v;
}

// The same for input columns read once: streaming loads (evict first), so the
// stream does not push the join index and the tables out of L2.
__device__ __forceinline__ Val load_stream(const void* data, int cls, int64_t i) {
  Val v;
  v.hi = 0;
  v.null = false;
  switch (cls) {
    case WG_CLS_I32: v.lo = (unsigned long long)(long long)__ldcs((const int32_t*)data + i); break;
    case WG_CLS_I64: v.lo = (unsigned long long)__ldcs((const long long*)data + i); break;
    case WG_CLS_F32: v.lo = as_w((double)__ldcs((const float*)data + i)); break;
    case WG_CLS_F64: v.lo = (unsigned long long)__ldcs((const long long*)data + i); break;
    case WG_CLS_DEC: {
      const longlong2 d = __ldcs((const longlong2*)data + i);  // .x = hi, .y = lo
      v.lo = (unsigned long long)d.y;
      v.hi = (unsigned long long)d.x;
      break;
    }
    default: v.lo = 0;
  }
  return v;
}

// The same from memory that may be shared (generic loads).
__device__ __forceinline__ Val load_generic(const char* p, int cls) {
  Val v;
  v.hi = 0;
  v.null = false;
  switch (cls) {
    case WG_CLS_I32: v.lo = (unsigned long long)(long long)*(const int32_t*)p; break;
    case WG_CLS_I64: case WG_CLS_F64: v.lo = *(const unsigned long long*)p; break;
    case WG_CLS_F32: v.lo = as_w((double)*(const float*)p); break;
    case WG_CLS_DEC: v.hi = ((const unsigned long long*)p)[0]; v.lo = ((const unsigned long long*)p)[1]; break;
    default: v.lo = 0;
  }
  return v;
}

__host__ __device__ __forceinline__ constexpr int cls_bytes(int cls) {
  return cls == WG_CLS_I32 || cls == WG_CLS_F32 ? 4 : cls == WG_CLS_DEC ? 16 : 8;
}

// Identity of an accumulator word (the empty-slot value the layout starts from).
__device__ __forceinline__ unsigned long long ident_word(int kind, int w) {
  switch (kind) {
    case K_MIN_I64: return 0x7FFFFFFFFFFFFFFFULL;
    case K_MAX_I64: return 0x8000000000000000ULL;
    case K_MIN_F64: return ~0ULL;
    case K_MAX_F64: return 0ULL;
    case K_MIN_DEC: return w == 0 ? ~0ULL : 0x7FFFFFFFFFFFFFFFULL;
    case K_MAX_DEC: return w == 0 ? 0ULL : 0x8000000000000000ULL;
    default: return 0ULL;
  }
}

// ---- shape accessors --------------------------------------------------------

// Layout facts of a table (folds, flushes, growth): always run time.
struct LayoutAcc {
  const Layout& L;
  __device__ __forceinline__ int key_words() const { return L.key_words; }
  __device__ __forceinline__ int slot_words() const { return L.slot_words; }
  __device__ __forceinline__ int n_aggs() const { return L.n_aggs; }
  __device__ __forceinline__ int agg_kind(int a) const { return L.agg[a].kind; }
  __device__ __forceinline__ int agg_off(int a) const { return L.agg[a].off; }
  __device__ __forceinline__ int agg_null_off(int a) const { return L.agg[a].null_off; }
};

// Everything from the plan at run time.
struct DynShape {
  static constexpr bool smem_ok = true;
  static constexpr int kBlock = 512, kMinBlocks = 2;  // launch shape of the plain fused kernel
  const Plan& P;
  __device__ __forceinline__ bool nullable() const { return true; }
  __device__ __forceinline__ int n_in() const { return P.n_in; }
  __device__ __forceinline__ int in_cls(int j) const { return P.in[j].cls; }
  __device__ __forceinline__ int n_filters() const { return P.n_filters; }
  __device__ __forceinline__ int filt_col(int f) const { return P.filt[f].col; }
  __device__ __forceinline__ int filt_cls(int f) const { return P.filt[f].cls; }
  __device__ __forceinline__ int filt_op(int f) const { return P.filt[f].op; }
  __device__ __forceinline__ int has_join() const { return P.has_join; }
  __device__ __forceinline__ int direct() const { return P.join.direct; }
  __device__ __forceinline__ int probe_col() const { return P.probe_col; }
  __device__ __forceinline__ int n_pay() const { return P.join.n_pay; }
  __device__ __forceinline__ int pay_cls(int i) const { return P.join.pay[i].cls; }
  __device__ __forceinline__ int n_exprs() const { return P.n_exprs; }
  __device__ __forceinline__ int expr_nops(int e) const { return P.expr[e].n_ops; }
  __device__ __forceinline__ int expr_opc(int e, int k) const { return P.expr[e].opc[k]; }
  __device__ __forceinline__ int expr_arg(int e, int k) const { return P.expr[e].arg[k]; }
  __device__ __forceinline__ int expr_cls(int e) const { return P.expr[e].result_cls; }
  __device__ __forceinline__ int vcls(int j) const { return P.vcls[j]; }
  __device__ __forceinline__ int key_words() const { return P.L.key_words; }
  __device__ __forceinline__ int slot_words() const { return P.L.slot_words; }
  __device__ __forceinline__ int n_keys() const { return P.L.n_keys; }
  __device__ __forceinline__ int key_vcol(int k) const { return P.L.key_vcol[k]; }
  __device__ __forceinline__ int key_i32(int k) const { return P.L.key_i32[k]; }
  __device__ __forceinline__ int key_word(int k) const { return P.L.key_word[k]; }
  __device__ __forceinline__ int key_shift(int k) const { return P.L.key_shift[k]; }
  __device__ __forceinline__ int n_aggs() const { return P.L.n_aggs; }
  __device__ __forceinline__ int agg_kind(int a) const { return P.L.agg[a].kind; }
  __device__ __forceinline__ int agg_off(int a) const { return P.L.agg[a].off; }
  __device__ __forceinline__ int agg_null_off(int a) const { return P.L.agg[a].null_off; }
  __device__ __forceinline__ int agg_vcol(int a) const { return P.L.agg[a].vcol; }
};

// Everything from compile-time constants (see wg_shapes.cuh for the C structs).
template <class C>
struct StatShape {
  static constexpr bool smem_ok = C::smem_ok;
  // straight-line code fits 40 registers: two 768-thread CTAs per SM (48 warps)
  static constexpr int kBlock = 768, kMinBlocks = 2;
  // vector kernel: evaluate all of a lane's rows before their table updates
  // when no projection program runs per row (short, independent chains the
  // scheduler interleaves); with one, row by row keeps fewer values live
  static constexpr bool kRowsTogether = C::n_exprs == 0;
  const Plan& P;
  // compiled shapes take inputs without validity bitmaps (shape_matches), so
  // no value they read is NULL
  __device__ __forceinline__ constexpr bool nullable() const { return false; }
  __device__ __forceinline__ constexpr int n_in() const { return C::n_in; }
  __device__ __forceinline__ constexpr int in_cls(int j) const { return C::in_cls(j); }
  __device__ __forceinline__ constexpr int n_filters() const { return C::n_filters; }
  __device__ __forceinline__ constexpr int filt_col(int f) const { return C::filt_col(f); }
  __device__ __forceinline__ constexpr int filt_cls(int f) const { return C::filt_cls(f); }
  __device__ __forceinline__ constexpr int filt_op(int f) const { return C::filt_op(f); }
  __device__ __forceinline__ constexpr int has_join() const { return C::has_join; }
  __device__ __forceinline__ constexpr int direct() const { return C::direct; }
  __device__ __forceinline__ constexpr int probe_col() const { return C::probe_col; }
  __device__ __forceinline__ constexpr int n_pay() const { return C::n_pay; }
  __device__ __forceinline__ constexpr int pay_cls(int i) const { return C::pay_cls(i); }
  __device__ __forceinline__ constexpr int n_exprs() const { return C::n_exprs; }
  __device__ __forceinline__ constexpr int expr_nops(int e) const { return C::expr_nops(e, 0); }
  __device__ __forceinline__ constexpr int expr_opc(int e, int k) const { return C::expr_opc(e, k); }
  __device__ __forceinline__ constexpr int expr_arg(int e, int k) const { return C::expr_arg(e, k); }
  __device__ __forceinline__ constexpr int expr_cls(int e) const { return C::expr_cls(e); }
  __device__ __forceinline__ constexpr int vcls(int j) const { return C::vcls(j); }
  __device__ __forceinline__ constexpr int key_words() const { return C::key_words; }
  __device__ __forceinline__ constexpr int slot_words() const { return C::slot_words; }
  __device__ __forceinline__ constexpr int n_keys() const { return C::n_keys; }
  __device__ __forceinline__ constexpr int key_vcol(int k) const { return C::key_vcol(k); }
  __device__ __forceinline__ constexpr int key_i32(int k) const { return C::key_i32(k); }
  __device__ __forceinline__ constexpr int key_word(int k) const { return C::key_word(k); }
  __device__ __forceinline__ constexpr int key_shift(int k) const { return C::key_shift(k); }
  __device__ __forceinline__ constexpr int n_aggs() const { return C::n_aggs; }
  __device__ __forceinline__ constexpr int agg_kind(int a) const { return C::agg_kind(a); }
  __device__ __forceinline__ constexpr int agg_off(int a) const { return C::agg_off(a); }
  __device__ __forceinline__ constexpr int agg_null_off(int a) const { return C::agg_null_off(a); }
  __device__ __forceinline__ constexpr int agg_vcol(int a) const { return C::agg_vcol(a); }
};

// ---- row sources --------------------------------------------------------------

// Input column j of one row, straight from HBM.
struct SrcGlobal {
  int64_t row;
  template <class Sh>
  __device__ __forceinline__ Val in(const Plan& P, const Sh& sh, int j) const {
    Val v = load_stream(P.in[j].data, sh.in_cls(j), row);
    v.null = sh.nullable() && is_null(P.in[j], row);
    return v;
  }
};

template <class Sh, class Src>
__device__ __forceinline__ Val fetch_base(const Plan& P, const Sh& sh, const Src& src, int j, int32_t brow) {
  if (j < sh.n_in()) return src.in(P, sh, j);
  if (sh.direct()) {  // brow already holds the payload's 32 bits
    Val v;
    v.hi = 0;
    v.null = false;
    v.lo = sh.pay_cls(0) == WG_CLS_F32 ? as_w((double)__int_as_float(brow)) : (unsigned long long)(long long)brow;
    return v;
  }
  const int p = j - sh.n_in();
  if (sh.nullable() && brow < 0) {  // LEFT join, unmatched probe row: NULL build columns
    Val v;
    v.lo = 0; v.hi = 0; v.null = true;
    return v;
  }
  Val v = load_typed(P.join.pay[p].data, sh.pay_cls(p), brow);
  v.null = sh.nullable() && is_null(P.join.pay[p], brow);
  return v;
}

// Postfix evaluation of a projection (expr.BinOpNumeric): integer ops wrap,
// float ops are single IEEE operations (no contraction), DECIMAL operands read
// as Int128.ToFloat64, a NULL operand makes the result NULL. The four-entry
// stack is addressed through selects so it stays in registers (and, for a
// static shape, folds to straight-line code).
template <class Sh, class Src>
__device__ __forceinline__ Val eval_expr(const Plan& P, const Sh& sh, int e, const Src& src, int32_t brow) {
  unsigned long long s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  unsigned fl = 0;  // bit i: stack entry i holds a float
  int sp = 0;
  bool null = false;
#pragma unroll
  for (int k = 0; k < WG_EXPR_OPS; ++k) {
    if (k >= sh.expr_nops(e)) break;
    const int opc = sh.expr_opc(e, k);
    unsigned long long w = 0;
    bool isf = false;
    if (opc == 0) {  // WG_EXPR_COL
      const int j = sh.expr_arg(e, k);
      Val v = fetch_base(P, sh, src, j, brow);
      null |= v.null;
      const int cls = sh.vcls(j);
      if (cls == WG_CLS_I32 || cls == WG_CLS_I64) { w = v.lo; isf = false; }
      else if (cls == WG_CLS_DEC) {
        w = as_w(div_by_recip(int128_to_f64((int64_t)v.hi, v.lo), P.vdiv_b[j], P.vdiv_y[j]));
        isf = true;
      }
      else { w = v.lo; isf = true; }
    } else if (opc == 1) {
      w = (unsigned long long)P.expr[e].imm[k]; isf = false;
    } else if (opc == 2) {
      w = (unsigned long long)P.expr[e].imm[k]; isf = true;
    } else {
      if (sp < 2) { set_error(P.err, WG_DERR_STACK); Val r; r.lo = 0; r.hi = 0; r.null = true; return r; }
      const unsigned long long b = sp == 1 ? s0 : sp == 2 ? s1 : sp == 3 ? s2 : s3;
      const unsigned long long a = sp == 2 ? s0 : sp == 3 ? s1 : s2;
      const bool bf = (fl >> (sp - 1)) & 1, af = (fl >> (sp - 2)) & 1;
      sp -= 2;
      if (opc == 7 || opc == 8) {  // SHR, AND (integers)
        w = opc == 7 ? (unsigned long long)((long long)a >> (b & 63)) : (a & b);
        isf = false;
      } else if (!af && !bf && opc != 6) {
        w = opc == 3 ? a + b : opc == 4 ? a - b : a * b;
        isf = false;
      } else {
        const double x = af ? as_f(a) : __ll2double_rn((long long)a);
        const double y = bf ? as_f(b) : __ll2double_rn((long long)b);
        double r = 0.0;
        switch (opc) {
          case 3: r = __dadd_rn(x, y); break;
          case 4: r = __dsub_rn(x, y); break;
          case 5: r = __dmul_rn(x, y); break;
          case 6: r = __ddiv_rn(x, y); break;
        }
        w = as_w(r);
        isf = true;
      }
    }
    if (sp >= 4) { set_error(P.err, WG_DERR_STACK); Val r; r.lo = 0; r.hi = 0; r.null = true; return r; }
    if (sp == 0) s0 = w; else if (sp == 1) s1 = w; else if (sp == 2) s2 = w; else s3 = w;
    fl = isf ? (fl | (1u << sp)) : (fl & ~(1u << sp));
    ++sp;
  }
  Val r;
  r.hi = 0;
  r.null = null;
  const unsigned long long top = sp == 1 ? s0 : sp == 2 ? s1 : sp == 3 ? s2 : s3;
  const bool tf = sp > 0 && ((fl >> (sp - 1)) & 1);
  if (sh.expr_cls(e) == WG_CLS_F64 && !tf) r.lo = as_w(__ll2double_rn((long long)top));
  else r.lo = top;
  return r;
}

// The projected columns of one (row, build row), evaluated once and then read
// by every key and aggregate that refers to them.
struct ExprVals {
  Val v[WG_MAX_EXPRS];
};

template <class Sh, class Src>
__device__ __forceinline__ void eval_exprs(const Plan& P, const Sh& sh, const Src& src, int32_t brow, ExprVals& ev) {
#pragma unroll
  for (int e = 0; e < WG_MAX_EXPRS; ++e) {
    if (e < sh.n_exprs()) ev.v[e] = eval_expr(P, sh, e, src, brow);
    else { ev.v[e].lo = 0; ev.v[e].hi = 0; ev.v[e].null = true; }
  }
}

template <class Sh, class Src>
__device__ __forceinline__ Val fetch(const Plan& P, const Sh& sh, const Src& src, int j, int32_t brow,
                                     const ExprVals& ev) {
  const int nb = sh.n_in() + (sh.has_join() ? sh.n_pay() : 0);
  if (j < nb) return fetch_base(P, sh, src, j, brow);
  return j == nb ? ev.v[0] : ev.v[1];
}

template <int NA>
struct Contrib {
  unsigned long long w0[NA], w1[NA];
  int nul[NA];
};

// One row's contribution to each aggregate (the scatter kernels' per-row
// update, internal/engine/exec/agg_scatter.go:178-510), as combinable words.
template <int NA, class Sh, class Src>
__device__ __forceinline__ void make_contrib(const Plan& P, const Sh& sh, const Src& src, int32_t brow,
                                             const ExprVals& ev, Contrib<NA>& c) {
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    c.w0[a] = 0; c.w1[a] = 0; c.nul[a] = 0;
    if (a >= sh.n_aggs()) continue;
    const int kind = sh.agg_kind(a), vcol = sh.agg_vcol(a);
    if (vcol < 0 || kind == K_COUNT) {
      if (vcol >= 0) c.nul[a] = fetch(P, sh, src, vcol, brow, ev).null ? 1 : 0;
      continue;
    }
    const Val v = fetch(P, sh, src, vcol, brow, ev);
    if (v.null) {
      c.nul[a] = 1;
      c.w0[a] = ident_word(kind, 0);
      c.w1[a] = ident_word(kind, 1);
      continue;
    }
    const int cls = sh.vcls(vcol);
    switch (kind) {
      case K_SUM_I64: case K_MIN_I64: case K_MAX_I64: c.w0[a] = v.lo; break;
      case K_SUM_F64:
        c.w0[a] = (cls == WG_CLS_I32 || cls == WG_CLS_I64) ? as_w(__ll2double_rn((long long)v.lo)) : v.lo;
        break;
      case K_MIN_F64: case K_MAX_F64: c.w0[a] = f64_to_ord(as_f(v.lo)); break;
      default: c.w0[a] = v.lo; c.w1[a] = v.hi; break;  // DECIMAL kinds
    }
  }
}

__device__ __forceinline__ void combine(int kind, unsigned long long& a0, unsigned long long& a1, unsigned long long b0,
                                        unsigned long long b1) {
  switch (kind) {
    case K_SUM_I64: a0 += b0; break;
    case K_SUM_F64: a0 = as_w(__dadd_rn(as_f(a0), as_f(b0))); break;
    case K_SUM_DEC: add128(a0, a1, b0, b1); break;
    case K_MIN_I64: if ((long long)b0 < (long long)a0) a0 = b0; break;
    case K_MAX_I64: if ((long long)b0 > (long long)a0) a0 = b0; break;
    case K_MIN_F64: if (b0 < a0) a0 = b0; break;
    case K_MAX_F64: if (b0 > a0) a0 = b0; break;
    case K_MIN_DEC: if (less128(b0, b1, a0, a1)) { a0 = b0; a1 = b1; } break;
    case K_MAX_DEC: if (less128(a0, a1, b0, b1)) { a0 = b0; a1 = b1; } break;
    default: break;
  }
}

// Add a two's-complement integer of `nlimbs` 32-bit limbs (lo, hi words) to the
// limbs at L with native 32-bit shared-memory atomics: each limb's carry out is
// read from the value its atomic replaced and added to the next limb, so the
// words end up holding the exact sum mod 2^(32*nlimbs) in any interleaving.
// (64-bit shared-memory atomic adds are compare-and-swap loops that replay
// while lanes of a warp hit the same hot group; 32-bit adds are not.)
// In 32-bit arithmetic: a = limb + carry wraps to 0 only for limb 2^32-1 with
// a carry, which adds nothing here and passes the carry on, and a = 0 without
// a carry passes none: either way the carry is unchanged and no atomic runs.
// The top limb's carry out is dropped (mod 2^(32*nlimbs)), so its atomic
// returns nothing.
__device__ __forceinline__ void smem_add_limbs(unsigned* L, int nlimbs, unsigned long long lo, unsigned long long hi) {
  const unsigned x[4] = {(unsigned)lo, (unsigned)(lo >> 32), (unsigned)hi, (unsigned)(hi >> 32)};
  unsigned carry = 0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    if (i >= nlimbs) break;
    const unsigned a = x[i] + carry;
    if (a == 0) continue;
    if (i == nlimbs - 1) {
      atomicAdd(L + i, a);
    } else {
      const unsigned old = atomicAdd(L + i, a);
      carry = old > ~a ? 1u : 0u;  // old + a overflowed 32 bits
    }
  }
}

// Float SUMs in a shared-memory table can accumulate exactly instead of in
// float: a finite x with 2^-12 <= |x| < 2^30 is a multiple of 2^-64 below 2^30,
// so x * 2^64 is an integer below 2^94, added into a 128-bit two's-complement
// accumulator with 32-bit shared-memory atomics (fast even when many lanes hit
// one hot group, where 64-bit shared atomics serialise). The sum is exact for
// fewer than 2^32 rows, and the flush rounds it to float64 once. Values
// outside that range (zero, tiny, huge, NaN, Inf) add into the slot's float
// word instead. The result is the correctly rounded sum of the in-range values
// plus the float sum of the rest: a different summation order from the
// reference, within the same bound as any reordered float sum.
__device__ __forceinline__ bool f64_to_fixed(double d, unsigned long long& lo, unsigned long long& hi) {
  const double ad = fabs(d);
  if (!(ad >= 0x1p-12 && ad < 0x1p30)) return false;
  const double y = __dmul_rn(d, 0x1p64);                 // exact: a power-of-two scaling, |y| < 2^94
  const double a = trunc(__dmul_rn(y, 0x1p-62));         // |a| < 2^32, exact
  const double r = __dsub_rn(y, __dmul_rn(a, 0x1p62));   // exact: y's bits below 2^62, |r| < 2^62
  const long long ai = (long long)a, ri = (long long)r;
  const unsigned long long l0 = (unsigned long long)ai << 62;
  const long long h0 = ai >> 2;                          // a * 2^62 as (h0:l0)
  lo = l0 + (unsigned long long)ri;
  hi = (unsigned long long)(h0 + (ri < 0 ? -1LL : 0LL) + (lo < l0 ? 1LL : 0LL));
  return true;
}

// The 128-bit two's-complement integer (hi:lo) times 2^-64, rounded to nearest
// even once: the top 64 significant bits with a sticky bit for the rest convert
// exactly as the whole would, then scale by a power of two.
__device__ __forceinline__ double fixed_to_f64(unsigned long long lo, unsigned long long hi) {
  if ((long long)hi == ((long long)lo >> 63)) return __dmul_rn(__ll2double_rn((long long)lo), 0x1p-64);
  const bool neg = (long long)hi < 0;
  if (neg) {  // magnitude
    lo = ~lo + 1ULL;
    hi = ~hi + (lo == 0 ? 1ULL : 0ULL);
  }
  double v;
  if (hi == 0) {  // a magnitude in [2^63, 2^64)
    v = __dmul_rn(__ull2double_rn(lo), 0x1p-64);
  } else {
    const int n = 64 - __clzll((long long)hi);           // bits of the high word, 1..64
    unsigned long long t = n == 64 ? hi : ((hi << (64 - n)) | (lo >> n));
    const unsigned long long dropped = n == 64 ? lo : (lo << (64 - n));
    if (dropped) t |= 1ULL;                               // sticky: only breaks ties
    v = scalbn(__ull2double_rn(t), n - 64);               // exact power-of-two scaling
  }
  return neg ? -v : v;
}

// Fold a combined contribution into a slot with atomics. SH: the slot is in a
// CTA-private shared-memory table, where the row count is a 32-bit counter in
// the low half of its word (a CTA applies fewer than 2^32 rows), integer and
// DECIMAL sums go limb by limb, and MIN/MAX skip the atomic when the slot
// already holds a value at least as good (slot values only ever improve).
// A float SUM has no native shared-memory atomic (it is a compare-and-swap
// loop that replays while lanes of a warp hit the same hot group), so a shared
// slot may hold `rep` copies of each float SUM: lane l adds into copy l % rep
// (copy 0 is the layout's word, copies 1.. follow the slot's regular words),
// which divides those replays by about `rep`; the flush adds the copies.
// rep < 0: float SUMs accumulate in fixed point (f64_to_fixed), in two words per
// float SUM after the slot's regular words.
template <int NA, bool SH, class Lay>
__device__ __forceinline__ void apply(const Lay& ly, unsigned long long* s, const Contrib<NA>& c,
                                      unsigned long long rows, int rep = 1, bool test_first = false) {
  const bool test = SH || test_first;  // MIN/MAX: read the slot, skip an atomic that cannot win
  if (SH) atomicAdd((unsigned*)(s + ly.key_words()), (unsigned)rows);
  else atomicAdd(s + ly.key_words(), rows);
  const bool fix = SH && rep < 0;
  const int copy = SH && rep > 1 ? (int)(threadIdx.x & 31) & (rep - 1) : 0;
  int nf = 0;  // float SUMs before aggregate a
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    if (a >= ly.n_aggs()) continue;
    const int kind = ly.agg_kind(a), off = ly.agg_off(a), noff = ly.agg_null_off(a);
    const unsigned long long w0 = c.w0[a], w1 = c.w1[a];
    unsigned long long* t = s + off;
    unsigned long long* tf = nullptr;
    if (SH && kind == K_SUM_F64) {
      if (fix) tf = s + ly.slot_words() + 2 * nf;
      else if (copy > 0) t = s + ly.slot_words() + nf * (rep - 1) + (copy - 1);
      ++nf;
    }
    switch (kind) {
      case K_SUM_I64:
        if (w0) { if (SH) smem_add_limbs((unsigned*)t, 2, w0, 0); else atomicAdd(t, w0); }
        break;
      case K_SUM_F64: {
        const double d = as_f(w0);
        unsigned long long flo, fhi;
        if (tf != nullptr && f64_to_fixed(d, flo, fhi)) smem_add_limbs((unsigned*)tf, 4, flo, fhi);
        else if (d != 0.0) atomicAdd((double*)t, d);
        break;
      }
      case K_SUM_DEC:
        if (SH) smem_add_limbs((unsigned*)t, 4, w0, w1);
        else atomic_add128(t, w0, w1);
        break;
      case K_MIN_I64:
        if (w0 != 0x7FFFFFFFFFFFFFFFULL && (!test || (long long)w0 < *(volatile long long*)t))
          atomicMin((long long*)t, (long long)w0);
        break;
      case K_MAX_I64:
        if (w0 != 0x8000000000000000ULL && (!test || (long long)w0 > *(volatile long long*)t))
          atomicMax((long long*)t, (long long)w0);
        break;
      case K_MIN_F64:
        if (w0 != ~0ULL && (!test || w0 < *(volatile unsigned long long*)t)) atomicMin(t, w0);
        break;
      case K_MAX_F64:
        if (w0 != 0ULL && (!test || w0 > *(volatile unsigned long long*)t)) atomicMax(t, w0);
        break;
      case K_MIN_DEC: atomic_min128((U128*)t, w0, w1); break;
      case K_MAX_DEC: atomic_max128((U128*)t, w0, w1); break;
      default: break;
    }
    if (noff >= 0 && c.nul[a]) atomicAdd(s + noff, (unsigned long long)c.nul[a]);
  }
}

// Contribution held by a whole slot (shared-memory flush, merge, migration).
template <int NA, class Lay>
__device__ __forceinline__ void slot_contrib(const Lay& ly, const unsigned long long* s, Contrib<NA>& c) {
#pragma unroll
  for (int a = 0; a < NA; ++a) {
    c.w0[a] = 0; c.w1[a] = 0; c.nul[a] = 0;
    if (a >= ly.n_aggs()) continue;
    const int off = ly.agg_off(a), noff = ly.agg_null_off(a);
    if (off >= 0) { c.w0[a] = s[off]; if (kind_words(ly.agg_kind(a)) == 2) c.w1[a] = s[off + 1]; }
    if (noff >= 0) c.nul[a] = (int)s[noff];
  }
}

// A thread's unused group reservations (Table::n_groups counts reserved groups;
// an insert must hold one). Taken credit_chunk at a time and handed back when
// the thread is done, so n_groups is exact again after the kernel.
struct Credit {
  unsigned long long n = 0;
  __device__ __forceinline__ bool take(const Table& T, int chunk) {
    if (n == 0) {
      const unsigned long long want = (unsigned long long)max(1, chunk);
      const unsigned long long r = atomicAdd(T.n_groups, want);
      if (r >= T.limit) {
        atomicAdd(T.n_groups, 0ULL - want);
        return false;
      }
      const unsigned long long ok = min(want, T.limit - r);
      if (ok < want) atomicAdd(T.n_groups, 0ULL - (want - ok));
      n = ok;
    }
    --n;
    return true;
  }
  __device__ __forceinline__ void give_back() { ++n; }
  __device__ __forceinline__ void release(const Table& T) {
    if (n) atomicAdd(T.n_groups, 0ULL - n);
    n = 0;
  }
};

// Find or insert the global slot of a key. Inserting claims a group
// reservation first; past T.limit the insert is refused and the overflow flag
// raised (the host then replays the launch on a larger table).
template <class Lay>
__device__ __forceinline__ unsigned long long* find_global(const Lay& ly, const Table& T, unsigned long long k0,
                                                           unsigned long long k1, bool keynull, int32_t* err,
                                                           Credit* cr = nullptr) {
  Credit local;  // without a caller's credit: exactly one reservation per insert
  Credit& c = cr ? *cr : local;
  const int chunk = cr ? T.credit_chunk : 1;
  const int sw = ly.slot_words();
  if (ly.key_words() == 0) return T.slots;
  const uint64_t cap = T.mask + 1;
  if (keynull) return T.slots + (cap + 1) * sw;
  if (ly.key_words() == 1) {
    if (k0 == WG_EMPTY_KEY) return T.slots + cap * sw;
    uint64_t h = fib_slot(k0, T.shift);
    for (uint64_t probe = 0; probe <= T.mask; ++probe) {
      unsigned long long* s = T.slots + h * sw;
      unsigned long long cur = *((volatile unsigned long long*)s);
      if (cur == k0) return s;
      if (cur == WG_EMPTY_KEY) {
        if (!c.take(T, chunk)) {
          *T.overflow = 1;
          return nullptr;
        }
        unsigned long long old = atomicCAS(s, WG_EMPTY_KEY, k0);
        if (old == WG_EMPTY_KEY) return s;
        c.give_back();
        if (!cr) c.release(T);
        if (old == k0) return s;
      }
      h = (h + 1) & T.mask;
    }
  } else {
    if (k0 == ~0ULL && k1 == ~0ULL) return T.slots + cap * sw;
    uint64_t h = packed_slot(k0, k1, T.shift);
    for (uint64_t probe = 0; probe <= T.mask; ++probe) {
      unsigned long long* s = T.slots + h * sw;
      // A slot's key words change once, from {~0,~0} to the key. A read with
      // neither word ~0 is therefore the complete key; anything else is settled
      // by the 128-bit CAS below.
      const U128 cur = read128(s);
      if (cur.lo != ~0ULL && cur.hi != ~0ULL) {
        if (cur.lo == k0 && cur.hi == k1) return s;
      } else {
        if (!c.take(T, chunk)) {
          *T.overflow = 1;
          return nullptr;
        }
        U128 e; e.lo = ~0ULL; e.hi = ~0ULL;
        U128 k; k.lo = k0; k.hi = k1;
        U128 old = cas128((U128*)s, e, k);
        if (old.lo == e.lo && old.hi == e.hi) return s;
        c.give_back();
        if (!cr) c.release(T);
        if (old.lo == k0 && old.hi == k1) return s;
      }
      h = (h + 1) & T.mask;
    }
  }
  set_error(err, WG_DERR_TABLE_FULL);
  return nullptr;
}

// Words per shared slot and copies of each float SUM in it.
__device__ __forceinline__ int smem_stride(const Plan& P) { return P.smem_sw > 0 ? P.smem_sw : P.L.slot_words; }
__device__ __forceinline__ int smem_copies(const Plan& P) { return P.smem_rep > 1 ? P.smem_rep : P.smem_rep < 0 ? -1 : 1; }

// CTA-private shared-memory table (single int64 key, no NULL words). Returns
// nullptr when the key is absent and the table has reached its fill limit.
__device__ __forceinline__ unsigned long long* find_smem(unsigned long long* sm, int S, int sw,
                                                         unsigned long long k0, int* s_groups, int s_limit) {
  if (k0 == WG_EMPTY_KEY) return nullptr;
  uint32_t h = (uint32_t)__umul64hi(k0 * 0x9E3779B97F4A7C15ULL, (unsigned long long)S);
  for (int p = 0; p < S; ++p) {
    unsigned long long* s = sm + (size_t)h * sw;
    unsigned long long cur = *((volatile unsigned long long*)s);
    if (cur == k0) return s;
    if (cur == WG_EMPTY_KEY) {
      if (*((volatile int*)s_groups) >= s_limit) return nullptr;
      unsigned long long old = atomicCAS(s, WG_EMPTY_KEY, k0);
      if (old == WG_EMPTY_KEY) { atomicAdd(s_groups, 1); return s; }
      if (old == k0) return s;
    }
    h = (h + 1 == (uint32_t)S) ? 0u : h + 1;
  }
  return nullptr;
}

// Shared-table lookups for rows already bucketed by the top `shift` bits of
// their key hash: the slot comes from the hash bits below those (the top bits
// are the same for every row of a bucket). One-word keys hash like fib_slot,
// packed keys like packed_slot; a packed key is installed with one 16-byte CAS
// (its words change once, from {~0, ~0} to the key, as in find_global).
__device__ __forceinline__ unsigned long long* find_smem_bucketed(unsigned long long* sm, int S, int sw, int kw,
                                                                  unsigned long long k0, unsigned long long k1,
                                                                  int shift, int* s_groups, int s_limit,
                                                                  uint32_t* list) {
  unsigned long long h;
  if (kw == 1) {
    if (k0 == WG_EMPTY_KEY) return nullptr;
    h = k0 * 0x9E3779B97F4A7C15ULL;
  } else {
    if (k0 == ~0ULL && k1 == ~0ULL) return nullptr;
    const unsigned long long a = k0 ^ 0x9E3779B97F4A7C15ULL, b = k1 ^ 0x517CC1B727220A95ULL;
    h = (__umul64hi(a, b) ^ (a * b) ^ (k0 + k1)) * 0x9E3779B97F4A7C15ULL;
  }
  uint32_t i = (uint32_t)__umul64hi(shift > 0 ? h << shift : h, (unsigned long long)S);
  for (int p = 0; p < S; ++p) {
    unsigned long long* s = sm + (size_t)i * sw;
    if (kw == 1) {
      const unsigned long long cur = *((volatile unsigned long long*)s);
      if (cur == k0) return s;
      if (cur == WG_EMPTY_KEY) {
        if (*((volatile int*)s_groups) >= s_limit) return nullptr;
        const unsigned long long old = atomicCAS(s, WG_EMPTY_KEY, k0);
        if (old == WG_EMPTY_KEY) {
          const int g = atomicAdd(s_groups, 1);
          if (list) list[g] = i;
          return s;
        }
        if (old == k0) return s;
      }
    } else {
      const U128 cur = read128(s);
      if (cur.lo != ~0ULL && cur.hi != ~0ULL) {  // a complete key (as in find_global)
        if (cur.lo == k0 && cur.hi == k1) return s;
      } else {
        if (*((volatile int*)s_groups) >= s_limit) return nullptr;
        U128 e; e.lo = ~0ULL; e.hi = ~0ULL;
        U128 k; k.lo = k0; k.hi = k1;
        const U128 old = cas128((U128*)s, e, k);
        if (old.lo == e.lo && old.hi == e.hi) {
          const int g = atomicAdd(s_groups, 1);
          if (list) list[g] = i;
          return s;
        }
        if (old.lo == k0 && old.hi == k1) return s;
      }
    }
    i = (i + 1 == (uint32_t)S) ? 0u : i + 1;
  }
  return nullptr;
}

// The shared slot of a key: direct (k0 - gmin) when the keys' range is known
// and fits the table, the bucketed table for rows of one hash bucket, else the
// hashed one-word table.
__device__ __forceinline__ unsigned long long* find_shared(const Plan& P, unsigned long long* sm, unsigned long long k0,
                                                           unsigned long long k1, int* s_groups, int s_limit) {
  if (P.gdense) {
    // every key lies in [gmin, gmin + smem_slots), fewer than 2^14 apart: the
    // low 32 bits give the exact offset
    const uint32_t d = (uint32_t)k0 - (uint32_t)P.gmin;
    return d < (uint32_t)P.smem_slots ? sm + d * (uint32_t)smem_stride(P) : nullptr;
  }
  if (P.smem_hash_shift > 0)
    return find_smem_bucketed(sm, P.smem_slots, smem_stride(P), P.L.key_words, k0, k1, P.smem_hash_shift, s_groups,
                              s_limit, P.smem_list > 0 ? (uint32_t*)(sm + P.smem_list) : nullptr);
  return find_smem(sm, P.smem_slots, smem_stride(P), k0, s_groups, s_limit);
}

// Update of one row per lane. Rows bound for the HBM table (no shared table, a
// NULL key, or a shared table at its fill limit) are combined first: lanes
// holding the same key pre-combine their contributions (__match_any_sync) and
// only the group's lowest lane touches the table, so a hot key costs one set
// of global atomics per warp instead of one per row. With a CTA-private
// shared-memory table each lane applies its own row there with shared-memory
// atomics, or, when P.smem_combine is set, the lanes combine first there too
// (fewer atomics on a hot group's words at the price of the shuffles).
template <int NA, bool SMEM, class Sh>
__device__ __forceinline__ void warp_update(const Plan& P, const Sh& sh, bool cur, unsigned long long k0,
                                            unsigned long long k1, bool knull, Contrib<NA>& c,
                                            unsigned long long* sm, int* s_groups, int s_limit, Credit& cr) {
  const bool combine_first = SMEM && P.smem_combine != 0;
  if (SMEM && !combine_first && cur && !knull) {
    unsigned long long* s = find_shared(P, sm, k0, k1, s_groups, s_limit);
    if (s != nullptr) {
      apply<NA, true>(sh, s, c, 1ULL, smem_copies(P));
      cur = false;
    }
  }
  const unsigned am = __ballot_sync(WG_FULL_MASK, cur);
  if (am == 0) return;
  const int lane = threadIdx.x & 31;
  unsigned peers = __match_any_sync(WG_FULL_MASK, k0);
  if (sh.key_words() == 2) peers &= __match_any_sync(WG_FULL_MASK, k1);
  peers &= __match_any_sync(WG_FULL_MASK, knull ? 1u : 0u);
  peers &= am;
  const int mysz = cur ? __popc(peers) : 0;
  const bool leader = cur && (__ffs(peers) - 1) == lane;
  const int maxsz = (int)__reduce_max_sync(WG_FULL_MASK, (unsigned)mysz);
  for (int i = 1; i < maxsz; ++i) {
    const bool take = leader && i < mysz;
    const int src = take ? (int)__fns(peers, 0, i + 1) : lane;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      if (a >= sh.n_aggs()) continue;
      const int kind = sh.agg_kind(a);
      const int kw = kind_words(kind);
      unsigned long long b0 = 0, b1 = 0;
      int bn = 0;
      if (kw >= 1) b0 = __shfl_sync(WG_FULL_MASK, c.w0[a], src);
      if (kw == 2) b1 = __shfl_sync(WG_FULL_MASK, c.w1[a], src);
      if (sh.agg_null_off(a) >= 0) bn = __shfl_sync(WG_FULL_MASK, c.nul[a], src);
      if (take) {
        combine(kind, c.w0[a], c.w1[a], b0, b1);
        c.nul[a] += bn;
      }
    }
  }
  if (leader) {
    if (combine_first && !knull) {
      unsigned long long* s = find_shared(P, sm, k0, k1, s_groups, s_limit);
      if (s != nullptr) {
        apply<NA, true>(sh, s, c, (unsigned long long)mysz, smem_copies(P));
        return;
      }
    }
    unsigned long long* s = find_global(sh, P.T, k0, k1, knull, P.err, &cr);
    if (s != nullptr) apply<NA, false>(sh, s, c, (unsigned long long)mysz, 1, P.minmax_test != 0);
  }
}

// Group key of one (row, build row): the int-key path widens to int64
// (consumeBatchIntGroup, aggregate.go:1908); the packed path places each column
// by buildPackedLayout (packed_hash.go:386) as packedKeyAt does (:456).
template <class Sh, class Src>
__device__ __forceinline__ bool make_key(const Plan& P, const Sh& sh, const Src& src, int32_t brow,
                                         const ExprVals& ev, unsigned long long& k0, unsigned long long& k1,
                                         bool& knull) {
  k0 = 0; k1 = 0; knull = false;
  if (sh.key_words() == 0) return true;
  if (sh.key_words() == 1) {
    Val v = fetch(P, sh, src, sh.key_vcol(0), brow, ev);
    knull = v.null;
    k0 = v.null ? 0 : v.lo;
    return true;
  }
#pragma unroll
  for (int k = 0; k < WG_MAX_KEYS; ++k) {
    if (k >= sh.n_keys()) break;
    Val v = fetch(P, sh, src, sh.key_vcol(k), brow, ev);
    if (v.null) {
      // a NULL composite-key column is its own value (the generic path's NULL,
      // aggregate.go:1822-1840): its bit in the NULL field, value bits 0
      if (P.L.null_word < 0) { set_error(P.err, WG_DERR_NULL_PACKED); return false; }
      const unsigned long long m = 1ULL << (P.L.null_shift + k);
      if (P.L.null_word == 0) k0 |= m; else k1 |= m;
      continue;
    }
    const unsigned long long w =
        sh.key_i32(k) ? ((unsigned long long)(uint32_t)(int32_t)v.lo) << sh.key_shift(k) : v.lo;
    if (sh.key_word(k) == 0) k0 |= w; else k1 |= w;
  }
  return true;
}

// `col OP const` on an already loaded value (compareFilterImpl, compare.go:47).
template <class Sh>
__device__ __forceinline__ bool pred_val(const Plan& P, const Sh& sh, int f, const Val& v) {
  if (v.null) return false;
  const int op = sh.filt_op(f);
  switch (sh.filt_cls(f)) {
    case WG_CLS_I32: return cmp_op<int32_t>((int32_t)(long long)v.lo, (int32_t)P.filt[f].ci, op);
    case WG_CLS_I64: return cmp_op<long long>((long long)v.lo, P.filt[f].ci, op);
    case WG_CLS_F32: return cmp_op<double>(as_f(v.lo), (double)(float)P.filt[f].cf, op);  // both exact in binary64
    case WG_CLS_F64: return cmp_op<double>(as_f(v.lo), P.filt[f].cf, op);
    default: return false;
  }
}

// One row per lane of a warp: KernelFilter chain → HashJoinProbe → Project →
// HashAggregate.Consume. All 32 lanes call it together (act = row present).
template <int NA, bool SMEM, class Sh, class Src>
__device__ __forceinline__ void process_rows(const Plan& P, const Sh& sh, const Src& src, bool act,
                                             unsigned long long* sm, int* s_groups, int s_limit, Credit& cr) {
#pragma unroll
  for (int f = 0; f < WG_MAX_FILTERS; ++f) {
    if (f >= sh.n_filters()) break;
    if (act) act = pred_val(P, sh, f, src.in(P, sh, sh.filt_col(f)));
  }
  int32_t brow = -1;
  // exec.JoinType: inner and left walk the chain; semi and anti only test it
  const int jt = sh.has_join() ? (sh.direct() ? WG_JOIN_INNER : P.join.jtype) : WG_JOIN_INNER;
  if (sh.has_join() && act) {
    const Val kv = src.in(P, sh, sh.probe_col());
    if (!join_pass_mine(P.join, kv.null, (long long)kv.lo)) act = false;  // another pass's row
  }
  if (sh.has_join() && act) {
    const Val kv = src.in(P, sh, sh.probe_col());
    bool found = false;
    if (kv.null) found = false;  // NULL keys never match (join.go:2700)
    else if (sh.direct()) found = join_direct(P.join, (int64_t)kv.lo, brow, P.err);
    else {
      brow = join_head(P.join, (int64_t)kv.lo, P.err);
      found = brow >= 0;
    }
    if (jt == WG_JOIN_INNER) act = found;
    else if (jt == WG_JOIN_LEFT) { if (!found) brow = -1; }     // kept; NULL build columns
    else { act = jt == WG_JOIN_SEMI ? found : !found; brow = -1; }  // executeSemiAntiJoin (join.go:3247)
  }
  for (;;) {
    if (!__any_sync(WG_FULL_MASK, act)) break;
    unsigned long long k0 = 0, k1 = 0;
    bool knull = false;
    Contrib<NA> c;
    bool cur = act;
    if (cur) {
      ExprVals ev;
      eval_exprs(P, sh, src, brow, ev);
      cur = make_key(P, sh, src, brow, ev, k0, k1, knull);
      make_contrib<NA>(P, sh, src, brow, ev, c);
    } else {
#pragma unroll
      for (int a = 0; a < NA; ++a) { c.w0[a] = 0; c.w1[a] = 0; c.nul[a] = 0; }
    }
    warp_update<NA, SMEM>(P, sh, cur, k0, k1, knull, c, sm, s_groups, s_limit, cr);
    if (!sh.has_join() || sh.direct()) break;  // unique keys: at most one match
    if (act) {
      if (brow < 0) act = false;                // semi, anti, or an unmatched left row: emitted once
      else {
        brow = __ldg(P.join.next + brow);       // arenaNext chain (join.go:2700)
        act = brow >= 0;
      }
    }
  }
}

// Shared slot of P.smem_sw words: the layout's slot words (empty pattern),
// then the extra float-SUM copies (+0.0).
__device__ __forceinline__ void smem_table_init(const Plan& P, unsigned long long* sm, int S, int* s_groups) {
  const int sw = P.L.slot_words, ssw = smem_stride(P);
  for (int i = threadIdx.x; i < S * ssw; i += blockDim.x) {
    const int w = i % ssw;
    sm[i] = w < sw ? P.L.init[w] : 0ULL;
  }
  if (threadIdx.x == 0) *s_groups = 0;
}

template <int NA>
__device__ __forceinline__ void smem_table_flush(const Plan& P, const unsigned long long* sm, int S, Credit& cr) {
  const LayoutAcc ly{P.L};
  const int sw = P.L.slot_words, ssw = smem_stride(P), rep = smem_copies(P);
  // CTAs start their pass at different slots: CTAs that finish together then
  // insert and update different groups at any moment instead of racing on the
  // same new keys, the same reservation counter and the same state words
  const int off = (int)(((long long)blockIdx.x * S) / max(1, (int)gridDim.x));
  for (int i0 = threadIdx.x; i0 < S; i0 += blockDim.x) {
    const int i = i0 + off < S ? i0 + off : i0 + off - S;
    const unsigned long long* s = sm + (size_t)i * ssw;
    unsigned long long key = s[0];
    if (P.gdense) {  // a direct slot is in use once it counted a row
      if (s[P.L.key_words] == 0) continue;
      key = (unsigned long long)P.gmin + (unsigned long long)i;
    } else if (key == WG_EMPTY_KEY) {
      continue;
    }
    unsigned long long* g = find_global(ly, P.T, key, 0, false, P.err, &cr);
    if (g == nullptr) continue;
    Contrib<NA> c;
    slot_contrib<NA>(ly, s, c);
    int nf = 0;
#pragma unroll
    for (int a = 0; a < NA; ++a) {
      if (a >= P.L.n_aggs || P.L.agg[a].kind != K_SUM_F64) continue;
      double d = as_f(c.w0[a]);
      if (rep < 0) d = __dadd_rn(fixed_to_f64(s[sw + 2 * nf], s[sw + 2 * nf + 1]), d);
      for (int r = 1; r < rep; ++r) d = __dadd_rn(d, as_f(s[sw + nf * (rep - 1) + (r - 1)]));
      c.w0[a] = as_w(d);
      ++nf;
    }
    apply<NA, false>(ly, g, c, s[P.L.key_words]);
  }
}

// One lane's share of the L2 prefetch of a grid-stride loop over chunks of
// ROWS rows: the lane's 128-byte line of one column, fixed for the whole loop
// (set up once, then one compare, one add and one prefetch per iteration).
template <int ROWS>
struct Prefetcher {
  const char* p = nullptr;   // next line to prefetch (nullptr: this lane has none)
  const char* end = nullptr;
  int64_t step = 0;          // bytes between this lane's lines in consecutive iterations
  template <class Sh>
  __device__ __forceinline__ void init(const Plan& P, const Sh& sh, int64_t first_row, int64_t rows_per_iter,
                                       int lane) {
    int first = 0;
#pragma unroll
    for (int j = 0; j < WG_MAX_IN; ++j) {
      if (j >= sh.n_in()) break;
      const int es = cls_bytes(sh.in_cls(j));
      const int lines = ROWS * es / 128;
      if (lane >= first && lane < first + lines) {
        p = (const char*)P.in[j].data + first_row * es + (int64_t)(lane - first) * 128;
        end = (const char*)P.in[j].data + P.n_items * es;
        step = rows_per_iter * es;
      }
      first += lines;
    }
  }
  __device__ __forceinline__ void next() {
    if (p != nullptr && p < end) asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
    p += step;
  }
};

// The fused pipeline reading HBM directly: one warp per 32 consecutive rows
// (or selection-vector entries), grid-stride.
template <int NA, bool SMEM, class Sh>
__global__ void __launch_bounds__(Sh::kBlock, Sh::kMinBlocks) pipeline_kernel(const __grid_constant__ Plan P) {
  extern __shared__ unsigned long long sm[];
  __shared__ int s_groups;
  const Sh sh{P};
  Credit cr;  // this thread's group reservations, handed back at the end
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  if (SMEM) {
    smem_table_init(P, sm, S, &s_groups);
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  const int64_t total_warps = (int64_t)gridDim.x * wpb;
  const int64_t ahead = (int64_t)P.prefetch * total_warps * 32;
  const int64_t base0 = ((int64_t)blockIdx.x * wpb + (threadIdx.x >> 5)) * 32;
  Prefetcher<32> pf;
  if (ahead > 0 && P.sel == nullptr) pf.init(P, sh, base0 + ahead, total_warps * 32, lane);
  for (int64_t base = base0; base < P.n_items; base += total_warps * 32) {
    pf.next();
    const int64_t item = base + lane;
    const bool act = item < P.n_items;
    SrcGlobal src{act ? (P.sel ? (int64_t)__ldg(P.sel + item) : item) : 0};
    process_rows<NA, SMEM>(P, sh, src, act, sm, &s_groups, s_limit, cr);
  }
  if (SMEM) {
    __syncthreads();
    smem_table_flush<NA>(P, sm, S, cr);
  }
  cr.release(P.T);
}

// ---------------------------------------------------------------------------
// Hash partitioning of the input for large tables. The table's slot is the top
// bits of a 64-bit key hash, so rows grouped by the top `pbits` bits of that
// hash touch one 1/2^pbits region of the table. Rows reordered that way and
// fed in order keep the aggregate's working set to an L2-sized region at any
// time. The order is a pure permutation of the input: every row is kept
// (filters still run in the aggregation pass) and NULL keys go to region 0.
// ---------------------------------------------------------------------------
// The partition is bits [pshift, pshift + pbits) of the 64-bit key hash: the
// top bits (pshift = 64 - pbits) for the in-HBM reorder, whose table regions
// they select; bits below any table's slot bits for the spill, whose
// per-partition table must spread a partition's keys over all its slots.
template <class Sh>
__device__ __forceinline__ uint32_t row_partition(const Plan& P, const Sh& sh, int64_t row, int pbits, int pshift) {
  const SrcGlobal src{row};
  ExprVals ev;
  eval_exprs(P, sh, src, -1, ev);
  const uint32_t mask = (1u << pbits) - 1u;
  if (sh.key_words() == 1) {
    const Val v = fetch(P, sh, src, sh.key_vcol(0), -1, ev);
    return v.null ? 0u : (uint32_t)(fib_slot(v.lo, 0) >> pshift) & mask;
  }
  unsigned long long k0 = 0, k1 = 0;
#pragma unroll
  for (int k = 0; k < WG_MAX_KEYS; ++k) {
    if (k >= sh.n_keys()) break;
    const Val v = fetch(P, sh, src, sh.key_vcol(k), -1, ev);
    if (v.null) return 0u;
    const unsigned long long w =
        sh.key_i32(k) ? ((unsigned long long)(uint32_t)(int32_t)v.lo) << sh.key_shift(k) : v.lo;
    if (sh.key_word(k) == 0) k0 |= w; else k1 |= w;
  }
  return (uint32_t)(packed_slot(k0, k1, 0) >> pshift) & mask;
}

// Both partition kernels walk the input in tiles of kPartTile rows, CTA c
// taking tiles c, c + gridDim.x, ...; so the rows a CTA counts per partition
// are exactly the rows it later scatters there.
constexpr int kPartThreads = 512;
constexpr int kPartTile = 16384;
static_assert(kPartTile <= 65536, "tile-local row indices are 16-bit");
__host__ __device__ constexpr size_t part_count_smem(int np) { return (size_t)np * 4; }
__host__ __device__ constexpr size_t part_scatter_smem(int np) {
  return (size_t)np * 8 + (size_t)np * 12 + (size_t)kPartTile * 4;
}

// Rows per partition seen by each CTA (counts[p * gridDim.x + cta]).
static __global__ void __launch_bounds__(kPartThreads) part_count_kernel(const __grid_constant__ Plan P, int pbits,
                                                                         int pshift, uint32_t* counts) {
  extern __shared__ uint32_t hist[];
  const int np = 1 << pbits;
  for (int i = threadIdx.x; i < np; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  const DynShape sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * kPartTile; t0 < P.n_items; t0 += (int64_t)gridDim.x * kPartTile) {
    const int m = (int)min((int64_t)kPartTile, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) atomicAdd(&hist[row_partition(P, sh, t0 + k, pbits, pshift)], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < np; i += blockDim.x) counts[(size_t)i * gridDim.x + blockIdx.x] = hist[i];
}

// Output columns of the reordered copy (one per input column of the plan).
struct PartOut {
  char* data[WG_MAX_IN];
  int32_t es[WG_MAX_IN];
  // side columns moved with the rows (4 bytes each, e.g. one validity flag per
  // row of a nullable input): side_src[k] + row, in the rows' order
  const int32_t* side_src[WG_MAX_IN];
  int32_t* side_dst[WG_MAX_IN];
  int32_t n_side;
};

// Exclusive prefix sums of v[0..n) in place (n <= 2 * blockDim.x, blockDim.x a
// multiple of 32, at most 32 warps); every thread of the CTA calls it.
__device__ __forceinline__ void block_exclusive_scan(uint32_t* v, int n, uint32_t* warp_tot) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5, nw = blockDim.x >> 5;
  const uint32_t a = 2 * t < n ? v[2 * t] : 0u, b = 2 * t + 1 < n ? v[2 * t + 1] : 0u;
  uint32_t x = a + b;  // inclusive scan of the pair sums within the warp
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(WG_FULL_MASK, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_tot[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t z = lane < nw ? warp_tot[lane] : 0u;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(WG_FULL_MASK, z, o);
      if (lane >= o) z += y;
    }
    if (lane < nw) warp_tot[lane] = z;  // inclusive warp totals
  }
  __syncthreads();
  const uint32_t before = (w > 0 ? warp_tot[w - 1] : 0u) + x - (a + b);
  if (2 * t < n) v[2 * t] = before;
  if (2 * t + 1 < n) v[2 * t + 1] = before + a;
  __syncthreads();
}

// Same tiles as part_count_kernel: CTA c writes its rows of partition p from
// offs[p * gridDim.x + c] on. Per tile, the rows are counting-sorted by
// partition in shared memory (tile-local row indices), then written column by
// column in that order, so consecutive threads store consecutive rows of one
// partition instead of one row each to scattered partitions.
static __global__ void __launch_bounds__(kPartThreads) part_scatter_kernel(const __grid_constant__ Plan P, int pbits,
                                                                           int pshift,
                                                                           const unsigned long long* offs,
                                                                           PartOut out) {
  extern __shared__ unsigned long long gcur[];  // np output cursors, then the arrays below
  __shared__ uint32_t warp_tot[32];
  const int np = 1 << pbits;
  uint32_t* hist = (uint32_t*)(gcur + np);      // rows of partition p in this tile
  uint32_t* loff = hist + np;                   // their first position in the tile order
  uint32_t* lcur = loff + np;
  uint16_t* part = (uint16_t*)(lcur + np);      // partition of tile row k
  uint16_t* perm = part + kPartTile;            // tile row at position k of the order
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    gcur[i] = offs[(size_t)i * gridDim.x + blockIdx.x];
    hist[i] = 0;
  }
  __syncthreads();
  const DynShape sh{P};
  for (int64_t t0 = (int64_t)blockIdx.x * kPartTile; t0 < P.n_items; t0 += (int64_t)gridDim.x * kPartTile) {
    const int m = (int)min((int64_t)kPartTile, P.n_items - t0);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t p = row_partition(P, sh, t0 + k, pbits, pshift);
      part[k] = (uint16_t)p;
      atomicAdd(&hist[p], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { loff[i] = hist[i]; lcur[i] = 0; }
    __syncthreads();
    block_exclusive_scan(loff, np, warp_tot);
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const uint32_t p = part[k];
      perm[loff[p] + atomicAdd(&lcur[p], 1u)] = (uint16_t)k;
    }
    __syncthreads();
    for (int j = 0; j < P.n_in; ++j) {
      const int es = out.es[j];
      const char* src = (const char*)P.in[j].data + t0 * es;
      char* dcol = out.data[j];
      for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int k = perm[q];
        const uint32_t p = part[k];
        char* d = dcol + (gcur[p] + (q - loff[p])) * es;
        if (es == 4) *(uint32_t*)d = __ldg((const uint32_t*)(src + (size_t)k * 4));
        else if (es == 8) *(unsigned long long*)d = __ldg((const unsigned long long*)(src + (size_t)k * 8));
        else *(longlong2*)d = __ldg((const longlong2*)(src + (size_t)k * 16));
      }
    }
    for (int j = 0; j < out.n_side; ++j) {
      const int32_t* src = out.side_src[j] + t0;
      for (int q = threadIdx.x; q < m; q += blockDim.x) {
        const int k = perm[q];
        const uint32_t p = part[k];
        out.side_dst[j][gcur[p] + (q - loff[p])] = __ldg(src + k);
      }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < np; i += blockDim.x) { gcur[i] += hist[i]; hist[i] = 0; }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Vector variant for compiled shapes: each lane takes U consecutive rows, loads
// each column's U values with 16-byte (or 8-byte) loads, evaluates all U
// filters and issues all U join lookups before the first aggregate update, so
// a warp keeps U times the bytes and lookups in flight of the one-row form.
// ---------------------------------------------------------------------------

// The input values of one row, held in registers.
struct SrcRow {
  Val v[WG_MAX_IN];
  template <class Sh>
  __device__ __forceinline__ Val in(const Plan&, const Sh&, int j) const { return v[j]; }
};

// Rows r0 .. r0+U-1 (r0 a multiple of U, column starts 16-byte aligned): one
// vector load per 16 bytes when all U rows exist, row by row at the end.
template <int U, class Sh>
__device__ __forceinline__ void load_rows(const Plan& P, const Sh& sh, int64_t r0, SrcRow (&rw)[U], int64_t n_end = -1) {
  const int64_t n = n_end >= 0 ? n_end : P.n_items;  // rows past n are absent
  const bool full = r0 + U <= n;
#pragma unroll
  for (int j = 0; j < WG_MAX_IN; ++j) {
    if (j >= sh.n_in()) break;
    const int cls = sh.in_cls(j);
    const int es = cls_bytes(cls);
    if (full) {
      const char* p = (const char*)P.in[j].data + r0 * es;
      unsigned long long w[2 * U];  // U*es bytes as 64-bit words (es <= 16)
      const int nbytes = U * es;
      if (nbytes == 4) {
        w[0] = (unsigned long long)(uint32_t)__ldcs((const int32_t*)p);
      } else if (nbytes == 8) {
        w[0] = (unsigned long long)__ldcs((const long long*)p);
      } else {
#pragma unroll
        for (int q = 0; q < 2 * U; q += 2) {
          if (q * 8 >= nbytes) break;
          const longlong2 d = __ldcs((const longlong2*)p + q / 2);
          w[q] = (unsigned long long)d.x;
          w[q + 1] = (unsigned long long)d.y;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        Val& v = rw[u].v[j];
        v.hi = 0;
        if (cls == WG_CLS_I32 || cls == WG_CLS_F32) {
          const uint32_t b = (uint32_t)(w[u >> 1] >> ((u & 1) * 32));
          v.lo = cls == WG_CLS_I32 ? (unsigned long long)(long long)(int32_t)b : as_w((double)__uint_as_float(b));
        } else if (cls == WG_CLS_DEC) {
          v.hi = w[2 * u];      // {int64 hi; uint64 lo}
          v.lo = w[2 * u + 1];
        } else {
          v.lo = w[u];
        }
        v.null = sh.nullable() && is_null(P.in[j], r0 + u);
      }
    } else {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int64_t row = r0 + u;
        if (row < n) {
          rw[u].v[j] = load_stream(P.in[j].data, cls, row);
          rw[u].v[j].null = sh.nullable() && is_null(P.in[j], row);
        } else {
          rw[u].v[j].lo = 0; rw[u].v[j].hi = 0; rw[u].v[j].null = true;
        }
      }
    }
  }
}

// Byte offset of input column j inside a staged chunk of CH rows (the columns
// one after another, each CH values long), and the chunk's size.
template <int CH, class Sh>
__device__ __forceinline__ constexpr int stage_col_off(const Sh& sh, int j) {
  int off = 0;
  for (int i = 0; i < WG_MAX_IN; ++i) {
    if (i >= j || i >= sh.n_in()) break;
    off += CH * cls_bytes(sh.in_cls(i));
  }
  return off;
}

// Rows l .. l+U-1 of a chunk staged in shared memory (all present).
template <int U, class Sh>
__device__ __forceinline__ void load_rows_staged(const Sh& sh, const unsigned char* stg, int l, SrcRow (&rw)[U]) {
#pragma unroll
  for (int j = 0; j < WG_MAX_IN; ++j) {
    if (j >= sh.n_in()) break;
    const int cls = sh.in_cls(j);
    const int es = cls_bytes(cls);
    const unsigned char* p = stg + stage_col_off<32 * U>(sh, j) + l * es;
    unsigned long long w[2 * U];
    const int nbytes = U * es;
    if (nbytes == 4) {
      w[0] = *(const uint32_t*)p;
    } else if (nbytes == 8) {
      w[0] = *(const unsigned long long*)p;
    } else {
#pragma unroll
      for (int q = 0; q < 2 * U; q += 2) {
        if (q * 8 >= nbytes) break;
        const ulonglong2 d = *((const ulonglong2*)p + q / 2);
        w[q] = d.x;
        w[q + 1] = d.y;
      }
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      Val& v = rw[u].v[j];
      v.hi = 0;
      v.null = false;
      if (cls == WG_CLS_I32 || cls == WG_CLS_F32) {
        const uint32_t b = (uint32_t)(w[u >> 1] >> ((u & 1) * 32));
        v.lo = cls == WG_CLS_I32 ? (unsigned long long)(long long)(int32_t)b : as_w((double)__uint_as_float(b));
      } else if (cls == WG_CLS_DEC) {
        v.hi = w[2 * u];      // {int64 hi; uint64 lo}
        v.lo = w[2 * u + 1];
      } else {
        v.lo = w[u];
      }
    }
  }
}

// U rows per lane (no join, or the direct-payload join) already loaded:
// filters and lookups for all rows first, then one warp-wide update per row.
template <int NA, bool SMEM, int U, class Sh>
__device__ __forceinline__ void process_loaded_vec(const Plan& P, const Sh& sh, int64_t r0, SrcRow (&rw)[U],
                                                   unsigned long long* sm, int* s_groups, int s_limit, Credit& cr,
                                                   int64_t n_end = -1) {
  bool act[U];
  int32_t brow[U];
  const int64_t n = n_end >= 0 ? n_end : P.n_items;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    act[u] = r0 + u < n;
    brow[u] = -1;
#pragma unroll
    for (int f = 0; f < WG_MAX_FILTERS; ++f) {
      if (f >= sh.n_filters()) break;
      if (act[u]) act[u] = pred_val(P, sh, f, rw[u].v[sh.filt_col(f)]);
    }
  }
  if (sh.has_join()) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const Val kv = rw[u].v[sh.probe_col()];
      if (act[u] && !join_pass_mine(P.join, kv.null, (long long)kv.lo)) act[u] = false;  // another pass's row
      if (act[u]) {
        if (sh.in_cls(sh.probe_col()) == WG_CLS_I32)
          act[u] = !kv.null && join_direct_i32(P.join, (int32_t)kv.lo, brow[u], P.err);
        else
          act[u] = !kv.null && join_direct(P.join, (int64_t)kv.lo, brow[u], P.err);
      }
    }
  }
  if (!Sh::kRowsTogether) {
#pragma unroll
    for (int u = 0; u < U; ++u) {
      if (!__any_sync(WG_FULL_MASK, act[u])) continue;
      unsigned long long k0 = 0, k1 = 0;
      bool knull = false;
      Contrib<NA> c;
      bool cur = act[u];
      if (cur) {
        ExprVals ev;
        eval_exprs(P, sh, rw[u], brow[u], ev);
        cur = make_key(P, sh, rw[u], brow[u], ev, k0, k1, knull);
        make_contrib<NA>(P, sh, rw[u], brow[u], ev, c);
      } else {
#pragma unroll
        for (int a = 0; a < NA; ++a) { c.w0[a] = 0; c.w1[a] = 0; c.nul[a] = 0; }
      }
      warp_update<NA, SMEM>(P, sh, cur, k0, k1, knull, c, sm, s_groups, s_limit, cr);
    }
    return;
  }
  // every row's key and contribution first (independent dependency chains
  // the scheduler can interleave), then the table updates
  unsigned long long k0[U], k1[U];
  bool knull[U];
  Contrib<NA> c[U];
#pragma unroll
  for (int u = 0; u < U; ++u) {
    k0[u] = 0; k1[u] = 0; knull[u] = false;
    if (act[u]) {
      ExprVals ev;
      eval_exprs(P, sh, rw[u], brow[u], ev);
      act[u] = make_key(P, sh, rw[u], brow[u], ev, k0[u], k1[u], knull[u]);
      make_contrib<NA>(P, sh, rw[u], brow[u], ev, c[u]);
    } else {
#pragma unroll
      for (int a = 0; a < NA; ++a) { c[u].w0[a] = 0; c[u].w1[a] = 0; c[u].nul[a] = 0; }
    }
  }
#pragma unroll
  for (int u = 0; u < U; ++u) {
    if (!__any_sync(WG_FULL_MASK, act[u])) continue;
    warp_update<NA, SMEM>(P, sh, act[u], k0[u], k1[u], knull[u], c[u], sm, s_groups, s_limit, cr);
  }
}

template <int NA, bool SMEM, int U, class Sh>
__device__ __forceinline__ void process_rows_vec(const Plan& P, const Sh& sh, int64_t r0, unsigned long long* sm,
                                                 int* s_groups, int s_limit, Credit& cr) {
  SrcRow rw[U];
  load_rows<U>(P, sh, r0, rw);
  process_loaded_vec<NA, SMEM, U>(P, sh, r0, rw, sm, s_groups, s_limit, cr);
}

// Grid-stride over chunks of 32*U rows; MB CTAs of BLK threads per SM.
template <int NA, bool SMEM, class Sh, int U, int MB, int BLK>
__global__ void __launch_bounds__(BLK, MB) pipeline_vec_kernel(const __grid_constant__ Plan P) {
  static_assert(U == 2 || U == 4, "rows per lane");
  extern __shared__ unsigned long long sm[];
  __shared__ int s_groups;
  const Sh sh{P};
  Credit cr;  // this thread's group reservations, handed back at the end
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  if (SMEM) {
    smem_table_init(P, sm, S, &s_groups);
    __syncthreads();
  }
  const int lane = threadIdx.x & 31;
  const int64_t wpb = blockDim.x >> 5;
  const int64_t step = (int64_t)gridDim.x * wpb * 32 * U;
  const int64_t ahead = (int64_t)P.prefetch * step;
  const int64_t base0 = ((int64_t)blockIdx.x * wpb + (threadIdx.x >> 5)) * 32 * U;
  // the 768-thread variant (48 warps per SM) hides HBM latency with warps and
  // leaves the prefetcher's registers to the rows (40 per thread)
  constexpr bool kPrefetch = BLK != 768;
  Prefetcher<32 * U> pf;
  if (kPrefetch && ahead > 0) pf.init(P, sh, base0 + ahead, step, lane);
  for (int64_t base = base0; base < P.n_items; base += step) {
    if (kPrefetch) pf.next();
    process_rows_vec<NA, SMEM, U>(P, sh, base + (int64_t)lane * U, sm, &s_groups, s_limit, cr);
  }
  if (SMEM) {
    __syncthreads();
    smem_table_flush<NA>(P, sm, S, cr);
  }
  cr.release(P.T);
}

// Self-staged vector kernel: one CTA of 1024 threads per SM with a shared
// table. Each warp copies its next chunk of 32*U rows (every input column, one
// bulk asynchronous copy per column, completing on the warp's own mbarrier)
// into one half of its shared-memory double buffer while it evaluates the
// current chunk out of the other half, so the warp's HBM reads for the next
// chunk are in flight during the current chunk's lookups and table updates.
// A warp's last chunk, when it is cut short by the end of the input, is read
// from HBM directly. Every wait is bounded (wg_tma.cuh); a timeout records
// WG_DERR_TIMEOUT, and the warp stops after waiting (bounded) for the copy it
// still has in flight.
template <int NA, class Sh, int U>
__global__ void __launch_bounds__(1024, 1) pipeline_stage_kernel(const __grid_constant__ Plan P) {
  extern __shared__ __align__(128) unsigned long long sm[];  // [shared table][staging]
  __shared__ int s_groups;
  __shared__ __align__(8) unsigned long long bars[64];      // two per warp
  constexpr int CH = 32 * U;
  const Sh sh{P};
  Credit cr;
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int cbytes = stage_col_off<CH>(sh, WG_MAX_IN);
  unsigned char* stg = (unsigned char*)sm + P.stage_off + (size_t)warp * 2 * cbytes;
  unsigned long long* bar = bars + 2 * warp;
  if (lane == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    mbar_init_fence();
  }
  smem_table_init(P, sm, S, &s_groups);
  __syncthreads();
  const int64_t wpb = blockDim.x >> 5;
  const int64_t step = (int64_t)gridDim.x * wpb * CH;
  const int64_t base0 = ((int64_t)blockIdx.x * wpb + warp) * CH;
  // chunk k of this warp (base0 + k * step) goes to stage k & 1 and completes
  // that stage's phase k >> 1
  auto issue = [&](int64_t k) {
    const int s = (int)(k & 1);
    const int64_t b = base0 + k * step;
    unsigned char* dst = stg + s * cbytes;
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // earlier reads of this half come first
    mbar_arrive_expect_tx(&bar[s], (uint32_t)cbytes);
#pragma unroll
    for (int j = 0; j < WG_MAX_IN; ++j) {
      if (j >= sh.n_in()) break;
      const int es = cls_bytes(sh.in_cls(j));
      bulk_g2s(dst + stage_col_off<CH>(sh, j), (const char*)P.in[j].data + b * es, (uint32_t)(CH * es), &bar[s]);
    }
  };
  // chunks [0, issued) have been started, chunks [0, landed) waited for
  int64_t issued = 0, landed = 0;
  if (base0 + CH <= P.n_items) {
    if (lane == 0) issue(0);
    issued = 1;
  }
  int64_t k = 0;
  for (int64_t base = base0; base < P.n_items; base += step, ++k) {
    const bool staged = base + CH <= P.n_items;
    if (base + step + CH <= P.n_items) {  // the next chunk is whole: start its copy now
      if (lane == 0) issue(k + 1);
      issued = k + 2;
    }
    SrcRow rw[U];
    const int64_t r0 = base + (int64_t)lane * U;
    if (staged) {
      const bool ok = __all_sync(WG_FULL_MASK, mbar_wait(&bar[k & 1], (uint32_t)((k >> 1) & 1), P.err));
      if (!ok) break;
      landed = k + 1;
      load_rows_staged<U>(sh, stg + (k & 1) * cbytes, lane * U, rw);
    } else {
      load_rows<U>(P, sh, r0, rw);
    }
    process_loaded_vec<NA, true, U>(P, sh, r0, rw, sm, &s_groups, s_limit, cr);
    __syncwarp();
  }
  // no copy outlives the CTA: after a timeout, wait (bounded) for what is in flight
  for (int64_t c = landed; c < issued; ++c) mbar_wait(&bar[c & 1], (uint32_t)((c >> 1) & 1), P.err);
  __syncthreads();
  smem_table_flush<NA>(P, sm, S, cr);
  cr.release(P.T);
}

// ---------------------------------------------------------------------------
// Tile-staged variant: a producer warp streams each tile's input columns into
// shared memory with bulk asynchronous copies (cp.async.bulk, completing on an
// mbarrier), STAGES tiles ahead; consumer warps evaluate the rows out of shared
// memory. HBM streaming then no longer waits on the probe's dependent loads.
// ---------------------------------------------------------------------------
struct TileCfg {
  int32_t rows;                // T: rows per tile (multiple of 64)
  int32_t stages;
  int32_t stage_bytes;
  int32_t consumers;           // consumer warps
  int32_t col_off[WG_MAX_IN];  // byte offset of column j inside a stage
  int32_t es[WG_MAX_IN];       // element size of column j
  int32_t table_off;           // byte offset of the shared-memory aggregate table
  int32_t _pad;
  int64_t n_tiles;
};

// Row i of the current tile: staged bytes come from shared memory, the ragged
// tail past the last whole 16-byte chunk from HBM.
struct SrcTile {
  const char* stage;
  int64_t row0;
  int32_t i;
  int32_t m;
  const TileCfg* C;
  template <class Sh>
  __device__ __forceinline__ Val in(const Plan& P, const Sh& sh, int j) const {
    const DCol& c = P.in[j];
    const int cls = sh.in_cls(j);
    const int es = cls_bytes(cls);
    const int staged = ((m * es) & ~15) / es;
    const int64_t row = row0 + i;
    const char* p = i < staged ? stage + C->col_off[j] + (size_t)i * es : (const char*)c.data + row * es;
    Val v = load_generic(p, cls);
    v.null = sh.nullable() && is_null(c, row);
    return v;
  }
};

template <int NA, bool SMEM, class Sh>
__global__ void __launch_bounds__(544, 1) tile_pipeline_kernel(const __grid_constant__ Plan P,
                                                               const __grid_constant__ TileCfg C) {
  extern __shared__ __align__(128) unsigned char tsm[];
  __shared__ int s_groups;
  __shared__ __align__(8) unsigned long long bars[16];  // full[0..7], empty[8..15]
  unsigned long long* full = bars;
  unsigned long long* empty = bars + 8;
  unsigned long long* table = (unsigned long long*)(tsm + C.table_off);
  const Sh sh{P};
  Credit cr;  // this thread's group reservations, handed back at the end
  const int S = P.smem_slots;
  const int s_limit = (S * 7) / 8;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C.stages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], C.consumers);
    }
    mbar_init_fence();
  }
  if (SMEM) smem_table_init(P, table, S, &s_groups);
  __syncthreads();

  if (warp == 0) {
    // producer: one lane issues every copy
    if (lane == 0) {
      int64_t it = 0;
      for (int64_t tile = blockIdx.x; tile < C.n_tiles; tile += gridDim.x, ++it) {
        const int s = (int)(it % C.stages);
        if (it >= C.stages && !mbar_wait(&empty[s], (uint32_t)(((it / C.stages) - 1) & 1), P.err)) break;
        const int64_t row0 = tile * C.rows;
        const int m = (int)min((int64_t)C.rows, P.n_items - row0);
        uint32_t total = 0;
        for (int j = 0; j < P.n_in; ++j) total += (uint32_t)((m * C.es[j]) & ~15);
        mbar_arrive_expect_tx(&full[s], total);
        unsigned char* st = tsm + (size_t)s * C.stage_bytes;
        for (int j = 0; j < P.n_in; ++j) {
          const uint32_t bytes = (uint32_t)((m * C.es[j]) & ~15);
          if (bytes) bulk_g2s(st + C.col_off[j], (const char*)P.in[j].data + row0 * C.es[j], bytes, &full[s]);
        }
      }
      // never leave with copies in flight: wait for the last issued tiles to land
      const int64_t issued = it;
      for (int64_t k = issued > C.stages ? issued - C.stages : 0; k < issued; ++k)
        mbar_wait(&full[k % C.stages], (uint32_t)((k / C.stages) & 1), P.err);
    }
  } else {
    const int cw = warp - 1;
    int64_t it = 0;
    for (int64_t tile = blockIdx.x; tile < C.n_tiles; tile += gridDim.x, ++it) {
      const int s = (int)(it % C.stages);
      if (!mbar_wait(&full[s], (uint32_t)((it / C.stages) & 1), P.err)) break;
      const int64_t row0 = tile * C.rows;
      const int m = (int)min((int64_t)C.rows, P.n_items - row0);
      const unsigned char* st = tsm + (size_t)s * C.stage_bytes;
      for (int base = cw * 32; base < m; base += C.consumers * 32) {
        const int i = base + lane;
        SrcTile src{(const char*)st, row0, i < m ? i : 0, m, &C};
        process_rows<NA, SMEM>(P, sh, src, i < m, table, &s_groups, s_limit, cr);
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(&empty[s]);
    }
  }
  __syncthreads();
  if (SMEM) smem_table_flush<NA>(P, table, S, cr);
  cr.release(P.T);
}

}  // namespace wgd
