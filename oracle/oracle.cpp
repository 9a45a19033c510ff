// oracle.cpp — TEST INFRASTRUCTURE ONLY: the CPU restatement of Wadjet's
// filter → hash-join → hash-aggregate semantics. It is the checker the GPU
// library is compared against and the CPU baseline timed beside it; the
// product never links or loads it. Parity of this restatement is pinned by the
// reference's own known-answer tests restated under tests/golden/.
//
// Built with -ffp-contract=off so binary64 expressions round exactly as Go
// evaluates them on amd64 (no fused multiply-add).

#include "oracle.h"
#include "../include/wadjet_synth.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

namespace {

thread_local std::string g_err;
int fail(const std::string& m) { g_err = m; return -1; }

// ---------------------------------------------------------------------------
// Int128 (internal/engine/batch/decimal.go:11-100)
// ---------------------------------------------------------------------------
struct I128 { int64_t hi; uint64_t lo; };

inline I128 i128_from(int64_t v) { return I128{v < 0 ? -1 : 0, (uint64_t)v}; }  // decimal.go:17

inline I128 i128_add(I128 d, I128 o) {  // decimal.go:78 (carry on lo < d.Lo)
  uint64_t lo = d.lo + o.lo;
  uint64_t hi = (uint64_t)d.hi + (uint64_t)o.hi;
  if (lo < d.lo) hi += 1;
  return I128{(int64_t)hi, lo};
}

inline bool i128_less(I128 a, I128 b) {  // decimal.go:93 (signed Hi, then unsigned Lo)
  if (a.hi != b.hi) return a.hi < b.hi;
  return a.lo < b.lo;
}

// math.Pow10 for the scales DECIMAL uses: pow10tab[n%32] * pow10postab32[n/32]
double pow10_go(int n) {
  static const double tab[32] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10,
                                 1e11, 1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21,
                                 1e22, 1e23, 1e24, 1e25, 1e26, 1e27, 1e28, 1e29, 1e30, 1e31};
  static const double post[4] = {1e0, 1e32, 1e64, 1e96};
  if (n < 0 || n >= 128) return n < 0 ? 1.0 / pow10_go(-n) : HUGE_VAL;
  return tab[n % 32] * post[n / 32];
}

inline double i128_to_f64(I128 d, int scale) {  // decimal.go:39-51
  if (d.hi == 0 && d.lo <= (uint64_t)INT64_MAX) return (double)(int64_t)d.lo / pow10_go(scale);
  if (d.hi == -1 && d.lo > (uint64_t)INT64_MAX) return (double)(int64_t)d.lo / pow10_go(scale);
  double f = (double)d.hi * 18446744073709551616.0 + (double)d.lo;
  return f / pow10_go(scale);
}

// ---------------------------------------------------------------------------
// Column access
// ---------------------------------------------------------------------------
enum Cls { C_I32, C_I64, C_F32, C_F64, C_DEC, C_BAD };

Cls cls_of(int t) {
  switch (t) {
    case WG_TYPE_INT32: case WG_TYPE_PORT: case WG_TYPE_PROTOCOL: case WG_TYPE_DATE: return C_I32;
    case WG_TYPE_INT64: case WG_TYPE_TIMESTAMP: case WG_TYPE_IPV4: case WG_TYPE_MAC:
    case WG_TYPE_DURATION: return C_I64;
    case WG_TYPE_FLOAT32: return C_F32;
    case WG_TYPE_FLOAT64: return C_F64;
    case WG_TYPE_DECIMAL: return C_DEC;
    default: return C_BAD;
  }
}
bool is_int_cls(int t) { Cls c = cls_of(t); return c == C_I32 || c == C_I64; }

inline bool is_null(const wg_column& c, int64_t i) {  // bitmap.go:84 (bit 0 = null)
  return c.valid_words && ((c.valid_words[i >> 6] >> (i & 63)) & 1ULL) == 0;
}
inline int64_t get_i64(const wg_column& c, int64_t i) {
  return cls_of(c.type_id) == C_I32 ? (int64_t)((const int32_t*)c.data)[i] : ((const int64_t*)c.data)[i];
}
inline double get_f64(const wg_column& c, int64_t i) {  // expr.ColRef.EvalFloat64, expr/expr.go:206
  switch (cls_of(c.type_id)) {
    case C_I32: return (double)((const int32_t*)c.data)[i];
    case C_I64: return (double)((const int64_t*)c.data)[i];
    case C_F32: return (double)((const float*)c.data)[i];
    case C_F64: return ((const double*)c.data)[i];
    case C_DEC: { const wg_int128 v = ((const wg_int128*)c.data)[i]; return i128_to_f64(I128{v.hi, v.lo}, c.scale); }
    default: return 0;
  }
}
inline I128 get_dec(const wg_column& c, int64_t i) {
  const wg_int128 v = ((const wg_int128*)c.data)[i];
  return I128{v.hi, v.lo};
}

// ---------------------------------------------------------------------------
// Filter constants (toInt64 / toFloat64 / toDateInt32, kernel/compare.go:580-640)
// ---------------------------------------------------------------------------
int64_t go_f64_to_i64(double f) {  // Go float64→int64 conversion on amd64 (CVTTSD2SQ)
  if (!(f >= -9223372036854775808.0 && f < 9223372036854775808.0)) return INT64_MIN;
  return (int64_t)f;
}
int64_t to_int64(const wg_predicate& p) { return p.const_kind == WG_CONST_FLOAT ? go_f64_to_i64(p.const_f64) : p.const_i64; }
double to_float64(const wg_predicate& p) { return p.const_kind == WG_CONST_FLOAT ? p.const_f64 : (double)p.const_i64; }

template <typename T>
inline bool cmp(T a, T b, int op) {  // resolveCompare, kernel/compare.go:27-44
  switch (op) {
    case WG_OP_EQ: return a == b;
    case WG_OP_NE: return a != b;
    case WG_OP_LT: return a < b;
    case WG_OP_LE: return a <= b;
    case WG_OP_GT: return a > b;
    case WG_OP_GE: return a >= b;
    default: return false;
  }
}

template <typename T>
int64_t filter_typed(const wg_column& c, const T* data, T val, int op, int64_t len, const uint32_t* sel,
                     int64_t sel_len, uint32_t* out) {  // compareFilterImpl, kernel/compare.go:47-90
  int64_t n = 0;
  if (sel) {
    for (int64_t k = 0; k < sel_len; ++k) {
      uint32_t idx = sel[k];
      if (!is_null(c, idx) && cmp<T>(data[idx], val, op)) out[n++] = idx;
    }
  } else {
    for (int64_t i = 0; i < len; ++i)
      if (!is_null(c, i) && cmp<T>(data[i], val, op)) out[n++] = (uint32_t)i;
  }
  return n;
}

int64_t filter_col(const wg_column& c, int64_t len, const uint32_t* sel, int64_t sel_len,
                   const wg_predicate& p, uint32_t* out) {  // ResolveFilterKernel, kernel/compare.go:145
  switch (c.type_id) {
    case WG_TYPE_INT64: case WG_TYPE_TIMESTAMP: case WG_TYPE_DURATION: case WG_TYPE_IPV4: case WG_TYPE_MAC:
      return filter_typed<int64_t>(c, (const int64_t*)c.data, to_int64(p), p.op, len, sel, sel_len, out);
    case WG_TYPE_INT32: case WG_TYPE_PORT: case WG_TYPE_PROTOCOL:
      return filter_typed<int32_t>(c, (const int32_t*)c.data, (int32_t)to_int64(p), p.op, len, sel, sel_len, out);
    case WG_TYPE_DATE:  // toDateInt32: integers truncate to int32; a float constant becomes 0
      return filter_typed<int32_t>(c, (const int32_t*)c.data,
                                   p.const_kind == WG_CONST_FLOAT ? 0 : (int32_t)p.const_i64, p.op, len, sel,
                                   sel_len, out);
    case WG_TYPE_FLOAT64:
      return filter_typed<double>(c, (const double*)c.data, to_float64(p), p.op, len, sel, sel_len, out);
    case WG_TYPE_FLOAT32:
      return filter_typed<float>(c, (const float*)c.data, (float)to_float64(p), p.op, len, sel, sel_len, out);
    default:
      return -1;
  }
}

// ---------------------------------------------------------------------------
// intHashTable (exec/int_hash.go): int64 → int32, fibHash, linear probing, 70% load
// ---------------------------------------------------------------------------
const int64_t kIntHashEmpty = -0x7FFFFFFFFFFFFFFFLL;  // int_hash.go:42
inline uint64_t fib_hash(int64_t k) { return (uint64_t)k * 11400714819323198485ULL; }  // int_hash.go:93

struct IntHashTable {
  struct E { int64_t key; int32_t val; };
  std::vector<E> e;
  uint64_t mask = 0;
  int64_t size = 0;
  explicit IntHashTable(int64_t n) {  // newIntHashTable, int_hash.go:47-60
    int64_t cap = 16, target = n + n / 3;
    while (cap < target) cap <<= 1;
    e.assign((size_t)cap, E{kIntHashEmpty, 0});
    mask = (uint64_t)cap - 1;
  }
  // PutNoGrow (int_hash.go:227): returns previous value and whether it existed
  std::pair<int32_t, bool> put(int64_t key, int32_t val) {
    uint64_t idx = fib_hash(key) & mask;
    for (;;) {
      E& x = e[idx];
      if (x.key == kIntHashEmpty) { x.key = key; x.val = val; ++size; return {0, false}; }
      if (x.key == key) { int32_t old = x.val; x.val = val; return {old, true}; }
      idx = (idx + 1) & mask;
    }
  }
  std::pair<int32_t, bool> get(int64_t key) const {  // Get, int_hash.go:133
    uint64_t idx = fib_hash(key) & mask;
    for (;;) {
      const E& x = e[idx];
      if (x.key == kIntHashEmpty) return {0, false};
      if (x.key == key) return {x.val, true};
      idx = (idx + 1) & mask;
    }
  }
  std::pair<int32_t, bool> get_or_insert(int64_t key, int32_t val) {  // GetOrInsertNoGrow, int_hash.go:167
    uint64_t idx = fib_hash(key) & mask;
    for (;;) {
      E& x = e[idx];
      if (x.key == kIntHashEmpty) { x.key = key; x.val = val; ++size; return {val, false}; }
      if (x.key == key) return {x.val, true};
      idx = (idx + 1) & mask;
    }
  }
  void check_grow() {  // CheckGrow, int_hash.go:255
    if (size * 10 > (int64_t)e.size() * 7) grow();
  }
  void grow() {  // int_hash.go:357
    std::vector<E> old;
    old.swap(e);
    size_t cap = old.size() * 2;
    e.assign(cap, E{kIntHashEmpty, 0});
    mask = cap - 1;
    for (const E& x : old) {
      if (x.key == kIntHashEmpty) continue;
      uint64_t idx = fib_hash(x.key) & mask;
      while (e[idx].key != kIntHashEmpty) idx = (idx + 1) & mask;
      e[idx] = x;
    }
  }
};

// ---------------------------------------------------------------------------
// packedHashTable (exec/packed_hash.go:64-320): 128-bit key → int32, val == -1 empty
// ---------------------------------------------------------------------------
inline uint64_t packed_hash(uint64_t lo, uint64_t hi) {  // packed_hash.go:155
  unsigned __int128 p = (unsigned __int128)(lo ^ 0x9E3779B97F4A7C15ULL) * (unsigned __int128)(hi ^ 0x517CC1B727220A95ULL);
  return (uint64_t)(p >> 64) ^ (uint64_t)p ^ (lo + hi);
}
struct PackedHashTable {
  struct E { uint64_t lo, hi; int32_t val; };
  std::vector<E> e;
  uint64_t mask = 0;
  int64_t size = 0;
  explicit PackedHashTable(int64_t n) {
    int64_t cap = 16, target = n + n / 3;
    while (cap < target) cap <<= 1;
    e.assign((size_t)cap, E{0, 0, -1});
    mask = (uint64_t)cap - 1;
  }
  int32_t get_or_insert(uint64_t lo, uint64_t hi, int32_t val) {  // packed_hash.go:198
    uint64_t idx = packed_hash(lo, hi) & mask;
    for (;;) {
      E& x = e[idx];
      if (x.val == -1) { x.lo = lo; x.hi = hi; x.val = val; ++size; return val; }
      if (x.lo == lo && x.hi == hi) return x.val;
      idx = (idx + 1) & mask;
    }
  }
  void check_grow() {
    if (size * 10 > (int64_t)e.size() * 7) {
      std::vector<E> old;
      old.swap(e);
      size_t cap = old.size() * 2;
      e.assign(cap, E{0, 0, -1});
      mask = cap - 1;
      for (const E& x : old) {
        if (x.val == -1) continue;
        uint64_t idx = packed_hash(x.lo, x.hi) & mask;
        while (e[idx].val != -1) idx = (idx + 1) & mask;
        e[idx] = x;
      }
    }
  }
};

// buildPackedLayout (packed_hash.go:386): widest-first placement into two words
struct PackedField { int word; int shift; bool i32; };
bool build_packed_layout(const std::vector<int>& types, std::vector<PackedField>& out) {
  if (types.size() < 2) return false;
  int total = 0;
  for (int t : types) {
    Cls c = cls_of(t);
    if (c == C_I32) total += 4; else if (c == C_I64) total += 8; else return false;
  }
  if (total > 16) return false;
  out.assign(types.size(), PackedField{0, 0, false});
  int next_wide = 0;
  for (size_t i = 0; i < types.size(); ++i)
    if (cls_of(types[i]) == C_I64) out[i] = PackedField{next_wide++, 0, false};
  std::vector<std::pair<int, int>> slots;
  for (int w = next_wide; w < 2; ++w) { slots.push_back({w, 0}); slots.push_back({w, 32}); }
  size_t nn = 0;
  for (size_t i = 0; i < types.size(); ++i)
    if (cls_of(types[i]) == C_I32) { out[i] = PackedField{slots[nn].first, slots[nn].second, true}; ++nn; }
  return true;
}

// ---------------------------------------------------------------------------
// HashJoin, int key (exec/join.go:520-575 build, 2670-2820 probe)
// ---------------------------------------------------------------------------
struct Join {
  int type = WG_JOIN_INNER;         // exec.JoinType (join.go:20-30)
  std::unique_ptr<IntHashTable> index;
  std::vector<int64_t> arena;       // build row of each arena entry (buildRef)
  std::vector<int32_t> arena_next;  // chain to the previously built row with the same key
  int64_t rows_seen = 0;
};

// ---------------------------------------------------------------------------
// HashAggregate
// ---------------------------------------------------------------------------
struct AggCol {
  int func, col, out_type;
  int in_cls = C_BAD, scale = 0;
  bool is_float = false, is_dec = false;
  // per-group SoA state (agg_scatter.go:16 flatAccumArrays)
  std::vector<int64_t> count, i64;
  std::vector<double> f64;
  std::vector<I128> dec;
  std::vector<uint8_t> has;
};

struct Agg {
  std::vector<int> key_cols;
  std::vector<AggCol> aggs;
  bool resolved = false;
  int mode = 0;  // 0 scalar, 1 int key, 2 packed key
  std::vector<int> key_types;
  std::vector<PackedField> layout;
  std::unique_ptr<IntHashTable> itab;
  std::unique_ptr<PackedHashTable> ptab;
  std::map<std::vector<std::pair<int, int64_t>>, int32_t> null_groups;  // processRow keys with a NULL
  int64_t ngroups = 0;
  std::vector<std::vector<int64_t>> keys;   // [key col][group] widened
  std::vector<std::vector<uint8_t>> kvalid; // [key col][group]
  bool consumed_any = false;

  void add_group() {
    ++ngroups;
    for (auto& a : aggs) {
      a.count.push_back(0); a.i64.push_back(0); a.f64.push_back(0.0); a.dec.push_back(I128{0, 0}); a.has.push_back(0);
    }
  }
};

bool default_out_type(AggCol& a) {  // aggOutputType (plan.go:9968) + minMaxOutputType (aggregate.go:4611)
  if (a.out_type != 0) return true;
  switch (a.func) {
    case WG_AGG_COUNT: a.out_type = WG_TYPE_INT64; return true;
    case WG_AGG_SUM: case WG_AGG_AVG: a.out_type = WG_TYPE_FLOAT64; return true;
    case WG_AGG_MIN: case WG_AGG_MAX:
      a.out_type = (a.in_cls == C_I32 || a.in_cls == C_I64) ? WG_TYPE_INT64 : WG_TYPE_FLOAT64;
      return true;
  }
  return false;
}

int resolve(Agg& g, const wg_batch_desc& b) {  // resolveIndices, aggregate.go:1296
  g.key_types.clear();
  for (int kc : g.key_cols) {
    if (kc < 0 || kc >= b.ncols) return fail("group column out of range");
    if (!is_int_cls(b.cols[kc].type_id)) return fail("group key is not an integer-class column");
    g.key_types.push_back(b.cols[kc].type_id);
  }
  for (auto& a : g.aggs) {
    if (a.col >= 0) {
      if (a.col >= b.ncols) return fail("aggregate column out of range");
      const wg_column& c = b.cols[a.col];
      a.in_cls = cls_of(c.type_id);
      a.scale = c.scale;
      if (a.in_cls == C_BAD && a.func != WG_AGG_COUNT) return fail("unsupported aggregate input type");
      // initFlatAccums, aggregate.go:6060-6118
      switch (a.func) {
        case WG_AGG_SUM: case WG_AGG_AVG:
          if (a.in_cls == C_F32 || a.in_cls == C_F64) a.is_float = true;
          else if (a.in_cls == C_DEC) a.is_dec = true;
          else if (a.in_cls == C_I64 && a.func == WG_AGG_AVG) a.is_float = true;
          break;
        case WG_AGG_MIN: case WG_AGG_MAX:
          if (a.in_cls == C_F32 || a.in_cls == C_F64) a.is_float = true;
          else if (a.in_cls == C_DEC) a.is_dec = true;
          break;
        default: break;
      }
    } else if (a.func != WG_AGG_COUNT) {
      return fail("only COUNT may omit its input column");
    }
    default_out_type(a);
  }
  if (g.key_cols.empty()) {
    g.mode = 0;
    if (g.ngroups == 0) { g.add_group(); }
  } else if (g.key_cols.size() == 1) {
    g.mode = 1;
    g.itab.reset(new IntHashTable(4096));
  } else {
    if (!build_packed_layout(g.key_types, g.layout) || g.key_cols.size() > 4)
      return fail("composite key does not pack into 128 bits");
    g.mode = 2;
    g.ptab.reset(new PackedHashTable(4096));
  }
  g.keys.assign(g.key_cols.size(), {});
  g.kvalid.assign(g.key_cols.size(), {});
  if (g.mode == 0) {}  // scalar group has no key
  g.resolved = true;
  return 0;
}

// One row into one group: the per-aggregate scatter kernels (agg_scatter.go:178-510)
inline void update(AggCol& a, const wg_batch_desc& b, int64_t row, int32_t gi) {
  if (a.col < 0) { a.count[gi]++; return; }  // scatterCountStar, agg_scatter.go:387
  const wg_column& c = b.cols[a.col];
  if (is_null(c, row)) return;
  switch (a.func) {
    case WG_AGG_COUNT: a.count[gi]++; return;  // scatterCount :369
    case WG_AGG_SUM: case WG_AGG_AVG:
      if (a.is_dec) a.dec[gi] = i128_add(a.dec[gi], get_dec(c, row));           // scatterSumDecimal :330
      else if (a.is_float) a.f64[gi] = a.f64[gi] + get_f64(c, row);               // scatterSumFloat :256
      else a.i64[gi] = (int64_t)((uint64_t)a.i64[gi] + (uint64_t)get_i64(c, row));  // scatterSumInt :178 (wraps)
      a.count[gi]++;
      return;
    case WG_AGG_MIN:
      a.count[gi]++;
      if (a.is_dec) { I128 v = get_dec(c, row); if (!a.has[gi] || i128_less(v, a.dec[gi])) { a.dec[gi] = v; a.has[gi] = 1; } }
      else if (a.is_float) { double v = get_f64(c, row); if (!a.has[gi] || v < a.f64[gi]) { a.f64[gi] = v; a.has[gi] = 1; } }  // :434
      else { int64_t v = get_i64(c, row); if (!a.has[gi] || v < a.i64[gi]) { a.i64[gi] = v; a.has[gi] = 1; } }  // :408
      return;
    case WG_AGG_MAX:
      a.count[gi]++;
      if (a.is_dec) { I128 v = get_dec(c, row); if (!a.has[gi] || i128_less(a.dec[gi], v)) { a.dec[gi] = v; a.has[gi] = 1; } }
      else if (a.is_float) { double v = get_f64(c, row); if (!a.has[gi] || v > a.f64[gi]) { a.f64[gi] = v; a.has[gi] = 1; } }  // :486
      else { int64_t v = get_i64(c, row); if (!a.has[gi] || v > a.i64[gi]) { a.i64[gi] = v; a.has[gi] = 1; } }  // :460
      return;
  }
}

int32_t group_of(Agg& g, const wg_batch_desc& b, int64_t row) {
  const size_t nk = g.key_cols.size();
  if (g.mode == 0) return 0;
  bool any_null = false;
  for (size_t k = 0; k < nk; ++k) any_null |= is_null(b.cols[g.key_cols[k]], row);
  if (any_null) {  // processRow, aggregate.go:3422: per-column (null flag, value)
    std::vector<std::pair<int, int64_t>> key;
    for (size_t k = 0; k < nk; ++k) {
      const wg_column& c = b.cols[g.key_cols[k]];
      if (is_null(c, row)) key.push_back({1, 0}); else key.push_back({0, get_i64(c, row)});
    }
    auto it = g.null_groups.find(key);
    if (it != g.null_groups.end()) return it->second;
    int32_t id = (int32_t)g.ngroups;
    g.null_groups.emplace(key, id);
    for (size_t k = 0; k < nk; ++k) { g.keys[k].push_back(key[k].second); g.kvalid[k].push_back(key[k].first ? 0 : 1); }
    g.add_group();
    return id;
  }
  if (g.mode == 1) {  // consumeBatchIntGroup, aggregate.go:1908
    int64_t key = get_i64(b.cols[g.key_cols[0]], row);
    auto r = g.itab->get_or_insert(key, (int32_t)g.ngroups);
    if (r.second) return r.first;
    g.itab->check_grow();
    g.keys[0].push_back(key); g.kvalid[0].push_back(1);
    g.add_group();
    return r.first;
  }
  // consumeBatchPackedGroup, aggregate.go:2326; packedKeyAt, packed_hash.go:456
  uint64_t lo = 0, hi = 0;
  for (size_t k = 0; k < nk; ++k) {
    const wg_column& c = b.cols[g.key_cols[k]];
    const PackedField& f = g.layout[k];
    uint64_t v = f.i32 ? ((uint64_t)(uint32_t)((const int32_t*)c.data)[row]) << f.shift
                       : (uint64_t)((const int64_t*)c.data)[row];
    if (f.word == 0) lo |= v; else hi |= v;
  }
  int32_t offer = (int32_t)g.ngroups;
  int32_t got = g.ptab->get_or_insert(lo, hi, offer);
  if (got != offer) return got;
  g.ptab->check_grow();
  for (size_t k = 0; k < nk; ++k) { g.keys[k].push_back(get_i64(b.cols[g.key_cols[k]], row)); g.kvalid[k].push_back(1); }
  g.add_group();
  return got;
}

int consume(Agg& g, const wg_batch_desc& b) {  // HashAggregate.Consume, aggregate.go:1075
  if (!g.resolved) { if (resolve(g, b) != 0) return -1; }
  g.consumed_any = true;
  const int64_t n = b.sel ? b.sel_len : b.len;
  std::vector<int32_t> gi((size_t)n);
  for (int64_t i = 0; i < n; ++i) gi[i] = group_of(g, b, b.sel ? (int64_t)b.sel[i] : i);  // phase 1
  for (auto& a : g.aggs)                                                                    // phase 2
    for (int64_t i = 0; i < n; ++i) update(a, b, b.sel ? (int64_t)b.sel[i] : i, gi[i]);
  return 0;
}

// Accumulator.Merge (kernel/types.go:106-175) per group
void merge_group(AggCol& d, int32_t dg, const AggCol& s, int32_t sg) {
  d.count[dg] += s.count[sg];
  switch (d.func) {
    case WG_AGG_SUM: case WG_AGG_AVG:
      if (d.is_dec) d.dec[dg] = i128_add(d.dec[dg], s.dec[sg]);
      else if (d.is_float) d.f64[dg] = d.f64[dg] + s.f64[sg];
      else d.i64[dg] = (int64_t)((uint64_t)d.i64[dg] + (uint64_t)s.i64[sg]);
      break;
    case WG_AGG_MIN:
      if (s.has[sg]) {
        if (!d.has[dg]) { d.i64[dg] = s.i64[sg]; d.f64[dg] = s.f64[sg]; d.dec[dg] = s.dec[sg]; d.has[dg] = 1; }
        else if (d.is_float) { if (s.f64[sg] < d.f64[dg]) d.f64[dg] = s.f64[sg]; }
        else if (d.is_dec) { if (i128_less(s.dec[sg], d.dec[dg])) d.dec[dg] = s.dec[sg]; }
        else { if (s.i64[sg] < d.i64[dg]) d.i64[dg] = s.i64[sg]; }
      }
      break;
    case WG_AGG_MAX:
      if (s.has[sg]) {
        if (!d.has[dg]) { d.i64[dg] = s.i64[sg]; d.f64[dg] = s.f64[sg]; d.dec[dg] = s.dec[sg]; d.has[dg] = 1; }
        else if (d.is_float) { if (s.f64[sg] > d.f64[dg]) d.f64[dg] = s.f64[sg]; }
        else if (d.is_dec) { if (i128_less(d.dec[dg], s.dec[sg])) d.dec[dg] = s.dec[sg]; }
        else { if (s.i64[sg] > d.i64[dg]) d.i64[dg] = s.i64[sg]; }
      }
      break;
    default: break;
  }
}

// Find-or-create the group of src group sg inside dst (MergeSink → mergeSinkState)
int32_t dst_group(Agg& d, const Agg& s, int32_t sg) {
  const size_t nk = d.key_cols.size();
  if (d.mode == 0) return 0;
  bool any_null = false;
  for (size_t k = 0; k < nk; ++k) any_null |= !s.kvalid[k][sg];
  if (any_null) {
    std::vector<std::pair<int, int64_t>> key;
    for (size_t k = 0; k < nk; ++k) key.push_back(s.kvalid[k][sg] ? std::make_pair(0, s.keys[k][sg]) : std::make_pair(1, (int64_t)0));
    auto it = d.null_groups.find(key);
    if (it != d.null_groups.end()) return it->second;
    int32_t id = (int32_t)d.ngroups;
    d.null_groups.emplace(key, id);
    for (size_t k = 0; k < nk; ++k) { d.keys[k].push_back(key[k].second); d.kvalid[k].push_back(key[k].first ? 0 : 1); }
    d.add_group();
    return id;
  }
  if (d.mode == 1) {
    auto r = d.itab->get_or_insert(s.keys[0][sg], (int32_t)d.ngroups);
    if (r.second) return r.first;
    d.itab->check_grow();
    d.keys[0].push_back(s.keys[0][sg]); d.kvalid[0].push_back(1);
    d.add_group();
    return r.first;
  }
  uint64_t lo = 0, hi = 0;
  for (size_t k = 0; k < nk; ++k) {
    const PackedField& f = d.layout[k];
    uint64_t v = f.i32 ? ((uint64_t)(uint32_t)(int32_t)s.keys[k][sg]) << f.shift : (uint64_t)s.keys[k][sg];
    if (f.word == 0) lo |= v; else hi |= v;
  }
  int32_t offer = (int32_t)d.ngroups;
  int32_t got = d.ptab->get_or_insert(lo, hi, offer);
  if (got != offer) return got;
  d.ptab->check_grow();
  for (size_t k = 0; k < nk; ++k) { d.keys[k].push_back(s.keys[k][sg]); d.kvalid[k].push_back(1); }
  d.add_group();
  return got;
}

int merge(Agg& d, Agg& s) {
  if (!s.resolved) return 0;
  if (!d.resolved) {
    d.key_types = s.key_types; d.layout = s.layout; d.mode = s.mode;
    for (size_t i = 0; i < d.aggs.size(); ++i) {
      d.aggs[i].in_cls = s.aggs[i].in_cls; d.aggs[i].scale = s.aggs[i].scale;
      d.aggs[i].is_float = s.aggs[i].is_float; d.aggs[i].is_dec = s.aggs[i].is_dec;
      d.aggs[i].out_type = s.aggs[i].out_type;
    }
    if (d.mode == 1) d.itab.reset(new IntHashTable(4096));
    if (d.mode == 2) d.ptab.reset(new PackedHashTable(4096));
    d.keys.assign(d.key_cols.size(), {});
    d.kvalid.assign(d.key_cols.size(), {});
    if (d.mode == 0 && d.ngroups == 0) d.add_group();
    d.resolved = true;
  }
  d.consumed_any = d.consumed_any || s.consumed_any;
  for (int32_t sg = 0; sg < (int32_t)s.ngroups; ++sg) {
    int32_t dg = dst_group(d, s, sg);
    for (size_t i = 0; i < d.aggs.size(); ++i) merge_group(d.aggs[i], dg, s.aggs[i], sg);
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Expressions (expr.ColRef.EvalFloat64 / BinOpNumeric), postfix
// ---------------------------------------------------------------------------
struct Val { bool is_f; int64_t i; double f; };

bool eval_expr(const wg_expr& e, const std::vector<const wg_column*>& cols, int64_t row, Val& out) {
  Val st[WG_EXPR_MAX_OPS];
  int sp = 0;
  for (int k = 0; k < e.n_ops; ++k) {
    const wg_expr_op& o = e.ops[k];
    switch (o.opcode) {
      case WG_EXPR_COL: {
        const wg_column& c = *cols[o.arg];
        if (is_null(c, row)) return false;  // a NULL operand makes the expression NULL
        Cls cl = cls_of(c.type_id);
        if (cl == C_I32 || cl == C_I64) st[sp++] = Val{false, get_i64(c, row), 0.0};
        else st[sp++] = Val{true, 0, get_f64(c, row)};
        break;
      }
      case WG_EXPR_CONST_I: st[sp++] = Val{false, o.imm_i64, 0.0}; break;
      case WG_EXPR_CONST_F: st[sp++] = Val{true, 0, o.imm_f64}; break;
      default: {
        Val b = st[--sp], a = st[--sp];
        if (o.opcode == WG_EXPR_SHR || o.opcode == WG_EXPR_AND) {
          if (a.is_f || b.is_f) return false;
          st[sp++] = Val{false, o.opcode == WG_EXPR_SHR ? (a.i >> (b.i & 63)) : (a.i & b.i), 0.0};
          break;
        }
        if (!a.is_f && !b.is_f && o.opcode != WG_EXPR_DIV) {
          uint64_t x = (uint64_t)a.i, y = (uint64_t)b.i, r = 0;
          if (o.opcode == WG_EXPR_ADD) r = x + y; else if (o.opcode == WG_EXPR_SUB) r = x - y; else r = x * y;
          st[sp++] = Val{false, (int64_t)r, 0.0};
          break;
        }
        double x = a.is_f ? a.f : (double)a.i, y = b.is_f ? b.f : (double)b.i, r = 0;
        switch (o.opcode) {
          case WG_EXPR_ADD: r = x + y; break;
          case WG_EXPR_SUB: r = x - y; break;
          case WG_EXPR_MUL: r = x * y; break;
          case WG_EXPR_DIV: r = x / y; break;
        }
        st[sp++] = Val{true, 0, r};
      }
    }
  }
  out = st[sp - 1];
  if (e.result_type == WG_TYPE_FLOAT64 && !out.is_f) { out.is_f = true; out.f = (double)out.i; }
  return true;
}

void set_valid(uint64_t* w, int64_t i, bool v) {
  if (v) w[i >> 6] |= (1ULL << (i & 63)); else w[i >> 6] &= ~(1ULL << (i & 63));
}

// One worker of Pipeline.runParallel: batches [b0, b1) of 2048 rows each
int run_worker(const wg_batch_desc& in, int32_t nf, const wg_predicate* filters, Join* join, int32_t probe_key,
               const wg_batch_desc* build, int32_t npay, const int32_t* pay, int32_t nexpr, const wg_expr* exprs,
               Agg& agg, int64_t b0, int64_t b1) {
  const int64_t BS = 2048;  // batch.DefaultBatchSize, batch.go:6
  const int ncols_virtual = in.ncols + (join ? npay : 0) + nexpr;
  std::vector<uint32_t> sel(BS), sel2(BS);
  std::vector<uint32_t> pr; std::vector<int64_t> br;
  // scratch for the joined / projected batch
  std::vector<std::vector<uint8_t>> bufs((size_t)ncols_virtual);
  std::vector<std::vector<uint64_t>> valid((size_t)ncols_virtual);
  std::vector<wg_column> vcols((size_t)ncols_virtual);
  for (int64_t bi = b0; bi < b1; ++bi) {
    const int64_t r0 = bi * BS;
    const int64_t len = std::min<int64_t>(BS, in.len - r0);
    if (len <= 0) break;
    // the batch's columns, offset to this batch
    std::vector<wg_column> cols((size_t)in.ncols);
    for (int c = 0; c < in.ncols; ++c) {
      cols[c] = in.cols[c];
      int64_t es = cls_of(cols[c].type_id) == C_DEC ? 16 : (cls_of(cols[c].type_id) == C_I32 || cls_of(cols[c].type_id) == C_F32) ? 4 : 8;
      cols[c].data = (const uint8_t*)in.cols[c].data + r0 * es;
      cols[c].len = len;
      if (in.cols[c].valid_words) {  // re-base the bitmap at r0 (r0 is a multiple of 64)
        cols[c].valid_words = in.cols[c].valid_words + (r0 >> 6);
      }
    }
    // KernelFilter chain (filter.go:373): compact sel in place
    const uint32_t* cur = nullptr; int64_t cur_n = len;
    for (int32_t f = 0; f < nf; ++f) {
      int64_t n = filter_col(cols[filters[f].col], len, cur, cur_n, filters[f], cur ? sel2.data() : sel.data());
      if (n < 0) return fail("unsupported filter column type");
      if (cur) { std::copy(sel2.begin(), sel2.begin() + n, sel.begin()); }
      cur = sel.data(); cur_n = n;
      if (n == 0) break;
    }
    if (nf > 0 && cur_n == 0) continue;  // fully filtered → nil batch
    wg_batch_desc vb;
    std::vector<const wg_column*> vptr((size_t)ncols_virtual);
    int64_t out_len = len;
    if (join) {
      // HashJoinProbe: match pairs then gatherVector per output column (sort.go:611)
      int64_t total = or_join_probe(join, &cols[probe_key], len, cur, cur_n, nullptr, nullptr, 0);
      pr.resize((size_t)total); br.resize((size_t)total);
      or_join_probe(join, &cols[probe_key], len, cur, cur_n, pr.data(), br.data(), total);
      out_len = total;
      if (total == 0) continue;
      for (int c = 0; c < in.ncols + npay; ++c) {
        const wg_column& src = c < in.ncols ? cols[c] : build->cols[pay[c - in.ncols]];
        int64_t es = cls_of(src.type_id) == C_DEC ? 16 : (cls_of(src.type_id) == C_I32 || cls_of(src.type_id) == C_F32) ? 4 : 8;
        bufs[c].resize((size_t)(total * es));
        // build columns of a LEFT join are NULL where a probe row found no match
        bool nullable = src.valid_words != nullptr || (c >= in.ncols && join->type == WG_JOIN_LEFT);
        if (nullable) valid[c].assign((size_t)((total + 63) / 64), 0);
        for (int64_t k = 0; k < total; ++k) {
          int64_t r = c < in.ncols ? (int64_t)pr[k] : br[k];
          if (r < 0) {
            std::memset(&bufs[c][k * es], 0, (size_t)es);
            continue;  // valid bit stays 0
          }
          std::memcpy(&bufs[c][k * es], (const uint8_t*)src.data + r * es, (size_t)es);
          if (nullable) set_valid(valid[c].data(), k, !is_null(src, r));
        }
        vcols[c] = wg_column{src.type_id, src.scale, bufs[c].data(), nullable ? valid[c].data() : nullptr, total};
      }
      cur = nullptr; cur_n = total;
    } else {
      for (int c = 0; c < in.ncols; ++c) vcols[c] = cols[c];
    }
    // Project (exprs append columns over the dense or selected rows)
    const int base = in.ncols + (join ? npay : 0);
    for (int e = 0; e < nexpr; ++e) {
      for (int c = 0; c < base + e; ++c) vptr[c] = &vcols[c];
      const int c = base + e;
      bufs[c].resize((size_t)(out_len * 8));
      valid[c].assign((size_t)((out_len + 63) / 64), 0);
      bool any_null = false;
      for (int64_t k = 0; k < (cur ? cur_n : out_len); ++k) {
        int64_t r = cur ? (int64_t)cur[k] : k;
        Val v;
        bool ok = eval_expr(exprs[e], vptr, r, v);
        set_valid(valid[c].data(), r, ok);
        any_null |= !ok;
        if (exprs[e].result_type == WG_TYPE_FLOAT64) ((double*)bufs[c].data())[r] = ok ? v.f : 0.0;
        else ((int64_t*)bufs[c].data())[r] = ok ? v.i : 0;
      }
      vcols[c] = wg_column{exprs[e].result_type, 0, bufs[c].data(), any_null ? valid[c].data() : nullptr, out_len};
    }
    vb.ncols = ncols_virtual; vb._pad = 0; vb.cols = vcols.data(); vb.len = out_len;
    vb.sel = cur; vb.sel_len = cur ? cur_n : 0;
    if (consume(agg, vb) != 0) return -1;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// Parquet page decode (internal/storage/parquet/rle.go, page_reader.go:607-690,
// engine/scan/columnar_native.go:470-640)
// ---------------------------------------------------------------------------
// decodeBitPackedRange (rle.go:214-250): value i of a run reads up to four
// little-endian bytes from its first byte, bytes past the run reading as zero.
void bitpacked_range(int32_t* dst, const uint8_t* data, int64_t len, int bw, int64_t from, int64_t n) {
  if (bw == 0) { for (int64_t i = 0; i < n; ++i) dst[i] = 0; return; }
  const int32_t mask = bw >= 32 ? -1 : (int32_t)((1u << bw) - 1u);
  int64_t bit = from * bw;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t byte = bit / 8;
    const int sh = (int)(bit % 8);
    uint32_t raw = 0;
    const int64_t rem = len - byte;
    for (int k = 0; k < 4; ++k)
      if (k < rem) raw |= (uint32_t)data[byte + k] << (8 * k);
    dst[i] = (int32_t)(raw >> sh) & mask;
    bit += bw;
  }
}

// DecodeRLEInt32Into / decodeAllBatch (rle.go:219-300): returns the values
// decoded (fewer than count when the stream ends), or -1 on a truncated varint
// or a repeated value missing its bytes.
int64_t rle_decode(const uint8_t* data, int64_t len, int bw, int64_t count, int32_t* dst) {
  int64_t off = 0, pos = 0;
  const int vbytes = (bw + 7) / 8;
  while (off < len && pos < count) {
    uint64_t h = 0;
    unsigned shift = 0;
    for (;;) {
      if (off >= len) return -1;                 // varint truncated
      const uint8_t b = data[off++];
      h |= (uint64_t)(b & 0x7F) << shift;
      if (!(b & 0x80)) break;
      shift += 7;
      if (shift >= 64) return -1;                // varint overflow
    }
    if ((h & 1) == 0) {
      const int64_t c = (int64_t)(h >> 1);
      if (off + vbytes > len) return -1;
      int32_t v = 0;
      for (int i = 0; i < vbytes; ++i) v |= (int32_t)data[off + i] << (8 * i);
      off += vbytes;
      const int64_t end = std::min(count, pos + c);
      for (int64_t i = pos; i < end; ++i) dst[i] = v;
      pos = end;
    } else {
      const int64_t groups = (int64_t)(h >> 1);
      if (groups <= 0) continue;
      if (groups > INT64_MAX / 8 || (bw > 0 && groups > INT64_MAX / bw)) return -1;
      int64_t nv = std::min(groups * 8, count - pos);
      int64_t bc = groups * bw;
      if (off + bc > len) bc = len - off;
      bitpacked_range(dst + pos, data + off, bc, bw, 0, nv);
      off += bc;
      pos += nv;
    }
  }
  return pos;
}

template <typename F>
void par_for(int64_t n, int32_t threads, F f) {
  if (threads <= 1 || n < 65536) { f(0, n); return; }
  std::vector<std::thread> ts;
  for (int t = 0; t < threads; ++t) ts.emplace_back([=] { f(n * t / threads, n * (t + 1) / threads); });
  for (auto& th : ts) th.join();
}

}  // namespace

// ===========================================================================
// extern "C"
// ===========================================================================
extern "C" {

const char* or_last_error(void) { return g_err.c_str(); }

double or_i128_to_f64(int64_t hi, uint64_t lo, int32_t scale) { return i128_to_f64(I128{hi, lo}, scale); }

int64_t or_rle_decode(const uint8_t* data, int64_t len, int32_t bw, int64_t count, int32_t* out) {
  return rle_decode(data, len, bw, count, out);
}

// One column chunk's pages into a host column (out: rows * element size;
// valid_words: (rows + 63) / 64 words or NULL): definition levels to validity
// (level 1 = a value), the values section decoded (PLAIN, or dictionary
// indices with the gather loops' bounds check, columnar_native.go:470-520) and
// written to the non-NULL rows in order, INT64 DECIMAL widened with
// Int128From (columnar_native.go:619-625). Returns 0, or -1 on a malformed page.
int or_page_decode(const wg_column_chunk* ch, void* out, uint64_t* valid_words) {
  const int cls = cls_of(ch->type_id);
  const int64_t es = ch->type_id == WG_TYPE_DECIMAL ? 8 : (cls == C_I32 || cls == C_F32) ? 4 : 8;
  const int64_t oes = ch->type_id == WG_TYPE_DECIMAL ? 16 : es;
  int64_t row0 = 0;
  for (int p = 0; p < ch->n_pages; ++p) {
    const wg_page& pg = ch->pages[p];
    const int64_t n = pg.num_values;
    std::vector<int32_t> lv((size_t)n, 1);
    if (pg.def_levels) {
      if (rle_decode(pg.def_levels, pg.def_len, 1, n, lv.data()) != n) return fail("definition levels end early");
    }
    int64_t nn = 0;
    for (int64_t i = 0; i < n; ++i) nn += lv[(size_t)i] == 1;
    std::vector<uint8_t> vals((size_t)(nn * es));
    if (pg.encoding == WG_ENC_PLAIN) {
      if (pg.data_len < nn * es) return fail("PLAIN data shorter than its values");
      if (nn) std::memcpy(vals.data(), pg.data, (size_t)(nn * es));
    } else if (nn > 0) {
      if (pg.data_len < 1 || pg.data[0] > 32) return fail("dictionary page without a bit width");
      std::vector<int32_t> idx((size_t)nn);
      if (rle_decode(pg.data + 1, pg.data_len - 1, pg.data[0], nn, idx.data()) != nn)
        return fail("fewer dictionary indices than values");
      for (int64_t k = 0; k < nn; ++k) {
        if ((uint64_t)(uint32_t)idx[(size_t)k] >= (uint64_t)ch->dict_len) return fail("dictionary index out of range");
        std::memcpy(&vals[(size_t)(k * es)], (const uint8_t*)ch->dict + (int64_t)(uint32_t)idx[(size_t)k] * es, (size_t)es);
      }
    }
    int64_t k = 0;
    for (int64_t i = 0; i < n; ++i) {
      const int64_t r = row0 + i;
      uint8_t* o = (uint8_t*)out + r * oes;
      const bool valid = lv[(size_t)i] == 1;
      if (valid_words) {
        if (valid) valid_words[r >> 6] |= 1ULL << (r & 63);
        else valid_words[r >> 6] &= ~(1ULL << (r & 63));
      }
      if (!valid) { std::memset(o, 0, (size_t)oes); continue; }
      if (ch->type_id == WG_TYPE_DECIMAL) {
        int64_t v;
        std::memcpy(&v, &vals[(size_t)(k * es)], 8);
        const wg_int128 d{v < 0 ? -1 : 0, (uint64_t)v};
        std::memcpy(o, &d, 16);
      } else {
        std::memcpy(o, &vals[(size_t)(k * es)], (size_t)es);
      }
      ++k;
    }
    row0 += n;
  }
  return 0;
}

int64_t or_filter(const wg_column* col, int64_t len, const uint32_t* sel, int64_t sel_len, const wg_predicate* p,
                  uint32_t* out_sel) {
  int64_t n = filter_col(*col, len, sel, sel_len, *p, out_sel);
  if (n < 0) fail("unsupported filter column type");
  return n;
}

// HashJoin.buildBloom (join.go:1441) over the join's distinct keys, then
// BloomFilterOp.Execute (bloom_filter_op.go:39) for one int key: the probe rows
// (or selection entries) with a non-NULL key that the bloom may contain, in
// order. bloomHashInt (join.go:1650), bloomSet (:1475), bloomContains
// (bloom_filter_op.go:268): 64-bit words, about 10 bits per distinct key
// rounded up to a power-of-two word count (at least 8), two bits per key.
static uint64_t bloom_hash_int(int64_t key) {
  const uint64_t x = (uint64_t)key * 0x9E3779B97F4A7C15ULL;
  return x ^ (x >> 32);
}

int64_t or_join_bloom_filter(void* jp, const wg_column* key, int64_t len, const uint32_t* sel, int64_t sel_len,
                             uint32_t* out_sel, int64_t* n_words) {
  Join* j = (Join*)jp;
  if (!is_int_cls(key->type_id)) return fail("bloom filter key is not an integer-class column");
  const int64_t n_keys = j->index->size;
  std::vector<uint64_t> bloom;
  uint64_t mask = 0;
  if (n_keys > 0) {
    const int64_t n_bits = n_keys * 10;
    int64_t slots = 1;
    while (slots * 64 < n_bits) slots *= 2;
    if (slots < 8) slots = 8;
    bloom.assign((size_t)slots, 0);
    mask = (uint64_t)slots - 1;
    for (const auto& e : j->index->e) {
      if (e.key == kIntHashEmpty) continue;
      const uint64_t h = bloom_hash_int(e.key);
      bloom[h & mask] |= 1ULL << (h & 63);
      bloom[(h >> 17) & mask] |= 1ULL << ((h >> 6) & 63);
    }
  }
  if (n_words) *n_words = (int64_t)bloom.size();
  const int64_t n = sel ? sel_len : len;
  int64_t m = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t row = sel ? (int64_t)sel[i] : i;
    if (is_null(*key, row)) continue;
    if (bloom.empty()) continue;  // no build keys: nothing may match
    const uint64_t h = bloom_hash_int(get_i64(*key, row));
    if (((bloom[h & mask] >> (h & 63)) & 1ULL) && ((bloom[(h >> 17) & mask] >> ((h >> 6) & 63)) & 1ULL))
      out_sel[m++] = (uint32_t)row;
  }
  return m;
}

void* or_join_new(int64_t hint) {
  Join* j = new Join();
  j->index.reset(new IntHashTable(hint > 0 ? hint : 64));
  return j;
}

int or_join_append(void* jp, const wg_column* key, int64_t base_row) {  // arenaAppendInt per row, join.go:551
  Join* j = (Join*)jp;
  if (!is_int_cls(key->type_id)) return fail("join key is not an integer-class column");
  for (int64_t i = 0; i < key->len; ++i) {
    if (is_null(*key, i)) continue;  // intKeyFromVector: NULL keys are not indexed
    int64_t k = get_i64(*key, i);
    int32_t idx = (int32_t)j->arena.size();
    j->arena.push_back(base_row + i);
    auto r = j->index->put(k, idx);
    j->arena_next.push_back(r.second ? r.first : -1);
    j->index->check_grow();  // per insert: a batch may hold more keys than the table has free slots
  }
  j->rows_seen += key->len;
  return 0;
}

int64_t or_join_rows(void* jp) { return (int64_t)((Join*)jp)->arena.size(); }
int64_t or_join_distinct(void* jp) { return ((Join*)jp)->index->size; }

void or_join_set_type(void* jp, int32_t type) { ((Join*)jp)->type = type; }

// inlineIntProbe for inner joins (join.go:2670-2820); the generic probe's
// LEFT emission of an unmatched row as one NULL-padded pair (join.go:3180-3186,
// NULL keys included since they never match); executeSemiAntiJoin's SEMI (a
// matched row once) and ANTI (an unmatched or NULL-key row once)
// (join.go:3247-3300). Pairs without a build row carry -1.
int64_t or_join_probe(void* jp, const wg_column* key, int64_t len, const uint32_t* sel, int64_t sel_len,
                      uint32_t* out_probe, int64_t* out_build, int64_t cap) {
  Join* j = (Join*)jp;
  int64_t n = 0;
  const int64_t cnt = sel ? sel_len : len;
  auto emit = [&](int64_t row, int64_t b) {
    if (n < cap) { out_probe[n] = (uint32_t)row; out_build[n] = b; }
    ++n;
  };
  for (int64_t p = 0; p < cnt; ++p) {
    int64_t row = sel ? (int64_t)sel[p] : p;
    std::pair<int32_t, bool> h{-1, false};
    if (!is_null(*key, row)) h = j->index->get(get_i64(*key, row));
    if (j->type == WG_JOIN_SEMI) { if (h.second) emit(row, -1); continue; }
    if (j->type == WG_JOIN_ANTI) { if (!h.second) emit(row, -1); continue; }
    if (!h.second) {
      if (j->type == WG_JOIN_LEFT) emit(row, -1);
      continue;
    }
    for (int32_t ref = h.first; ref >= 0; ref = j->arena_next[(size_t)ref]) emit(row, j->arena[(size_t)ref]);
  }
  return n;
}

void or_join_free(void* jp) { delete (Join*)jp; }

void* or_agg_new(int32_t n_keys, const int32_t* key_cols, int32_t n_aggs, const wg_agg_spec* aggs) {
  Agg* g = new Agg();
  for (int i = 0; i < n_keys; ++i) g->key_cols.push_back(key_cols[i]);
  for (int i = 0; i < n_aggs; ++i) {
    AggCol a;
    a.func = aggs[i].func; a.col = aggs[i].input_col; a.out_type = aggs[i].out_type;
    g->aggs.push_back(a);
  }
  return g;
}

void* or_agg_clone(void* ap) {  // CloneSink: same shape, fresh state
  Agg* s = (Agg*)ap;
  Agg* g = new Agg();
  g->key_cols = s->key_cols;
  for (auto& a : s->aggs) { AggCol c; c.func = a.func; c.col = a.col; c.out_type = a.out_type; g->aggs.push_back(c); }
  return g;
}

int or_agg_consume(void* ap, const wg_batch_desc* b) { return consume(*(Agg*)ap, *b); }

int64_t or_agg_groups(void* ap) {
  Agg* g = (Agg*)ap;
  if (!g->resolved && g->key_cols.empty()) return 1;  // scalar aggregate over no input emits one row
  return g->ngroups;
}

int or_agg_export(void* ap, const wg_group_export* o) {
  Agg* g = (Agg*)ap;
  const int64_t n = g->ngroups;
  for (size_t k = 0; k < g->key_cols.size(); ++k)
    for (int64_t i = 0; i < n; ++i) {
      if (o->keys) o->keys[k * n + i] = g->keys[k][i];
      if (o->key_valid) o->key_valid[k * n + i] = g->kvalid[k][i];
    }
  for (size_t a = 0; a < g->aggs.size(); ++a) {
    const AggCol& c = g->aggs[a];
    for (int64_t i = 0; i < n; ++i) {
      if (o->count) o->count[a * n + i] = c.count[i];
      if (o->i64) o->i64[a * n + i] = c.i64[i];
      if (o->f64) o->f64[a * n + i] = c.f64[i];
      if (o->dec) o->dec[a * n + i] = wg_int128{c.dec[i].hi, c.dec[i].lo};
      if (o->has) o->has[a * n + i] = (c.func == WG_AGG_MIN || c.func == WG_AGG_MAX) ? c.has[i] : (c.count[i] > 0);
    }
  }
  return 0;
}

int or_agg_emit(void* ap, wg_column* out) {  // writeAccToColumn, aggregate_partial_spill.go:1855
  Agg* g = (Agg*)ap;
  const size_t nk = g->key_cols.size();
  if (!g->resolved) {
    if (nk != 0) return 0;
    // Scalar aggregate with no input (aggregate.go:4270): COUNT 0, others NULL
    for (size_t a = 0; a < g->aggs.size(); ++a) {
      wg_column& c = out[a];
      AggCol& s = g->aggs[a];
      default_out_type(s);
      if (s.func == WG_AGG_COUNT) { ((int64_t*)c.data)[0] = 0; if (c.valid_words) set_valid((uint64_t*)c.valid_words, 0, true); }
      else if (c.valid_words) set_valid((uint64_t*)c.valid_words, 0, false);
    }
    return 0;
  }
  const int64_t n = g->ngroups;
  for (size_t k = 0; k < nk; ++k) {
    wg_column& c = out[k];
    for (int64_t i = 0; i < n; ++i) {
      if (cls_of(g->key_types[k]) == C_I32) ((int32_t*)c.data)[i] = (int32_t)g->keys[k][i];
      else ((int64_t*)c.data)[i] = g->keys[k][i];
      if (c.valid_words) set_valid((uint64_t*)c.valid_words, i, g->kvalid[k][i] != 0);
    }
  }
  for (size_t a = 0; a < g->aggs.size(); ++a) {
    wg_column& c = out[nk + a];
    const AggCol& s = g->aggs[a];
    for (int64_t i = 0; i < n; ++i) {
      bool valid = true;
      double f = 0; int64_t iv = 0;
      switch (s.func) {
        case WG_AGG_SUM:
          if (s.count[i] == 0) { valid = false; break; }
          f = s.is_dec ? i128_to_f64(s.dec[i], s.scale) : s.is_float ? s.f64[i] : (double)s.i64[i];
          iv = s.i64[i];
          break;
        case WG_AGG_AVG:
          if (s.count[i] == 0) { valid = false; break; }
          f = s.is_dec ? i128_to_f64(s.dec[i], s.scale) / (double)s.count[i]
              : s.is_float ? s.f64[i] / (double)s.count[i] : (double)s.i64[i] / (double)s.count[i];
          break;
        case WG_AGG_COUNT: iv = s.count[i]; f = (double)iv; break;
        case WG_AGG_MIN: case WG_AGG_MAX:
          if (!s.has[i]) { valid = false; break; }
          f = s.is_dec ? i128_to_f64(s.dec[i], s.scale) : s.is_float ? s.f64[i] : (double)s.i64[i];
          iv = s.i64[i];
          break;
      }
      if (s.out_type == WG_TYPE_INT64) ((int64_t*)c.data)[i] = valid ? iv : 0;
      else ((double*)c.data)[i] = valid ? f : 0.0;
      if (c.valid_words) set_valid((uint64_t*)c.valid_words, i, valid);
    }
  }
  return 0;
}

int or_agg_merge(void* dp, void* sp) { return merge(*(Agg*)dp, *(Agg*)sp); }

void or_agg_free(void* ap) { delete (Agg*)ap; }

int or_pipeline_run(const wg_batch_desc* input, int32_t n_filters, const wg_predicate* filters, void* join,
                    int32_t probe_key_col, const wg_batch_desc* build, int32_t n_payload, const int32_t* payload_cols,
                    int32_t n_exprs, const wg_expr* exprs, void* agg, int32_t threads) {
  if (input->sel) return fail("pipeline input must not carry a selection vector");
  const int64_t BS = 2048;
  const int64_t nb = (input->len + BS - 1) / BS;
  if (threads < 1) threads = 1;
  if (threads > nb) threads = (int32_t)std::max<int64_t>(1, nb);
  std::vector<void*> clones((size_t)threads);
  std::vector<int> rc((size_t)threads, 0);
  std::vector<std::thread> ts;
  std::vector<std::string> errs((size_t)threads);
  for (int t = 0; t < threads; ++t) {
    clones[t] = or_agg_clone(agg);
    int64_t b0 = nb * t / threads, b1 = nb * (t + 1) / threads;
    ts.emplace_back([&, t, b0, b1] {
      rc[t] = run_worker(*input, n_filters, filters, (Join*)join, probe_key_col, build, n_payload, payload_cols,
                         n_exprs, exprs, *(Agg*)clones[t], b0, b1);
      if (rc[t] != 0) errs[t] = g_err;
    });
  }
  for (auto& th : ts) th.join();
  int status = 0;
  for (int t = 0; t < threads; ++t) {
    if (rc[t] != 0 && status == 0) { status = -1; g_err = errs[t]; }
    if (status == 0) merge(*(Agg*)agg, *(Agg*)clones[t]);
    delete (Agg*)clones[t];
  }
  return status;
}

// ---- generators -----------------------------------------------------------
void or_gen_starjoin_fact(uint64_t seed, int64_t row0, int64_t n, int32_t* fk, int32_t* qty, wg_int128* price,
                          double* disc, int32_t threads) {
  const int bits = WG_SYN_SJ_DIM_BITS;
  std::vector<double> cdf((size_t)1 << bits);
  wg_syn_zipf_cdf(cdf.data(), (int64_t)cdf.size(), WG_SYN_SJ_ZIPF_S);
  const double* c = cdf.data();
  par_for(n, threads, [=](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; ++i) {
      uint64_t r = (uint64_t)(row0 + i);
      if (fk) fk[i] = wg_syn_sj_fk(seed, r, c, bits);
      if (qty) qty[i] = wg_syn_sj_qty(seed, r);
      if (price) price[i] = wg_int128{0, (uint64_t)wg_syn_sj_price(seed, r)};
      if (disc) disc[i] = wg_syn_sj_disc(seed, r);
    }
  });
}

void or_gen_starjoin_dim(uint64_t seed, int64_t n, int32_t* key, int32_t* grp) {
  for (int64_t i = 0; i < n; ++i) {
    key[i] = wg_syn_sj_dim_key((uint64_t)i, WG_SYN_SJ_DIM_BITS);
    grp[i] = wg_syn_sj_grp(seed, (uint64_t)i);
  }
}

void or_gen_groupby(uint64_t seed, int64_t row0, int64_t n, int64_t ngroups, int64_t* k, int64_t* v, double* f,
                    int32_t* flag, int32_t threads) {
  par_for(n, threads, [=](int64_t a, int64_t b) {
    for (int64_t i = a; i < b; ++i) {
      uint64_t r = (uint64_t)(row0 + i);
      if (k) k[i] = wg_syn_gb_k(seed, r, ngroups);
      if (v) v[i] = wg_syn_gb_v(seed, r);
      if (f) f[i] = wg_syn_gb_f(seed, r);
      if (flag) flag[i] = wg_syn_gb_flag(seed, r);
    }
  });
}

void or_gen_highcard(uint64_t seed, int64_t row0, int64_t n, int32_t* a, int64_t* b, wg_int128* amt, double* x,
                     int32_t threads) {
  par_for(n, threads, [=](int64_t s, int64_t e) {
    for (int64_t i = s; i < e; ++i) {
      uint64_t r = (uint64_t)(row0 + i);
      int64_t bv = wg_syn_hc_b(seed, r, WG_SYN_HC_B_BITS);
      if (b) b[i] = bv;
      if (a) a[i] = wg_syn_hc_a(bv);
      if (amt) { int64_t v = wg_syn_hc_amt(seed, r); amt[i] = wg_int128{v < 0 ? -1 : 0, (uint64_t)v}; }
      if (x) x[i] = wg_syn_hc_x(seed, r);
    }
  });
}

// ---- string GROUP BY keys (consumeBatchStrGroup, exec/aggregate.go:3038) ----
// strIdx.GetOrInsertRefAt hands out len(h.strGroupStates) to a string it has not
// seen (aggregate.go:3083-3090), i.e. group indexes in first-appearance order;
// NULL rows take strNullGroupSlot (aggregate.go:3078), the NULL key here.
struct StrIndex {
  std::unordered_map<std::string, int32_t> index;
  std::vector<std::string> strings;
};

void* or_strindex_new(void) { return new StrIndex(); }

int64_t or_strindex_map(void* h, const uint32_t* offs, const uint8_t* bytes, const uint64_t* valid, int64_t len,
                        const uint32_t* sel, int64_t sel_len, int32_t* ids) {
  StrIndex* x = (StrIndex*)h;
  const int64_t n = sel ? sel_len : len;
  for (int64_t i = 0; i < n; ++i) {
    const int64_t r = sel ? (int64_t)sel[i] : i;
    if (valid && !((valid[r >> 6] >> (r & 63)) & 1)) { ids[r] = 0; continue; }
    std::string key((const char*)bytes + offs[r], offs[r + 1] - offs[r]);
    auto it = x->index.find(key);
    if (it == x->index.end()) {
      const int32_t g = (int32_t)x->strings.size();
      x->strings.push_back(key);
      it = x->index.emplace(std::move(key), g).first;
    }
    ids[r] = it->second;
  }
  return (int64_t)x->strings.size();
}

int64_t or_strindex_get(void* h, int64_t id, uint8_t* out, int64_t cap) {
  StrIndex* x = (StrIndex*)h;
  if (id < 0 || id >= (int64_t)x->strings.size()) return -1;
  const std::string& s = x->strings[(size_t)id];
  if (out) std::memcpy(out, s.data(), std::min<size_t>(s.size(), (size_t)cap));
  return (int64_t)s.size();
}

void or_strindex_free(void* h) { delete (StrIndex*)h; }

}  // extern "C"
