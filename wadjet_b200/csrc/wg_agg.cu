// wg_agg.cu — exec.HashAggregate and the fused pipeline on the GPU.
//
// Host policy around the device table (see wg_agg.cuh for the slot layout):
//  - The table is an open-addressing array of (cap + 2) slots, cap a power of
//    two, at most 75% of cap regular groups (inserts beyond are refused and
//    flagged, never silently dropped).
//  - A launch that provably cannot reach the limit (groups known so far + rows
//    in the launch) runs straight through. Otherwise a small table is
//    snapshotted, the launch runs, and on an overflow the snapshot is restored,
//    the table grown 4x and the launch replayed; a large table is fed in chunks
//    that each fit, growing between chunks. Either way every row is applied
//    exactly once.
//  - Low-cardinality int keys use a CTA-private shared-memory table flushed to
//    the global table at the end of the kernel.
#include "wg_internal.h"
#include "wg_launch.cuh"
#include "wg_hc.cuh"

#include <algorithm>
#include <type_traits>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace wg {
wg_status resolve_pred(const wg_predicate& p, int32_t type_id, wgd::Pred* out);
wg_status join_view_fused(wg_join* j, wgd::JoinView* v);
int32_t join_probe_key_col(wg_join* j);
int32_t join_n_payload(wg_join* j);
int32_t join_payload_type(wg_join* j, int i);
int32_t join_payload_scale(wg_join* j, int i);
bool join_payload_nullable(wg_join* j, int i);
bool join_payload_range(wg_join* j, int i, long long* lo, long long* hi);
bool join_is_grace(wg_join* j);
int join_grace_passes(wg_join* j);
wg_status join_grace_pass(wg_join* j, int g, wg_join** out);
int64_t join_max_fanout(wg_join* j);
int32_t join_type_of(wg_join* j);
}  // namespace wg

using namespace wgd;

namespace {

constexpr int64_t kSnapshotMaxBytes = 256LL << 20;
constexpr double kMaxLoad = 0.75;
// spill partitions take hash bits [20, 30): below the slot bits of any table up
// to 2^34 slots, so each partition's keys spread over its whole table
constexpr int kSpillPartShift = 20;

__global__ void init_table_kernel(unsigned long long* slots, int64_t words, int sw, Layout L) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < words; i += (int64_t)gridDim.x * blockDim.x)
    slots[i] = L.init[i % sw];
}

__device__ __forceinline__ bool slot_used(const Layout& L, const unsigned long long* s, uint64_t idx, uint64_t cap) {
  if (L.key_words == 0) return idx == 0;
  if (idx >= cap) return s[L.key_words] != 0;  // special slots: any rows
  if (L.key_words == 1) return s[0] != WG_EMPTY_KEY;
  return !(s[0] == ~0ULL && s[1] == ~0ULL);
}

// Fold every group of table (Ls, Ts) into (Ld, Td): MergeSink, table growth and
// layout upgrades are all this one kernel.
// compact_n >= 0: the source is a compact result of compact_n groups, slot
// list[i] for group i (every listed slot a group; a key equal to the empty
// pattern is that key's group, and the slot at the view's capacity + 1, when
// listed, is the NULL-key group).
template <int NA>
__global__ void fold_kernel(Layout Ls, Table Ts, Layout Ld, Table Td, int32_t* err, int64_t compact_n,
                            const int64_t* list) {
  Credit cr;
  const uint64_t cap = Ts.mask + 1;
  const uint64_t n = compact_n >= 0 ? (uint64_t)compact_n : Ls.key_words == 0 ? 1 : cap + 2;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = compact_n >= 0 ? (uint64_t)list[i] : i;
    const unsigned long long* s = Ts.slots + idx * Ls.slot_words;
    if (compact_n < 0 && !slot_used(Ls, s, idx, cap)) continue;
    unsigned long long k0 = 0, k1 = 0;
    bool knull = false;
    if (Ls.key_words >= 1) {
      if (idx == cap + 1) knull = true;
      else if (compact_n < 0 && idx == cap) { k0 = Ls.key_words == 1 ? WG_EMPTY_KEY : ~0ULL; k1 = ~0ULL; }
      else { k0 = s[0]; if (Ls.key_words == 2) k1 = s[1]; }
    }
    const LayoutAcc ls{Ls}, ld{Ld};
    unsigned long long* d = find_global(ld, Td, k0, k1, knull, err, &cr);
    if (!d) continue;
    Contrib<NA> c;
    slot_contrib<NA>(ls, s, c);
    apply<NA, false>(ld, d, c, s[Ls.key_words]);
  }
  cr.release(Td);
}

// out[i] = the slot list[i] of a table (slot_words words each): one partition's
// groups appended to a spilled aggregate's compact result.
__global__ void gather_slots_kernel(const unsigned long long* slots, int sw, const int64_t* list, int64_t n,
                                    unsigned long long* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n * sw; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = i / sw;
    out[i] = slots[list[g] * sw + (i - g * sw)];
  }
}

// Spill input normalisation. The rows a selection vector keeps, gathered into
// a contiguous column (es = 4, 8 or 16 bytes).
__global__ void spill_gather_kernel(const char* src, int es, const uint32_t* sel, int64_t n, char* dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = sel ? (int64_t)sel[i] : i;
    if (es == 4) ((uint32_t*)dst)[i] = __ldg((const uint32_t*)src + row);
    else if (es == 8) ((unsigned long long*)dst)[i] = __ldg((const unsigned long long*)src + row);
    else ((longlong2*)dst)[i] = __ldg((const longlong2*)src + row);
  }
}

// One validity flag per row (1 = a value; every row when `valid` is null), of
// the rows a selection vector keeps.
__global__ void spill_valid_kernel(const uint64_t* valid, const uint32_t* sel, int64_t n, int32_t* ok) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = sel ? (int64_t)sel[i] : i;
    ok[i] = valid ? (int32_t)((__ldg(valid + (row >> 6)) >> (row & 63)) & 1ULL) : 1;
  }
}

// Validity words (LSB first) from per-row flags.
__global__ void pack_valid_kernel(const int32_t* ok, int64_t n, uint64_t* words) {
  const int64_t nw = (n + 63) / 64;
  for (int64_t w = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x) {
    uint64_t bits = 0;
    for (int b = 0; b < 64; ++b) {
      const int64_t r = w * 64 + b;
      if (r < n && ok[r]) bits |= 1ULL << b;
    }
    words[w] = bits;
  }
}

__global__ void iota_kernel(int64_t* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) out[i] = i;
}

// The used slots' indices into `list` (any order). Each thread checks
// kCompactK slots per pass (coalesced per step), the CTA sums its finds with a
// block scan and takes one range of `list` with a single atomic per pass,
// instead of one atomic per warp on the shared counter.
constexpr int kCompactK = 8;
__global__ void compact_kernel(Layout L, Table T, int64_t* list, unsigned long long* count) {
  __shared__ unsigned warp_sum[32];
  __shared__ unsigned long long s_base;
  const uint64_t cap = T.mask + 1;
  const uint64_t n = L.key_words == 0 ? 1 : cap + 2;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const uint64_t span = (uint64_t)blockDim.x * kCompactK;
  for (uint64_t base = (uint64_t)blockIdx.x * span; base < n; base += (uint64_t)gridDim.x * span) {
    unsigned bits = 0, c = 0;
#pragma unroll
    for (int j = 0; j < kCompactK; ++j) {
      const uint64_t i = base + (uint64_t)j * blockDim.x + threadIdx.x;
      if (i < n && slot_used(L, T.slots + i * L.slot_words, i, cap)) { bits |= 1u << j; ++c; }
    }
    unsigned x = c;  // inclusive scan within the warp
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned y = __shfl_up_sync(WG_FULL_MASK, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
      unsigned z = lane < nw ? warp_sum[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(WG_FULL_MASK, z, o);
        if (lane >= o) z += y;
      }
      if (lane < nw) warp_sum[lane] = z;
      if (lane == nw - 1) s_base = z ? atomicAdd(count, (unsigned long long)z) : 0ULL;
    }
    __syncthreads();
    unsigned long long off = s_base + (w > 0 ? warp_sum[w - 1] : 0u) + x - c;
#pragma unroll
    for (int j = 0; j < kCompactK; ++j)
      if (bits >> j & 1u) list[off++] = (int64_t)(base + (uint64_t)j * blockDim.x + threadIdx.x);
    __syncthreads();  // warp_sum and s_base are reused by the next pass
  }
}

struct FinalArgs {
  Layout L;
  Table T;
  const int64_t* list;
  int64_t start, n;
  int32_t key_cls[WG_MAX_KEYS];
  int32_t agg_func[WG_MAX_AGGS];
  int32_t agg_out[WG_MAX_AGGS];   // 0 = int64 out, 1 = float64 out
  int32_t agg_scale[WG_MAX_AGGS];
  // export (raw)
  int64_t* keys; uint8_t* key_valid; int64_t* count; int64_t* i64; double* f64; wg_int128* dec; uint8_t* has;
  int64_t stride;                 // n_groups (rows per key / aggregate block)
  // emit (finalized)
  void* out[WG_MAX_KEYS + WG_MAX_AGGS];
  uint8_t* out_valid[WG_MAX_KEYS + WG_MAX_AGGS];
};

__device__ __forceinline__ void slot_agg_state(const Layout& L, const unsigned long long* s, int a, int64_t& cnt,
                                               int64_t& iv, double& fv, unsigned long long& dlo,
                                               unsigned long long& dhi, bool& has) {
  const AggD g = L.agg[a];
  const unsigned long long rows = s[L.key_words];
  const unsigned long long nulls = g.null_off >= 0 ? s[g.null_off] : 0;
  cnt = (int64_t)(rows - nulls);
  has = cnt > 0;
  iv = 0; fv = 0.0; dlo = 0; dhi = 0;
  switch (g.kind) {
    case K_SUM_I64: case K_MIN_I64: case K_MAX_I64: iv = (int64_t)s[g.off]; break;
    case K_SUM_F64: fv = as_f(s[g.off]); break;
    case K_MIN_F64: case K_MAX_F64: fv = ord_to_f64(s[g.off]); break;
    case K_SUM_DEC: case K_MIN_DEC: case K_MAX_DEC: dlo = s[g.off]; dhi = s[g.off + 1]; break;
    default: break;
  }
  if (!has && g.kind >= K_MIN_I64) { iv = 0; fv = 0.0; dlo = 0; dhi = 0; }
}

__device__ __forceinline__ int64_t slot_key(const Layout& L, const unsigned long long* s, int k) {
  if (L.key_words == 1) return (int64_t)s[0];
  const unsigned long long w = s[L.key_word[k]];
  return L.key_i32[k] ? (int64_t)(int32_t)(uint32_t)(w >> L.key_shift[k]) : (int64_t)w;
}

// Whether key column k of a packed slot is NULL (its bit in the NULL field).
__device__ __forceinline__ bool slot_key_null(const Layout& L, const unsigned long long* s, uint64_t idx, uint64_t cap,
                                              int k) {
  if (L.key_words == 1) return idx == cap + 1;
  if (L.key_words != 2 || L.null_word < 0 || idx == cap) return false;
  return (s[L.null_word] >> (L.null_shift + k)) & 1ULL;
}

__global__ void export_kernel(FinalArgs A) {
  const Layout& L = A.L;
  const uint64_t cap = A.T.mask + 1;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < A.n; g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = (uint64_t)A.list[A.start + g];
    const unsigned long long* s = A.T.slots + idx * L.slot_words;
    const int64_t o = g;
    for (int k = 0; k < L.n_keys; ++k) {
      const bool valid = !slot_key_null(L, s, idx, cap, k);
      if (A.keys) A.keys[k * A.stride + o] = valid ? slot_key(L, s, k) : 0;
      if (A.key_valid) A.key_valid[k * A.stride + o] = valid ? 1 : 0;
    }
    for (int a = 0; a < L.n_aggs; ++a) {
      int64_t cnt, iv; double fv; unsigned long long dlo, dhi; bool has;
      slot_agg_state(L, s, a, cnt, iv, fv, dlo, dhi, has);
      if (A.count) A.count[a * A.stride + o] = cnt;
      if (A.i64) A.i64[a * A.stride + o] = iv;
      if (A.f64) A.f64[a * A.stride + o] = fv;
      if (A.dec) { wg_int128 d; d.hi = (int64_t)dhi; d.lo = dlo; A.dec[a * A.stride + o] = d; }
      if (A.has) A.has[a * A.stride + o] = has ? 1 : 0;
    }
  }
}

// writeAccToColumn (internal/engine/exec/aggregate_partial_spill.go:1855-1960)
__global__ void emit_kernel(FinalArgs A) {
  const Layout& L = A.L;
  const uint64_t cap = A.T.mask + 1;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < A.n; g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = (uint64_t)A.list[A.start + g];
    const unsigned long long* s = A.T.slots + idx * L.slot_words;
    for (int k = 0; k < L.n_keys; ++k) {
      const bool valid = !slot_key_null(L, s, idx, cap, k);
      const int64_t v = valid ? slot_key(L, s, k) : 0;
      if (A.key_cls[k] == WG_CLS_I32) ((int32_t*)A.out[k])[g] = (int32_t)v;
      else ((int64_t*)A.out[k])[g] = v;
      A.out_valid[k][g] = valid ? 1 : 0;
    }
    for (int a = 0; a < L.n_aggs; ++a) {
      int64_t cnt, iv; double fv; unsigned long long dlo, dhi; bool has;
      slot_agg_state(L, s, a, cnt, iv, fv, dlo, dhi, has);
      const int kind = L.agg[a].kind;
      const int func = A.agg_func[a];
      const bool dec = kind == K_SUM_DEC || kind == K_MIN_DEC || kind == K_MAX_DEC;
      const bool flt = kind == K_SUM_F64 || kind == K_MIN_F64 || kind == K_MAX_F64;
      bool valid = true;
      double f = 0.0;
      int64_t i = 0;
      if (func == WG_AGG_COUNT) {
        i = cnt; f = __ll2double_rn(cnt);
      } else if (func == WG_AGG_SUM || func == WG_AGG_AVG) {
        if (cnt == 0) valid = false;
        else {
          f = dec ? dec_to_f64((int64_t)dhi, dlo, A.agg_scale[a]) : flt ? fv : __ll2double_rn(iv);
          if (func == WG_AGG_AVG) f = __ddiv_rn(f, __ll2double_rn(cnt));
          i = iv;
        }
      } else {  // MIN / MAX
        if (!has) valid = false;
        else {
          f = dec ? dec_to_f64((int64_t)dhi, dlo, A.agg_scale[a]) : flt ? fv : __ll2double_rn(iv);
          i = dec ? (int64_t)dlo : flt ? (int64_t)fv : iv;
        }
      }
      const int c = L.n_keys + a;
      if (A.agg_out[a] == 0) ((int64_t*)A.out[c])[g] = valid ? i : 0;
      else ((double*)A.out[c])[g] = valid ? f : 0.0;
      A.out_valid[c][g] = valid ? 1 : 0;
    }
  }
}

// ---------------------------------------------------------------------------
// Exchange of partial group state between ranks (one process per GPU). A
// state row is [flag][the group's slot words]: flag 0 = a regular key, 1 = the
// group whose key equals the table's empty pattern, 2 = the NULL-key group.
// Rows are routed like partitionFor (internal/engine/exec/partitioned_agg.go:221):
// owner = high 64 bits of route_hash * parts, with route_hash = fibHash(key)
// for one int key (routeHashInt64, :515), packedHash(lo, hi) for a packed key
// (routeHashPacked, :529) and routeNullHash for a NULL key (:197).
// ---------------------------------------------------------------------------
constexpr unsigned long long kRouteNullHash = 0x9ae16a3b2f90404fULL;

__device__ __forceinline__ int state_flag(const Layout& L, const unsigned long long* s, uint64_t idx, uint64_t cap) {
  if (L.key_words == 0) return 0;
  if (idx == cap + 1) return 2;
  if (idx == cap) return 1;
  if (L.key_words == 1) return s[0] == WG_EMPTY_KEY ? 1 : 0;
  return (s[0] == ~0ULL && s[1] == ~0ULL) ? 1 : 0;
}

__device__ __forceinline__ uint32_t state_owner(const Layout& L, const unsigned long long* s, int flag, int parts) {
  unsigned long long h = 0;
  if (L.key_words == 0) return 0;
  if (flag == 2) h = kRouteNullHash;
  else if (L.key_words == 1) h = (flag == 1 ? WG_EMPTY_KEY : s[0]) * 0x9E3779B97F4A7C15ULL;
  else if (flag == 0 && L.null_word >= 0 && ((s[L.null_word] >> L.null_shift) & 0xFULL) != 0) {
    h = kRouteNullHash;  // routeHashPacked: a row with any NULL key column (partitioned_agg.go:530)
  } else {
    const unsigned long long lo = flag == 1 ? ~0ULL : s[0], hi = flag == 1 ? ~0ULL : s[1];
    const unsigned long long a = lo ^ 0x9E3779B97F4A7C15ULL, b = hi ^ 0x517CC1B727220A95ULL;
    h = __umul64hi(a, b) ^ (a * b) ^ (lo + hi);
  }
  return (uint32_t)__umul64hi(h, (unsigned long long)parts);
}

// Rows per owner (counts[p], zeroed by the caller).
__global__ void state_count_kernel(Layout L, Table T, const int64_t* list, int64_t n, int parts,
                                   unsigned long long* counts) {
  const uint64_t cap = T.mask + 1;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = (uint64_t)list[g];
    const unsigned long long* s = T.slots + idx * L.slot_words;
    atomicAdd(&counts[state_owner(L, s, state_flag(L, s, idx, cap), parts)], 1ULL);
  }
}

// Every group's state row at cursor[owner] (cursor starts at each owner's
// first row; rows of one owner come out in any order).
__global__ void state_scatter_kernel(Layout L, Table T, const int64_t* list, int64_t n, int parts,
                                     unsigned long long* cursor, unsigned long long* rows) {
  const uint64_t cap = T.mask + 1;
  const int W = 1 + L.slot_words;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t idx = (uint64_t)list[g];
    const unsigned long long* s = T.slots + idx * L.slot_words;
    const int flag = state_flag(L, s, idx, cap);
    const unsigned long long at = atomicAdd(&cursor[state_owner(L, s, flag, parts)], 1ULL);
    unsigned long long* r = rows + at * W;
    r[0] = (unsigned long long)flag;
    for (int w = 0; w < L.slot_words; ++w) r[1 + w] = s[w];
  }
}

// MergeSink of state rows laid out by Ls into the table (Ld, Td).
template <int NA>
__global__ void state_merge_kernel(Layout Ls, const unsigned long long* rows, int64_t n, Layout Ld, Table Td,
                                   int32_t* err) {
  Credit cr;
  const int W = 1 + Ls.slot_words;
  const LayoutAcc ls{Ls}, ld{Ld};
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < n; g += (int64_t)gridDim.x * blockDim.x) {
    const unsigned long long* r = rows + g * W;
    const unsigned long long* s = r + 1;
    const int flag = (int)r[0];
    unsigned long long k0 = 0, k1 = 0;
    bool knull = false;
    if (Ls.key_words >= 1) {
      if (flag == 2) knull = true;
      else if (flag == 1) { k0 = Ls.key_words == 1 ? WG_EMPTY_KEY : ~0ULL; k1 = ~0ULL; }
      else { k0 = s[0]; if (Ls.key_words == 2) k1 = s[1]; }
    }
    unsigned long long* d = find_global(ld, Td, k0, k1, knull, err, &cr);
    if (!d) continue;
    Contrib<NA> c;
    slot_contrib<NA>(ls, s, c);
    apply<NA, false>(ld, d, c, s[Ls.key_words]);
  }
  cr.release(Td);
}

template <int NA>
void launch_fold(const Layout& Ls, const Table& Ts, const Layout& Ld, const Table& Td, int32_t* err, unsigned grid,
                 cudaStream_t st, int64_t compact_n = -1, const int64_t* list = nullptr) {
  fold_kernel<NA><<<grid, 256, 0, st>>>(Ls, Ts, Ld, Td, err, compact_n, list);
}

unsigned grid_cap(wg::Ctx* ctx, int64_t n, int block, int per_sm = 16) {
  int64_t b = (n + block - 1) / block;
  b = std::min<int64_t>(b, (int64_t)ctx->sm_count * per_sm);
  return (unsigned)std::max<int64_t>(b, 1);
}

int env_int(const char* name, int dflt) {
  const char* v = std::getenv(name);
  return v && *v ? std::atoi(v) : dflt;
}

}  // namespace

// ---------------------------------------------------------------------------
// host aggregate object
// ---------------------------------------------------------------------------
struct wg_agg {
  wg::Ctx* ctx;
  std::vector<int32_t> key_cols;
  std::vector<wg_agg_spec> specs;
  int64_t hint = 0;
  bool resolved = false;
  bool finalized = false;
  // resolved schema (from the first batch's virtual schema)
  std::vector<int32_t> key_types;
  std::vector<int32_t> in_cls, in_scale, out_type, kind;
  std::vector<bool> nullable;
  wgd::Layout L{};
  // table
  wg::DevBuf table, backup, ctr;   // ctr: [0] n_groups, [1] overflow flag
  uint64_t cap = 0;
  int shift = 0;
  int64_t known_groups = 0;        // regular groups, exact as of the last read-back
  int64_t upper_groups = 0;        // upper bound since then
  // the keys of every group in the table lie in [dom_lo, dom_hi]: dom 0 = no
  // group yet, 1 = so bounded, 2 = unknown (a launch whose keys had no known
  // range, a merge, a partitioned or spilled run)
  int dom = 0;
  long long dom_lo = 0, dom_hi = -1;
  // finalize
  wg::DevBuf list, cnt;
  int64_t n_out = 0;
  std::vector<wg::DevBuf> emit_bufs, emit_valid;
  bool emitted = false;
  int32_t last_shape = -1;         // compiled shape of the last fused launch
  // a single STRING / BYTES key: the dictionary whose ids the table groups by
  // (str_keyed -1 no input yet, 0 an integer key, 1 a string key)
  wg::StrDict* sdict = nullptr;
  int str_keyed = -1;
  // Spill (the table for the expected groups does not fit the HBM ledger): the
  // consume calls partition their rows by the key hash's top bits into runs in
  // pinned host memory; finalize aggregates one partition at a time into a
  // small table and appends its groups to a compact result, which then stands
  // in for the table (`spilled`).
  bool spill = false;
  bool spilled = false;
  int spill_pbits = 0;
  uint64_t small_cap = 0;
  struct SpillRun {
    int64_t rows = 0;
    std::vector<int64_t> off;        // start of each partition in the run (np + 1)
    std::vector<char*> col;          // pinned host copy of each plan input column
    std::vector<char*> ok;           // pinned host copy of each nullable input's validity flags
  };
  std::vector<SpillRun> runs;
  std::vector<std::pair<char*, int64_t>> host_blocks;  // pinned arena (kept for the next query)
  size_t block_idx = 0;
  int64_t block_used = 0, host_bytes = 0;
  // the spilled consume calls' shape, replayed per partition at finalize
  std::vector<wg_column> sp_cols;
  std::vector<int> sp_map, sp_es;    // caller column -> plan input, plan input element size
  std::vector<wg_predicate> sp_filters;
  std::vector<wg_expr> sp_exprs;
  std::vector<wg::DevBuf> sp_dev;    // device staging per plan input column
  // NULLs and selection vectors: per plan input whether it is nullable; the
  // gathered rows, validity flags (int32 per row, moved with the rows) and
  // packed words of a consume call; the flags' and words' staging at finalize
  std::vector<bool> sp_null;
  std::vector<wg::DevBuf> sp_norm, sp_ok, sp_words, sp_okdev;
  // export staging (kept for the next export): every output field of a chunk
  // side by side on the device, read back in one copy through pinned memory
  wg::DevBuf exp_dev;
  // the in-HBM key-hash reorder's copy of the input and its counters (kept for
  // the next query: allocating and freeing GBs per query costs milliseconds)
  std::vector<wg::DevBuf> part_bufs;
  wg::DevBuf part_counts, part_offs;
  char* exp_host = nullptr;
  int64_t exp_host_bytes = 0;
  // Two-level partitioned mode (wg_hc.cuh), for tables far larger than L2:
  // each consume call writes its filtered rows, as the columns the aggregate
  // reads, to a first-level run in HBM; finalize re-partitions the runs into
  // buckets and aggregates each bucket in one SM's shared memory, leaving a
  // compact result that stands in for the table (`spilled`).
  bool hc = false;
  int hc_b1 = 0, hc_b2 = 0;
  int hc_tile = 8192;               // rows per tile of the partition kernels
  std::vector<int32_t> hc_cols;     // copy columns: caller-numbered virtual columns (keys, then agg inputs)
  std::vector<int32_t> hc_es, hc_cls;
  struct HcRun {
    int64_t rows = 0;
    std::vector<int64_t> off1;      // first-level partition starts (np1 + 1)
    std::vector<wg::DevBuf> cols;
    wg::DevBuf bucket;              // per row: its bucket within the partition
  };
  std::vector<HcRun> hc_runs;
  std::vector<HcRun> hc_free;       // runs of earlier queries, kept for reuse
  std::vector<wg::DevBuf> hc_copy2;
  wg::DevBuf hc_hist, hc_counts1, hc_offs1, hc_dev, hc_out, hc_scalars;
  wg::DevBuf hc_hll;                // distinct-key sketch of the rows consumed so far
  ~wg_agg() {
    for (auto& b : host_blocks) cudaFreeHost(b.first);
    if (exp_host) cudaFreeHost(exp_host);
  }
};

namespace wg {

// Most threads one aggregate launch runs (pipeline grids of up to 4 CTAs of
// 768 threads per SM; the batched mode checks its tables after the run).
static int64_t max_launch_threads(Ctx* ctx) { return (int64_t)ctx->sm_count * 4 * 768; }

static wgd::Table table_view(wg_agg* a) {
  wgd::Table T;
  T.slots = a->table.as<unsigned long long>();
  T.n_groups = a->ctr.as<unsigned long long>();
  T.overflow = (int32_t*)(a->ctr.as<unsigned long long>() + 1);
  T.shift = a->shift;
  T.mask = a->cap - 1;
  T.limit = (unsigned long long)((double)a->cap * kMaxLoad);
  // Large tables: a thread reserves up to 16 groups at a time, so the
  // reservation counter is not one contended atomic per new group. Unused
  // reservations held by running threads read as groups, so the chunk is kept
  // to where they stay under 1/8 of the limit (credit_slack); small tables
  // reserve one group per insert.
  const int64_t per = (int64_t)T.limit / (8 * max_launch_threads(a->ctx));
  T.credit_chunk = (int32_t)std::max<int64_t>(1, std::min<int64_t>(16, 1 + per));
  return T;
}

// Reservations that running threads may hold beyond the groups they inserted.
static int64_t credit_slack(wg_agg* a) {
  return (int64_t)(table_view(a).credit_chunk - 1) * max_launch_threads(a->ctx);
}

static int64_t table_words(const wg_agg* a, uint64_t cap) {
  return a->L.key_words == 0 ? a->L.slot_words : (int64_t)(cap + 2) * a->L.slot_words;
}

// Build the slot layout from kinds/nullability.
static void build_layout(wg_agg* a) {
  wgd::Layout& L = a->L;
  const int nk = (int)a->key_cols.size();
  int w = L.key_words;
  const int rows_at = w++;
  bool need_even = L.key_words == 2;
  for (size_t i = 0; i < a->specs.size(); ++i) {
    wgd::AggD& g = L.agg[i];
    g.kind = a->kind[i];
    const int kw = wgd::kind_words(g.kind);
    if (g.kind == wgd::K_MIN_DEC || g.kind == wgd::K_MAX_DEC) { if (w & 1) ++w; need_even = true; }
    g.off = kw > 0 ? w : -1;
    w += kw;
    g.null_off = (a->nullable[i] && a->specs[i].input_col >= 0) ? w++ : -1;
    g.vcol = a->specs[i].input_col;
  }
  if (need_even && (w & 1)) ++w;
  L.slot_words = w;
  L.n_keys = nk;
  L.n_aggs = (int)a->specs.size();
  for (int i = 0; i < WG_MAX_SLOT_WORDS; ++i) L.init[i] = 0;
  if (L.key_words == 1) L.init[0] = WG_EMPTY_KEY;
  if (L.key_words == 2) { L.init[0] = ~0ULL; L.init[1] = ~0ULL; }
  L.init[rows_at] = 0;
  for (size_t i = 0; i < a->specs.size(); ++i) {
    const wgd::AggD& g = L.agg[i];
    switch (g.kind) {
      case wgd::K_MIN_I64: L.init[g.off] = 0x7FFFFFFFFFFFFFFFULL; break;
      case wgd::K_MAX_I64: L.init[g.off] = 0x8000000000000000ULL; break;
      case wgd::K_MIN_F64: L.init[g.off] = ~0ULL; break;
      case wgd::K_MAX_F64: L.init[g.off] = 0ULL; break;
      case wgd::K_MIN_DEC: L.init[g.off] = ~0ULL; L.init[g.off + 1] = 0x7FFFFFFFFFFFFFFFULL; break;
      case wgd::K_MAX_DEC: L.init[g.off] = 0ULL; L.init[g.off + 1] = 0x8000000000000000ULL; break;
      default: break;
    }
  }
}

static wg_status init_table(wg_agg* a, DevBuf& buf, uint64_t cap) {
  Ctx* ctx = a->ctx;
  const int64_t words = table_words(a, cap);
  WG_TRY(buf.alloc(ctx, words * 8));
  init_table_kernel<<<grid_cap(ctx, words, 256), 256, 0, ctx->stream>>>(buf.as<unsigned long long>(), words,
                                                                       a->L.slot_words, a->L);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  return WG_OK;
}

static uint64_t cap_for(int64_t groups) {
  uint64_t cap = 1024;
  while ((double)cap * kMaxLoad < (double)groups * 1.34) cap <<= 1;  // target ~56% load
  return cap;
}

static int log2u(uint64_t v) { int l = 0; while ((1ULL << l) < v) ++l; return l; }

static void run_fold(wg_agg* a, const wgd::Layout& Ls, const wgd::Table& Ts, const wgd::Layout& Ld, const wgd::Table& Td,
                     int64_t compact_n = -1, const int64_t* list = nullptr) {
  Ctx* ctx = a->ctx;
  const int64_t n = compact_n >= 0 ? std::max<int64_t>(compact_n, 1) : Ls.key_words == 0 ? 1 : (int64_t)(Ts.mask + 3);
  const unsigned grid = grid_cap(ctx, n, 256);
  if (Ls.n_aggs <= 4) launch_fold<4>(Ls, Ts, Ld, Td, ctx->dev_error, grid, ctx->stream, compact_n, list);
  else launch_fold<8>(Ls, Ts, Ld, Td, ctx->dev_error, grid, ctx->stream, compact_n, list);
  ctx->count_launch();
}

// Re-create the table with capacity new_cap and/or a new layout, folding every
// group across.
static wg_status rebuild_table(wg_agg* a, uint64_t new_cap, const wgd::Layout& new_layout) {
  Ctx* ctx = a->ctx;
  const wgd::Layout old_L = a->L;
  const wgd::Table old_T = table_view(a);
  DevBuf old_table = std::move(a->table);
  DevBuf old_ctr = std::move(a->ctr);
  a->L = new_layout;
  a->cap = a->L.key_words == 0 ? 1 : new_cap;
  a->shift = 64 - log2u(a->cap);
  WG_TRY(init_table(a, a->table, a->cap));
  WG_TRY(a->ctr.alloc(ctx, 64));
  WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, ctx->stream));
  wgd::Table old_view = old_T;
  old_view.slots = old_table.as<unsigned long long>();
  old_view.n_groups = old_ctr.as<unsigned long long>();
  old_view.overflow = (int32_t*)(old_ctr.as<unsigned long long>() + 1);
  run_fold(a, old_L, old_view, a->L, table_view(a));
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  a->backup.reset();
  return WG_OK;
}

static int agg_kind(int func, int cls) {
  switch (func) {
    case WG_AGG_COUNT: return wgd::K_COUNT;
    case WG_AGG_SUM: case WG_AGG_AVG:  // initFlatAccums, aggregate.go:6060-6090
      if (cls == WG_CLS_F32 || cls == WG_CLS_F64) return wgd::K_SUM_F64;
      if (cls == WG_CLS_DEC) return wgd::K_SUM_DEC;
      if (cls == WG_CLS_I64 && func == WG_AGG_AVG) return wgd::K_SUM_F64;
      return wgd::K_SUM_I64;
    case WG_AGG_MIN:
      return (cls == WG_CLS_F32 || cls == WG_CLS_F64) ? wgd::K_MIN_F64 : cls == WG_CLS_DEC ? wgd::K_MIN_DEC : wgd::K_MIN_I64;
    case WG_AGG_MAX:
      return (cls == WG_CLS_F32 || cls == WG_CLS_F64) ? wgd::K_MAX_F64 : cls == WG_CLS_DEC ? wgd::K_MAX_DEC : wgd::K_MAX_I64;
  }
  return -1;
}

// Virtual schema of one launch: type, scale and nullability per virtual column.
struct VSchema {
  std::vector<int32_t> type, scale;
  std::vector<bool> nullable;
};

// resolveIndices (aggregate.go:1296): fix the path and the accumulators from the
// first batch's schema.
static wg_status agg_resolve(wg_agg* a, const VSchema& vs) {
  const int nk = (int)a->key_cols.size();
  a->key_types.clear();
  for (int k = 0; k < nk; ++k) {
    const int kc = a->key_cols[k];
    if (kc < 0 || kc >= (int)vs.type.size()) return fail(WG_E_INVALID, "group column out of range");
    const int cls = class_of(vs.type[kc]);
    if (cls != WG_CLS_I32 && cls != WG_CLS_I64)
      return fail(WG_E_UNSUPPORTED, "GROUP BY key is not an integer-class column (string keys are not on the GPU path)");
    a->key_types.push_back(vs.type[kc]);
  }
  std::memset(&a->L, 0, sizeof(a->L));
  if (nk == 0) a->L.key_words = 0;
  else if (nk == 1) a->L.key_words = 1;
  else {
    // buildPackedLayout (packed_hash.go:386): widest-first into two 64-bit words
    int total = 0;
    for (int k = 0; k < nk; ++k) total += class_of(a->key_types[k]) == WG_CLS_I32 ? 4 : 8;
    if (nk > WG_MAX_KEYS || total > 16) return fail(WG_E_UNSUPPORTED, "composite key does not pack into 128 bits");
    a->L.key_words = 2;
    int next_wide = 0;
    for (int k = 0; k < nk; ++k)
      if (class_of(a->key_types[k]) == WG_CLS_I64) { a->L.key_word[k] = next_wide++; a->L.key_shift[k] = 0; a->L.key_i32[k] = 0; }
    std::vector<std::pair<int, int>> slots;
    for (int w = next_wide; w < 2; ++w) { slots.push_back({w, 0}); slots.push_back({w, 32}); }
    size_t nn = 0;
    for (int k = 0; k < nk; ++k)
      if (class_of(a->key_types[k]) == WG_CLS_I32) {
        a->L.key_word[k] = slots[nn].first; a->L.key_shift[k] = slots[nn].second; a->L.key_i32[k] = 1; ++nn;
      }
    // the first 32-bit half the packing leaves unused holds the NULL field
    a->L.null_word = -1;
    a->L.null_shift = 0;
    if (nn < slots.size()) { a->L.null_word = slots[nn].first; a->L.null_shift = slots[nn].second; }
  }
  for (int k = 0; k < nk; ++k) a->L.key_vcol[k] = a->key_cols[k];
  const size_t na = a->specs.size();
  a->in_cls.assign(na, WG_CLS_BAD); a->in_scale.assign(na, 0); a->out_type.assign(na, 0); a->kind.assign(na, 0);
  a->nullable.assign(na, false);
  for (size_t i = 0; i < na; ++i) {
    const wg_agg_spec& s = a->specs[i];
    if (s.func < WG_AGG_SUM || s.func > WG_AGG_AVG) return fail(WG_E_UNSUPPORTED, "aggregate function is not on the GPU path");
    if (s.input_col < 0) {
      if (s.func != WG_AGG_COUNT) return fail(WG_E_INVALID, "only COUNT may omit its input column");
    } else {
      if (s.input_col >= (int)vs.type.size()) return fail(WG_E_INVALID, "aggregate column out of range");
      a->in_cls[i] = class_of(vs.type[s.input_col]);
      a->in_scale[i] = vs.scale[s.input_col];
      if (a->in_cls[i] == WG_CLS_BAD) return fail(WG_E_UNSUPPORTED, "aggregate input type is not on the GPU path");
      a->nullable[i] = vs.nullable[s.input_col];
    }
    a->kind[i] = agg_kind(s.func, a->in_cls[i]);
    int ot = s.out_type;
    if (ot == 0) {  // aggOutputType (plan.go:9968) / minMaxOutputType (aggregate.go:4611)
      if (s.func == WG_AGG_COUNT) ot = WG_TYPE_INT64;
      else if (s.func == WG_AGG_SUM || s.func == WG_AGG_AVG) ot = WG_TYPE_FLOAT64;
      else ot = (a->in_cls[i] == WG_CLS_I32 || a->in_cls[i] == WG_CLS_I64) ? WG_TYPE_INT64 : WG_TYPE_FLOAT64;
    }
    if (ot != WG_TYPE_INT64 && ot != WG_TYPE_FLOAT64) return fail(WG_E_UNSUPPORTED, "aggregate output type must be INT64 or FLOAT64");
    a->out_type[i] = ot;
  }
  if (na > WG_MAX_AGGS) return fail(WG_E_UNSUPPORTED, "more than 8 aggregates");
  build_layout(a);
  if (a->L.slot_words > WG_MAX_SLOT_WORDS) return fail(WG_E_UNSUPPORTED, "aggregate state too wide");
  // the two-level mode keeps only the groups that outgrow a bucket's shared
  // table in HBM: a small table, grown on demand
  a->cap = a->L.key_words == 0 ? 1 : cap_for(a->hc ? (int64_t(1) << 16) : std::max<int64_t>(a->hint, 1024));
  if (a->hc) a->small_cap = a->cap;
  a->shift = 64 - log2u(a->cap);
  wg_status st = init_table(a, a->table, a->cap);
  if (st == WG_E_NOMEM && a->L.key_words >= 1 && a->ctx->pinned_spill_bytes > 0 && env_int("WG_AGG_SPILL", 1) != 0) {
    // spill: one small table per hash partition, each holding about 1/16 of
    // what the ledger has left
    const int64_t left = a->ctx->ledger.budget() > 0 ? a->ctx->ledger.budget() - a->ctx->ledger.used() : (int64_t(1) << 40);
    const int64_t full = (int64_t)a->cap * a->L.slot_words * 8;
    int pbits = 1;
    while (pbits < 10 && (full >> pbits) > left / 16) ++pbits;
    a->spill = true;
    a->spill_pbits = pbits;
    a->small_cap = cap_for(std::max<int64_t>(1024, std::max<int64_t>(a->hint, 1024) >> pbits));
    a->cap = a->small_cap;
    a->shift = 64 - log2u(a->cap);
    st = init_table(a, a->table, a->cap);
  }
  WG_TRY(st);
  WG_TRY(a->ctr.alloc(a->ctx, 64));
  WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, a->ctx->stream));
  a->known_groups = 0;
  a->upper_groups = 0;
  a->dom = 0;
  a->resolved = true;
  return WG_OK;
}

// Upgrade the layout when a batch brings NULLs to an aggregate whose state has
// no null counter yet.
static wg_status agg_check_nullable(wg_agg* a, const VSchema& vs) {
  bool need = false;
  std::vector<bool> nn = a->nullable;
  for (size_t i = 0; i < a->specs.size(); ++i) {
    const int c = a->specs[i].input_col;
    if (c >= 0 && vs.nullable[c] && !nn[i]) { nn[i] = true; need = true; }
  }
  if (!need) return WG_OK;
  wg_agg tmp;  // compute the new layout on a scratch copy of the shape
  tmp.key_cols = a->key_cols; tmp.specs = a->specs; tmp.kind = a->kind; tmp.nullable = nn;
  tmp.L = a->L;
  build_layout(&tmp);
  for (int k = 0; k < WG_MAX_KEYS; ++k) tmp.L.key_vcol[k] = a->L.key_vcol[k];
  if (tmp.L.slot_words > WG_MAX_SLOT_WORDS) return fail(WG_E_UNSUPPORTED, "aggregate state too wide");
  a->nullable = nn;
  return rebuild_table(a, a->cap, tmp.L);
}

static wg_status refresh_groups(wg_agg* a) {
  int64_t v[2];
  WG_TRY(read_back_i64(a->ctx, (const int64_t*)a->ctr.get(), v, 2));
  a->known_groups = v[0];
  a->upper_groups = v[0];
  return WG_OK;
}

// Launch on the compiled shape of the plan (ls.P.shape), or the generic kernel.
static void launch_pipeline_shape(const LaunchSpec& ls, cudaStream_t st) {
  if (ls.P.shape != wgd::SHAPE_GENERIC) {
    launch_static_shape(ls, st);
    return;
  }
  if (ls.P.L.n_aggs <= 4) launch_pipeline_t<4, wgd::DynShape>(ls, st);
  else launch_pipeline_t<8, wgd::DynShape>(ls, st);
}

// The compiled shape to launch a finished plan with; WG_SPECIALIZE=0 forces
// the generic kernel.
static int32_t pick_shape(const wgd::Plan& P) {
  if (env_int("WG_SPECIALIZE", 1) == 0) return wgd::SHAPE_GENERIC;
  return wgd::shape_of(P);
}

// The table's layout with a plan's compact column numbering.
static wgd::Layout launch_layout(const wg_agg* a, const wgd::Plan& P) {
  wgd::Layout L = a->L;
  for (int k = 0; k < WG_MAX_KEYS; ++k) L.key_vcol[k] = P.L.key_vcol[k];
  for (int i = 0; i < WG_MAX_AGGS; ++i) L.agg[i].vcol = P.L.agg[i].vcol;
  return L;
}

static wg_status launch_pipeline(wg_agg* a, const LaunchSpec& ls, int64_t n_items) {
  Ctx* ctx = a->ctx;
  LaunchSpec l2 = ls;
  wgd::Plan& P = l2.P;
  P.T = table_view(a);
  // a launch with more threads than the launch policy's slack assumes takes
  // one reservation per insert
  const int64_t threads = (int64_t)ls.grid * (ls.tile ? 32 * (1 + ls.cfg.consumers) : ls.block);
  if (threads > max_launch_threads(ctx)) P.T.credit_chunk = 1;
  P.L = launch_layout(a, ls.P);
  P.n_items = n_items;
  if (l2.tile) l2.cfg.n_tiles = (n_items + l2.cfg.rows - 1) / l2.cfg.rows;
  P.shape = pick_shape(P);
  a->last_shape = P.shape;
  launch_pipeline_shape(l2, ctx->stream);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  return WG_OK;
}

}  // namespace wg

// Everything the fused pipeline needs to run one device-resident input.
struct PipelineRun {
  wg_agg* agg;
  const wg_batch_desc* in;      // device descriptors
  int32_t n_filters;
  const wg_predicate* filters;
  wg_join* join;
  int32_t n_exprs;
  const wg_expr* exprs;
  bool no_partition = false;    // set on the reordered copy (hash partitioning runs once)
  bool defer_check = false;     // a launch that needs no read-back returns without waiting for it
                                // (windowed host input checks the device error word once, at the end)
  bool str_ids = false;         // the key column holds a string dictionary's ids
};

namespace wg {

// Column rebasing for a row window without a selection vector: the kernel sees
// rows [0, n); data pointers move by row0 (row0 is a multiple of 64 so the
// validity bitmap moves by whole words).
static void rebase_cols(wgd::Plan& P, int64_t row0) {
  for (int j = 0; j < P.n_in; ++j) {
    const int64_t es = P.in[j].cls == WG_CLS_I32 || P.in[j].cls == WG_CLS_F32 ? 4 : P.in[j].cls == WG_CLS_DEC ? 16 : 8;
    P.in[j].data = (const char*)P.in[j].data + row0 * es;
    if (P.in[j].valid) P.in[j].valid += row0 >> 6;
  }
}

static wg_status build_plan(const PipelineRun& r, wgd::Plan& P, VSchema& vs, std::vector<int>& in_map) {
  std::memset(&P, 0, sizeof(P));
  const wg_batch_desc* in = r.in;
  const int ncols = in->ncols;
  const int npay = r.join ? join_n_payload(r.join) : 0;
  // virtual schema in caller numbering
  vs.type.clear(); vs.scale.clear(); vs.nullable.clear();
  for (int c = 0; c < ncols; ++c) {
    vs.type.push_back(in->cols[c].type_id); vs.scale.push_back(in->cols[c].scale);
    vs.nullable.push_back(in->cols[c].valid_words != nullptr);
  }
  // an unmatched LEFT-join row carries NULL build columns
  const bool outer = r.join && join_type_of(r.join) == WG_JOIN_LEFT;
  for (int p = 0; p < npay; ++p) {
    vs.type.push_back(join_payload_type(r.join, p)); vs.scale.push_back(join_payload_scale(r.join, p));
    vs.nullable.push_back(outer || join_payload_nullable(r.join, p));
  }
  if (r.n_exprs < 0 || r.n_exprs > WG_MAX_EXPRS) return fail(WG_E_UNSUPPORTED, "at most 2 projection expressions");
  for (int e = 0; e < r.n_exprs; ++e) {
    const wg_expr& x = r.exprs[e];
    if (x.result_type != WG_TYPE_INT64 && x.result_type != WG_TYPE_FLOAT64) return fail(WG_E_INVALID, "expression result type must be INT64 or FLOAT64");
    bool nul = false;
    for (int k = 0; k < x.n_ops && k < WG_EXPR_MAX_OPS; ++k)
      if (x.ops[k].opcode == WG_EXPR_COL) {
        if (x.ops[k].arg < 0 || x.ops[k].arg >= ncols + npay) return fail(WG_E_INVALID, "expression column out of range");
        nul = nul || vs.nullable[x.ops[k].arg];
      }
    vs.type.push_back(x.result_type); vs.scale.push_back(0); vs.nullable.push_back(nul);
  }
  // referenced input columns → compact indices
  in_map.assign(ncols, -1);
  std::vector<int> order;
  auto use = [&](int c) -> wg_status {
    if (c < 0) return WG_OK;
    if (c >= ncols) return WG_OK;
    if (in_map[c] < 0) {
      if ((int)order.size() >= WG_MAX_IN) return fail(WG_E_UNSUPPORTED, "more than 8 input columns referenced");
      in_map[c] = (int)order.size();
      order.push_back(c);
    }
    return WG_OK;
  };
  if (r.n_filters < 0 || r.n_filters > WG_MAX_FILTERS) return fail(WG_E_UNSUPPORTED, "at most 4 filter predicates");
  for (int f = 0; f < r.n_filters; ++f) {
    if (r.filters[f].col < 0 || r.filters[f].col >= ncols)
      return fail(WG_E_INVALID, "filter column " + std::to_string(r.filters[f].col) + " does not exist in the input schema");
    WG_TRY(use(r.filters[f].col));
  }
  if (r.join) {
    const int pk = join_probe_key_col(r.join);
    if (pk < 0 || pk >= ncols) return fail(WG_E_INVALID, "probe key column out of range");
    const int pcls = class_of(in->cols[pk].type_id);
    if (pcls != WG_CLS_I32 && pcls != WG_CLS_I64) return fail(WG_E_UNSUPPORTED, "probe key is not an integer-class column");
    WG_TRY(use(pk));
  }
  for (int e = 0; e < r.n_exprs; ++e)
    for (int k = 0; k < r.exprs[e].n_ops && k < WG_EXPR_MAX_OPS; ++k)
      if (r.exprs[e].ops[k].opcode == WG_EXPR_COL) WG_TRY(use(r.exprs[e].ops[k].arg));
  for (int32_t kc : r.agg->key_cols) WG_TRY(use(kc));
  for (const wg_agg_spec& s : r.agg->specs) WG_TRY(use(s.input_col));
  const int nin = (int)order.size();
  auto vmap = [&](int c) -> int {  // caller vcol → compact vcol
    if (c < 0) return -1;
    if (c < ncols) return in_map[c];
    return nin + (c - ncols);
  };
  P.n_in = nin;
  for (int j = 0; j < nin; ++j) {
    const wg_column& c = in->cols[order[j]];
    const int cls = class_of(c.type_id);
    if (cls == WG_CLS_BAD) return fail(WG_E_UNSUPPORTED, "input column type is not on the GPU path");
    P.in[j] = wgd::DCol{c.data, c.valid_words, cls, c.scale};
    P.vcls[j] = cls; P.vscale[j] = c.scale;
  }
  P.n_filters = r.n_filters;
  for (int f = 0; f < r.n_filters; ++f) {
    WG_TRY(resolve_pred(r.filters[f], in->cols[r.filters[f].col].type_id, &P.filt[f]));
    P.filt[f].col = in_map[r.filters[f].col];
  }
  if (r.join) {
    P.has_join = 1;
    WG_TRY(join_view_fused(r.join, &P.join));
    P.probe_col = in_map[join_probe_key_col(r.join)];
    for (int p = 0; p < npay; ++p) { P.vcls[nin + p] = class_of(vs.type[ncols + p]); P.vscale[nin + p] = vs.scale[ncols + p]; }
  } else {
    P.join.n_pay = 0;
  }
  P.n_exprs = r.n_exprs;
  for (int e = 0; e < r.n_exprs; ++e) {
    const wg_expr& x = r.exprs[e];
    wgd::ExprD& d = P.expr[e];
    if (x.n_ops < 1 || x.n_ops > WG_EXPR_MAX_OPS) return fail(WG_E_INVALID, "expression needs 1..12 operations");
    d.n_ops = x.n_ops;
    d.result_cls = x.result_type == WG_TYPE_INT64 ? WG_CLS_I64 : WG_CLS_F64;
    int depth = 0;
    for (int k = 0; k < x.n_ops; ++k) {
      const wg_expr_op& o = x.ops[k];
      d.opc[k] = o.opcode;
      d.arg[k] = o.opcode == WG_EXPR_COL ? vmap(o.arg) : 0;
      if (o.opcode == WG_EXPR_CONST_F) std::memcpy(&d.imm[k], &o.imm_f64, 8);
      else d.imm[k] = o.imm_i64;
      if (o.opcode <= WG_EXPR_CONST_F) ++depth;
      else if (o.opcode <= WG_EXPR_AND) { if (depth < 2) return fail(WG_E_INVALID, "expression stack underflow"); --depth; }
      else return fail(WG_E_INVALID, "unknown expression opcode");
      if (depth > 4) return fail(WG_E_UNSUPPORTED, "expression deeper than 4 stack entries");
    }
    if (depth != 1) return fail(WG_E_INVALID, "expression must leave exactly one value");
    P.vcls[nin + npay + e] = d.result_cls;
    P.vscale[nin + npay + e] = 0;
  }
  for (int j = 0; j < nin + npay + r.n_exprs; ++j) pow10_divisor_host(P.vscale[j], &P.vdiv_b[j], &P.vdiv_y[j]);
  for (int k = 0; k < (int)r.agg->key_cols.size(); ++k) P.L.key_vcol[k] = vmap(r.agg->key_cols[k]);
  for (size_t i = 0; i < r.agg->specs.size(); ++i) P.L.agg[i].vcol = vmap(r.agg->specs[i].input_col);
  P.sel = in->sel;
  P.n_items = in->sel ? in->sel_len : in->len;
  return WG_OK;
}

static wg_status run_partitioned(const PipelineRun& r, const wgd::Plan& P0, const std::vector<int>& in_map,
                                 bool* done);
static wg_status spill_consume(const PipelineRun& r, const wgd::Plan& P0, const std::vector<int>& in_map);
static bool hc_eligible(const PipelineRun& r, const wgd::Plan& P);
static wg_status hc_consume(const PipelineRun& r, const wgd::Plan& P0);
static wg_status agg_compact(wg_agg* a);

// Run the fused kernel over a device-resident input with the overflow policy.
static bool is_str_type(int32_t t) { return t == WG_TYPE_STRING || t == WG_TYPE_BYTES; }

// The batch column holding the aggregate's single string GROUP BY key, or -1.
static int str_key_col(const wg_agg* a, const wg_batch_desc* in) {
  if (a->key_cols.size() != 1 || in->ncols < 0 || (in->ncols > 0 && !in->cols)) return -1;
  const int kc = a->key_cols[0];
  return kc >= 0 && kc < in->ncols && is_str_type(in->cols[kc].type_id) ? kc : -1;
}

static wg_status run_device(const PipelineRun& r) {
  wg_agg* a = r.agg;
  Ctx* ctx = a->ctx;
  if (a->finalized) return fail(WG_E_STATE, "aggregate already finalized");
  // a string key reaches the table as its dictionary's ids (the consume entry
  // points map it first)
  for (int kc : a->key_cols)
    if (kc >= 0 && kc < r.in->ncols && is_str_type(r.in->cols[kc].type_id))
      return fail(WG_E_UNSUPPORTED, a->key_cols.size() == 1
                                        ? "a string GROUP BY key of a windowed host pipeline run"
                                        : "a string column in a composite GROUP BY key is not on the GPU path");
  if (a->str_keyed >= 0 && a->str_keyed != (r.str_ids ? 1 : 0))
    return fail(WG_E_INVALID, "the GROUP BY column changed between a string and an integer type");
  a->str_keyed = r.str_ids ? 1 : 0;
  LaunchSpec ls;
  VSchema vs;
  std::vector<int> in_map;
  WG_TRY(build_plan(r, ls.P, vs, in_map));
  if (!a->resolved) {
    a->hc = hc_eligible(r, ls.P);
    WG_TRY(agg_resolve(a, vs));
  } else {
    WG_TRY(agg_check_nullable(a, vs));
  }
  ls.P.err = ctx->dev_error;
  const int64_t n_items = ls.P.n_items;
  if (n_items == 0) return WG_OK;
  const int64_t fan = r.join ? std::max<int64_t>(1, join_max_fanout(r.join)) : 1;
  if (a->hc && !r.no_partition) { a->dom = 2; return hc_consume(r, ls.P); }
  if (a->spill && !r.no_partition) { a->dom = 2; return spill_consume(r, ls.P, in_map); }
  if (!r.no_partition) {
    bool done = false;
    WG_TRY(run_partitioned(r, ls.P, in_map, &done));
    if (done) { a->dom = 2; return WG_OK; }
  }

  // kernel shape: shared-memory table for low-cardinality single int keys
  bool any_null_words = false, any_dec_minmax = false;
  for (int i = 0; i < a->L.n_aggs; ++i) {
    any_null_words |= a->L.agg[i].null_off >= 0;
    any_dec_minmax |= a->L.agg[i].kind == wgd::K_MIN_DEC || a->L.agg[i].kind == wgd::K_MAX_DEC;
  }
  // a kernel compiled for this query shape runs 768-thread CTAs (48 warps per
  // SM), the generic one 512-thread CTAs
  wgd::Plan probe = ls.P;
  probe.L = launch_layout(a, ls.P);
  const bool stat = pick_shape(probe) != wgd::SHAPE_GENERIC;
  // vector kernel (U rows per lane): compiled shapes over contiguous input whose
  // columns start on 16-byte boundaries, no join or the direct-payload one
  bool vec_ok = stat && ls.P.sel == nullptr && ls.P.n_in > 0 && (!ls.P.has_join || ls.P.join.direct);
  for (int j = 0; j < ls.P.n_in; ++j) vec_ok = vec_ok && ((uintptr_t)ls.P.in[j].data % 16 == 0);
  ls.vec = vec_ok && env_int("WG_VEC", 2) != 0 ? 2 : 0;
  const int env_bps = env_int("WG_AGG_BLOCKS_PER_SM", 0);
  const int pref_bps = env_bps > 0 ? env_bps : 2;
  int blocks_per_sm = pref_bps;
  // vector kernel: 768-thread CTAs (48 warps per SM, no L2 prefetcher: 2.57 ms
  // against 2.81 ms for 512 threads with it on the 2^28-row star join);
  // WG_VEC_BLOCK=512 selects the prefetching variant
  ls.block = ls.vec ? (env_int("WG_VEC_BLOCK", 768) == 512 ? 512 : 768)
                    : stat ? wgd::StatShape<wgd::ShapeStarJoin>::kBlock : wgd::DynShape::kBlock;
  // copies of each float SUM per shared slot (lane-striped, see apply)
  int n_fsum = 0;
  for (int i = 0; i < a->L.n_aggs; ++i) n_fsum += a->L.agg[i].kind == wgd::K_SUM_F64;
  // float SUMs in a shared table: `rep` lane-striped float copies, or
  // (WG_SMEM_FIXED=1) exact fixed-point accumulation in two words each with
  // 32-bit atomics, order-independent but measured slower on the star join
  // (3 dependent limb atomics per row against one float atomic)
  const bool fixed = n_fsum > 0 && env_int("WG_SMEM_FIXED", 0) != 0;
  const int max_rep = n_fsum > 0 && !fixed ? std::max(1, std::min(8, env_int("WG_SMEM_REPLICAS", 4))) : 1;
  // an odd number of 8-byte words per shared slot spreads the slots over all
  // 16 bank pairs (an even stride maps them onto a few)
  auto stride_for = [&](int rep) { return (a->L.slot_words + n_fsum * (fixed ? 2 : rep - 1)) | 1; };
  auto slots_for = [&](int bps, int rep) {
    return (int)std::min<int64_t>(((int64_t)ctx->max_smem_optin / bps - 2048) / (stride_for(rep) * 8), 16384);
  };
  // a shared table runs at most 5/8 full for the expected groups, 3/4 when it
  // fills a whole SM (one CTA per SM)
  auto fits = [&](int64_t groups, int slots) {
    return slots >= 256 && groups * (blocks_per_sm == 1 ? 4 : 8) <= (int64_t)slots * (blocks_per_sm == 1 ? 3 : 5);
  };
  // a string dictionary's ids: the groups are at most its strings and the NULL key
  const int64_t expect = r.str_ids ? strdict_size(a->sdict) + 1 : std::max<int64_t>(a->hint, a->known_groups);
  const bool smem_ok = env_int("WG_AGG_SMEM", 1) != 0 && a->L.key_words == 1 && !any_null_words && !any_dec_minmax &&
                       expect > 0;
  // prefer the kernel's CTAs per SM, then as many float-SUM copies as still
  // fit; a table too large for that takes a whole SM (one CTA)
  int S = 0, rep = 1;
  bool found = false;
  const int bps_try[2] = {pref_bps, 1};
  for (int t = 0; t < 2 && smem_ok && !found; ++t) {
    if (t == 1 && (env_bps > 0 || pref_bps == 1)) break;
    blocks_per_sm = bps_try[t];
    for (int r = max_rep; r >= 1 && !found; r /= 2)
      if (fits(expect, slots_for(blocks_per_sm, r))) { S = slots_for(blocks_per_sm, r); rep = r; found = true; }
  }
  if (!found) {
    blocks_per_sm = pref_bps;
    S = slots_for(blocks_per_sm, 1);
  }
  // dense GROUP BY: the key is a join payload column whose value range is known
  // and small, or a small string dictionary's ids, so the shared table is indexed by key - min (no hashing, no key
  // compare, no insert) and holds exactly one slot per possible key
  {
    long long glo = 0, ghi = -1;
    const int kv = ls.P.L.key_vcol[0];
    const int npay = r.join ? join_n_payload(r.join) : 0;
    bool ranged = false;
    if (r.join != nullptr && join_type_of(r.join) == WG_JOIN_INNER && kv >= ls.P.n_in && kv < ls.P.n_in + npay)
      ranged = join_payload_range(r.join, kv - ls.P.n_in, &glo, &ghi);
    else if (r.str_ids && kv < ls.P.n_in) {  // a string dictionary's ids: [0, its strings)
      glo = 0;
      ghi = strdict_size(a->sdict) - 1;
      ranged = true;
    }
    const bool cand = smem_ok && env_int("WG_GROUP_DENSE", 1) != 0 && a->L.n_keys == 1 && ranged && ghi >= glo &&
                      ghi - glo < 16384;
    bool placed = false;
    for (int t = 0; t < 2 && cand && !placed; ++t) {
      if (t == 1 && (env_bps > 0 || pref_bps == 1)) break;
      const int bps = bps_try[t];
      const int64_t budget = (int64_t)ctx->max_smem_optin / bps - 2048;
      for (int r2 = max_rep; r2 >= 1 && !placed; r2 /= 2)
        if ((ghi - glo + 1) * stride_for(r2) * 8 <= budget) {
          blocks_per_sm = bps;
          rep = r2;
          S = (int)(ghi - glo + 1);
          placed = true;
        }
    }
    if (placed) {
      found = true;
      ls.P.gdense = 1;
      ls.P.gmin = glo;
    }
  }
  ls.smem = found;
  // a shared table that takes a whole SM: one CTA of 1024 threads for the vector kernel
  if (ls.vec && ls.smem && blocks_per_sm == 1 && env_int("WG_VEC_WIDE", 1) != 0) ls.block = 1024;
  // self-staged vector kernel (WG_STAGE=1; off by default: on the star join
  // it measured slower than the plain vector kernel, whose L2 prefetch already
  // hides the HBM latency): one CTA of 1024 threads whose 32 warps each
  // double-buffer a 64-row chunk of every input column next to the shared
  // table, when the table (as many float-SUM copies as still fit) leaves room
  int64_t stage_bytes = 0;
  if (ls.vec && ls.smem && env_int("WG_STAGE", 0) != 0) {
    int64_t chunk = 0;
    for (int j = 0; j < ls.P.n_in; ++j) chunk += 64 * wgd::cls_bytes(ls.P.in[j].cls);
    const int64_t sb = 32 * 2 * chunk;
    const int64_t budget = (int64_t)ctx->max_smem_optin - sb - 2048;
    int S2 = 0, rep2 = 0;
    const int save_bps = blocks_per_sm;
    blocks_per_sm = 1;  // the 3/4 fill rule of a table that has the SM to itself
    for (int r2 = max_rep; r2 >= 1 && rep2 == 0 && budget > 0; r2 /= 2) {
      if (ls.P.gdense) {
        if ((int64_t)S * stride_for(r2) * 8 <= budget) { S2 = S; rep2 = r2; }
      } else {
        const int cand = (int)std::min<int64_t>(budget / (stride_for(r2) * 8), 16384);
        if (fits(expect, cand)) { S2 = cand; rep2 = r2; }
      }
    }
    blocks_per_sm = save_bps;
    if (rep2 > 0) {
      ls.stage = true;
      ls.block = 1024;
      blocks_per_sm = 1;
      S = S2;
      rep = rep2;
      stage_bytes = sb;
    }
  }
  ls.P.smem_slots = ls.smem ? S : 0;
  ls.P.smem_rep = fixed ? -1 : rep;
  ls.P.smem_sw = stride_for(rep);
  ls.smem_bytes = ls.smem ? (size_t)S * ls.P.smem_sw * 8 : 0;
  if (ls.stage) {
    ls.P.stage_off = (int32_t)((ls.smem_bytes + 127) & ~size_t(127));
    ls.smem_bytes = (size_t)ls.P.stage_off + (size_t)stage_bytes;
  }
  ls.P.prefetch = std::max(0, env_int("WG_PREFETCH", 2));
  ls.P.smem_combine = env_int("WG_SMEM_COMBINE", 0) != 0;
  // many rows per group: most MIN/MAX updates cannot win, so read before the atomic
  const int mm = env_int("WG_MINMAX_TEST", -1);
  ls.P.minmax_test = mm >= 0 ? (mm != 0) : (n_items >= 8 * std::max<int64_t>(expect, 1));
  int64_t rows_per_cta = (int64_t)ls.block * (ls.vec ? ls.vec : 1);
  // a CTA with a shared table flushes up to all of its slots into the HBM table
  // at the end, every CTA onto the same hot groups: a small input takes fewer
  // CTAs, each with at least four rows per slot (16K rows at least), so the
  // flushes do not outweigh the rows (a 2^20-row query over 4096 groups: 80 us
  // on 148 CTAs, all flushing every group)
  if (ls.smem) {
    const int64_t floor_rows = env_int("WG_SMEM_ROWS_PER_CTA", 0) > 0 ? env_int("WG_SMEM_ROWS_PER_CTA", 0)
                                                                       : std::max<int64_t>(16384, 4 * (int64_t)S);
    rows_per_cta = std::max(rows_per_cta, floor_rows);
  }
  const int64_t want_ctas = (n_items + rows_per_cta - 1) / rows_per_cta + 1;
  ls.grid = (unsigned)std::min<int64_t>((int64_t)ctx->sm_count * blocks_per_sm, want_ctas);
  if (!ls.smem && !stat) ls.grid = (unsigned)std::min<int64_t>((int64_t)ctx->sm_count * 4, (n_items + 1023) / 1024 + 1);

  // TMA-staged tile kernel: contiguous input (no selection vector) whose columns
  // start on 16-byte boundaries; one persistent CTA per SM.
  bool aligned = ls.P.sel == nullptr && ls.P.n_in > 0;
  for (int j = 0; j < ls.P.n_in; ++j) aligned = aligned && ((uintptr_t)ls.P.in[j].data % 16 == 0);
  if (aligned && env_int("WG_TILE", 0) != 0 && n_items >= 4096) {
    wgd::TileCfg& c = ls.cfg;
    std::memset(&c, 0, sizeof(c));
    c.consumers = std::max(1, std::min(31, env_int("WG_TILE_CONSUMERS", 16)));
    c.stages = std::max(2, std::min(8, env_int("WG_TILE_STAGES", 2)));
    const int64_t budget = (int64_t)ctx->max_smem_optin - 1024;
    // the tile kernel's shared table keeps one copy of each float SUM and hashes
    ls.P.smem_rep = 1;
    if (ls.P.gdense) {
      ls.P.gdense = 0;
      ls.smem = smem_ok && fits(expect, S);
      ls.P.smem_slots = ls.smem ? S : 0;
    }
    ls.P.smem_sw = a->L.slot_words;
    const int64_t table_bytes = ls.smem ? (int64_t)S * a->L.slot_words * 8 : 0;
    for (int rows = std::max(64, env_int("WG_TILE_ROWS", 2048) & ~63); rows >= 64; rows /= 2) {
      int64_t off = 0;
      for (int j = 0; j < ls.P.n_in; ++j) {
        const int cls = ls.P.in[j].cls;
        c.es[j] = cls == WG_CLS_I32 || cls == WG_CLS_F32 ? 4 : cls == WG_CLS_DEC ? 16 : 8;
        c.col_off[j] = (int32_t)off;
        off += ((int64_t)rows * c.es[j] + 15) & ~int64_t(15);
      }
      // the shared-memory aggregate table shrinks to what the stages leave over
      int64_t tb = table_bytes;
      if (ls.smem && off * c.stages + tb > budget) {
        const int64_t s2 = (budget - off * c.stages) / (a->L.slot_words * 8);
        if (fits(expect, (int)s2)) { ls.P.smem_slots = (int)s2; tb = s2 * a->L.slot_words * 8; }
      }
      if (off * c.stages + tb <= budget) {
        c.rows = rows;
        c.stage_bytes = (int32_t)off;
        c.table_off = (int32_t)(off * c.stages);
        ls.tile = true;
        if (ls.smem && tb != table_bytes) ls.smem_bytes = (size_t)tb;
        break;
      }
    }
    if (ls.tile) {
      if (ls.smem && (int64_t)c.table_off + (int64_t)ls.P.smem_slots * a->L.slot_words * 8 > budget) {
        ls.smem = false;
        ls.P.smem_slots = 0;
      }
      ls.grid = (unsigned)ctx->sm_count;
    }
  }

  // shared-table row counters are 32-bit: a CTA's share of the rows stays below 2^31
  if (ls.smem && n_items / std::max<int64_t>(1, ls.grid) >= (int64_t(1) << 31)) {
    ls.smem = false;
    ls.P.smem_slots = 0;
    ls.smem_bytes = 0;
  }
  const wgd::Plan base = ls.P;
  // the room the launch policy plans with: the table's limit less the
  // reservations threads may hold unused
  auto limit = [&]() { return (int64_t)((double)a->cap * kMaxLoad) - credit_slack(a); };

  // The groups after this launch are at most the groups before it plus its
  // rows (times the join's fan-out), and, when every key so far and every key
  // of this launch lies in a known range (a group key that is an inner join's
  // payload column with a known value range), at most that range's size.
  bool dom_ok = false;
  long long dlo = 0, dhi = -1;
  if (a->L.key_words == 1 && a->L.n_keys == 1 && a->dom != 2 && r.join && join_type_of(r.join) == WG_JOIN_INNER) {
    const int kv = ls.P.L.key_vcol[0];
    const int npay = join_n_payload(r.join);
    if (kv >= ls.P.n_in && kv < ls.P.n_in + npay && join_payload_range(r.join, kv - ls.P.n_in, &dlo, &dhi) &&
        dhi >= dlo) {
      if (a->dom == 1) { dlo = std::min(dlo, a->dom_lo); dhi = std::max(dhi, a->dom_hi); }
      dom_ok = dhi - dlo < (int64_t(1) << 40);
    }
  }
  if (r.str_ids && a->L.key_words == 1 && a->dom != 2) {
    // a string dictionary's ids are dense: [0, its distinct strings)
    dlo = 0;
    dhi = std::max<int64_t>(0, strdict_size(a->sdict) - 1);
    if (a->dom == 1) { dlo = std::min(dlo, a->dom_lo); dhi = std::max(dhi, a->dom_hi); }
    dom_ok = true;
  }
  auto note_domain = [&]() {
    if (a->L.key_words == 0) return;
    if (dom_ok) { a->dom = 1; a->dom_lo = dlo; a->dom_hi = dhi; }
    else a->dom = 2;
  };
  int64_t bound = a->upper_groups + n_items * fan;
  // Threads that race to insert the same new key each hold a reservation until
  // they lose: a bound below the launch's rows must leave room for one per
  // launched thread beside the groups.
  int64_t race = 0;
  if (dom_ok && (int64_t)(dhi - dlo) + 2 < bound) {
    bound = (int64_t)(dhi - dlo) + 2;  // + a NULL key's group
    race = (int64_t)ls.grid * (ls.tile ? 32 * (1 + ls.cfg.consumers) : ls.block);
    if (bound + race > limit() && !a->spill) {  // a table that holds them, when it is small
      const int64_t nb = (int64_t)table_words(a, cap_for(bound + race)) * 8;
      const int64_t budget = ctx->ledger.budget();
      if (nb <= kSnapshotMaxBytes && (budget <= 0 || 2 * nb <= budget - ctx->ledger.used())) {
        WG_TRY(rebuild_table(a, cap_for(bound + race), a->L));
        WG_TRY(refresh_groups(a));
      }
    }
  }

  // 1) provably safe: one launch
  if (a->L.key_words == 0 || bound + race <= limit()) {
    WG_TRY(launch_pipeline(a, ls, n_items));
    a->upper_groups = a->L.key_words == 0 ? 0 : bound;
    note_domain();
    return r.defer_check ? WG_OK : check_device_error(ctx);
  }
  note_domain();  // the launches below insert this run's keys whatever they find
  // 2) small table: snapshot, run, replay on overflow. Threads that race to
  // insert the same new key each hold a reservation until they lose, so the
  // table leaves room for one per launched thread beside the expected groups
  // (else a first run over few hot keys could be refused and replayed).
  // Best effort: not for a spilled aggregate's partition tables, and only
  // within the snapshot size and half of what the HBM ledger has left.
  if (!a->spill) {
    const int64_t want = std::max<int64_t>(a->hint, a->known_groups) + (int64_t)ls.grid * ls.block;
    const int64_t nb = (int64_t)table_words(a, cap_for(want)) * 8;
    const int64_t budget = ctx->ledger.budget();
    if (limit() < want && nb <= kSnapshotMaxBytes && (budget <= 0 || 2 * nb <= budget - ctx->ledger.used())) {
      WG_TRY(rebuild_table(a, cap_for(want), a->L));
      WG_TRY(refresh_groups(a));
    }
  }
  const int64_t tbytes = table_words(a, a->cap) * 8;
  if (tbytes <= kSnapshotMaxBytes) {
    for (int attempt = 0; attempt < 16; ++attempt) {
      const int64_t tb = table_words(a, a->cap) * 8;
      WG_TRY(a->backup.ensure(ctx, tb + 64));
      WG_CUDA_TRY(cudaMemcpyAsync(a->backup.get(), a->table.get(), (size_t)tb, cudaMemcpyDeviceToDevice, ctx->stream));
      WG_CUDA_TRY(cudaMemcpyAsync(a->backup.as<char>() + tb, a->ctr.get(), 64, cudaMemcpyDeviceToDevice, ctx->stream));
      WG_TRY(launch_pipeline(a, ls, n_items));
      int64_t v[2];
      WG_TRY(read_back_checked(ctx, (const int64_t*)a->ctr.get(), v, 2));
      if ((int32_t)v[1] == 0) {
        a->known_groups = a->upper_groups = v[0];
        return WG_OK;
      }
      // overflow: restore, grow 4x, replay
      WG_CUDA_TRY(cudaMemcpyAsync(a->table.get(), a->backup.get(), (size_t)tb, cudaMemcpyDeviceToDevice, ctx->stream));
      WG_CUDA_TRY(cudaMemcpyAsync(a->ctr.get(), a->backup.as<char>() + tb, 64, cudaMemcpyDeviceToDevice, ctx->stream));
      WG_TRY(rebuild_table(a, a->cap * 4, a->L));
      WG_TRY(refresh_groups(a));
      const int64_t expect2 = std::max<int64_t>(a->hint, a->known_groups);
      if (ls.smem && !ls.P.gdense && !fits(expect2, S)) { ls.smem = false; ls.P.smem_slots = 0; ls.smem_bytes = 0; }
      if (table_words(a, a->cap) * 8 > kSnapshotMaxBytes) break;
    }
  }
  // 3) large table: chunks that each fit, growing between chunks
  WG_TRY(refresh_groups(a));
  if (ls.smem) { ls.smem = false; ls.P.smem_slots = 0; ls.smem_bytes = 0; if (!ls.tile) ls.grid = (unsigned)(ctx->sm_count * 4); }
  int64_t done = 0;
  const int64_t min_chunk = 1 << 20;
  while (done < n_items) {
    int64_t room = (limit() - a->known_groups) / fan;
    if (room < min_chunk && room < n_items - done) {
      WG_TRY(rebuild_table(a, cap_for(a->known_groups + std::min<int64_t>(n_items - done, 64LL << 20) * fan), a->L));
      WG_TRY(refresh_groups(a));
      room = (limit() - a->known_groups) / fan;
    }
    int64_t m = std::min<int64_t>(room, n_items - done);
    if (!ls.P.sel) m = std::max<int64_t>(64, m & ~int64_t(63));
    m = std::min<int64_t>(m, n_items - done);
    LaunchSpec lc = ls;
    lc.P = base;
    if (lc.P.sel) lc.P.sel = base.sel + done;
    else rebase_cols(lc.P, done);
    WG_TRY(launch_pipeline(a, lc, m));
    WG_TRY(refresh_groups(a));
    WG_TRY(check_device_error(ctx));
    int64_t v[2];
    WG_TRY(read_back_i64(ctx, (const int64_t*)a->ctr.get(), v, 2));
    if ((int32_t)v[1] != 0) return fail(WG_E_NOMEM, "aggregate table overflow on a checked chunk");
    done += m;
  }
  return WG_OK;
}

// Large tables: reorder the input by the top bits of the group key's table hash
// (part_count_kernel / part_scatter_kernel) and aggregate the reordered copy in
// order, so the atomics of any stretch of the run land in one L2-sized region
// of the table instead of all over HBM. Applies to inputs of at least 2^22
// rows, without a join, selection vector or NULL bitmaps, whose table is at
// least 64 MB (WG_AGG_PARTITION=0 turns it off; on the 2^28-row, 65.9M-group
// case it takes 40 ms against 59 ms direct). The reordered copy is kept on the
// aggregate for the next query; when the ledger has no room for it the input
// runs directly. *done says whether it ran.
static wg_status run_partitioned(const PipelineRun& r, const wgd::Plan& P0, const std::vector<int>& in_map,
                                 bool* done) {
  *done = false;
  wg_agg* a = r.agg;
  Ctx* ctx = a->ctx;
  const int64_t n = P0.n_items;
  // a string dictionary's ids are dense and its table small per id: the
  // reorder does not pay for them (2.85 against 3.28 ms at 2^24 rows, 2^20 ids)
  if (env_int("WG_AGG_PARTITION", 1) == 0 || r.join || r.str_ids || P0.sel || a->L.key_words == 0 ||
      n < (int64_t(1) << 22))
    return WG_OK;
  for (int j = 0; j < P0.n_in; ++j)
    if (P0.in[j].valid) return WG_OK;
  const int64_t expect = std::max<int64_t>(a->hint, a->known_groups);
  const int64_t tbytes = std::max<int64_t>(table_words(a, a->cap), (int64_t)cap_for(expect) * a->L.slot_words) * 8;
  if (tbytes < (int64_t(64) << 20)) return WG_OK;
  int pbits = 1;
  while (pbits < 10 && (tbytes >> pbits) > (int64_t(32) << 20)) ++pbits;
  const int np = 1 << pbits;
  wgd::Plan P = P0;
  P.L = launch_layout(a, P0);
  P.err = ctx->dev_error;
  const unsigned grid = (unsigned)(ctx->sm_count * 2);
  DevBuf& counts = a->part_counts;
  DevBuf& offs = a->part_offs;
  WG_TRY(counts.ensure(ctx, (int64_t)np * grid * 4));
  WG_TRY(offs.ensure(ctx, (int64_t)np * grid * 8));
  wgd::part_count_kernel<<<grid, wgd::kPartThreads, wgd::part_count_smem(np), ctx->stream>>>(P, pbits, 64 - pbits, counts.as<uint32_t>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  std::vector<uint32_t> hc((size_t)np * grid);
  std::vector<unsigned long long> ho((size_t)np * grid);
  WG_CUDA_TRY(cudaMemcpyAsync(hc.data(), counts.get(), hc.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  unsigned long long acc = 0;
  for (size_t i = 0; i < hc.size(); ++i) { ho[i] = acc; acc += hc[i]; }  // partition-major, then CTA
  if ((int64_t)acc != n) return fail(WG_E_CUDA, "partition counts do not add up to the input rows");
  WG_CUDA_TRY(cudaMemcpyAsync(offs.get(), ho.data(), ho.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  std::vector<DevBuf>& bufs = a->part_bufs;
  if ((int)bufs.size() < P.n_in) bufs.resize((size_t)P.n_in);
  wgd::PartOut po{};
  for (int j = 0; j < P.n_in; ++j) {
    const int cls = P.in[j].cls;
    const int es = cls == WG_CLS_I32 || cls == WG_CLS_F32 ? 4 : cls == WG_CLS_DEC ? 16 : 8;
    if (bufs[(size_t)j].ensure(ctx, n * es) != WG_OK) {  // no room for the copy: run directly
      bufs.clear();
      set_error("");  // the ledger's refusal is handled here, not reported
      return WG_OK;
    }
    po.data[j] = bufs[(size_t)j].as<char>();
    po.es[j] = es;
  }
  if (cudaFuncSetAttribute(wgd::part_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)wgd::part_scatter_smem(np)) != cudaSuccess) {
    cudaGetLastError();  // the scatter's shared memory is refused: run directly
    return WG_OK;
  }
  wgd::part_scatter_kernel<<<grid, wgd::kPartThreads, wgd::part_scatter_smem(np), ctx->stream>>>(P, pbits, 64 - pbits,
                                                                        offs.as<unsigned long long>(), po);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  // the caller's batch with its referenced columns replaced by the reordered copy
  wg_batch_desc d2 = *r.in;
  std::vector<wg_column> c2(r.in->cols, r.in->cols + r.in->ncols);
  for (int c = 0; c < r.in->ncols; ++c)
    if (in_map[(size_t)c] >= 0) {
      c2[(size_t)c].data = bufs[(size_t)in_map[(size_t)c]].get();
      c2[(size_t)c].valid_words = nullptr;
      c2[(size_t)c].len = n;
    }
  d2.cols = c2.data();
  d2.len = n;
  d2.sel = nullptr;
  d2.sel_len = 0;
  PipelineRun r2 = r;
  r2.in = &d2;
  r2.no_partition = true;
  WG_TRY(run_device(r2));
  *done = true;
  return WG_OK;
}

// ---------------------------------------------------------------------------
// Two-level partitioned mode (wg_hc.cuh)
// ---------------------------------------------------------------------------
// Rows the mode needs before it pays (smaller inputs fit the direct path).
constexpr int64_t kHcMinRows = int64_t(1) << 22;
// Bucket CTAs per SM (WG_HC_BUCKET_CTAS, 1 or 2): two CTAs, each with half of
// the SM's shared memory and half as many groups per bucket, overlap one
// bucket's table sweeps with the other's row updates.
static int hc_bucket_ctas() { return env_int("WG_HC_BUCKET_CTAS", 2) == 1 ? 1 : 2; }

// The bucket kernel's shared table: slot stride (words) and slots per CTA. An
// odd stride spreads slots over the banks, but a packed key (and an Int128
// MIN/MAX) is updated with 16-byte atomics, which need 16-byte aligned slots.
static void hc_table_shape(const wg_agg* a, int* ssw_out, int* slots_out, int* rep_out) {
  const int sw = a->L.slot_words;
  int n_fsum = 0;
  for (int i = 0; i < a->L.n_aggs; ++i) n_fsum += a->L.agg[i].kind == wgd::K_SUM_F64;
  const int rep = n_fsum > 0 ? 2 : 1;
  bool wide = a->L.key_words == 2;
  for (int i = 0; i < a->L.n_aggs; ++i)
    wide |= a->L.agg[i].kind == wgd::K_MIN_DEC || a->L.agg[i].kind == wgd::K_MAX_DEC;
  const int ssw = wide ? ((sw + n_fsum * (rep - 1) + 1) & ~1) : ((sw + n_fsum * (rep - 1)) | 1);
  const int ctas = hc_bucket_ctas();
  // per CTA: its share of the SM, less the 1 KB the runtime reserves per CTA and room for static shared memory
  const int64_t bytes = std::min<int64_t>(a->ctx->max_smem_optin, a->ctx->smem_per_sm / ctas - 1024) - 1024;
  *ssw_out = ssw;
  *slots_out = (int)std::min<int64_t>(bytes / (ssw * 8 + 4), 1 << 14);  // slot words and a used-slot list entry
  *rep_out = rep;
}

// Large-table GROUP BY on a plain input: no join, no selection vector, no
// validity bitmaps (a NULL key has no bucket), one or more integer keys, and a
// table for the expected groups of at least 64 MB (WG_AGG_HC=0 turns it off).
static bool hc_eligible(const PipelineRun& r, const wgd::Plan& P) {
  wg_agg* a = r.agg;
  if (env_int("WG_AGG_HC", 1) == 0 || r.join || P.sel || a->key_cols.empty() || P.n_items < kHcMinRows) return false;
  for (int j = 0; j < P.n_in; ++j)
    if (P.in[j].valid) return false;
  if ((int)a->specs.size() > WG_MAX_AGGS) return false;
  const int64_t words = (int64_t)a->key_cols.size() + 1 + 2 * (int64_t)a->specs.size();
  if ((int64_t)cap_for(std::max<int64_t>(a->hint, 1024)) * words * 8 < (int64_t(64) << 20)) return false;
  // room for the first-level run and the second-level copy of the input, and the result
  int64_t row_bytes = 0;
  for (int j = 0; j < P.n_in; ++j) row_bytes += wgd::cls_bytes(P.in[j].cls);
  const int64_t need = 2 * P.n_items * row_bytes + std::max<int64_t>(a->hint, 1024) * words * 8 * 5 / 4;
  const Ledger& L = a->ctx->ledger;
  return L.budget() <= 0 || L.budget() - L.used() >= need;
}

// The copy's column j as a plan input: class and element size from the plan
// that wrote it.
static wg_status hc_setup(wg_agg* a, const PipelineRun& r, const wgd::Plan& P0) {
  a->hc_cols.clear();
  auto add = [&](int32_t c) {
    if (c < 0) return;
    for (int32_t x : a->hc_cols) if (x == c) return;
    a->hc_cols.push_back(c);
  };
  for (int32_t k : a->key_cols) add(k);
  for (const wg_agg_spec& sp : a->specs) add(sp.input_col);
  if ((int)a->hc_cols.size() > WG_MAX_IN) return fail(WG_E_UNSUPPORTED, "more than 8 grouped or aggregated columns");
  a->hc_cls.clear();
  a->hc_es.clear();
  (void)r;
  (void)P0;
  // 256 first-level partitions; the second level's bits are chosen at finalize
  // from the distinct-key sketch
  a->hc_b1 = 8;
  a->hc_b2 = 0;
  a->hc_tile = env_int("WG_HC_TILE", 8192) == 4096 ? 4096 : 8192;
  WG_TRY(a->hc_hll.ensure(a->ctx, (int64_t(1) << wgd::kHllBits) * 4));
  WG_CUDA_TRY(cudaMemsetAsync(a->hc_hll.get(), 0, (size_t(1) << wgd::kHllBits) * 4, a->ctx->stream));
  return WG_OK;
}

// A plan over the copy's columns: inputs are the copy columns, keys and
// aggregates point at them, no filters, projections or join.
static wgd::Plan hc_plan(wg_agg* a, const std::vector<wg::DevBuf>& cols, int64_t n) {
  wgd::Plan P;
  std::memset(&P, 0, sizeof(P));
  P.n_in = (int32_t)a->hc_cols.size();
  for (int j = 0; j < P.n_in; ++j) {
    P.in[j] = wgd::DCol{cols[(size_t)j].get(), nullptr, a->hc_cls[(size_t)j], 0};
    P.vcls[j] = a->hc_cls[(size_t)j];
    pow10_divisor_host(0, &P.vdiv_b[j], &P.vdiv_y[j]);
  }
  P.L = a->L;
  auto idx = [&](int32_t c) -> int32_t {
    for (size_t j = 0; j < a->hc_cols.size(); ++j) if (a->hc_cols[j] == c) return (int32_t)j;
    return -1;
  };
  for (size_t k = 0; k < a->key_cols.size(); ++k) P.L.key_vcol[k] = idx(a->key_cols[k]);
  for (size_t i = 0; i < a->specs.size(); ++i) P.L.agg[i].vcol = idx(a->specs[i].input_col);
  P.n_items = n;
  P.err = a->ctx->dev_error;
  return P;
}

// The first level's kernels for one tile size and shape (hc_count_kernel and
// hc_scatter1_kernel on the same grid).
template <int TILE, class Sh>
static wg_status hc_first_level(wg_agg* a, const wgd::Plan& P, unsigned grid, int phase, const wgd::HcCols& out,
                                int n_pre, uint8_t* bucket_out) {
  Ctx* ctx = a->ctx;
  const int np1 = 1 << a->hc_b1;
  constexpr int threads = wgd::HcGeom<TILE>::threads;
  if (phase == 0) {
    wgd::hc_count_kernel<TILE, Sh><<<grid, threads, wgd::hc_count_smem(np1), ctx->stream>>>(
        P, a->hc_b1, a->hc_counts1.as<uint32_t>(), a->hc_hll.as<uint32_t>());
  } else {
    const size_t ss = wgd::hc_scatter_smem(TILE, np1, true);
    WG_CUDA_TRY(cudaFuncSetAttribute(wgd::hc_scatter1_kernel<TILE, Sh>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)ss));
    wgd::hc_scatter1_kernel<TILE, Sh><<<grid, threads, ss, ctx->stream>>>(P, a->hc_b1, a->hc_offs1.as<unsigned long long>(),
                                                                          out, n_pre, bucket_out);
  }
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  return WG_OK;
}

static wg_status hc_first_level_any(wg_agg* a, const wgd::Plan& P, bool stat, unsigned grid, int phase,
                                    const wgd::HcCols& out, int n_pre, uint8_t* bucket_out) {
  using HC = wgd::StatShape<wgd::ShapeHighCard>;
  if (a->hc_tile == 4096)
    return stat ? hc_first_level<4096, HC>(a, P, grid, phase, out, n_pre, bucket_out)
                : hc_first_level<4096, wgd::DynShape>(a, P, grid, phase, out, n_pre, bucket_out);
  return stat ? hc_first_level<8192, HC>(a, P, grid, phase, out, n_pre, bucket_out)
              : hc_first_level<8192, wgd::DynShape>(a, P, grid, phase, out, n_pre, bucket_out);
}

// One consume call: count the rows per partition and bucket, then write them
// to a first-level run.
static wg_status hc_consume(const PipelineRun& r, const wgd::Plan& P0) {
  wg_agg* a = r.agg;
  Ctx* ctx = a->ctx;
  if (a->hc_cols.empty()) WG_TRY(hc_setup(a, r, P0));
  wgd::Plan P = P0;
  P.L = launch_layout(a, P0);
  P.err = ctx->dev_error;
  const int np1 = 1 << a->hc_b1;
  // the copy columns in this call's compact numbering
  wgd::HcCols out{};
  out.n = (int32_t)a->hc_cols.size();
  std::vector<int32_t> cls((size_t)out.n);
  for (int j = 0; j < out.n; ++j) {
    const int32_t c = a->hc_cols[(size_t)j];
    int32_t v = -1;
    for (size_t k = 0; k < a->key_cols.size(); ++k) if (a->key_cols[k] == c) v = P.L.key_vcol[k];
    for (size_t i = 0; i < a->specs.size() && v < 0; ++i) if (a->specs[i].input_col == c) v = P.L.agg[i].vcol;
    if (v < 0) return fail(WG_E_INVALID, "grouped column missing from the plan");
    out.vcol[j] = v;
    cls[(size_t)j] = P.vcls[v];
    out.es[j] = wgd::cls_bytes(P.vcls[v]);
  }
  if (a->hc_cls.empty()) { a->hc_cls = cls; for (int j = 0; j < out.n; ++j) a->hc_es.push_back(out.es[j]); }
  else if (a->hc_cls != cls) return fail(WG_E_INVALID, "column classes changed between consume calls");
  // count and scatter1 share the grid: one CTA per SM (8192-row tiles) or two (4096)
  const unsigned grid = (unsigned)ctx->sm_count * (a->hc_tile == 4096 ? 2u : 1u);
  WG_TRY(a->hc_counts1.ensure(ctx, (int64_t)np1 * grid * 4));
  WG_TRY(a->hc_offs1.ensure(ctx, (int64_t)np1 * grid * 8));
  // the compiled high-cardinality shape when the input matches it
  wgd::Plan probe = P;
  const bool stat = wgd::shape_matches<wgd::ShapeHighCard>(probe) && env_int("WG_SPECIALIZE", 1) != 0;
  WG_TRY(hc_first_level_any(a, P, stat, grid, 0, out, 0, nullptr));
  std::vector<uint32_t> hc((size_t)np1 * grid);
  std::vector<unsigned long long> ho((size_t)np1 * grid);
  WG_CUDA_TRY(cudaMemcpyAsync(hc.data(), a->hc_counts1.get(), hc.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  wg_agg::HcRun run;
  if (!a->hc_free.empty()) { run = std::move(a->hc_free.back()); a->hc_free.pop_back(); }
  run.off1.assign((size_t)np1 + 1, 0);
  unsigned long long acc = 0;
  for (int p = 0; p < np1; ++p) {
    run.off1[(size_t)p] = (int64_t)acc;
    for (unsigned c = 0; c < grid; ++c) { ho[(size_t)p * grid + c] = acc; acc += hc[(size_t)p * grid + c]; }
  }
  run.off1[(size_t)np1] = (int64_t)acc;
  run.rows = (int64_t)acc;
  if (run.rows > P.n_items) return fail(WG_E_CUDA, "partition counts exceed the input rows");
  WG_CUDA_TRY(cudaMemcpyAsync(a->hc_offs1.get(), ho.data(), ho.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
  if ((int)run.cols.size() < out.n) run.cols.resize((size_t)out.n);
  for (int j = 0; j < out.n; ++j) {
    WG_TRY(run.cols[(size_t)j].ensure(ctx, std::max<int64_t>(run.rows, 1) * out.es[j]));
    out.data[j] = run.cols[(size_t)j].as<char>();
  }
  WG_TRY(run.bucket.ensure(ctx, std::max<int64_t>(run.rows, 1)));
  // the leading copy columns that are input columns of 4 or 8 bytes (the keys
  // come first) are staged while the rows are hashed
  int n_pre = 0;
  for (int j = 0, bytes = 0; j < out.n; ++j) {
    if (out.vcol[j] >= P.n_in || (out.es[j] != 4 && out.es[j] != 8) || bytes + a->hc_tile * out.es[j] > a->hc_tile * 16)
      break;
    bytes += a->hc_tile * out.es[j];
    n_pre = j + 1;
  }
  if (n_pre > (int)a->key_cols.size()) n_pre = (int)a->key_cols.size();
  WG_TRY(hc_first_level_any(a, P, stat, grid, 1, out, n_pre, run.bucket.as<uint8_t>()));
  a->hc_runs.push_back(std::move(run));
  return check_device_error(ctx);
}

template <int NA, class Sh>
static cudaError_t launch_hc_bucket(const wgd::Plan& P, size_t smem, const int64_t* boff, int64_t nb,
                                    unsigned long long* out, unsigned long long* cursor, int64_t cap, int32_t* over,
                                    int sms, int ctas, cudaStream_t st) {
  if (ctas == 1) {
    const cudaError_t e =
        cudaFuncSetAttribute(wgd::hc_bucket_kernel<NA, Sh, 1024>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    wgd::hc_bucket_kernel<NA, Sh, 1024><<<sms, 1024, smem, st>>>(P, boff, nb, out, cursor, cap, over);
  } else {
    const cudaError_t e =
        cudaFuncSetAttribute(wgd::hc_bucket_kernel<NA, Sh, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    wgd::hc_bucket_kernel<NA, Sh, 512><<<sms * 2, 512, smem, st>>>(P, boff, nb, out, cursor, cap, over);
  }
  return cudaGetLastError();
}

// Finalize of the two-level mode: the runs re-partitioned into buckets, the
// buckets aggregated into a compact result, the groups that outgrew their
// bucket's shared table appended from the HBM table; the result then stands
// in for the table.
// Distinct keys estimated from the sketch (HyperLogLog: the harmonic mean of
// 2^-rank over the registers, with the small-range linear-counting estimate
// while registers are still empty).
static wg_status hc_estimate_groups(wg_agg* a, double* out) {
  const int m = 1 << wgd::kHllBits;
  std::vector<uint32_t> reg((size_t)m);
  WG_CUDA_TRY(cudaMemcpyAsync(reg.data(), a->hc_hll.get(), (size_t)m * 4, cudaMemcpyDeviceToHost, a->ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(a->ctx->stream));
  double z = 0.0;
  int zeros = 0;
  for (uint32_t r : reg) { z += std::ldexp(1.0, -(int)r); zeros += r == 0; }
  const double alpha = 0.7213 / (1.0 + 1.079 / m);
  double e = alpha * m * m / z;
  if (e <= 2.5 * m && zeros > 0) e = m * std::log((double)m / zeros);
  *out = e;
  return WG_OK;
}

static wg_status hc_finish(wg_agg* a) {
  Ctx* ctx = a->ctx;
  // second-level bits: buckets of about half a shared table of groups (the
  // sketch's estimate plus 10%, its error being about 3% at 1024 registers)
  {
    double groups = 0.0;
    WG_TRY(hc_estimate_groups(a, &groups));
    int ssw = 0, slots = 0, rep = 0;
    hc_table_shape(a, &ssw, &slots, &rep);
    const double per_bucket = (double)std::max(16, env_int("WG_HC_BUCKET_GROUPS", slots / 2));
    const double want = groups * 1.1 / per_bucket;
    int b2 = 0;
    while (b2 < wgd::kHcByteBits && std::ldexp(1.0, a->hc_b1 + b2) < want) ++b2;
    a->hc_b2 = b2;
  }
  const int b1 = a->hc_b1, b2 = a->hc_b2;
  const int np1 = 1 << b1, np2 = 1 << b2;
  const int64_t nb = int64_t(1) << (b1 + b2);
  const int ncol = (int)a->hc_cols.size();
  const int sw = a->L.slot_words;
  int64_t rows = 0;
  for (const auto& r : a->hc_runs) rows += r.rows;
  // device scratch: boff (nb + 1), cursors (nb), then per run off1 and item0 (np1 + 1 each)
  const int64_t scal = (nb + 1) + nb + 2 * ((int64_t)np1 + 1) * (int64_t)std::max<size_t>(a->hc_runs.size(), 1);
  WG_TRY(a->hc_dev.ensure(ctx, scal * 8));
  int64_t* d_boff = a->hc_dev.as<int64_t>();
  unsigned long long* d_cur = (unsigned long long*)(d_boff + nb + 1);
  // per run: its partition starts and first work items (tiles of hc_tile rows) on the device
  std::vector<int64_t> run_items(a->hc_runs.size(), 0);
  for (size_t ri = 0; ri < a->hc_runs.size(); ++ri) {
    const auto& run = a->hc_runs[ri];
    std::vector<int64_t> item0((size_t)np1 + 1);
    int64_t items = 0;
    for (int p = 0; p < np1; ++p) {
      item0[(size_t)p] = items;
      items += (run.off1[(size_t)p + 1] - run.off1[(size_t)p] + a->hc_tile - 1) / a->hc_tile;
    }
    item0[(size_t)np1] = items;
    run_items[ri] = items;
    int64_t* d_off1 = (int64_t*)(d_cur + nb) + 2 * ((int64_t)np1 + 1) * (int64_t)ri;
    WG_CUDA_TRY(cudaMemcpyAsync(d_off1, run.off1.data(), (size_t)(np1 + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    WG_CUDA_TRY(cudaMemcpyAsync(d_off1 + np1 + 1, item0.data(), (size_t)(np1 + 1) * 8, cudaMemcpyHostToDevice,
                                ctx->stream));
  }
  // rows per bucket, from the runs' bucket bytes
  WG_TRY(a->hc_hist.ensure(ctx, nb * 8));
  WG_CUDA_TRY(cudaMemsetAsync(a->hc_hist.get(), 0, (size_t)nb * 8, ctx->stream));
  for (size_t ri = 0; ri < a->hc_runs.size(); ++ri) {
    if (a->hc_runs[ri].rows == 0) continue;
    const int64_t* d_off1 = (const int64_t*)(d_cur + nb) + 2 * ((int64_t)np1 + 1) * (int64_t)ri;
    const unsigned grid = (unsigned)std::min<int64_t>((int64_t)ctx->sm_count * 4, run_items[ri]);
    if (a->hc_tile == 4096)
      wgd::hc_count2_kernel<4096><<<grid, wgd::kHcThreads, 0, ctx->stream>>>(
          a->hc_runs[ri].bucket.as<uint8_t>(), b2, d_off1, d_off1 + np1 + 1, np1, run_items[ri],
          a->hc_hist.as<unsigned long long>());
    else
      wgd::hc_count2_kernel<8192><<<grid, wgd::kHcThreads, 0, ctx->stream>>>(
          a->hc_runs[ri].bucket.as<uint8_t>(), b2, d_off1, d_off1 + np1 + 1, np1, run_items[ri],
          a->hc_hist.as<unsigned long long>());
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  // bucket starts in the second copy
  std::vector<unsigned long long> hist((size_t)nb);
  WG_CUDA_TRY(cudaMemcpyAsync(hist.data(), a->hc_hist.get(), (size_t)nb * 8, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  std::vector<int64_t> boff((size_t)nb + 1);
  int64_t acc = 0;
  for (int64_t b = 0; b < nb; ++b) { boff[(size_t)b] = acc; acc += (int64_t)hist[(size_t)b]; }
  boff[(size_t)nb] = acc;
  if (acc != rows) return fail(WG_E_CUDA, "bucket counts do not add up to the partitioned rows");
  WG_CUDA_TRY(cudaMemcpyAsync(d_boff, boff.data(), (size_t)(nb + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
  WG_CUDA_TRY(cudaMemcpyAsync(d_cur, boff.data(), (size_t)nb * 8, cudaMemcpyHostToDevice, ctx->stream));
  if ((int)a->hc_copy2.size() < ncol) a->hc_copy2.resize((size_t)ncol);
  wgd::HcCols out2{};
  out2.n = ncol;
  for (int j = 0; j < ncol; ++j) {
    WG_TRY(a->hc_copy2[(size_t)j].ensure(ctx, std::max<int64_t>(rows, 1) * a->hc_es[(size_t)j]));
    out2.data[j] = a->hc_copy2[(size_t)j].as<char>();
    out2.es[j] = a->hc_es[(size_t)j];
    out2.vcol[j] = j;
  }
  const size_t ss = wgd::hc_scatter_smem(a->hc_tile, np2, false);
  if (a->hc_tile == 4096)
    WG_CUDA_TRY(cudaFuncSetAttribute(wgd::hc_scatter2_kernel<4096>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  else
    WG_CUDA_TRY(cudaFuncSetAttribute(wgd::hc_scatter2_kernel<8192>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ss));
  for (size_t ri = 0; ri < a->hc_runs.size(); ++ri) {
    auto& run = a->hc_runs[ri];
    if (run.rows == 0) continue;
    const int64_t* d_off1 = (const int64_t*)(d_cur + nb) + 2 * ((int64_t)np1 + 1) * (int64_t)ri;
    wgd::Plan Pc = hc_plan(a, run.cols, run.rows);
    const int64_t slots = (int64_t)ctx->sm_count * (a->hc_tile == 4096 ? 2 : 1);
    const unsigned grid = (unsigned)std::min<int64_t>(slots, run_items[ri]);
    if (a->hc_tile == 4096)
      wgd::hc_scatter2_kernel<4096><<<grid, wgd::HcGeom<4096>::threads, ss, ctx->stream>>>(
          Pc, b2, run.bucket.as<uint8_t>(), d_off1, d_off1 + np1 + 1, np1, run_items[ri], d_cur, out2);
    else
      wgd::hc_scatter2_kernel<8192><<<grid, wgd::HcGeom<8192>::threads, ss, ctx->stream>>>(
          Pc, b2, run.bucket.as<uint8_t>(), d_off1, d_off1 + np1 + 1, np1, run_items[ri], d_cur, out2);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  // buckets into the compact result
  wgd::Plan Pb = hc_plan(a, a->hc_copy2, rows);
  int ssw = 0, S = 0, rep = 0;
  hc_table_shape(a, &ssw, &S, &rep);
  const int ctas = hc_bucket_ctas();
  Pb.smem_slots = S;
  Pb.smem_sw = ssw;
  Pb.smem_rep = rep;
  Pb.smem_hash_shift = b1 + b2;
  Pb.smem_list = S * ssw;
  const size_t smem = (size_t)S * ssw * 8 + (size_t)S * 4;
  WG_TRY(a->hc_scalars.ensure(ctx, 64));
  unsigned long long* d_ocur = a->hc_scalars.as<unsigned long long>();
  int32_t* d_over = (int32_t*)(d_ocur + 1);
  int64_t cap = std::max<int64_t>(1024, std::min<int64_t>(rows, std::max<int64_t>(a->hint, a->known_groups) * 5 / 4 + 65536));
  if (env_int("WG_HC_OUT_CAP", 0) > 0) cap = env_int("WG_HC_OUT_CAP", 0);  // a small first guess (replay paths)
  wgd::Plan probe = Pb;
  const bool stat = wgd::shape_matches<wgd::ShapeHighCard>(probe) && env_int("WG_SPECIALIZE", 1) != 0;
  a->last_shape = stat ? wgd::SHAPE_HIGHCARD : wgd::SHAPE_GENERIC;
  for (int attempt = 0; attempt < 8; ++attempt) {
    WG_TRY(a->hc_out.ensure(ctx, cap * sw * 8));
    WG_CUDA_TRY(cudaMemsetAsync(a->hc_scalars.get(), 0, 64, ctx->stream));
    Pb.T = table_view(a);
    const int sms = ctx->sm_count;
    if (stat)
      WG_CUDA_TRY((launch_hc_bucket<4, wgd::StatShape<wgd::ShapeHighCard>>(
          Pb, smem, d_boff, nb, a->hc_out.as<unsigned long long>(), d_ocur, cap, d_over, sms, ctas, ctx->stream)));
    else if (a->L.n_aggs <= 4)
      WG_CUDA_TRY((launch_hc_bucket<4, wgd::DynShape>(Pb, smem, d_boff, nb, a->hc_out.as<unsigned long long>(), d_ocur,
                                                      cap, d_over, sms, ctas, ctx->stream)));
    else
      WG_CUDA_TRY((launch_hc_bucket<8, wgd::DynShape>(Pb, smem, d_boff, nb, a->hc_out.as<unsigned long long>(), d_ocur,
                                                      cap, d_over, sms, ctas, ctx->stream)));
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    int64_t v[2], t[2];
    WG_TRY(read_back_i64(ctx, (const int64_t*)a->hc_scalars.get(), v, 2));
    WG_TRY(read_back_i64(ctx, (const int64_t*)a->ctr.get(), t, 2));
    WG_TRY(check_device_error(ctx));
    const bool out_over = (int32_t)v[1] != 0, tab_over = (int32_t)t[1] != 0;
    if (!out_over && !tab_over) {
      // the groups that outgrew their bucket's shared table, appended from the HBM table
      WG_TRY(agg_compact(a));
      const int64_t n_sm = v[0], n_tab = a->n_out;
      if (n_sm + n_tab > cap) {
        DevBuf bigger;
        WG_TRY(bigger.alloc(ctx, (n_sm + n_tab) * sw * 8));
        WG_CUDA_TRY(cudaMemcpyAsync(bigger.get(), a->hc_out.get(), (size_t)(n_sm * sw * 8), cudaMemcpyDeviceToDevice,
                                    ctx->stream));
        a->hc_out = std::move(bigger);
      }
      if (n_tab > 0) {
        gather_slots_kernel<<<grid_cap(ctx, n_tab * sw, 256), 256, 0, ctx->stream>>>(
            a->table.as<unsigned long long>(), sw, a->list.as<int64_t>(), n_tab,
            a->hc_out.as<unsigned long long>() + n_sm * sw);
        ctx->count_launch();
        WG_CUDA_TRY(cudaGetLastError());
      }
      const int64_t n_res = n_sm + n_tab;
      // the compact result becomes the table (every slot a group, no NULL-key slot)
      std::swap(a->table, a->hc_out);
      a->cap = uint64_t(1) << 62;
      a->spilled = true;
      WG_TRY(a->list.ensure(ctx, std::max<int64_t>(n_res, 1) * 8));
      iota_kernel<<<grid_cap(ctx, std::max<int64_t>(n_res, 1), 256), 256, 0, ctx->stream>>>(a->list.as<int64_t>(), n_res);
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
      a->n_out = n_res;
      for (auto& r : a->hc_runs) a->hc_free.push_back(std::move(r));
      a->hc_runs.clear();
      return check_device_error(ctx);
    }
    // replay: a larger result, or a larger HBM table for the groups that outgrew their buckets
    if (out_over) cap = std::max<int64_t>(cap * 2, v[0] + 1024);
    if (tab_over) WG_TRY(rebuild_table(a, a->cap * 4, a->L));
    const int64_t words = table_words(a, a->cap);
    init_table_kernel<<<grid_cap(ctx, words, 256), 256, 0, ctx->stream>>>(a->table.as<unsigned long long>(), words,
                                                                         a->L.slot_words, a->L);
    ctx->count_launch();
    WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, ctx->stream));
    a->known_groups = a->upper_groups = 0;
    a->dom = 0;
  }
  return fail(WG_E_NOMEM, "two-level aggregation did not converge");
}

// Rows of the partition kernels' plan: the aggregate's key layout, the caller's
// columns rebased to row r0, m rows.
static wgd::Plan part_plan(wg_agg* a, const wgd::Plan& P0, int64_t r0, int64_t m) {
  wgd::Plan P = P0;
  for (int j = 0; j < P.n_in; ++j) {
    const int cls = P.in[j].cls;
    const int64_t es = cls == WG_CLS_I32 || cls == WG_CLS_F32 ? 4 : cls == WG_CLS_DEC ? 16 : 8;
    P.in[j].data = (const char*)P.in[j].data + r0 * es;
    if (P.in[j].valid) P.in[j].valid += r0 / 64;  // windows start on 64-row boundaries
  }
  P.n_items = m;
  P.L = launch_layout(a, P0);
  P.err = a->ctx->dev_error;
  return P;
}

// Pinned host memory for spilled runs, from blocks of at least 256 MB, within
// the context's pinned spill budget.
static wg_status spill_host_alloc(wg_agg* a, int64_t bytes, char** out) {
  bytes = (bytes + 255) & ~int64_t(255);
  while (a->block_idx < a->host_blocks.size() && a->block_used + bytes > a->host_blocks[a->block_idx].second) {
    ++a->block_idx;  // the rest of this block stays unused until the arena is rewound
    a->block_used = 0;
  }
  if (a->block_idx == a->host_blocks.size()) {
    const int64_t blk = std::max<int64_t>(bytes, int64_t(256) << 20);
    if (a->host_bytes + blk > a->ctx->pinned_spill_bytes)
      return fail(WG_E_NOMEM, "pinned spill budget exceeded by the spilled aggregation");
    void* p = nullptr;
    if (cudaMallocHost(&p, (size_t)blk) != cudaSuccess) return fail(WG_E_NOMEM, "pinned spill allocation failed");
    a->host_blocks.push_back({(char*)p, blk});
    a->host_bytes += blk;
    a->block_used = 0;
  }
  *out = a->host_blocks[a->block_idx].first + a->block_used;
  a->block_used += bytes;
  return WG_OK;
}

// A spilled consume call: the input, in windows of up to 2^24 rows, reordered
// on the device by partition (part_count_kernel / part_scatter_kernel) and
// copied to pinned host runs. Filters and projections run later, per
// partition, so every row is kept here.
static wg_status spill_consume(const PipelineRun& r, const wgd::Plan& P0in, const std::vector<int>& in_map) {
  wg_agg* a = r.agg;
  Ctx* ctx = a->ctx;
  if (r.join) return fail(WG_E_UNSUPPORTED, "a spilled aggregation takes no join");
  if (a->sp_map.empty()) {  // remember the consume calls' shape for the per-partition runs
    a->sp_cols.assign(r.in->cols, r.in->cols + r.in->ncols);
    a->sp_map = in_map;
    a->sp_es.assign((size_t)P0in.n_in, 0);
    a->sp_null.assign((size_t)P0in.n_in, false);
    for (int j = 0; j < P0in.n_in; ++j) {
      const int cls = P0in.in[j].cls;
      a->sp_es[(size_t)j] = cls == WG_CLS_I32 || cls == WG_CLS_F32 ? 4 : cls == WG_CLS_DEC ? 16 : 8;
      a->sp_null[(size_t)j] = P0in.in[j].valid != nullptr;
    }
    a->sp_filters.assign(r.filters, r.filters + r.n_filters);
    a->sp_exprs.assign(r.exprs, r.exprs + r.n_exprs);
    a->sp_dev.resize((size_t)P0in.n_in);
    a->sp_norm.resize((size_t)P0in.n_in);
    a->sp_ok.resize((size_t)P0in.n_in);
    a->sp_words.resize((size_t)P0in.n_in);
    a->sp_okdev.resize((size_t)P0in.n_in);
  } else {
    bool same = (int)a->sp_cols.size() == r.in->ncols && a->sp_map == in_map &&
                (int)a->sp_filters.size() == r.n_filters && (int)a->sp_exprs.size() == r.n_exprs;
    for (int c = 0; same && c < r.in->ncols; ++c)
      same = a->sp_cols[(size_t)c].type_id == r.in->cols[c].type_id && a->sp_cols[(size_t)c].scale == r.in->cols[c].scale;
    if (!same) return fail(WG_E_UNSUPPORTED, "every consume call of a spilled aggregation must have the same shape");
    for (int j = 0; j < P0in.n_in; ++j)
      if (P0in.in[j].valid && !a->sp_null[(size_t)j])
        return fail(WG_E_UNSUPPORTED, "NULLs in a column the spilled aggregation's first call had none in");
  }
  // The rows a selection vector keeps, gathered; each nullable input's
  // validity as one flag per row (moved with the rows into the runs) and as
  // packed words the partition kernels read (NULL keys hash like the table).
  wgd::Plan P0 = P0in;
  bool any_null = false;
  for (int j = 0; j < P0in.n_in; ++j) any_null = any_null || a->sp_null[(size_t)j];
  if (P0in.sel || any_null) {
    const int64_t nn = P0in.n_items;
    for (int j = 0; j < P0in.n_in; ++j) {
      const int64_t es = a->sp_es[(size_t)j];
      if (P0in.sel) {
        WG_TRY(a->sp_norm[(size_t)j].ensure(ctx, std::max<int64_t>(nn, 1) * es));
        spill_gather_kernel<<<grid_cap(ctx, nn, 256), 256, 0, ctx->stream>>>(
            (const char*)P0in.in[j].data, (int)es, P0in.sel, nn, a->sp_norm[(size_t)j].as<char>());
        ctx->count_launch();
        WG_CUDA_TRY(cudaGetLastError());
        P0.in[j].data = a->sp_norm[(size_t)j].get();
      }
      P0.in[j].valid = nullptr;
      if (a->sp_null[(size_t)j]) {
        WG_TRY(a->sp_ok[(size_t)j].ensure(ctx, std::max<int64_t>(nn, 1) * 4));
        WG_TRY(a->sp_words[(size_t)j].ensure(ctx, ((nn + 63) / 64 + 1) * 8));
        spill_valid_kernel<<<grid_cap(ctx, nn, 256), 256, 0, ctx->stream>>>(P0in.in[j].valid, P0in.sel, nn,
                                                                           a->sp_ok[(size_t)j].as<int32_t>());
        ctx->count_launch();
        pack_valid_kernel<<<grid_cap(ctx, (nn + 63) / 64, 256), 256, 0, ctx->stream>>>(
            a->sp_ok[(size_t)j].as<int32_t>(), nn, a->sp_words[(size_t)j].as<uint64_t>());
        ctx->count_launch();
        WG_CUDA_TRY(cudaGetLastError());
        P0.in[j].valid = a->sp_words[(size_t)j].as<uint64_t>();
      }
    }
    P0.sel = nullptr;
  }
  const int pbits = a->spill_pbits, np = 1 << pbits;
  const unsigned grid = (unsigned)(ctx->sm_count * 2);
  DevBuf counts, offs;
  WG_TRY(counts.ensure(ctx, (int64_t)np * grid * 4));
  WG_TRY(offs.ensure(ctx, (int64_t)np * grid * 8));
  // windows of up to 2^24 rows, or what a quarter of the ledger's room holds
  int64_t row_bytes = 0;
  for (int e : a->sp_es) row_bytes += e;
  const int64_t room = ctx->ledger.budget() > 0 ? ctx->ledger.budget() - ctx->ledger.used() : (int64_t(1) << 40);
  const int64_t n = P0.n_items;
  for (int j = 0; j < P0.n_in; ++j) row_bytes += a->sp_null[(size_t)j] ? 4 : 0;
  const int64_t win = std::max<int64_t>(int64_t(1) << 16, std::min<int64_t>(int64_t(1) << 24, room / 4 / std::max<int64_t>(row_bytes, 1))) &
                      ~int64_t(63);  // validity words stay whole
  std::vector<uint32_t> hc((size_t)np * grid);
  std::vector<unsigned long long> ho((size_t)np * grid);
  for (int64_t r0 = 0; r0 < n; r0 += win) {
    const int64_t m = std::min(win, n - r0);
    const wgd::Plan P = part_plan(a, P0, r0, m);
    wgd::part_count_kernel<<<grid, wgd::kPartThreads, wgd::part_count_smem(np), ctx->stream>>>(P, pbits, kSpillPartShift,
                                                                       counts.as<uint32_t>());
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    WG_CUDA_TRY(cudaMemcpyAsync(hc.data(), counts.get(), hc.size() * 4, cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    wg_agg::SpillRun run;
    run.rows = m;
    run.off.assign((size_t)np + 1, 0);
    unsigned long long acc = 0;
    for (int p = 0; p < np; ++p) {
      run.off[(size_t)p] = (int64_t)acc;
      for (unsigned c = 0; c < grid; ++c) { ho[(size_t)p * grid + c] = acc; acc += hc[(size_t)p * grid + c]; }
    }
    run.off[(size_t)np] = (int64_t)acc;
    if ((int64_t)acc != m) return fail(WG_E_CUDA, "partition counts do not add up to the input rows");
    WG_CUDA_TRY(cudaMemcpyAsync(offs.get(), ho.data(), ho.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
    wgd::PartOut po{};
    for (int j = 0; j < P.n_in; ++j) {
      WG_TRY(a->sp_dev[(size_t)j].ensure(ctx, win * a->sp_es[(size_t)j]));
      po.data[j] = a->sp_dev[(size_t)j].as<char>();
      po.es[j] = a->sp_es[(size_t)j];
      if (a->sp_null[(size_t)j]) {  // the validity flags move with the rows
        WG_TRY(a->sp_okdev[(size_t)j].ensure(ctx, win * 4));
        po.side_src[po.n_side] = a->sp_ok[(size_t)j].as<int32_t>() + r0;
        po.side_dst[po.n_side] = a->sp_okdev[(size_t)j].as<int32_t>();
        ++po.n_side;
      }
    }
    WG_CUDA_TRY(cudaFuncSetAttribute(wgd::part_scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)wgd::part_scatter_smem(np)));
    wgd::part_scatter_kernel<<<grid, wgd::kPartThreads, wgd::part_scatter_smem(np), ctx->stream>>>(P, pbits, kSpillPartShift,
                                                                          offs.as<unsigned long long>(), po);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    run.col.assign((size_t)P.n_in, nullptr);
    run.ok.assign((size_t)P.n_in, nullptr);
    for (int j = 0; j < P.n_in; ++j) {
      WG_TRY(spill_host_alloc(a, m * a->sp_es[(size_t)j], &run.col[(size_t)j]));
      WG_CUDA_TRY(cudaMemcpyAsync(run.col[(size_t)j], po.data[j], (size_t)(m * a->sp_es[(size_t)j]),
                                  cudaMemcpyDeviceToHost, ctx->stream));
      if (a->sp_null[(size_t)j]) {
        WG_TRY(spill_host_alloc(a, m * 4, &run.ok[(size_t)j]));
        WG_CUDA_TRY(cudaMemcpyAsync(run.ok[(size_t)j], a->sp_okdev[(size_t)j].get(), (size_t)(m * 4),
                                    cudaMemcpyDeviceToHost, ctx->stream));
      }
    }
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    a->runs.push_back(std::move(run));
  }
  return check_device_error(ctx);
}

static wg_status agg_compact(wg_agg* a);

// Finalize of a spilled aggregation: per partition, its rows from every run
// back to the device, the fused kernel into the small table, and the groups
// appended to the compact result; the result then stands in for the table.
static wg_status spill_finish(wg_agg* a) {
  Ctx* ctx = a->ctx;
  const int np = 1 << a->spill_pbits;
  const int nin = (int)a->sp_es.size();
  const int sw = a->L.slot_words;
  int64_t max_rows = 0;
  for (int p = 0; p < np; ++p) {
    int64_t rows = 0;
    for (const auto& run : a->runs) rows += run.off[(size_t)p + 1] - run.off[(size_t)p];
    max_rows = std::max(max_rows, rows);
  }
  for (int j = 0; j < nin; ++j) {  // staging for one partition (the consume windows' buffers go first)
    a->sp_dev[(size_t)j].reset();
    a->sp_norm[(size_t)j].reset();
    a->sp_ok[(size_t)j].reset();
    WG_TRY(a->sp_dev[(size_t)j].alloc(ctx, std::max<int64_t>(max_rows, 1) * a->sp_es[(size_t)j]));
    if (a->sp_null[(size_t)j]) {
      a->sp_okdev[(size_t)j].reset();
      a->sp_words[(size_t)j].reset();
      WG_TRY(a->sp_okdev[(size_t)j].alloc(ctx, std::max<int64_t>(max_rows, 1) * 4));
      WG_TRY(a->sp_words[(size_t)j].alloc(ctx, ((max_rows + 63) / 64 + 1) * 8));
    }
  }
  DevBuf res, null_slot;
  bool has_null = false;
  int64_t res_cap = std::max<int64_t>(a->hint, 1024), n_res = 0;
  WG_TRY(res.alloc(ctx, res_cap * sw * 8));
  std::vector<wg_column> cols = a->sp_cols;
  wg_batch_desc d{};
  d.ncols = (int32_t)cols.size();
  d.cols = cols.data();
  for (int p = 0; p < np; ++p) {
    int64_t rows = 0;
    for (const auto& run : a->runs) {
      const int64_t c = run.off[(size_t)p + 1] - run.off[(size_t)p];
      for (int j = 0; j < nin && c > 0; ++j) {
        const int64_t es = a->sp_es[(size_t)j];
        WG_CUDA_TRY(cudaMemcpyAsync(a->sp_dev[(size_t)j].as<char>() + rows * es, run.col[(size_t)j] + run.off[(size_t)p] * es,
                                    (size_t)(c * es), cudaMemcpyHostToDevice, ctx->stream));
        if (a->sp_null[(size_t)j])
          WG_CUDA_TRY(cudaMemcpyAsync(a->sp_okdev[(size_t)j].as<char>() + rows * 4, run.ok[(size_t)j] + run.off[(size_t)p] * 4,
                                      (size_t)(c * 4), cudaMemcpyHostToDevice, ctx->stream));
      }
      rows += c;
    }
    if (rows == 0) continue;
    for (int j = 0; j < nin; ++j) {  // the partition's validity words from its rows' flags
      if (!a->sp_null[(size_t)j]) continue;
      pack_valid_kernel<<<grid_cap(ctx, (rows + 63) / 64, 256), 256, 0, ctx->stream>>>(
          a->sp_okdev[(size_t)j].as<int32_t>(), rows, a->sp_words[(size_t)j].as<uint64_t>());
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
    }
    for (size_t c = 0; c < cols.size(); ++c) {
      cols[c].len = rows;
      cols[c].valid_words = nullptr;
      const int j = a->sp_map[c];
      if (j >= 0) {
        cols[c].data = a->sp_dev[(size_t)j].get();
        if (a->sp_null[(size_t)j]) cols[c].valid_words = a->sp_words[(size_t)j].as<uint64_t>();
      }
    }
    d.len = rows;
    // the small table, empty again
    const int64_t words = table_words(a, a->cap);
    init_table_kernel<<<grid_cap(ctx, words, 256), 256, 0, ctx->stream>>>(a->table.as<unsigned long long>(), words,
                                                                         sw, a->L);
    ctx->count_launch();
    WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, ctx->stream));
    a->known_groups = a->upper_groups = 0;
    a->dom = 0;
    PipelineRun rp{a, &d, (int32_t)a->sp_filters.size(), a->sp_filters.data(), nullptr, (int32_t)a->sp_exprs.size(),
                   a->sp_exprs.data()};
    rp.no_partition = true;
    WG_TRY(run_device(rp));
    if (a->L.key_words == 1) {
      // the NULL-key group (single-word keys: the table's slot cap + 1; every
      // NULL-key row is in partition 0) is kept aside and appended last
      const unsigned long long* ns = a->table.as<unsigned long long>() + (a->cap + 1) * (uint64_t)sw;
      int64_t rows_null = 0;
      WG_TRY(read_back_i64(ctx, (const int64_t*)(ns + a->L.key_words), &rows_null, 1));
      if (rows_null != 0) {
        if (has_null) return fail(WG_E_CUDA, "NULL-key rows in more than one spill partition");
        WG_TRY(null_slot.ensure(ctx, sw * 8));
        WG_CUDA_TRY(cudaMemcpyAsync(null_slot.get(), ns, (size_t)(sw * 8), cudaMemcpyDeviceToDevice, ctx->stream));
        WG_CUDA_TRY(cudaMemsetAsync((void*)(ns + a->L.key_words), 0, 8, ctx->stream));  // out of this compaction
        has_null = true;
      }
    }
    WG_TRY(agg_compact(a));
    if (n_res + a->n_out > res_cap) {  // grow the result, keeping what it holds
      const int64_t cap2 = std::max<int64_t>(res_cap * 2, n_res + a->n_out);
      DevBuf bigger;
      WG_TRY(bigger.alloc(ctx, cap2 * sw * 8));
      if (n_res > 0)
        WG_CUDA_TRY(cudaMemcpyAsync(bigger.get(), res.get(), (size_t)(n_res * sw * 8), cudaMemcpyDeviceToDevice, ctx->stream));
      WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      res = std::move(bigger);
      res_cap = cap2;
    }
    if (a->n_out > 0) {
      gather_slots_kernel<<<grid_cap(ctx, a->n_out * sw, 256), 256, 0, ctx->stream>>>(
          a->table.as<unsigned long long>(), sw, a->list.as<int64_t>(), a->n_out, res.as<unsigned long long>() + n_res * sw);
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
    }
    n_res += a->n_out;
  }
  // The compact result becomes the table: every listed slot a group. With a
  // NULL-key group the slots are [groups][unused][NULL group] and the view's
  // capacity is the number of groups, so the NULL group sits at capacity + 1
  // where the readers of a table look for it; the list skips the unused slot.
  if (has_null) {
    if (n_res + 2 > res_cap) {
      DevBuf bigger;
      WG_TRY(bigger.alloc(ctx, (n_res + 2) * sw * 8));
      if (n_res > 0)
        WG_CUDA_TRY(cudaMemcpyAsync(bigger.get(), res.get(), (size_t)(n_res * sw * 8), cudaMemcpyDeviceToDevice, ctx->stream));
      WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
      res = std::move(bigger);
    }
    WG_CUDA_TRY(cudaMemcpyAsync(res.as<unsigned long long>() + (n_res + 1) * sw, null_slot.get(), (size_t)(sw * 8),
                                cudaMemcpyDeviceToDevice, ctx->stream));
  }
  a->table = std::move(res);
  a->cap = has_null ? (uint64_t)n_res : uint64_t(1) << 62;
  a->spilled = true;
  const int64_t n_list = n_res + (has_null ? 1 : 0);
  WG_TRY(a->list.ensure(ctx, std::max<int64_t>(n_list, 1) * 8));
  iota_kernel<<<grid_cap(ctx, std::max<int64_t>(n_res, 1), 256), 256, 0, ctx->stream>>>(a->list.as<int64_t>(), n_res);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  if (has_null) {
    const int64_t at = n_res + 1;
    WG_CUDA_TRY(cudaMemcpyAsync(a->list.as<int64_t>() + n_res, &at, 8, cudaMemcpyHostToDevice, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // `at` is on this stack
  }
  a->n_out = n_list;
  a->runs.clear();
  for (auto& b : a->sp_dev) b.reset();  // staging and snapshots go back to the ledger
  a->backup.reset();
  a->block_idx = 0;  // rewind the arena for the next query on this aggregate
  a->block_used = 0;
  return check_device_error(ctx);
}

// Compact the occupied slots once; the list drives export and emit.
static wg_status agg_compact(wg_agg* a) {
  Ctx* ctx = a->ctx;
  const int64_t n = a->L.key_words == 0 ? 1 : (int64_t)a->cap + 2;
  WG_TRY(a->list.ensure(ctx, n * 8));
  WG_TRY(a->cnt.ensure(ctx, 64));
  WG_CUDA_TRY(cudaMemsetAsync(a->cnt.get(), 0, 8, ctx->stream));
  compact_kernel<<<grid_cap(ctx, n, 256), 256, 0, ctx->stream>>>(a->L, table_view(a), a->list.as<int64_t>(),
                                                                  a->cnt.as<unsigned long long>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  int64_t c = 0;
  WG_TRY(read_back_checked(ctx, a->cnt.as<int64_t>(), &c, 1));
  a->n_out = c;
  return WG_OK;
}

static void fill_final_args(wg_agg* a, FinalArgs& A) {
  std::memset(&A, 0, sizeof(A));
  A.L = a->L;
  A.T = table_view(a);
  A.list = a->list.as<int64_t>();
  for (size_t k = 0; k < a->key_types.size(); ++k) A.key_cls[k] = class_of(a->key_types[k]);
  for (size_t i = 0; i < a->specs.size(); ++i) {
    A.agg_func[i] = a->specs[i].func;
    A.agg_out[i] = a->out_type[i] == WG_TYPE_INT64 ? 0 : 1;
    A.agg_scale[i] = a->in_scale[i];
  }
}

}  // namespace wg

using namespace wg;

namespace wg {
// Access for the pipeline entry points (wg_pipeline.cu).
// The aggregate's single string GROUP BY key in column `col` of `in` mapped to
// its dictionary's ids (*out: the INT32 id column on the device).
wg_status agg_map_str_key(wg_agg* a, const wg_batch_desc* in, int col, bool host, wg_column* out) {
  if (a->finalized) return fail(WG_E_STATE, "aggregate already finalized");
  return strdict_map(a->ctx, &a->sdict, in, col, host, a->hint, out);
}
int agg_str_key_col(wg_agg* a, const wg_batch_desc* in) { return str_key_col(a, in); }

wg_status agg_run_device(wg_agg* a, const wg_batch_desc* in, int32_t nf, const wg_predicate* f, wg_join* j, int32_t ne,
                         const wg_expr* e, bool defer_check, bool str_ids) {
  // a string key column of a device batch: its ids first, for every row the
  // fused launch reads (rows its filters or join drop keep their strings in the
  // dictionary without forming a group)
  std::vector<wg_column> cols;
  wg_batch_desc mapped;
  const int sk = str_ids ? -1 : str_key_col(a, in);
  if (sk >= 0) {
    cols.assign(in->cols, in->cols + in->ncols);
    WG_TRY(agg_map_str_key(a, in, sk, false, &cols[(size_t)sk]));
    mapped = *in;
    mapped.cols = cols.data();
    in = &mapped;
    str_ids = true;
  }
  if (j && join_is_grace(j)) {
    // a partitioned build: one pass per group of its partitions, each probe row
    // taking part in the pass of its key's partition
    for (int g = 0; g < join_grace_passes(j); ++g) {
      wg_join* pj = nullptr;
      WG_TRY(join_grace_pass(j, g, &pj));
      PipelineRun r{a, in, nf, f, pj, ne, e};
      r.str_ids = str_ids;
      WG_TRY(run_device(r));
    }
    return WG_OK;
  }
  PipelineRun r{a, in, nf, f, j, ne, e};
  r.defer_check = defer_check;
  r.str_ids = str_ids;
  return run_device(r);
}
Ctx* agg_ctx(wg_agg* a) { return a->ctx; }
// Frees what an aggregate keeps only to speed up its next query (the
// reordered input copy and its counters), for an aggregate parked in a pool.
void agg_trim(wg_agg* a) {
  if (a->part_bufs.empty() && !a->part_counts.get()) return;
  ensure_device(a->ctx);
  cudaStreamSynchronize(a->ctx->stream);  // no launch still reads them
  a->part_bufs.clear();
  a->part_counts.reset();
  a->part_offs.reset();
}
std::vector<int32_t> agg_input_cols(wg_agg* a) {
  std::vector<int32_t> r = a->key_cols;
  for (const wg_agg_spec& s : a->specs) r.push_back(s.input_col);
  return r;
}
}  // namespace wg

extern "C" {

wg_status wg_agg_create(wg_ctx* ctx, int32_t n_keys, const int32_t* key_cols, int32_t n_aggs, const wg_agg_spec* aggs,
                        int64_t group_ndv_hint, wg_agg** out) {
  if (!ctx || !out || n_keys < 0 || n_aggs < 0 || (n_keys > 0 && !key_cols) || (n_aggs > 0 && !aggs))
    return fail(WG_E_INVALID, "bad aggregate arguments");
  if (n_keys > WG_MAX_KEYS) return fail(WG_E_UNSUPPORTED, "more than 4 GROUP BY columns");
  if (n_aggs > WG_MAX_AGGS) return fail(WG_E_UNSUPPORTED, "more than 8 aggregates");
  wg_agg* a = new wg_agg();
  a->ctx = ctx;
  a->key_cols.assign(key_cols, key_cols + n_keys);
  a->specs.assign(aggs, aggs + n_aggs);
  a->hint = group_ndv_hint;
  *out = a;
  return WG_OK;
}

wg_status wg_agg_consume_device(wg_agg* a, const wg_batch_desc* in) {
  if (!a || !in) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(a->ctx));
  const int sk = str_key_col(a, in);
  if (sk >= 0) {
    // consumeBatchStrGroup (aggregate.go:3038): the strings become dense ids,
    // which the table groups by
    if (a->finalized) return fail(WG_E_STATE, "aggregate already finalized");
    std::vector<wg_column> cols(in->cols, in->cols + in->ncols);
    WG_TRY(strdict_map(a->ctx, &a->sdict, in, sk, false, a->hint, &cols[(size_t)sk]));
    wg_batch_desc d = *in;
    d.cols = cols.data();
    PipelineRun r{a, &d, 0, nullptr, nullptr, 0, nullptr};
    r.str_ids = true;
    return run_device(r);
  }
  PipelineRun r{a, in, 0, nullptr, nullptr, 0, nullptr};
  return run_device(r);
}

wg_status wg_agg_consume(wg_agg* a, const wg_batch_desc* in) {
  if (!a || !in) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(a->ctx));
  const int sk = str_key_col(a, in);
  if (sk >= 0 && a->finalized) return fail(WG_E_STATE, "aggregate already finalized");
  StagedBatch sb;
  WG_TRY(stage_batch(a->ctx, in, &sb));  // a string column is left for the dictionary
  if (sk >= 0) WG_TRY(strdict_map(a->ctx, &a->sdict, in, sk, true, a->hint, &sb.cols[(size_t)sk]));
  PipelineRun r{a, &sb.desc, 0, nullptr, nullptr, 0, nullptr};
  r.str_ids = sk >= 0;
  WG_TRY(run_device(r));
  WG_CUDA_TRY(cudaStreamSynchronize(a->ctx->stream));
  return WG_OK;
}

wg_status wg_agg_clone(wg_agg* a, wg_agg** out) {
  if (!a || !out) return fail(WG_E_INVALID, "NULL argument");
  return wg_agg_create(static_cast<wg_ctx*>(a->ctx), (int32_t)a->key_cols.size(), a->key_cols.data(), (int32_t)a->specs.size(),
                       a->specs.data(), a->hint, out);
}

wg_status wg_agg_merge(wg_agg* d, wg_agg* s) {
  if (!d || !s) return fail(WG_E_INVALID, "NULL argument");
  if (d->ctx != s->ctx) return fail(WG_E_INVALID, "aggregates belong to different contexts");
  if (d->key_cols != s->key_cols || d->specs.size() != s->specs.size()) return fail(WG_E_INVALID, "aggregate shapes differ");
  // two dictionaries number their strings independently
  if (d->str_keyed == 1 || s->str_keyed == 1) return fail(WG_E_UNSUPPORTED, "string-keyed aggregates are not merged");
  // a destination that parks its input in runs (spill, two-level mode) takes no
  // merges; a source of either kind merges once finalized (its compact result)
  if (d->spill || d->hc) return fail(WG_E_UNSUPPORTED, "a spilled or two-level aggregation takes no merges");
  if ((s->spill || s->hc) && !s->spilled) return fail(WG_E_STATE, "finalize a spilled or two-level source first");
  WG_TRY(ensure_device(d->ctx));
  if (d->finalized) return fail(WG_E_STATE, "aggregate already finalized");
  if (!s->resolved) return WG_OK;
  Ctx* ctx = d->ctx;
  if (!d->resolved) {
    // adopt the source's resolved schema (mergeSinkState inherits it, aggregate.go:4722)
    d->key_types = s->key_types; d->in_cls = s->in_cls; d->in_scale = s->in_scale; d->out_type = s->out_type;
    d->kind = s->kind; d->nullable = s->nullable; d->L = s->L;
    d->cap = d->L.key_words == 0 ? 1 : cap_for(std::max<int64_t>(d->hint, 1024));
    d->shift = 64 - log2u(d->cap);
    WG_TRY(init_table(d, d->table, d->cap));
    WG_TRY(d->ctr.alloc(ctx, 64));
    WG_CUDA_TRY(cudaMemsetAsync(d->ctr.get(), 0, 64, ctx->stream));
    d->resolved = true;
  }
  if (d->kind != s->kind) return fail(WG_E_INVALID, "aggregate input types differ");
  d->dom = 2;  // the source's keys have no range this side tracks
  // destination must carry every null counter the source has
  bool upgrade = false;
  std::vector<bool> nn = d->nullable;
  for (size_t i = 0; i < nn.size(); ++i) if (s->nullable[i] && !nn[i]) { nn[i] = true; upgrade = true; }
  if (upgrade) {
    wg_agg tmp;
    tmp.key_cols = d->key_cols; tmp.specs = d->specs; tmp.kind = d->kind; tmp.nullable = nn; tmp.L = d->L;
    build_layout(&tmp);
    for (int k = 0; k < WG_MAX_KEYS; ++k) tmp.L.key_vcol[k] = d->L.key_vcol[k];
    d->nullable = nn;
    WG_TRY(rebuild_table(d, d->cap, tmp.L));
  }
  WG_TRY(refresh_groups(d));
  int64_t s_groups = s->n_out;
  if (!s->spilled) {
    WG_TRY(refresh_groups(s));
    s_groups = s->known_groups;
  }
  const int64_t need = d->known_groups + s_groups + credit_slack(d);
  if (d->L.key_words != 0 && need > (int64_t)((double)d->cap * kMaxLoad)) WG_TRY(rebuild_table(d, cap_for(need), d->L));
  run_fold(d, s->L, table_view(s), d->L, table_view(d), s->spilled ? s->n_out : -1,
           s->spilled ? s->list.as<int64_t>() : nullptr);
  WG_CUDA_TRY(cudaGetLastError());
  WG_TRY(refresh_groups(d));
  return check_device_error(ctx);
}

wg_status wg_agg_finalize(wg_agg* a, int64_t* n_groups) {
  if (!a) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(a->ctx));
  if (!a->resolved) {
    // never fed: a scalar aggregate still emits its one identity row (aggregate.go:4270)
    a->finalized = true;
    a->n_out = a->key_cols.empty() ? 1 : 0;
    if (n_groups) *n_groups = a->n_out;
    return WG_OK;
  }
  if (!a->finalized) {
    if (a->hc) WG_TRY(hc_finish(a));
    else if (a->spill) WG_TRY(spill_finish(a));
    else WG_TRY(agg_compact(a));  // its read-back checks the device error word
    a->finalized = true;
    if (n_groups) *n_groups = a->n_out;
    return a->hc || a->spill ? check_device_error(a->ctx) : WG_OK;
  }
  if (n_groups) *n_groups = a->n_out;
  return check_device_error(a->ctx);
}

wg_status wg_agg_export(wg_agg* a, const wg_group_export* o) {
  if (!a || !o) return fail(WG_E_INVALID, "NULL argument");
  if (!a->finalized) return fail(WG_E_STATE, "aggregate not finalized");
  Ctx* ctx = a->ctx;
  WG_TRY(ensure_device(ctx));
  if (!a->resolved || a->n_out == 0) return WG_OK;
  const int64_t n = a->n_out;
  const int nk = (int)a->key_cols.size(), na = (int)a->specs.size();
  // in chunks of at most 2^16 groups, so the export's staging stays small
  const int64_t C = std::min<int64_t>(n, int64_t(1) << 16);
  FinalArgs A;
  fill_final_args(a, A);
  // the fields the caller asked for, each a block of (keys or aggregates) x C
  // values at a 256-byte aligned offset of one staging buffer
  struct Field { void* dst; int blocks; int64_t es; int64_t off; };
  Field f[7] = {{o->keys, nk, 8, 0}, {o->key_valid, nk, 1, 0}, {o->count, na, 8, 0}, {o->i64, na, 8, 0},
                {o->f64, na, 8, 0}, {o->dec, na, 16, 0}, {o->has, na, 1, 0}};
  int64_t total = 0;
  for (Field& x : f) {
    if (!x.dst || x.blocks == 0) { x.dst = nullptr; continue; }
    x.off = total;
    total += (x.blocks * C * x.es + 255) & ~int64_t(255);
  }
  if (total == 0) return WG_OK;
  WG_TRY(a->exp_dev.ensure(ctx, total));
  if (a->exp_host_bytes < total) {
    if (a->exp_host) cudaFreeHost(a->exp_host);
    a->exp_host = nullptr;
    a->exp_host_bytes = 0;
    if (cudaMallocHost((void**)&a->exp_host, (size_t)total) != cudaSuccess) {
      cudaGetLastError();
      return fail(WG_E_NOMEM, "pinned export staging allocation failed");
    }
    a->exp_host_bytes = total;
  }
  char* dev = a->exp_dev.as<char>();
  A.keys = f[0].dst ? (int64_t*)(dev + f[0].off) : nullptr;
  A.key_valid = f[1].dst ? (uint8_t*)(dev + f[1].off) : nullptr;
  A.count = f[2].dst ? (int64_t*)(dev + f[2].off) : nullptr;
  A.i64 = f[3].dst ? (int64_t*)(dev + f[3].off) : nullptr;
  A.f64 = f[4].dst ? (double*)(dev + f[4].off) : nullptr;
  A.dec = f[5].dst ? (wg_int128*)(dev + f[5].off) : nullptr;
  A.has = f[6].dst ? (uint8_t*)(dev + f[6].off) : nullptr;
  for (int64_t s0 = 0; s0 < n; s0 += C) {
    const int64_t c = std::min(C, n - s0);
    A.start = s0;
    A.n = c;
    A.stride = c;
    export_kernel<<<grid_cap(ctx, c, 256), 256, 0, ctx->stream>>>(A);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    // the chunk's fields sit at their offsets with block stride c: one copy up
    // to the end of the last field in use
    int64_t used = 0;
    for (const Field& x : f)
      if (x.dst) used = x.off + x.blocks * c * x.es;
    WG_CUDA_TRY(cudaMemcpyAsync(a->exp_host, dev, (size_t)used, cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the staging is reused by the next chunk
    // block b of the chunk (c rows at stride c) to rows [s0, s0 + c) of block b on the host (stride n)
    for (const Field& x : f) {
      if (!x.dst) continue;
      for (int b = 0; b < x.blocks; ++b)
        std::memcpy((char*)x.dst + (b * n + s0) * x.es, a->exp_host + x.off + b * c * x.es, (size_t)(c * x.es));
    }
  }
  return check_device_error(ctx);
}

wg_status wg_agg_emit(wg_agg* a, int64_t start, int64_t max_rows, wg_column* out_cols, int64_t* n_out) {
  if (!a || !n_out || (max_rows > 0 && !out_cols)) return fail(WG_E_INVALID, "NULL argument");
  if (!a->finalized) return fail(WG_E_STATE, "aggregate not finalized");
  Ctx* ctx = a->ctx;
  WG_TRY(ensure_device(ctx));
  const int nk = (int)a->key_cols.size(), na = (int)a->specs.size();
  *n_out = 0;
  if (start < 0 || start >= a->n_out || max_rows <= 0) return WG_OK;
  const int64_t m = std::min<int64_t>(max_rows, a->n_out - start);
  if (!a->resolved) {  // scalar aggregate over no input: COUNT 0, everything else NULL
    for (int i = 0; i < na; ++i) {
      wg_column& c = out_cols[i];
      const bool is_count = a->specs[i].func == WG_AGG_COUNT;
      int ot = a->specs[i].out_type ? a->specs[i].out_type : (is_count ? WG_TYPE_INT64 : WG_TYPE_FLOAT64);
      if (ot == WG_TYPE_INT64) ((int64_t*)c.data)[0] = 0; else ((double*)c.data)[0] = 0.0;
      if (c.valid_words) {
        uint64_t* w = (uint64_t*)c.valid_words;
        w[0] = is_count ? (w[0] | 1ULL) : (w[0] & ~1ULL);
      }
    }
    *n_out = 1;
    return WG_OK;
  }
  FinalArgs A;
  fill_final_args(a, A);
  A.start = start; A.n = m;
  std::vector<DevBuf> bufs((size_t)(nk + na)), vals((size_t)(nk + na));
  std::vector<int64_t> es((size_t)(nk + na));
  for (int c = 0; c < nk + na; ++c) {
    es[c] = c < nk ? (class_of(a->key_types[c]) == WG_CLS_I32 ? 4 : 8) : 8;
    WG_TRY(bufs[c].alloc(ctx, m * es[c]));
    WG_TRY(vals[c].alloc(ctx, m));
    A.out[c] = bufs[c].get();
    A.out_valid[c] = vals[c].as<uint8_t>();
  }
  emit_kernel<<<grid_cap(ctx, m, 256), 256, 0, ctx->stream>>>(A);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  std::vector<std::vector<uint8_t>> hv((size_t)(nk + na), std::vector<uint8_t>((size_t)m));
  for (int c = 0; c < nk + na; ++c) {
    WG_CUDA_TRY(cudaMemcpyAsync((void*)out_cols[c].data, bufs[c].get(), (size_t)(m * es[c]), cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaMemcpyAsync(hv[c].data(), vals[c].get(), (size_t)m, cudaMemcpyDeviceToHost, ctx->stream));
  }
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int c = 0; c < nk + na; ++c) {
    uint64_t* w = (uint64_t*)out_cols[c].valid_words;
    if (!w) continue;
    for (int64_t i = 0; i < m; ++i) {
      if (hv[c][i]) w[i >> 6] |= 1ULL << (i & 63);
      else w[i >> 6] &= ~(1ULL << (i & 63));
    }
  }
  *n_out = m;
  return check_device_error(ctx);
}

wg_status wg_agg_reset(wg_agg* a) {
  if (!a) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(a->ctx));
  a->finalized = false;
  a->n_out = 0;
  strdict_reset(a->sdict, a->ctx);  // the schema (and str_keyed) stays resolved
  if (!a->resolved) return WG_OK;
  Ctx* ctx = a->ctx;
  if (a->spill) {
    a->runs.clear();
    a->block_idx = 0;
    a->block_used = 0;
  }
  if (a->hc) {  // the runs' buffers are kept for the next query; the sketch starts over
    for (auto& r : a->hc_runs) a->hc_free.push_back(std::move(r));
    a->hc_runs.clear();
    if (a->hc_hll.get())
      WG_CUDA_TRY(cudaMemsetAsync(a->hc_hll.get(), 0, (size_t(1) << wgd::kHllBits) * 4, ctx->stream));
  }
  if (a->spilled) {  // the table holds a compact result: back to an empty small table
    // a two-level aggregate keeps the result buffer for its next finalize (as
    // it keeps its runs), instead of freeing and allocating gigabytes per query
    if (a->hc && a->table.bytes() > a->hc_out.bytes()) a->hc_out = std::move(a->table);
    a->table.reset();
    a->cap = a->small_cap;
    a->shift = 64 - log2u(a->cap);
    WG_TRY(a->table.alloc(ctx, table_words(a, a->cap) * 8));
    a->spilled = false;
  }
  const int64_t words = table_words(a, a->cap);
  init_table_kernel<<<grid_cap(ctx, words, 256), 256, 0, ctx->stream>>>(a->table.as<unsigned long long>(), words,
                                                                       a->L.slot_words, a->L);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, ctx->stream));
  a->known_groups = 0;
  a->upper_groups = 0;
  a->dom = 0;
  return WG_OK;
}

// ---- exchange of partial state between ranks -------------------------------

wg_status wg_agg_state_layout(wg_agg* a, wg_state_layout* out) {
  if (!a || !out) return fail(WG_E_INVALID, "NULL argument");
  if (!a->resolved) return fail(WG_E_STATE, "aggregate has no state yet (nothing consumed or merged)");
  std::memset(out, 0, sizeof(*out));
  out->key_words = a->L.key_words;
  out->slot_words = a->L.slot_words;
  out->n_keys = (int32_t)a->key_cols.size();
  out->n_aggs = (int32_t)a->specs.size();
  out->null_word = a->L.key_words == 2 ? a->L.null_word : -1;
  out->null_shift = a->L.null_shift;
  for (int k = 0; k < out->n_keys; ++k) {
    out->key_type[k] = a->key_types[(size_t)k];
    out->key_i32[k] = a->L.key_i32[k];
    out->key_word[k] = a->L.key_word[k];
    out->key_shift[k] = a->L.key_shift[k];
  }
  for (int i = 0; i < out->n_aggs; ++i) {
    out->agg_kind[i] = a->L.agg[i].kind;
    out->agg_off[i] = a->L.agg[i].off;
    out->agg_null_off[i] = a->L.agg[i].null_off;
    out->agg_in_cls[i] = a->in_cls[(size_t)i];
    out->agg_in_scale[i] = a->in_scale[(size_t)i];
    out->agg_out_type[i] = a->out_type[(size_t)i];
    out->agg_nullable[i] = a->nullable[(size_t)i] ? 1 : 0;
  }
  return WG_OK;
}

wg_status wg_agg_partition_state(wg_agg* a, int32_t n_parts, void* rows_dev, int64_t rows_cap, int64_t* part_rows) {
  if (!a || !part_rows || n_parts < 1 || n_parts > 4096) return fail(WG_E_INVALID, "bad partition arguments");
  if (!a->finalized) return fail(WG_E_STATE, "aggregate not finalized");
  if (a->str_keyed == 1) return fail(WG_E_UNSUPPORTED, "string-keyed aggregates are not exchanged");
  Ctx* ctx = a->ctx;
  WG_TRY(ensure_device(ctx));
  for (int p = 0; p < n_parts; ++p) part_rows[p] = 0;
  if (!a->resolved || a->n_out == 0) return WG_OK;
  if (a->n_out > rows_cap) return fail(WG_E_INVALID, "rows_cap is smaller than the aggregate's group count");
  if (!rows_dev) return fail(WG_E_INVALID, "rows_dev is NULL");
  DevBuf cnt;
  WG_TRY(cnt.alloc(ctx, (int64_t)n_parts * 8));
  WG_CUDA_TRY(cudaMemsetAsync(cnt.get(), 0, (size_t)n_parts * 8, ctx->stream));
  const Table T = table_view(a);
  const unsigned grid = grid_cap(ctx, a->n_out, 256);
  state_count_kernel<<<grid, 256, 0, ctx->stream>>>(a->L, T, a->list.as<int64_t>(), a->n_out, n_parts,
                                                    cnt.as<unsigned long long>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  std::vector<unsigned long long> c((size_t)n_parts), cur((size_t)n_parts);
  WG_CUDA_TRY(cudaMemcpyAsync(c.data(), cnt.get(), (size_t)n_parts * 8, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  unsigned long long acc = 0;
  for (int p = 0; p < n_parts; ++p) { cur[(size_t)p] = acc; acc += c[(size_t)p]; part_rows[p] = (int64_t)c[(size_t)p]; }
  if ((int64_t)acc != a->n_out) return fail(WG_E_CUDA, "state partition counts do not add up to the group count");
  WG_CUDA_TRY(cudaMemcpyAsync(cnt.get(), cur.data(), (size_t)n_parts * 8, cudaMemcpyHostToDevice, ctx->stream));
  state_scatter_kernel<<<grid, 256, 0, ctx->stream>>>(a->L, T, a->list.as<int64_t>(), a->n_out, n_parts,
                                                      cnt.as<unsigned long long>(), (unsigned long long*)rows_dev);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

wg_status wg_agg_merge_state(wg_agg* a, const wg_state_layout* src, const void* rows_dev, int64_t n_rows) {
  if (!a || !src || n_rows < 0 || (n_rows > 0 && !rows_dev)) return fail(WG_E_INVALID, "NULL argument");
  if (a->finalized) return fail(WG_E_STATE, "aggregate already finalized");
  if (a->spill) return fail(WG_E_UNSUPPORTED, "spilled aggregations are not merged");
  if (a->str_keyed == 1) return fail(WG_E_UNSUPPORTED, "string-keyed aggregates are not merged");
  if (src->n_keys != (int32_t)a->key_cols.size() || src->n_aggs != (int32_t)a->specs.size() ||
      src->n_aggs > WG_MAX_AGGS || src->n_keys > WG_MAX_KEYS || src->slot_words > WG_MAX_SLOT_WORDS)
    return fail(WG_E_INVALID, "state layout does not match the aggregate's shape");
  Ctx* ctx = a->ctx;
  WG_TRY(ensure_device(ctx));
  a->dom = 2;  // merged keys have no tracked range
  // the layout a source with these kinds and null counters has
  wg_agg ref;
  ref.key_cols = a->key_cols;
  ref.specs = a->specs;
  ref.kind.assign(src->agg_kind, src->agg_kind + src->n_aggs);
  ref.nullable.assign((size_t)src->n_aggs, false);
  for (int i = 0; i < src->n_aggs; ++i) ref.nullable[(size_t)i] = src->agg_nullable[i] != 0;
  std::memset(&ref.L, 0, sizeof(ref.L));
  ref.L.key_words = src->key_words;
  build_layout(&ref);
  ref.L.null_word = src->null_word;
  ref.L.null_shift = src->null_shift;
  for (int k = 0; k < src->n_keys; ++k) {
    ref.L.key_i32[k] = src->key_i32[k];
    ref.L.key_word[k] = src->key_word[k];
    ref.L.key_shift[k] = src->key_shift[k];
    ref.L.key_vcol[k] = a->key_cols[(size_t)k];
  }
  bool same = ref.L.slot_words == src->slot_words;
  for (int i = 0; i < src->n_aggs && same; ++i)
    same = ref.L.agg[i].off == src->agg_off[i] && ref.L.agg[i].null_off == src->agg_null_off[i];
  if (!same) return fail(WG_E_INVALID, "state layout is inconsistent with its aggregate kinds");
  if (!a->resolved) {
    // adopt the source's resolved schema (mergeSinkState inherits it, aggregate.go:4722)
    a->key_types.assign(src->key_type, src->key_type + src->n_keys);
    a->in_cls.assign(src->agg_in_cls, src->agg_in_cls + src->n_aggs);
    a->in_scale.assign(src->agg_in_scale, src->agg_in_scale + src->n_aggs);
    a->out_type.assign(src->agg_out_type, src->agg_out_type + src->n_aggs);
    a->kind = ref.kind;
    a->nullable = ref.nullable;
    a->L = ref.L;
    a->cap = a->L.key_words == 0 ? 1 : cap_for(std::max<int64_t>(std::max<int64_t>(a->hint, n_rows), 1024));
    a->shift = 64 - log2u(a->cap);
    WG_TRY(init_table(a, a->table, a->cap));
    WG_TRY(a->ctr.alloc(ctx, 64));
    WG_CUDA_TRY(cudaMemsetAsync(a->ctr.get(), 0, 64, ctx->stream));
    a->known_groups = a->upper_groups = 0;
    a->dom = 0;
    a->resolved = true;
  }
  if (a->L.key_words != src->key_words || a->kind != ref.kind)
    return fail(WG_E_INVALID, "aggregate input types differ");
  // the destination must carry every null counter the source has
  bool upgrade = false;
  std::vector<bool> nn = a->nullable;
  for (size_t i = 0; i < nn.size(); ++i) if (ref.nullable[i] && !nn[i]) { nn[i] = true; upgrade = true; }
  if (upgrade) {
    wg_agg tmp;
    tmp.key_cols = a->key_cols; tmp.specs = a->specs; tmp.kind = a->kind; tmp.nullable = nn; tmp.L = a->L;
    build_layout(&tmp);
    for (int k = 0; k < WG_MAX_KEYS; ++k) tmp.L.key_vcol[k] = a->L.key_vcol[k];
    a->nullable = nn;
    WG_TRY(rebuild_table(a, a->cap, tmp.L));
  }
  if (n_rows == 0) return WG_OK;
  WG_TRY(refresh_groups(a));
  const int64_t need = a->known_groups + n_rows + credit_slack(a);
  if (a->L.key_words != 0 && need > (int64_t)((double)a->cap * kMaxLoad)) WG_TRY(rebuild_table(a, cap_for(need), a->L));
  const unsigned grid = grid_cap(ctx, n_rows, 256);
  if (ref.L.n_aggs <= 4) state_merge_kernel<4><<<grid, 256, 0, ctx->stream>>>(ref.L, (const unsigned long long*)rows_dev,
                                                                          n_rows, a->L, table_view(a), ctx->dev_error);
  else state_merge_kernel<8><<<grid, 256, 0, ctx->stream>>>(ref.L, (const unsigned long long*)rows_dev, n_rows, a->L,
                                                           table_view(a), ctx->dev_error);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_TRY(refresh_groups(a));
  int64_t v[2];
  WG_TRY(read_back_i64(ctx, (const int64_t*)a->ctr.get(), v, 2));
  if ((int32_t)v[1] != 0) return fail(WG_E_NOMEM, "aggregate table overflow while merging state rows");
  return check_device_error(ctx);
}

int32_t wg_agg_kernel_shape(const wg_agg* a) { return a ? a->last_shape : -1; }

wg_status wg_agg_destroy(wg_agg* a) {
  if (!a) return WG_OK;
  ensure_device(a->ctx);
  cudaStreamSynchronize(a->ctx->stream);
  strdict_free(a->sdict);
  delete a;
  return WG_OK;
}

wg_status wg_agg_key_strings(wg_agg* a, const int64_t* ids, int64_t n, uint32_t* out_offsets, uint8_t* out_bytes,
                             int64_t bytes_cap, int64_t* need_bytes) {
  if (!a || n < 0 || (n > 0 && !ids) || !out_offsets || !need_bytes || bytes_cap < 0 || (bytes_cap > 0 && !out_bytes))
    return fail(WG_E_INVALID, "bad key-string arguments");
  if (a->str_keyed != 1) return fail(WG_E_STATE, "the aggregate is not grouped by a string column");
  WG_TRY(ensure_device(a->ctx));
  return strdict_strings(a->ctx, a->sdict, ids, n, out_offsets, out_bytes, bytes_cap, need_bytes);
}

}  // extern "C"

// ===========================================================================
// Batched mode: many small filter + GROUP BY queries in one persistent launch.
//
// Every query keeps its own aggregate (table, layout, launch plan); a work list
// of (query, row window) items is drained by persistent CTAs through an atomic
// cursor. Queries expecting few groups pre-combine each work item in a
// shared-memory table flushed to their HBM table at the end of the item. The
// whole run — table resets, the kernel, the group counts and their copy to the
// host — is captured once in a CUDA graph and replayed.
// ===========================================================================
namespace {

struct BatchItem {
  int32_t q;
  int32_t rows;
  int64_t row0;
};

struct ResetDesc {
  unsigned long long* slots;
  int64_t words;
  int32_t sw;
  int32_t key_words;
  unsigned long long* ctr;
  uint64_t cap;
  unsigned long long init[WG_MAX_SLOT_WORDS];
};

__global__ void batched_reset_kernel(const ResetDesc* rd, int n) {
  for (int q = blockIdx.x; q < n; q += gridDim.x) {
    const ResetDesc& r = rd[q];
    for (int64_t i = threadIdx.x; i < r.words; i += blockDim.x) r.slots[i] = r.init[i % r.sw];
    if (threadIdx.x < 8) r.ctr[threadIdx.x] = 0;
  }
}

// groups per query: regular slots taken + the two special slots when used; -1 on overflow
__global__ void batched_count_kernel(const ResetDesc* rd, int n, long long* out) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const ResetDesc& r = rd[q];
    if (((const int32_t*)(r.ctr + 1))[0] != 0) { out[q] = -1; continue; }
    if (r.key_words == 0) { out[q] = 1; continue; }
    long long g = (long long)r.ctr[0];
    g += r.slots[r.cap * r.sw + r.key_words] != 0;
    g += r.slots[(r.cap + 1) * r.sw + r.key_words] != 0;
    out[q] = g;
  }
}

// One work item (a window of one query's rows) on shape Sh.
// The rows of one work item: 2 consecutive rows per lane with vector loads
// (every row's loads in flight before its updates) when the query has a
// compiled shape and vector-aligned columns (P.vec_rows, set by the host), one
// row per lane otherwise.
template <int NA, bool SMEM, class Sh>
__device__ __forceinline__ void batched_rows(const Plan& P, const Sh& sh, const BatchItem& w, unsigned long long* sm,
                                             int* s_groups, int s_limit, Credit& cr) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if constexpr (!std::is_same<Sh, DynShape>::value) {
    if (P.vec_rows) {
      constexpr int U = 2;
      const int64_t end = w.row0 + w.rows;
      for (int64_t base = w.row0 + (int64_t)warp * 32 * U; base < end; base += (int64_t)nw * 32 * U) {
        const int64_t r0 = base + (int64_t)lane * U;
        SrcRow rw[U];
        load_rows<U>(P, sh, r0, rw, end);
        process_loaded_vec<NA, SMEM, U>(P, sh, r0, rw, sm, s_groups, s_limit, cr, end);
      }
      return;
    }
  }
  for (int base = warp * 32; base < w.rows; base += nw * 32) {
    const int i = base + lane;
    SrcGlobal src{w.row0 + (i < w.rows ? i : 0)};
    process_rows<NA, SMEM>(P, sh, src, i < w.rows, sm, s_groups, s_limit, cr);
  }
}

template <int NA, class Sh>
__device__ __forceinline__ void batched_item(const Plan& P, const BatchItem& w, unsigned long long* sm,
                                             int* s_groups) {
  const Sh sh{P};
  Credit cr;  // reservations in this query's table, handed back before the next item
  const int S = P.smem_slots;
  if (Sh::smem_ok && S > 0) {
    smem_table_init(P, sm, S, s_groups);
    __syncthreads();
    batched_rows<NA, Sh::smem_ok>(P, sh, w, sm, s_groups, (S * 7) / 8, cr);
    __syncthreads();
    smem_table_flush<NA>(P, sm, S, cr);
  } else {
    batched_rows<NA, false>(P, sh, w, sm, s_groups, 0, cr);
  }
  cr.release(P.T);
}

// STATIC_ONLY: every query has a compiled shape, so the generic path (and its
// registers) is left out and MB CTAs of 512 threads fit an SM.
template <int NA, bool STATIC_ONLY, int MB>
__global__ void __launch_bounds__(512, MB) batched_kernel(const Plan* plans, const BatchItem* items, int64_t n_items,
                                                          unsigned long long* cursor) {
  extern __shared__ unsigned long long sm[];
  __shared__ int s_groups;
  __shared__ long long s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = (long long)atomicAdd(cursor, 1ULL);
    __syncthreads();
    const long long it = s_item;
    if (it >= n_items) break;
    const BatchItem w = items[it];
    const Plan& P = plans[w.q];
    switch (P.shape) {
      case SHAPE_BATCH_I64: batched_item<ShapeBatchI64::n_aggs, StatShape<ShapeBatchI64>>(P, w, sm, &s_groups); break;
      case SHAPE_BATCH_F64: batched_item<ShapeBatchF64::n_aggs, StatShape<ShapeBatchF64>>(P, w, sm, &s_groups); break;
      default:
        if constexpr (!STATIC_ONLY) batched_item<NA, DynShape>(P, w, sm, &s_groups);
        break;
    }
    __syncthreads();
  }
}

}  // namespace

struct wg_batched {
  wg::Ctx* ctx;
  std::vector<wg_agg*> aggs;
  std::vector<wg_batch_desc> inputs;
  std::vector<std::vector<wg_column>> cols;
  std::vector<std::vector<wg_predicate>> filters;
  std::vector<wg_join*> joins;
  std::vector<std::vector<wg_expr>> exprs;
  wg_tune_params tp{};
  int max_na = 4;
  bool all_static = false;   // every query runs a compiled shape
  size_t dyn_smem = 0;
  std::vector<wgd::Plan> plans_h;
  std::vector<BatchItem> items_h;
  std::vector<ResetDesc> reset_h;
  wg::DevBuf plans, items, resets, cursor, counts;
  long long* counts_host = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace wg {

static wg_status batched_plan(wg_batched* b) {
  Ctx* ctx = b->ctx;
  const int n = (int)b->aggs.size();
  b->plans_h.assign((size_t)n, wgd::Plan{});
  b->reset_h.assign((size_t)n, ResetDesc{});
  b->max_na = 4;
  b->all_static = true;
  int64_t max_smem_words = 0;
  for (int q = 0; q < n; ++q) {
    wg_agg* a = b->aggs[q];
    PipelineRun r{a, &b->inputs[q], (int32_t)b->filters[q].size(), b->filters[q].data(), b->joins[q],
                  (int32_t)b->exprs[q].size(), b->exprs[q].data()};
    LaunchSpec ls;
    VSchema vs;
    std::vector<int> in_map;
    WG_TRY(build_plan(r, ls.P, vs, in_map));
    if (ls.P.sel) return fail(WG_E_INVALID, "batched inputs must not carry a selection vector");
    wgd::Plan& P = b->plans_h[q];
    P = ls.P;
    P.T = table_view(a);
    wgd::Layout L = a->L;
    for (int k = 0; k < WG_MAX_KEYS; ++k) L.key_vcol[k] = ls.P.L.key_vcol[k];
    for (int i = 0; i < WG_MAX_AGGS; ++i) L.agg[i].vcol = ls.P.L.agg[i].vcol;
    P.L = L;
    P.err = ctx->dev_error;
    bool plain = a->L.key_words == 1;
    for (int i = 0; i < a->L.n_aggs; ++i)
      plain = plain && a->L.agg[i].null_off < 0 && a->L.agg[i].kind != wgd::K_MIN_DEC && a->L.agg[i].kind != wgd::K_MAX_DEC;
    const int64_t smax = b->tp.smem_max_groups;
    int S = 0;
    if (plain && a->hint > 0 && a->hint <= smax) {
      // at most the shared memory one CTA may take; a table that would then run
      // more than 3/4 full stays in HBM
      const int64_t fit = ((int64_t)ctx->max_smem_optin - 1024) / (a->L.slot_words * 8);
      S = (int)std::min<int64_t>(fit, std::max<int64_t>(256, std::min<int64_t>(16384, a->hint * 2)));
      if ((int64_t)S * 3 < a->hint * 4) S = 0;
      max_smem_words = std::max<int64_t>(max_smem_words, (int64_t)S * a->L.slot_words);
    }
    P.smem_slots = S;
    {
      const int mm = env_int("WG_MINMAX_TEST", -1);
      P.minmax_test = mm >= 0 ? (mm != 0) : (b->inputs[q].len >= 8 * std::max<int64_t>(a->hint, 1));
    }
    P.shape = pick_shape(P);
    if (P.shape != wgd::SHAPE_BATCH_I64 && P.shape != wgd::SHAPE_BATCH_F64) P.shape = wgd::SHAPE_GENERIC;
    // compiled shapes over 16-byte aligned columns take 2 rows per lane with vector loads
    {
      bool vec = P.shape != wgd::SHAPE_GENERIC && !P.has_join && env_int("WG_BATCH_VEC", 1) != 0;
      for (int j = 0; j < P.n_in; ++j) vec = vec && ((uintptr_t)P.in[j].data % 16 == 0);
      P.vec_rows = vec ? 1 : 0;
    }
    a->last_shape = P.shape;
    if (a->L.n_aggs > 4) b->max_na = 8;
    if (P.shape == wgd::SHAPE_GENERIC) b->all_static = false;
    ResetDesc& rd = b->reset_h[q];
    rd.slots = a->table.as<unsigned long long>();
    rd.words = table_words(a, a->cap);
    rd.sw = a->L.slot_words;
    rd.key_words = a->L.key_words;
    rd.ctr = a->ctr.as<unsigned long long>();
    rd.cap = a->cap;
    for (int i = 0; i < WG_MAX_SLOT_WORDS; ++i) rd.init[i] = a->L.init[i];
  }
  b->dyn_smem = (size_t)max_smem_words * 8;
  if ((int64_t)b->dyn_smem > (int64_t)ctx->max_smem_optin - 1024) return fail(WG_E_INVALID, "shared-memory table too large");
  WG_TRY(b->plans.ensure(ctx, (int64_t)sizeof(wgd::Plan) * n));
  WG_TRY(b->resets.ensure(ctx, (int64_t)sizeof(ResetDesc) * n));
  WG_CUDA_TRY(cudaMemcpy(b->plans.get(), b->plans_h.data(), sizeof(wgd::Plan) * n, cudaMemcpyHostToDevice));
  WG_CUDA_TRY(cudaMemcpy(b->resets.get(), b->reset_h.data(), sizeof(ResetDesc) * n, cudaMemcpyHostToDevice));
  // work items: tile_rows-row windows of every query, largest queries first
  std::vector<int> order((size_t)n);
  for (int q = 0; q < n; ++q) order[q] = q;
  std::sort(order.begin(), order.end(), [&](int x, int y) { return b->inputs[x].len > b->inputs[y].len; });
  b->items_h.clear();
  for (int q : order)
    for (int64_t r0 = 0; r0 < b->inputs[q].len; r0 += b->tp.tile_rows)
      b->items_h.push_back(BatchItem{q, (int32_t)std::min<int64_t>(b->tp.tile_rows, b->inputs[q].len - r0), r0});
  WG_TRY(b->items.ensure(ctx, (int64_t)(sizeof(BatchItem) * std::max<size_t>(1, b->items_h.size()))));
  if (!b->items_h.empty())
    WG_CUDA_TRY(cudaMemcpy(b->items.get(), b->items_h.data(), sizeof(BatchItem) * b->items_h.size(), cudaMemcpyHostToDevice));
  WG_TRY(b->cursor.ensure(ctx, 64));
  WG_TRY(b->counts.ensure(ctx, 8 * (int64_t)std::max(1, n)));
  return WG_OK;
}

static void batched_enqueue(wg_batched* b, cudaStream_t st) {
  Ctx* ctx = b->ctx;
  const int n = (int)b->aggs.size();
  batched_reset_kernel<<<std::min(n, ctx->sm_count * 8), 256, 0, st>>>(b->resets.as<ResetDesc>(), n);
  cudaMemsetAsync(b->cursor.get(), 0, 8, st);
  const unsigned grid = (unsigned)(ctx->sm_count * std::max(1, b->tp.ctas_per_sm));
  if (b->all_static) {
    batched_kernel<4, true, 2><<<grid, b->tp.block, b->dyn_smem, st>>>(
        b->plans.as<wgd::Plan>(), b->items.as<BatchItem>(), (int64_t)b->items_h.size(), b->cursor.as<unsigned long long>());
  } else if (b->max_na <= 4) {
    batched_kernel<4, false, 2><<<grid, b->tp.block, b->dyn_smem, st>>>(
        b->plans.as<wgd::Plan>(), b->items.as<BatchItem>(), (int64_t)b->items_h.size(), b->cursor.as<unsigned long long>());
  } else {
    batched_kernel<8, false, 2><<<grid, b->tp.block, b->dyn_smem, st>>>(
        b->plans.as<wgd::Plan>(), b->items.as<BatchItem>(), (int64_t)b->items_h.size(), b->cursor.as<unsigned long long>());
  }
  batched_count_kernel<<<(n + 255) / 256, 256, 0, st>>>(b->resets.as<ResetDesc>(), n, b->counts.as<long long>());
  cudaMemcpyAsync(b->counts_host, b->counts.get(), 8 * (size_t)n, cudaMemcpyDeviceToHost, st);
}

static wg_status batched_capture(wg_batched* b) {
  Ctx* ctx = b->ctx;
  if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
  if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
  WG_CUDA_TRY(cudaFuncSetAttribute(batched_kernel<4, true, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->dyn_smem));
  WG_CUDA_TRY(cudaFuncSetAttribute(batched_kernel<4, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->dyn_smem));
  WG_CUDA_TRY(cudaFuncSetAttribute(batched_kernel<8, false, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)b->dyn_smem));
  WG_CUDA_TRY(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
  batched_enqueue(b, ctx->stream);
  WG_CUDA_TRY(cudaStreamEndCapture(ctx->stream, &b->graph));
  WG_CUDA_TRY(cudaGraphInstantiate(&b->exec, b->graph, 0));
  return WG_OK;
}

}  // namespace wg

extern "C" {

wg_status wg_batched_create(wg_ctx* ctx, int32_t n, const wg_batched_query* qs, const wg_tune_params* params,
                            wg_batched** out) {
  if (!ctx || !out || n < 1 || !qs) return fail(WG_E_INVALID, "bad batched arguments");
  WG_TRY(ensure_device(ctx));
  wg_batched* b = new wg_batched();
  b->ctx = ctx;
  wg_tune_params tp{};
  if (params) tp = *params;
  if (tp.tile_rows <= 0) tp.tile_rows = 1 << 15;
  tp.tile_rows = std::max(64, tp.tile_rows & ~63);
  if (tp.block <= 0) tp.block = 512;
  tp.block = std::max(64, std::min(512, tp.block & ~31));
  if (tp.ctas_per_sm <= 0) tp.ctas_per_sm = 2;
  if (tp.smem_max_groups == 0) tp.smem_max_groups = 2048;  // negative: never use shared memory
  if (tp.smem_max_groups < 0) tp.smem_max_groups = 0;
  if (tp.max_load <= 0.0 || tp.max_load > kMaxLoad) tp.max_load = 0.5;
  b->tp = tp;
  b->aggs.resize((size_t)n, nullptr);
  b->inputs.resize((size_t)n);
  b->cols.resize((size_t)n);
  b->filters.resize((size_t)n);
  b->joins.assign((size_t)n, nullptr);
  b->exprs.resize((size_t)n);
  auto cleanup = [&](wg_status s) { wg_batched_destroy(b); return s; };
  for (int q = 0; q < n; ++q) {
    const wg_batched_query& x = qs[q];
    if (!x.input || x.input->sel || x.n_filters < 0 || x.n_filters > WG_MAX_FILTERS)
      return cleanup(fail(WG_E_INVALID, "batched query " + std::to_string(q) + ": bad input or filters"));
    b->cols[q].assign(x.input->cols, x.input->cols + x.input->ncols);
    b->inputs[q] = *x.input;
    b->inputs[q].cols = b->cols[q].data();
    b->filters[q].assign(x.filters, x.filters + x.n_filters);
    if (x.n_exprs < 0 || x.n_exprs > WG_MAX_EXPRS || (x.n_exprs > 0 && !x.exprs))
      return cleanup(fail(WG_E_INVALID, "batched query " + std::to_string(q) + ": bad projections"));
    b->exprs[q].assign(x.exprs, x.exprs + x.n_exprs);
    if (x.join && join_is_grace(x.join))
      return cleanup(fail(WG_E_UNSUPPORTED, "batched query " + std::to_string(q) +
                                                ": a partitioned join build runs through the pipeline entry points"));
    b->joins[q] = x.join;
    wg_status s = wg_agg_create(ctx, x.n_keys, x.key_cols, x.n_aggs, x.aggs, x.ndv_hint, &b->aggs[q]);
    if (s != WG_OK) return cleanup(s);
    wg_agg* a = b->aggs[q];
    // resolve the aggregate against the query's schema, sized for its hint
    PipelineRun r{a, &b->inputs[q], (int32_t)b->filters[q].size(), b->filters[q].data(), b->joins[q],
                  (int32_t)b->exprs[q].size(), b->exprs[q].data()};
    LaunchSpec ls;
    VSchema vs;
    std::vector<int> in_map;
    s = build_plan(r, ls.P, vs, in_map);
    if (s == WG_OK) s = agg_resolve(a, vs);
    if (s == WG_OK && a->L.key_words != 0) {
      uint64_t cap = 1024;
      while ((double)cap * tp.max_load < (double)std::max<int64_t>(1, x.ndv_hint)) cap <<= 1;
      if (cap != a->cap) s = rebuild_table(a, cap, a->L);
    }
    if (s != WG_OK) return cleanup(s);
  }
  if (cudaMallocHost((void**)&b->counts_host, 8 * (size_t)n) != cudaSuccess)
    return cleanup(fail(WG_E_CUDA, "pinned counts"));
  wg_status s = batched_plan(b);
  if (s == WG_OK) s = batched_capture(b);
  if (s != WG_OK) return cleanup(s);
  *out = b;
  return WG_OK;
}

wg_status wg_batched_run(wg_batched* b, int64_t* n_groups) {
  if (!b) return fail(WG_E_INVALID, "batched is NULL");
  Ctx* ctx = b->ctx;
  WG_TRY(ensure_device(ctx));
  WG_CUDA_TRY(cudaGraphLaunch(b->exec, ctx->stream));
  ctx->count_launch(4);
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  WG_TRY(check_device_error(ctx));
  const int n = (int)b->aggs.size();
  bool replan = false;
  for (int q = 0; q < n; ++q) {
    wg_agg* a = b->aggs[q];
    a->finalized = false;
    if (b->counts_host[q] >= 0) continue;
    // this query outgrew its hint: rerun it alone on a 4x table
    WG_TRY(rebuild_table(a, a->cap * 4, a->L));
    WG_TRY(wg_agg_reset(a));
    PipelineRun r{a, &b->inputs[q], (int32_t)b->filters[q].size(), b->filters[q].data(), nullptr, 0, nullptr};
    WG_TRY(run_device(r));
    int64_t g = 0;
    WG_TRY(wg_agg_finalize(a, &g));
    a->finalized = false;
    b->counts_host[q] = g;
    replan = true;
  }
  if (n_groups)
    for (int q = 0; q < n; ++q) n_groups[q] = b->counts_host[q];
  if (replan) {  // tables moved: the graph must point at the new ones
    WG_TRY(batched_plan(b));
    WG_TRY(batched_capture(b));
  }
  return WG_OK;
}

wg_status wg_batched_export(wg_batched* b, int32_t q, const wg_group_export* out) {
  if (!b || q < 0 || q >= (int32_t)b->aggs.size()) return fail(WG_E_INVALID, "bad query index");
  wg_agg* a = b->aggs[q];
  a->finalized = false;
  int64_t g = 0;
  WG_TRY(wg_agg_finalize(a, &g));
  wg_status s = wg_agg_export(a, out);
  a->finalized = false;
  return s;
}

wg_status wg_batched_destroy(wg_batched* b) {
  if (!b) return WG_OK;
  ensure_device(b->ctx);
  cudaStreamSynchronize(b->ctx->stream);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->counts_host) cudaFreeHost(b->counts_host);
  for (wg_agg* a : b->aggs)
    if (a) wg_agg_destroy(a);
  delete b;
  return WG_OK;
}

}  // extern "C"
