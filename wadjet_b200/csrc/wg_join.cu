// wg_join.cu — exec.HashJoin (inner, int key) on the GPU.
//
// Build (HashJoin.Build, internal/engine/exec/join.go:771 → arenaAppendInt :551):
// build batches are appended to device-resident key/payload columns; finish
// sizes an open-addressing table at <= 50% load and inserts every non-NULL key
// with one thread per build row. A 64-bit (or 128-bit) atomicCAS swaps the
// slot's head to the inserting row and the replaced head becomes next[row] —
// the chained arena of the reference, built in parallel. Chains hold the same
// rows as the reference's; their order among equal keys is the order the
// atomics landed in, which a canonical sort of the join output makes moot.
//
// Probe (HashJoinProbe.Execute → inlineIntProbe, join.go:2306,2670) with the
// bounded-output protocol (operators.go:86): pairs are counted per probe row,
// scanned, and the window [cursor, cursor + cap) of the ordered pair list is
// written.
#include "wg_internal.h"
#include "wg_join.cuh"

#include <cub/cub.cuh>

#include <climits>
#include <cstdlib>

namespace {

using namespace wgd;

constexpr long long kCasLimit = 1LL << 24;

struct BuildArgs {
  DCol key;
  int64_t n;
  int32_t flavor;
  int32_t shift;
  uint64_t mask;
  void* slots;
  int32_t* next;
  unsigned long long* distinct;
  int32_t* dup;
  int32_t* err;
};

__global__ void join_build_kernel(const BuildArgs a) {
  for (int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; row < a.n;
       row += (int64_t)gridDim.x * blockDim.x) {
    if (is_null(a.key, row)) continue;
    const int64_t key = ld_i64(a.key, row);
    uint64_t h = fib_slot((uint64_t)key, a.shift);
    uint64_t probes = 0;
    long long spins = 0;
    bool done = false;
    if (a.flavor == 0) {
      unsigned long long* s = (unsigned long long*)a.slots;
      const unsigned long long mine = ((unsigned long long)(uint32_t)row << 32) | (uint32_t)(int32_t)key;
      unsigned long long cur = *((volatile unsigned long long*)(s + h));
      while (!done) {
        if (++spins > kCasLimit) { set_error(a.err, WG_DERR_TIMEOUT); break; }
        const int32_t head = (int32_t)(cur >> 32);
        if (head == -1 || (uint32_t)cur == (uint32_t)(int32_t)key) {
          unsigned long long old = atomicCAS(s + h, cur, mine);
          if (old == cur) {
            a.next[row] = head;
            if (head == -1) atomicAdd(a.distinct, 1ULL); else *a.dup = 1;
            done = true;
          } else {
            cur = old;  // lost a race on this slot: re-examine it
          }
        } else {
          if (++probes > a.mask) { set_error(a.err, WG_DERR_TABLE_FULL); break; }
          h = (h + 1) & a.mask;
          cur = *((volatile unsigned long long*)(s + h));
        }
      }
    } else {
      U128* s = (U128*)a.slots;
      U128 mine;
      mine.lo = (unsigned long long)key;
      mine.hi = (unsigned long long)(uint32_t)row;
      U128 cur = read128(s + h);  // may be torn; every decision is confirmed by a CAS
      while (!done) {
        if (++spins > kCasLimit) { set_error(a.err, WG_DERR_TIMEOUT); break; }
        const int32_t head = (int32_t)(uint32_t)cur.hi;
        if (head == -1 || (int64_t)cur.lo == key) {
          U128 old = cas128(s + h, cur, mine);
          if (old.lo == cur.lo && old.hi == cur.hi) {
            a.next[row] = head;
            if (head == -1) atomicAdd(a.distinct, 1ULL); else *a.dup = 1;
            done = true;
          } else {
            cur = old;
          }
        } else {
          const U128 chk = cas128(s + h, cur, cur);  // the slot really holds another key?
          if (chk.lo != cur.lo || chk.hi != cur.hi) { cur = chk; continue; }
          if (++probes > a.mask) { set_error(a.err, WG_DERR_TABLE_FULL); break; }
          h = (h + 1) & a.mask;
          cur = read128(s + h);
        }
      }
    }
  }
}

struct ProbeArgs {
  JoinView j;
  DCol key;
  const uint32_t* sel;
  int64_t n;
  int64_t* counts;
  const int64_t* offs;
  int64_t cursor;
  int64_t cap;
  uint32_t* out_probe;
  int64_t* out_build;
  int32_t* err;
};

// Output pairs of one probe row by join type: inner = the chain's length;
// left = at least one (an unmatched row once, NULL-padded, join.go:3180);
// semi = one when the chain is not empty; anti = one when it is (a NULL key
// never matches, so it passes an anti join, join.go:3290).
__device__ __forceinline__ int32_t probe_head(const ProbeArgs& a, int64_t row) {
  return is_null(a.key, row) ? -1 : join_head(a.j, ld_i64(a.key, row), a.err);
}

__global__ void join_probe_count_kernel(const ProbeArgs a) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = a.sel ? (int64_t)a.sel[p] : p;
    const int32_t head = probe_head(a, row);
    int64_t c = 0;
    if (a.j.jtype == WG_JOIN_SEMI) c = head >= 0;
    else if (a.j.jtype == WG_JOIN_ANTI) c = head < 0;
    else {
      for (int32_t ref = head; ref >= 0; ref = __ldg(a.j.next + ref)) ++c;
      if (a.j.jtype == WG_JOIN_LEFT && c == 0) c = 1;
    }
    a.counts[p] = c;
  }
}

__global__ void join_probe_emit_kernel(const ProbeArgs a) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < a.n; p += (int64_t)gridDim.x * blockDim.x) {
    if (a.counts[p] == 0) continue;
    int64_t j = a.offs[p];
    if (j >= a.cursor + a.cap || j + a.counts[p] <= a.cursor) continue;
    const int64_t row = a.sel ? (int64_t)a.sel[p] : p;
    const int32_t head = probe_head(a, row);
    if (a.j.jtype == WG_JOIN_SEMI || a.j.jtype == WG_JOIN_ANTI || head < 0) {  // one pair, no build row
      a.out_probe[j - a.cursor] = (uint32_t)row;
      a.out_build[j - a.cursor] = -1;
      continue;
    }
    for (int32_t ref = head; ref >= 0 && j < a.cursor + a.cap; ref = __ldg(a.j.next + ref), ++j) {
      if (j >= a.cursor) {
        a.out_probe[j - a.cursor] = (uint32_t)row;
        a.out_build[j - a.cursor] = ref;
      }
    }
  }
}

// Smallest and largest non-NULL value of an integer column (the build key's,
// to pick a sentinel that is not a key; a payload's, for dense GROUP BY).
// Reduced per warp and per CTA, then one atomic pair per CTA.
__global__ void key_range_kernel(DCol key, int64_t n, long long* mn, long long* mx) {
  long long lo = LLONG_MAX, hi = LLONG_MIN;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (is_null(key, i)) continue;
    const long long k = ld_i64(key, i);
    lo = k < lo ? k : lo;
    hi = k > hi ? k : hi;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const long long l2 = __shfl_down_sync(WG_FULL_MASK, lo, o), h2 = __shfl_down_sync(WG_FULL_MASK, hi, o);
    lo = l2 < lo ? l2 : lo;
    hi = h2 > hi ? h2 : hi;
  }
  __shared__ long long s_lo[32], s_hi[32];
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = (blockDim.x + 31) >> 5;
  if (l == 0) { s_lo[w] = lo; s_hi[w] = hi; }
  __syncthreads();
  if (w == 0) {
    lo = l < nw ? s_lo[l] : LLONG_MAX;
    hi = l < nw ? s_hi[l] : LLONG_MIN;
    for (int o = 16; o > 0; o >>= 1) {
      const long long l2 = __shfl_down_sync(WG_FULL_MASK, lo, o), h2 = __shfl_down_sync(WG_FULL_MASK, hi, o);
      lo = l2 < lo ? l2 : lo;
      hi = h2 > hi ? h2 : hi;
    }
    if (l == 0) {
      atomicMin(mn, lo);
      atomicMax(mx, hi);
    }
  }
}

// Rewrite a unique-key table as {key32, payload32} slots (empty = sentinel key).
__global__ void direct_table_kernel(const unsigned long long* slots, uint64_t cap, const uint32_t* pay,
                                    int32_t sentinel, unsigned long long* out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
    const unsigned long long v = slots[i];
    const int32_t head = (int32_t)(v >> 32);
    out[i] = head < 0 ? (unsigned long long)(uint32_t)sentinel
                      : ((unsigned long long)pay[head] << 32) | (uint32_t)v;
  }
}

// Dense direct table: slot (key - base) = {key32, payload32}; slots without a
// key keep {sentinel, 0} from the fill before this kernel.
__global__ void dense_table_kernel(DCol key, int64_t n, const uint32_t* pay, long long base,
                                   unsigned long long* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (is_null(key, i)) continue;
    const long long k = ld_i64(key, i);
    out[k - base] = ((unsigned long long)pay[i] << 32) | (uint32_t)(int32_t)k;
  }
}

// Dense direct table built straight from the build rows, before any hash index
// exists: each key claims its slot with a compare-and-swap from the empty word,
// so a second row with the same key finds the slot taken and flags `dup`.
__global__ void dense_build_kernel(DCol key, int64_t n, const uint32_t* pay, long long base,
                                   unsigned long long empty, unsigned long long* out, int32_t* dup) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const long long k = ld_i64(key, i);
    const unsigned long long mine = ((unsigned long long)__ldg(pay + i) << 32) | (uint32_t)(int32_t)k;
    if (atomicCAS(out + (k - base), empty, mine) != empty) *dup = 1;
  }
}

// The bloom's bits for every build row with a key (duplicates set the same
// bits as their key's first row, so this is the bloom over distinct keys).
__global__ void bloom_build_kernel(DCol key, int64_t n, unsigned long long* bloom, unsigned long long mask) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (is_null(key, i)) continue;
    const unsigned long long h = bloom_hash_int(ld_i64(key, i));
    atomicOr(bloom + (h & mask), 1ULL << (h & 63));
    atomicOr(bloom + ((h >> 17) & mask), 1ULL << ((h >> 6) & 63));
  }
}

// BloomFilterOp over a probe key column: per item (row, or selection entry),
// its row number and whether the bloom may contain its (non-NULL) key.
__global__ void bloom_probe_kernel(DCol key, const uint32_t* sel, int64_t n, const unsigned long long* bloom,
                                   unsigned long long mask, uint32_t* rows, uint8_t* flags) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = sel ? (int64_t)sel[i] : i;
    rows[i] = (uint32_t)row;
    flags[i] = !is_null(key, row) && bloom_contains(bloom, mask, bloom_hash_int(ld_i64(key, row))) ? 1 : 0;
  }
}

// Payload-only dense table from a full dense direct table (every slot used).
__global__ void dense_payload_kernel(const unsigned long long* slots, int64_t n, uint32_t* out) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (uint32_t)(__ldg(slots + i) >> 32);
}

__global__ void fill_u64_kernel(unsigned long long* out, int64_t n, unsigned long long v) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = v;
}

// Longest chain (max build rows sharing one key): the join's worst fan-out.
__global__ void join_fanout_kernel(JoinView j, unsigned long long* max_len) {
  const uint64_t cap = j.mask + 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
    int32_t head;
    if (j.flavor == 0) head = (int32_t)(((const unsigned long long*)j.slots)[i] >> 32);
    else head = (int32_t)(uint32_t)((const longlong2*)j.slots)[i].y;
    if (head < 0) continue;
    unsigned long long c = 0;
    for (int32_t r = head; r >= 0; r = j.next[r]) ++c;
    atomicMax(max_len, c);
  }
}

__global__ void gather_kernel(const char* src, int64_t es, const uint64_t* valid, const int64_t* rows, int64_t n,
                              char* dst, uint8_t* dst_valid) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = rows[i];
    if (r < 0) {  // no build row (an unmatched LEFT row): NULL
      for (int64_t b = 0; b < es; ++b) dst[i * es + b] = 0;
      if (dst_valid) dst_valid[i] = 0;
      continue;
    }
    for (int64_t b = 0; b < es; ++b) dst[i * es + b] = src[r * es + b];
    if (dst_valid) dst_valid[i] = valid ? (uint8_t)((valid[r >> 6] >> (r & 63)) & 1ULL) : (uint8_t)1;
  }
}

// Clear the bits of NULL rows of src into dst (all-ones initialised) at bit offset off.
__global__ void append_valid_kernel(uint32_t* dst, int64_t off, const uint64_t* src, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (((src[i >> 6] >> (i & 63)) & 1ULL) == 0) {
      const int64_t b = off + i;
      atomicAnd(dst + (b >> 5), ~(1u << (b & 31)));
    }
  }
}

unsigned grid_for(wg::Ctx* ctx, int64_t n, int block) {
  int64_t blocks = (n + block - 1) / block;
  int64_t cap = (int64_t)ctx->sm_count * 16;
  if (blocks > cap) blocks = cap;
  if (blocks < 1) blocks = 1;
  return (unsigned)blocks;
}

}  // namespace

// A growable device column of the build side.
struct BuildCol {
  int32_t type_id = 0, scale = 0;
  int64_t es = 0;
  wg::DevBuf data, valid;   // valid allocated lazily, all ones = valid
  int64_t cap_rows = 0;
  bool has_valid = false;
};

struct wg_join {
  wg::Ctx* ctx;
  int32_t jtype = WG_JOIN_INNER;  // exec.JoinType (join.go:20-30)
  int32_t build_key_col, probe_key_col;
  std::vector<int32_t> payload_cols;
  int64_t hint;
  int64_t rows = 0;
  BuildCol key;
  std::vector<BuildCol> pay;
  bool finished = false;
  bool schema_set = false;
  // index
  int32_t flavor = 0;
  int32_t shift = 0;
  uint64_t capacity = 0;
  wg::DevBuf slots, next, scratch, counts, offs, outp, outb, rows_dev, gath, gath_valid;
  int64_t distinct = 0;
  bool unique = true;
  int64_t max_fanout = 1;
  bool hashed = false;  // the hash index (slots/next) is built; a dense unique build defers it to first use
  // direct-payload copy of the table for the fused kernel (see JoinView)
  wg::DevBuf dslots, dpay;
  bool direct = false;
  bool full = false;  // dense and every key of the range present: dpay holds the payloads
  int32_t sentinel = 0;
  bool dense = false;
  long long dense_base = 0;
  int64_t dense_slots = 0;
  // value range of each integer payload column without NULLs (for dense GROUP BY)
  std::vector<long long> pay_lo, pay_hi;
  std::vector<bool> pay_range;
  wg::StagedBatch staged;
  // Partitioned build (the partition-on-arrival grace build of
  // join_partition_arrival.go:48): when the HBM ledger refuses the build's
  // columns or index, its rows move to host memory split into 64 partitions by
  // key hash (join_partition, NULL keys dropped: they match nothing), and the
  // fused pipeline probes in passes, each over a group of consecutive
  // partitions whose rows and index fit half of what the ledger has left,
  // built into `pass` (an ordinary join) for that pass. Probe rows take part
  // only in the pass of their key's partition (JoinView.part_*).
  bool grace = false;
  struct HostPart {
    int64_t rows = 0;
    std::vector<char> key;
    std::vector<std::vector<char>> pay;
    std::vector<std::vector<uint8_t>> ok;  // per payload column and row: 1 = not NULL
  };
  std::vector<HostPart> parts;
  std::vector<std::pair<int, int>> passes;  // partition ranges [lo, hi)
  wg_join* pass = nullptr;
  int pass_built = -1;
  // on a pass join: the partitions it covers (part_shift 0 = all)
  int32_t pass_shift = 0, pass_lo = 0, pass_hi = 0;
  // the bloom pre-filter (HashJoin.buildBloom), built on first use
  wg::DevBuf bloom, bloom_rows, bloom_flags, bloom_out, bloom_tmp;
  uint64_t bloom_mask = 0;
  bool bloom_built = false;
  ~wg_join() { delete pass; }
};

namespace wg {

static wg_status grow_col(Ctx* ctx, BuildCol& c, int64_t need_rows, int64_t used_rows) {
  if (need_rows <= c.cap_rows) return WG_OK;
  int64_t cap = std::max<int64_t>(need_rows, std::max<int64_t>(c.cap_rows * 2, 1024));
  DevBuf nd;
  WG_TRY(nd.alloc(ctx, cap * c.es));
  if (used_rows > 0)
    WG_CUDA_TRY(cudaMemcpyAsync(nd.get(), c.data.get(), (size_t)(used_rows * c.es), cudaMemcpyDeviceToDevice, ctx->stream));
  if (c.has_valid) {
    DevBuf nv;
    int64_t words = (cap + 63) / 64;
    WG_TRY(nv.alloc(ctx, words * 8));
    WG_CUDA_TRY(cudaMemsetAsync(nv.get(), 0xFF, (size_t)(words * 8), ctx->stream));
    if (used_rows > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(nv.get(), c.valid.get(), (size_t)(((used_rows + 63) / 64) * 8), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    c.valid = std::move(nv);
  }
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  c.data = std::move(nd);
  c.cap_rows = cap;
  return WG_OK;
}

static wg_status append_col(Ctx* ctx, BuildCol& c, const wg_column& src, int64_t n, int64_t at) {
  WG_TRY(grow_col(ctx, c, at + n, at));
  if (n > 0)
    WG_CUDA_TRY(cudaMemcpyAsync((char*)c.data.get() + at * c.es, src.data, (size_t)(n * c.es), cudaMemcpyDefault,
                                ctx->stream));
  if (src.valid_words) {
    if (!c.has_valid) {
      int64_t words = (c.cap_rows + 63) / 64;
      WG_TRY(c.valid.alloc(ctx, words * 8));
      WG_CUDA_TRY(cudaMemsetAsync(c.valid.get(), 0xFF, (size_t)(words * 8), ctx->stream));
      c.has_valid = true;
    }
    // src bitmap may live on the host: bring it over first
    DevBuf tmp;
    const uint64_t* sv = src.valid_words;
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, sv) != cudaSuccess || attr.type != cudaMemoryTypeDevice) {
      cudaGetLastError();
      int64_t words = (n + 63) / 64;
      WG_TRY(tmp.alloc(ctx, std::max<int64_t>(words * 8, 16)));
      WG_CUDA_TRY(cudaMemcpyAsync(tmp.get(), sv, (size_t)(words * 8), cudaMemcpyHostToDevice, ctx->stream));
      sv = tmp.as<uint64_t>();
    }
    if (n > 0) {
      append_valid_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(c.valid.as<uint32_t>(), at, sv, n);
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
    }
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  return WG_OK;
}

static bool grace_allowed(const wg_join* j);
static wg_status grace_convert(wg_join* j);
static wg_status grace_append(wg_join* j, const wg_batch_desc* b);
static wg_status grace_plan(wg_join* j);

static wg_status join_append(wg_join* j, const wg_batch_desc* b) {
  Ctx* ctx = j->ctx;
  if (j->finished) return fail(WG_E_STATE, "join build already finished");
  if (!b || j->build_key_col < 0 || j->build_key_col >= b->ncols) return fail(WG_E_INVALID, "build key column out of range");
  if (b->sel) return fail(WG_E_INVALID, "build batches must be flattened (no selection vector)");
  const wg_column& kc = b->cols[j->build_key_col];
  int kcls = class_of(kc.type_id);
  if (kcls != WG_CLS_I32 && kcls != WG_CLS_I64) return fail(WG_E_UNSUPPORTED, "join key is not an integer-class column");
  if (!j->schema_set) {
    j->key.type_id = kc.type_id; j->key.es = elem_size(kc.type_id);
    j->pay.resize(j->payload_cols.size());
    for (size_t i = 0; i < j->payload_cols.size(); ++i) {
      int pc = j->payload_cols[i];
      if (pc < 0 || pc >= b->ncols) return fail(WG_E_INVALID, "payload column out of range");
      const wg_column& c = b->cols[pc];
      if (elem_size(c.type_id) == 0) return fail(WG_E_UNSUPPORTED, "payload column type is not on the GPU path");
      j->pay[i].type_id = c.type_id; j->pay[i].scale = c.scale; j->pay[i].es = elem_size(c.type_id);
    }
    j->flavor = kcls == WG_CLS_I32 ? 0 : 1;
    j->schema_set = true;
  } else if (kc.type_id != j->key.type_id) {
    return fail(WG_E_INVALID, "build key type changed between batches");
  }
  const int64_t n = b->len;
  for (size_t i = 0; i < j->pay.size(); ++i)
    if (b->cols[j->payload_cols[i]].type_id != j->pay[i].type_id)
      return fail(WG_E_INVALID, "payload type changed between batches");
  if (j->grace) return grace_append(j, b);
  int64_t hint = std::max<int64_t>(j->hint, j->rows + n);
  wg_status st = grow_col(ctx, j->key, hint, j->rows);
  if (st == WG_OK) st = append_col(ctx, j->key, kc, n, j->rows);
  for (size_t i = 0; i < j->pay.size() && st == WG_OK; ++i) {
    const wg_column& c = b->cols[j->payload_cols[i]];
    st = grow_col(ctx, j->pay[i], hint, j->rows);
    if (st == WG_OK) st = append_col(ctx, j->pay[i], c, n, j->rows);
  }
  if (st == WG_E_NOMEM && grace_allowed(j)) {  // the ledger refused: partition the build into host memory
    WG_TRY(grace_convert(j));
    return grace_append(j, b);
  }
  WG_TRY(st);
  j->rows += n;
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

// ---- partitioned (grace) build ---------------------------------------------
constexpr int kJoinPartBits = 6;  // 64 partitions, as the reference's partitioned build
constexpr int kJoinPartShift = 64 - kJoinPartBits;

static bool grace_allowed(const wg_join* j) {
  const char* v = std::getenv("WG_JOIN_GRACE");
  return j->ctx->ledger.budget() > 0 && (!v || std::atoi(v) != 0);
}

// `bytes` of host or device memory into a host vector.
static wg_status to_host(Ctx* ctx, const void* src, int64_t bytes, std::vector<char>& out) {
  out.resize((size_t)std::max<int64_t>(bytes, 0));
  if (bytes <= 0) return WG_OK;
  WG_CUDA_TRY(cudaMemcpyAsync(out.data(), src, (size_t)bytes, cudaMemcpyDefault, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

static inline bool bit_at(const std::vector<char>& words, int64_t i) {
  return words.empty() || ((((const uint64_t*)words.data())[i >> 6] >> (i & 63)) & 1ULL);
}

// n rows (host copies of the key, its validity words, each payload column and
// its validity words; empty validity = no NULLs) appended to their partitions.
static void grace_partition(wg_join* j, const std::vector<char>& key, const std::vector<char>& key_valid,
                            const std::vector<std::vector<char>>& pay, const std::vector<std::vector<char>>& pay_valid,
                            int64_t n) {
  const int np = 1 << kJoinPartBits;
  if ((int)j->parts.size() != np) j->parts.assign((size_t)np, wg_join::HostPart{});
  const int kes = (int)j->key.es;
  std::vector<uint8_t> part((size_t)n);
  std::vector<int64_t> cnt((size_t)np, 0);
  for (int64_t i = 0; i < n; ++i) {
    if (!bit_at(key_valid, i)) { part[(size_t)i] = 0xFF; continue; }  // a NULL key matches nothing
    const long long k = kes == 4 ? (long long)((const int32_t*)key.data())[i] : ((const long long*)key.data())[i];
    part[(size_t)i] = (uint8_t)wgd::join_partition(k, kJoinPartShift);
    ++cnt[part[(size_t)i]];
  }
  const size_t npay = j->pay.size();
  std::vector<int64_t> at((size_t)np);
  for (int p = 0; p < np; ++p) {
    wg_join::HostPart& hp = j->parts[(size_t)p];
    at[(size_t)p] = hp.rows;
    hp.rows += cnt[(size_t)p];
    hp.key.resize((size_t)(hp.rows * kes));
    hp.pay.resize(npay);
    hp.ok.resize(npay);
    for (size_t c = 0; c < npay; ++c) {
      hp.pay[c].resize((size_t)(hp.rows * j->pay[c].es));
      hp.ok[c].resize((size_t)hp.rows, 1);
    }
  }
  for (int64_t i = 0; i < n; ++i) {
    const uint8_t p = part[(size_t)i];
    if (p == 0xFF) continue;
    wg_join::HostPart& hp = j->parts[p];
    const int64_t r = at[p]++;
    std::memcpy(hp.key.data() + r * kes, key.data() + i * kes, (size_t)kes);
    for (size_t c = 0; c < npay; ++c) {
      const int64_t es = j->pay[c].es;
      std::memcpy(hp.pay[c].data() + r * es, pay[c].data() + i * es, (size_t)es);
      hp.ok[c][(size_t)r] = bit_at(pay_valid[c], i) ? 1 : 0;
    }
  }
}

// The build rows already on the device moved to host partitions; the device
// columns and index freed.
static wg_status grace_convert(wg_join* j) {
  Ctx* ctx = j->ctx;
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int64_t n = j->rows;
  std::vector<char> key, key_valid;
  std::vector<std::vector<char>> pay(j->pay.size()), pay_valid(j->pay.size());
  WG_TRY(to_host(ctx, j->key.data.get(), n * j->key.es, key));
  if (j->key.has_valid) WG_TRY(to_host(ctx, j->key.valid.get(), (n + 63) / 64 * 8, key_valid));
  for (size_t c = 0; c < j->pay.size(); ++c) {
    WG_TRY(to_host(ctx, j->pay[c].data.get(), n * j->pay[c].es, pay[c]));
    if (j->pay[c].has_valid) WG_TRY(to_host(ctx, j->pay[c].valid.get(), (n + 63) / 64 * 8, pay_valid[c]));
  }
  j->grace = true;
  j->parts.clear();
  grace_partition(j, key, key_valid, pay, pay_valid, n);
  auto drop = [](BuildCol& c) { c.data.reset(); c.valid.reset(); c.cap_rows = 0; };
  drop(j->key);
  for (BuildCol& c : j->pay) drop(c);
  j->slots.reset(); j->next.reset(); j->dslots.reset(); j->dpay.reset();
  j->counts.reset(); j->offs.reset(); j->outp.reset(); j->outb.reset();
  return WG_OK;
}

// A batch appended to the host partitions.
static wg_status grace_append(wg_join* j, const wg_batch_desc* b) {
  Ctx* ctx = j->ctx;
  const int64_t n = b->len;
  const wg_column& kc = b->cols[j->build_key_col];
  std::vector<char> key, key_valid;
  std::vector<std::vector<char>> pay(j->pay.size()), pay_valid(j->pay.size());
  WG_TRY(to_host(ctx, kc.data, n * j->key.es, key));
  if (kc.valid_words) WG_TRY(to_host(ctx, kc.valid_words, (n + 63) / 64 * 8, key_valid));
  for (size_t c = 0; c < j->pay.size(); ++c) {
    const wg_column& pc = b->cols[j->payload_cols[c]];
    WG_TRY(to_host(ctx, pc.data, n * j->pay[c].es, pay[c]));
    if (pc.valid_words) WG_TRY(to_host(ctx, pc.valid_words, (n + 63) / 64 * 8, pay_valid[c]));
  }
  grace_partition(j, key, key_valid, pay, pay_valid, n);
  j->rows += n;
  return WG_OK;
}

// Passes: consecutive partitions grouped while their rows, stored and indexed
// on the device, fit half of what the ledger has left.
static wg_status grace_plan(wg_join* j) {
  Ctx* ctx = j->ctx;
  // per build row: the key, its chain link, the hash index (at most 4 slots of
  // 16 bytes per row: capacity is the power of two at or above twice the rows)
  // and the direct table (at most 4 slots of 8 bytes), and each payload column
  int64_t row_bytes = j->key.es + 4 + 64 + 32;
  for (const BuildCol& c : j->pay) row_bytes += c.es + 1;
  const int64_t left = ctx->ledger.budget() - ctx->ledger.used();
  const int64_t room = std::max<int64_t>(left / 2, 1 << 20);
  j->passes.clear();
  const int np = (int)j->parts.size();
  int lo = 0;
  int64_t bytes = 0;
  for (int p = 0; p < np; ++p) {
    const int64_t b = j->parts[(size_t)p].rows * row_bytes;
    if (b > room) return fail(WG_E_NOMEM, "a join build partition does not fit the HBM budget");
    if (bytes + b > room && p > lo) {
      j->passes.push_back({lo, p});
      lo = p;
      bytes = 0;
    }
    bytes += b;
  }
  j->passes.push_back({lo, np});
  j->pass_built = -1;
  j->distinct = -1;  // not counted across partitions
  return WG_OK;
}

// The join for pass g: an ordinary join over that pass's partitions, whose
// probe view admits only rows of those partitions.
wg_status join_grace_pass(wg_join* j, int g, wg_join** out) {
  Ctx* ctx = j->ctx;
  if (j->pass_built == g && j->pass) { *out = j->pass; return WG_OK; }
  delete j->pass;
  j->pass = nullptr;
  j->pass_built = -1;
  const int lo = j->passes[(size_t)g].first, hi = j->passes[(size_t)g].second;
  int64_t n = 0;
  for (int p = lo; p < hi; ++p) n += j->parts[(size_t)p].rows;
  const int npay = (int)j->pay.size();
  std::vector<int32_t> pcols((size_t)npay);
  for (int c = 0; c < npay; ++c) pcols[(size_t)c] = c + 1;
  wg_join* pj = nullptr;
  // every context is created as a wg_ctx (ctx_make)
  WG_TRY(wg_join_create(static_cast<wg_ctx*>(ctx), j->jtype, 0, j->probe_key_col, npay, pcols.data(),
                        std::max<int64_t>(n, 1), &pj));
  j->pass = pj;
  pj->pass_shift = kJoinPartShift;
  pj->pass_lo = lo;
  pj->pass_hi = hi;
  // the pass's rows as one host batch (key, then the payload columns with their validity words)
  std::vector<char> key((size_t)(n * j->key.es));
  std::vector<std::vector<char>> pay((size_t)npay);
  std::vector<std::vector<uint64_t>> valid((size_t)npay);
  std::vector<bool> any_null((size_t)npay, false);
  for (int c = 0; c < npay; ++c) {
    pay[(size_t)c].resize((size_t)(n * j->pay[(size_t)c].es));
    valid[(size_t)c].assign((size_t)((n + 63) / 64 + 1), ~0ULL);
  }
  int64_t r0 = 0;
  for (int p = lo; p < hi; ++p) {
    const wg_join::HostPart& hp = j->parts[(size_t)p];
    if (hp.rows == 0) continue;
    std::memcpy(key.data() + r0 * j->key.es, hp.key.data(), (size_t)(hp.rows * j->key.es));
    for (int c = 0; c < npay; ++c) {
      const int64_t es = j->pay[(size_t)c].es;
      std::memcpy(pay[(size_t)c].data() + r0 * es, hp.pay[(size_t)c].data(), (size_t)(hp.rows * es));
      for (int64_t i = 0; i < hp.rows; ++i)
        if (!hp.ok[(size_t)c][(size_t)i]) {
          const int64_t r = r0 + i;
          valid[(size_t)c][(size_t)(r >> 6)] &= ~(1ULL << (r & 63));
          any_null[(size_t)c] = true;
        }
    }
    r0 += hp.rows;
  }
  std::vector<wg_column> cols((size_t)npay + 1);
  cols[0] = wg_column{j->key.type_id, 0, key.data(), nullptr, n};
  for (int c = 0; c < npay; ++c)
    cols[(size_t)c + 1] = wg_column{j->pay[(size_t)c].type_id, j->pay[(size_t)c].scale, pay[(size_t)c].data(),
                                    any_null[(size_t)c] ? valid[(size_t)c].data() : nullptr, n};
  wg_batch_desc d{npay + 1, 0, cols.data(), n, nullptr, 0};
  if (n > 0) WG_TRY(join_append(pj, &d));
  else {  // an empty pass still needs the schema
    pj->key.type_id = j->key.type_id; pj->key.es = j->key.es;
    pj->pay.resize((size_t)npay);
    for (int c = 0; c < npay; ++c) {
      pj->pay[(size_t)c].type_id = j->pay[(size_t)c].type_id;
      pj->pay[(size_t)c].scale = j->pay[(size_t)c].scale;
      pj->pay[(size_t)c].es = j->pay[(size_t)c].es;
    }
    pj->flavor = j->flavor;
    pj->schema_set = true;
  }
  WG_TRY(wg_join_build_finish(pj));
  j->pass_built = g;
  *out = pj;
  return WG_OK;
}
bool join_is_grace(wg_join* j) { return j->grace; }
int join_grace_passes(wg_join* j) { return (int)j->passes.size(); }

// Device view for the fused pipeline and the probe kernels.
static wg_status build_hash(wg_join* j);

static wg_status join_view_fields(wg_join* j, wgd::JoinView* v) {
  if (!j->finished) return fail(WG_E_STATE, "join build not finished");
  v->flavor = j->flavor;
  v->shift = j->shift;
  v->mask = j->capacity - 1;
  v->slots = j->slots.get();
  v->next = j->next.as<int32_t>();
  v->n_pay = (int32_t)j->pay.size();
  v->jtype = j->jtype;
  v->part_shift = j->pass_shift;
  v->part_lo = j->pass_lo;
  v->part_hi = j->pass_hi;
  v->bloom = nullptr;
  v->bloom_mask = 0;
  v->direct = 0;
  v->sentinel = 0;
  v->dense = 0;
  v->l2keep = 0;
  v->base = 0;
  for (size_t i = 0; i < j->pay.size() && i < WG_MAX_PAYLOAD; ++i)
    v->pay[i] = wgd::DCol{j->pay[i].data.get(), j->pay[i].has_valid ? j->pay[i].valid.as<uint64_t>() : nullptr,
                          class_of(j->pay[i].type_id), j->pay[i].scale};
  return WG_OK;
}

// The bloom over the build side's distinct keys (HashJoin.buildBloom,
// join.go:1441): about 10 bits per key, a power-of-two count of 64-bit words,
// at least 8; built once per build.
static wg_status build_bloom(wg_join* j) {
  if (j->bloom_built) return WG_OK;
  Ctx* ctx = j->ctx;
  const int64_t nk = j->distinct;
  j->bloom_mask = 0;
  if (nk > 0) {
    int64_t slots = 1;
    while (slots * 64 < nk * 10) slots *= 2;
    if (slots < 8) slots = 8;
    WG_TRY(j->bloom.ensure(ctx, slots * 8));
    WG_CUDA_TRY(cudaMemsetAsync(j->bloom.get(), 0, (size_t)(slots * 8), ctx->stream));
    j->bloom_mask = (uint64_t)slots - 1;
    wgd::DCol kd{j->key.data.get(), j->key.has_valid ? j->key.valid.as<uint64_t>() : nullptr, class_of(j->key.type_id), 0};
    bloom_build_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(kd, j->rows, j->bloom.as<unsigned long long>(),
                                                                           j->bloom_mask);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  j->bloom_built = true;
  return WG_OK;
}

// Whether the hash probe checks the bloom first: WG_JOIN_BLOOM=1 always, 0
// never; by default when the hash index is larger than half of L2 (64 MB), so
// a key the bloom rules out saves a random HBM read.
static bool bloom_for_probe(const wg_join* j) {
  const char* v = std::getenv("WG_JOIN_BLOOM");
  if (v) return std::atoi(v) != 0;
  const int64_t index_bytes = (int64_t)j->capacity * (j->flavor == 0 ? 8 : 16);
  return index_bytes >= (int64_t(64) << 20);
}

wg_status join_view(wg_join* j, wgd::JoinView* v) {
  if (j->finished && !j->hashed) WG_TRY(build_hash(j));
  WG_TRY(join_view_fields(j, v));
  if (j->finished && j->distinct > 0 && bloom_for_probe(j)) {
    WG_TRY(build_bloom(j));
    v->bloom = j->bloom.as<unsigned long long>();
    v->bloom_mask = j->bloom_mask;
  }
  return WG_OK;
}

// The view the fused pipeline probes: the direct-payload table when one was built.
wg_status join_view_fused(wg_join* j, wgd::JoinView* v) {
  // the direct-payload table answers "which payload", not "was there a match":
  // outer, semi and anti joins probe the hash index
  if (!j->direct || j->jtype != WG_JOIN_INNER) return join_view(j, v);
  WG_TRY(join_view_fields(j, v));
  {
    v->slots = j->dslots.get();
    v->direct = 1;
    v->sentinel = j->sentinel;
    if (j->dense) {
      v->dense = 1;
      const char* keep = std::getenv("WG_JOIN_L2_KEEP");
      v->l2keep = !keep || std::atoi(keep) != 0;
      v->base = j->dense_base;
      v->mask = (uint64_t)j->dense_slots;
      if (j->full) {
        v->dense = 2;
        v->slots = j->dpay.get();
      }
    }
  }
  return WG_OK;
}
int32_t join_probe_key_col(wg_join* j) { return j->probe_key_col; }
int32_t join_n_payload(wg_join* j) { return (int32_t)j->pay.size(); }
int32_t join_payload_type(wg_join* j, int i) { return j->pay[i].type_id; }
int32_t join_payload_scale(wg_join* j, int i) { return j->pay[i].scale; }
bool join_payload_nullable(wg_join* j, int i) { return j->pay[i].has_valid; }
bool join_payload_range(wg_join* j, int i, long long* lo, long long* hi) {
  if (i < 0 || i >= (int)j->pay_range.size() || !j->pay_range[i]) return false;
  *lo = j->pay_lo[i];
  *hi = j->pay_hi[i];
  return true;
}
bool join_unique(wg_join* j) { return j->unique; }
int32_t join_type_of(wg_join* j) { return j->jtype; }
int64_t join_max_fanout(wg_join* j) { return j->max_fanout; }

// The hash index (slots/next): one CAS insert per build row, heads chained
// through `next`; counts distinct keys and flags duplicates.
static wg_status build_hash(wg_join* j) {
  Ctx* ctx = j->ctx;
  const uint64_t cap = j->capacity;
  const int64_t slot_bytes = j->flavor == 0 ? 8 : 16;
  WG_TRY(j->slots.ensure(ctx, (int64_t)cap * slot_bytes));
  WG_TRY(j->next.ensure(ctx, std::max<int64_t>(j->rows, 1) * 4));
  WG_TRY(j->scratch.ensure(ctx, 64));
  WG_CUDA_TRY(cudaMemsetAsync(j->slots.get(), 0xFF, (size_t)(cap * slot_bytes), ctx->stream));
  WG_CUDA_TRY(cudaMemsetAsync(j->scratch.get(), 0, 64, ctx->stream));
  if (j->rows > 0) {
    BuildArgs a;
    a.key = wgd::DCol{j->key.data.get(), j->key.has_valid ? j->key.valid.as<uint64_t>() : nullptr,
                      class_of(j->key.type_id), 0};
    a.n = j->rows;
    a.flavor = j->flavor;
    a.shift = j->shift;
    a.mask = cap - 1;
    a.slots = j->slots.get();
    a.next = j->next.as<int32_t>();
    a.distinct = j->scratch.as<unsigned long long>();
    a.dup = (int32_t*)(j->scratch.as<char>() + 8);
    a.err = ctx->dev_error;
    join_build_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(a);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
  }
  int64_t back[2] = {0, 0};
  WG_TRY(read_back_i64(ctx, j->scratch.as<int64_t>(), back, 2));
  WG_TRY(check_device_error(ctx));
  j->distinct = back[0];
  j->unique = (int32_t)back[1] == 0;
  j->hashed = true;
  return WG_OK;
}

// Unique int32 build keys without NULLs, spanning at most 4x the build rows,
// and one 4-byte payload column without NULLs: the dense direct table is built
// straight from the rows and the hash index is deferred to its first use (the
// fused probe never needs it). *done is false when this shape does not apply
// or a duplicate key turned up; the caller then builds the hash index.
static bool env_full_dense() {
  const char* e = std::getenv("WG_JOIN_FULL_DENSE");
  return !e || std::atoi(e) != 0;
}

static wg_status build_dense_unique(wg_join* j, bool* done) {
  *done = false;
  Ctx* ctx = j->ctx;
  const char* dsw = std::getenv("WG_JOIN_DIRECT");
  const char* dns = std::getenv("WG_JOIN_DENSE");
  if ((dsw && std::atoi(dsw) == 0) || (dns && std::atoi(dns) == 0) || j->rows <= 0 || j->flavor != 0 ||
      j->key.has_valid || j->pay.size() != 1 || j->pay[0].es != 4 || j->pay[0].has_valid)
    return WG_OK;
  const int pcls = class_of(j->pay[0].type_id);
  const bool pay_int = pcls == WG_CLS_I32 || pcls == WG_CLS_I64;
  long long* mm = (long long*)(j->scratch.as<char>() + 16);  // key lo, hi, payload lo, hi
  const long long init[4] = {LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN};
  WG_CUDA_TRY(cudaMemcpyAsync(mm, init, 32, cudaMemcpyHostToDevice, ctx->stream));
  wgd::DCol kd{j->key.data.get(), nullptr, class_of(j->key.type_id), 0};
  key_range_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(kd, j->rows, mm, mm + 1);
  ctx->count_launch();
  if (pay_int) {
    wgd::DCol pd{j->pay[0].data.get(), nullptr, pcls, 0};
    key_range_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(pd, j->rows, mm + 2, mm + 3);
    ctx->count_launch();
  }
  WG_CUDA_TRY(cudaGetLastError());
  int64_t r[4];
  WG_TRY(read_back_i64(ctx, (const int64_t*)mm, r, 4));
  int32_t sentinel;
  if (r[0] > INT32_MIN) sentinel = (int32_t)(r[0] - 1);
  else if (r[1] < INT32_MAX) sentinel = (int32_t)(r[1] + 1);
  else return WG_OK;
  const int64_t span = r[1] - r[0] + 1;
  if (!(span > 0 && span <= std::max<int64_t>(4 * j->rows, 1024) && span <= (int64_t(1) << 30))) return WG_OK;
  const unsigned long long empty = (unsigned long long)(uint32_t)sentinel;
  WG_TRY(j->dslots.ensure(ctx, span * 8));
  WG_CUDA_TRY(cudaMemsetAsync(j->scratch.get(), 0, 8, ctx->stream));
  fill_u64_kernel<<<grid_for(ctx, span, 256), 256, 0, ctx->stream>>>(j->dslots.as<unsigned long long>(), span, empty);
  ctx->count_launch();
  dense_build_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(
      kd, j->rows, j->pay[0].data.as<uint32_t>(), r[0], empty, j->dslots.as<unsigned long long>(),
      j->scratch.as<int32_t>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  int64_t dup = 0;
  WG_TRY(read_back_i64(ctx, j->scratch.as<int64_t>(), &dup, 1));
  if ((int32_t)dup != 0) return WG_OK;
  j->pay_lo.assign(1, pay_int ? r[2] : 0);
  j->pay_hi.assign(1, pay_int ? r[3] : 0);
  j->pay_range.assign(1, pay_int);
  j->distinct = j->rows;
  j->unique = true;
  j->max_fanout = 1;
  j->direct = true;
  j->dense = true;
  j->sentinel = sentinel;
  j->dense_base = r[0];
  j->dense_slots = span;
  // unique keys filling their whole range: the payloads alone (half the bytes a probe's cache lines carry)
  j->full = false;
  if (span == j->rows && env_full_dense()) {
    WG_TRY(j->dpay.ensure(ctx, span * 4));
    dense_payload_kernel<<<grid_for(ctx, span, 256), 256, 0, ctx->stream>>>(j->dslots.as<unsigned long long>(), span,
                                                                          j->dpay.as<uint32_t>());
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    j->full = true;
  }
  *done = true;
  return WG_OK;
}

}  // namespace wg

using namespace wg;

extern "C" {

wg_status wg_join_create(wg_ctx* ctx, int32_t join_type, int32_t build_key_col, int32_t probe_key_col,
                         int32_t n_payload, const int32_t* payload_cols, int64_t build_row_hint, wg_join** out) {
  if (!ctx || !out) return fail(WG_E_INVALID, "NULL argument");
  if (join_type != WG_JOIN_INNER && join_type != WG_JOIN_LEFT && join_type != WG_JOIN_SEMI &&
      join_type != WG_JOIN_ANTI)
    return fail(WG_E_UNSUPPORTED, "join type is not on the GPU path (inner, left, semi and anti are)");
  if (n_payload < 0 || n_payload > WG_MAX_PAYLOAD || (n_payload > 0 && !payload_cols))
    return fail(WG_E_INVALID, "at most 4 payload columns");
  if ((join_type == WG_JOIN_SEMI || join_type == WG_JOIN_ANTI) && n_payload > 0)
    return fail(WG_E_INVALID, "a semi or anti join returns probe rows only: no payload columns");
  wg_join* j = new wg_join();
  j->ctx = ctx;
  j->jtype = join_type;
  j->build_key_col = build_key_col;
  j->probe_key_col = probe_key_col;
  j->payload_cols.assign(payload_cols, payload_cols + n_payload);
  j->hint = build_row_hint > 0 ? build_row_hint : 1024;
  *out = j;
  return WG_OK;
}

wg_status wg_join_build_append(wg_join* j, const wg_batch_desc* b) {
  if (!j) return fail(WG_E_INVALID, "join is NULL");
  WG_TRY(ensure_device(j->ctx));
  return join_append(j, b);
}

wg_status wg_join_build_append_device(wg_join* j, const wg_batch_desc* b) {
  if (!j) return fail(WG_E_INVALID, "join is NULL");
  WG_TRY(ensure_device(j->ctx));
  return join_append(j, b);
}

static wg_status build_finish_device(wg_join* j);

wg_status wg_join_build_finish(wg_join* j) {
  if (!j) return fail(WG_E_INVALID, "join is NULL");
  if (j->finished) return WG_OK;
  WG_TRY(ensure_device(j->ctx));
  if (!j->grace) {
    const wg_status st = build_finish_device(j);
    if (st != WG_E_NOMEM || !grace_allowed(j) || !j->schema_set) return st;
    WG_TRY(grace_convert(j));  // the index did not fit: partition the build into host memory
  }
  WG_TRY(grace_plan(j));
  j->finished = true;
  return WG_OK;
}

static wg_status build_finish_device(wg_join* j) {
  Ctx* ctx = j->ctx;
  if (!j->schema_set) { j->flavor = 0; j->key.type_id = WG_TYPE_INT32; j->key.es = 4; }
  uint64_t cap = 1024;
  while (cap < (uint64_t)std::max<int64_t>(2 * j->rows, 1)) cap <<= 1;
  int log2 = 0;
  while ((1ULL << log2) < cap) ++log2;
  j->capacity = cap;
  j->shift = 64 - log2;
  j->hashed = false;
  WG_TRY(j->scratch.ensure(ctx, 64));
  bool done = false;
  WG_TRY(build_dense_unique(j, &done));
  if (done) {
    j->finished = true;
    return check_device_error(ctx);
  }
  WG_TRY(build_hash(j));
  j->finished = true;
  j->max_fanout = 1;
  if (!j->unique) {
    wgd::JoinView v;
    WG_TRY(join_view(j, &v));
    WG_CUDA_TRY(cudaMemsetAsync(j->scratch.get(), 0, 8, ctx->stream));
    join_fanout_kernel<<<grid_for(ctx, (int64_t)cap, 256), 256, 0, ctx->stream>>>(v, j->scratch.as<unsigned long long>());
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    int64_t mf = 1;
    WG_TRY(read_back_i64(ctx, j->scratch.as<int64_t>(), &mf, 1));
    j->max_fanout = std::max<int64_t>(1, mf);
  }
  // value range of the integer payload columns without NULLs
  j->pay_lo.assign(j->pay.size(), 0);
  j->pay_hi.assign(j->pay.size(), 0);
  j->pay_range.assign(j->pay.size(), false);
  for (size_t p = 0; p < j->pay.size() && j->rows > 0; ++p) {
    const int cls = class_of(j->pay[p].type_id);
    if (j->pay[p].has_valid || (cls != WG_CLS_I32 && cls != WG_CLS_I64)) continue;
    long long* mm = (long long*)(j->scratch.as<char>() + 32);
    const long long init[2] = {LLONG_MAX, LLONG_MIN};
    WG_CUDA_TRY(cudaMemcpyAsync(mm, init, 16, cudaMemcpyHostToDevice, ctx->stream));
    wgd::DCol pd{j->pay[p].data.get(), nullptr, cls, 0};
    key_range_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(pd, j->rows, mm, mm + 1);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    int64_t r[2];
    WG_TRY(read_back_i64(ctx, (const int64_t*)mm, r, 2));
    j->pay_lo[p] = r[0];
    j->pay_hi[p] = r[1];
    j->pay_range[p] = true;
  }
  // Direct-payload table for the fused probe: unique int32 keys, exactly one
  // 4-byte payload column without NULLs, and an int32 value that is no key.
  j->direct = false;
  j->dense = false;
  j->full = false;
  const char* dsw = std::getenv("WG_JOIN_DIRECT");
  if ((!dsw || std::atoi(dsw) != 0) && j->unique && j->flavor == 0 && j->pay.size() == 1 && j->pay[0].es == 4 &&
      !j->pay[0].has_valid && j->rows > 0) {
    long long* mm = (long long*)(j->scratch.as<char>() + 16);
    const long long init[2] = {LLONG_MAX, LLONG_MIN};
    WG_CUDA_TRY(cudaMemcpyAsync(mm, init, 16, cudaMemcpyHostToDevice, ctx->stream));
    wgd::DCol kd{j->key.data.get(), j->key.has_valid ? j->key.valid.as<uint64_t>() : nullptr, class_of(j->key.type_id), 0};
    key_range_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(kd, j->rows, mm, mm + 1);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    int64_t r[2];
    WG_TRY(read_back_i64(ctx, (const int64_t*)mm, r, 2));
    bool ok = true;
    if (r[0] > INT32_MIN) j->sentinel = (int32_t)(r[0] - 1);
    else if (r[1] < INT32_MAX) j->sentinel = (int32_t)(r[1] + 1);
    else ok = false;
    // keys spanning at most 4x the build rows: index by key - min instead of hashing
    const char* dns = std::getenv("WG_JOIN_DENSE");
    const int64_t span = r[1] - r[0] + 1;
    if (ok && (!dns || std::atoi(dns) != 0) && span > 0 && span <= std::max<int64_t>(4 * j->rows, 1024) &&
        span <= (int64_t(1) << 30)) {
      WG_TRY(j->dslots.ensure(ctx, span * 8));
      fill_u64_kernel<<<grid_for(ctx, span, 256), 256, 0, ctx->stream>>>(j->dslots.as<unsigned long long>(), span,
                                                                          (unsigned long long)(uint32_t)j->sentinel);
      ctx->count_launch();
      dense_table_kernel<<<grid_for(ctx, j->rows, 256), 256, 0, ctx->stream>>>(
          kd, j->rows, j->pay[0].data.as<uint32_t>(), r[0], j->dslots.as<unsigned long long>());
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
      j->direct = true;
      j->dense = true;
      j->dense_base = r[0];
      j->dense_slots = span;
    } else if (ok) {
      WG_TRY(j->dslots.ensure(ctx, (int64_t)cap * 8));
      direct_table_kernel<<<grid_for(ctx, (int64_t)cap, 256), 256, 0, ctx->stream>>>(
          j->slots.as<unsigned long long>(), cap, j->pay[0].data.as<uint32_t>(), j->sentinel,
          j->dslots.as<unsigned long long>());
      ctx->count_launch();
      WG_CUDA_TRY(cudaGetLastError());
      j->direct = true;
    }
  }
  return check_device_error(ctx);
}

wg_status wg_join_build_stats(wg_join* j, int64_t* build_rows, int64_t* distinct_keys) {
  if (!j) return fail(WG_E_INVALID, "join is NULL");
  if (build_rows) *build_rows = j->rows;
  if (distinct_keys) *distinct_keys = j->distinct;
  return WG_OK;
}

wg_status wg_join_probe(wg_join* j, const wg_batch_desc* probe, uint32_t* out_probe_rows, int64_t* out_build_rows,
                        int64_t cap, int64_t* cursor, int64_t* out_n) {
  if (!j || !probe || !cursor || !out_n || cap < 0) return fail(WG_E_INVALID, "NULL argument");
  Ctx* ctx = j->ctx;
  WG_TRY(ensure_device(ctx));
  if (!j->finished) return fail(WG_E_STATE, "join build not finished");
  if (j->grace) return fail(WG_E_UNSUPPORTED, "a partitioned build is probed through the fused pipeline");
  if (j->probe_key_col < 0 || j->probe_key_col >= probe->ncols) return fail(WG_E_INVALID, "probe key column out of range");
  const wg_column& kc = probe->cols[j->probe_key_col];
  if (class_of(kc.type_id) != WG_CLS_I32 && class_of(kc.type_id) != WG_CLS_I64)
    return fail(WG_E_UNSUPPORTED, "probe key is not an integer-class column");
  wg_column only = kc;
  wg_batch_desc one{1, 0, &only, probe->len, probe->sel, probe->sel_len};
  WG_TRY(stage_batch(ctx, &one, &j->staged));
  const int64_t n = probe->sel ? probe->sel_len : probe->len;
  *out_n = 0;
  if (n == 0) return WG_OK;
  WG_TRY(j->counts.ensure(ctx, n * 8));
  WG_TRY(j->offs.ensure(ctx, n * 8));
  ProbeArgs a;
  WG_TRY(join_view(j, &a.j));
  a.key = wgd::DCol{j->staged.cols[0].data, j->staged.cols[0].valid_words, class_of(kc.type_id), 0};
  a.sel = j->staged.desc.sel;
  a.n = n;
  a.counts = j->counts.as<int64_t>();
  a.offs = j->offs.as<int64_t>();
  a.cursor = *cursor;
  a.cap = cap;
  a.err = ctx->dev_error;
  join_probe_count_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(a);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, a.counts, j->offs.as<int64_t>(), (int)n, ctx->stream);
  WG_TRY(j->scratch.ensure(ctx, std::max<int64_t>((int64_t)tmp_bytes, 64)));
  cub::DeviceScan::ExclusiveSum(j->scratch.get(), tmp_bytes, a.counts, j->offs.as<int64_t>(), (int)n, ctx->stream);
  ctx->count_launch();
  int64_t last[2] = {0, 0};
  WG_TRY(read_back_i64(ctx, j->offs.as<int64_t>() + (n - 1), &last[0], 1));
  WG_TRY(read_back_i64(ctx, j->counts.as<int64_t>() + (n - 1), &last[1], 1));
  const int64_t total = last[0] + last[1];
  const int64_t m = std::max<int64_t>(0, std::min<int64_t>(cap, total - *cursor));
  if (m > 0) {
    WG_TRY(j->outp.ensure(ctx, m * 4));
    WG_TRY(j->outb.ensure(ctx, m * 8));
    a.out_probe = j->outp.as<uint32_t>();
    a.out_build = j->outb.as<int64_t>();
    join_probe_emit_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(a);
    ctx->count_launch();
    WG_CUDA_TRY(cudaGetLastError());
    WG_CUDA_TRY(cudaMemcpyAsync(out_probe_rows, j->outp.get(), (size_t)(m * 4), cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaMemcpyAsync(out_build_rows, j->outb.get(), (size_t)(m * 8), cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  WG_TRY(check_device_error(ctx));
  *cursor += m;
  *out_n = m;
  return WG_OK;
}

wg_status wg_join_gather(wg_join* j, int32_t payload_idx, const int64_t* build_rows, int64_t n, void* out,
                         uint8_t* out_valid) {
  if (!j || (n > 0 && (!build_rows || !out))) return fail(WG_E_INVALID, "NULL argument");
  if (payload_idx < 0 || payload_idx >= (int32_t)j->pay.size()) return fail(WG_E_INVALID, "payload index out of range");
  Ctx* ctx = j->ctx;
  WG_TRY(ensure_device(ctx));
  if (j->grace) return fail(WG_E_UNSUPPORTED, "a partitioned build is probed through the fused pipeline");
  if (n == 0) return WG_OK;
  for (int64_t i = 0; i < n; ++i)
    if (build_rows[i] < -1 || build_rows[i] >= j->rows) return fail(WG_E_INVALID, "build row out of range");
  BuildCol& c = j->pay[payload_idx];
  WG_TRY(j->rows_dev.ensure(ctx, n * 8));
  WG_TRY(j->gath.ensure(ctx, n * c.es));
  WG_TRY(j->gath_valid.ensure(ctx, n));
  WG_CUDA_TRY(cudaMemcpyAsync(j->rows_dev.get(), build_rows, (size_t)(n * 8), cudaMemcpyHostToDevice, ctx->stream));
  gather_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(
      c.data.as<char>(), c.es, c.has_valid ? c.valid.as<uint64_t>() : nullptr, j->rows_dev.as<int64_t>(), n,
      j->gath.as<char>(), j->gath_valid.as<uint8_t>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaMemcpyAsync(out, j->gath.get(), (size_t)(n * c.es), cudaMemcpyDeviceToHost, ctx->stream));
  if (out_valid) WG_CUDA_TRY(cudaMemcpyAsync(out_valid, j->gath_valid.get(), (size_t)n, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

wg_status wg_join_bloom_filter(wg_join* j, const wg_batch_desc* probe, uint32_t* out_sel, int64_t* n_out) {
  if (!j || !probe || !n_out) return fail(WG_E_INVALID, "NULL argument");
  Ctx* ctx = j->ctx;
  WG_TRY(ensure_device(ctx));
  if (!j->finished) return fail(WG_E_STATE, "join build not finished");
  if (j->grace) return fail(WG_E_UNSUPPORTED, "a partitioned build has no bloom filter");
  if (j->probe_key_col < 0 || j->probe_key_col >= probe->ncols) return fail(WG_E_INVALID, "probe key column out of range");
  const wg_column& kc = probe->cols[j->probe_key_col];
  if (class_of(kc.type_id) != WG_CLS_I32 && class_of(kc.type_id) != WG_CLS_I64)
    return fail(WG_E_UNSUPPORTED, "probe key is not an integer-class column");
  const int64_t n = probe->sel ? probe->sel_len : probe->len;
  *n_out = 0;
  if (n == 0 || j->distinct == 0) return WG_OK;
  if (!out_sel) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(build_bloom(j));
  wg_column only = kc;
  wg_batch_desc one{1, 0, &only, probe->len, probe->sel, probe->sel_len};
  WG_TRY(stage_batch(ctx, &one, &j->staged));
  WG_TRY(j->bloom_rows.ensure(ctx, n * 4));
  WG_TRY(j->bloom_flags.ensure(ctx, n));
  const int64_t count_off = (n * 4 + 7) & ~int64_t(7);  // the count's 8-byte word after the rows
  WG_TRY(j->bloom_out.ensure(ctx, count_off + 16));
  const wgd::DCol key{j->staged.cols[0].data, j->staged.cols[0].valid_words, class_of(kc.type_id), 0};
  bloom_probe_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(key, j->staged.desc.sel, n,
                                                                      j->bloom.as<unsigned long long>(), j->bloom_mask,
                                                                      j->bloom_rows.as<uint32_t>(),
                                                                      j->bloom_flags.as<uint8_t>());
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  // order-preserving compaction of the kept rows
  int64_t* d_count = (int64_t*)(j->bloom_out.as<char>() + count_off);
  size_t tmp = 0;
  cub::DeviceSelect::Flagged(nullptr, tmp, j->bloom_rows.as<uint32_t>(), j->bloom_flags.as<uint8_t>(),
                             j->bloom_out.as<uint32_t>(), d_count, (int)n, ctx->stream);
  WG_TRY(j->bloom_tmp.ensure(ctx, std::max<int64_t>((int64_t)tmp, 16)));
  cub::DeviceSelect::Flagged(j->bloom_tmp.get(), tmp, j->bloom_rows.as<uint32_t>(), j->bloom_flags.as<uint8_t>(),
                             j->bloom_out.as<uint32_t>(), d_count, (int)n, ctx->stream);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  int64_t m = 0;
  WG_TRY(read_back_i64(ctx, d_count, &m, 1));
  if (m > 0)
    WG_CUDA_TRY(cudaMemcpyAsync(out_sel, j->bloom_out.get(), (size_t)(m * 4), cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  WG_TRY(check_device_error(ctx));
  *n_out = m;
  return WG_OK;
}

wg_status wg_join_reset(wg_join* j) {
  if (!j) return fail(WG_E_INVALID, "join is NULL");
  WG_TRY(ensure_device(j->ctx));
  WG_CUDA_TRY(cudaStreamSynchronize(j->ctx->stream));
  j->rows = 0;
  j->finished = false;
  j->key.has_valid = false;
  j->key.valid.reset();
  for (BuildCol& c : j->pay) { c.has_valid = false; c.valid.reset(); }
  j->distinct = 0;
  j->unique = true;
  j->max_fanout = 1;
  j->bloom_built = false;
  j->grace = false;
  j->parts.clear();
  j->passes.clear();
  delete j->pass;
  j->pass = nullptr;
  j->pass_built = -1;
  return WG_OK;
}

wg_status wg_join_destroy(wg_join* j) {
  if (!j) return WG_OK;
  ensure_device(j->ctx);
  cudaStreamSynchronize(j->ctx->stream);
  delete j;
  return WG_OK;
}

}  // extern "C"
