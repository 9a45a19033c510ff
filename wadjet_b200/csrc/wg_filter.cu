// wg_filter.cu — exec.KernelFilter on the GPU (internal/engine/exec/filter.go:347-425).
//
// One pass over the column: each thread evaluates 4 × V rows with 128-bit
// vector loads (V = 16 / element size), every row's verdict becomes a bit of a
// warp ballot-style count, a block-wide scan orders the survivors, and the
// tile's position in the output comes from a decoupled look-back over the
// preceding tiles (Merrill & Garland, "Single-pass Parallel Prefix Scan with
// Decoupled Look-back", NVIDIA TR 2016). Output is the ascending selection
// vector the reference's compaction produces, so the result is bit-exact.
// Every wait on a predecessor tile is bounded; on expiry the kernel records
// WG_DERR_TIMEOUT and publishes its own state so no successor waits forever.
#include "wg_internal.h"
#include "wg_pred.cuh"

#include <algorithm>
#include <cstdlib>

namespace wg {

// Resolve a predicate constant against the column type (ResolveFilterKernel,
// internal/engine/exec/kernel/compare.go:145-182; toInt64/toFloat64/toDateInt32 :580-640).
wg_status resolve_pred(const wg_predicate& p, int32_t type_id, wgd::Pred* out) {
  if (p.op < WG_OP_EQ || p.op > WG_OP_GE) return fail(WG_E_INVALID, "unknown compare op");
  auto to_i64 = [&]() -> long long {
    if (p.const_kind == WG_CONST_FLOAT) {
      double f = p.const_f64;  // Go float64→int64 on amd64: out of range gives MinInt64
      if (!(f >= -9223372036854775808.0 && f < 9223372036854775808.0)) return INT64_MIN;
      return (long long)f;
    }
    return p.const_i64;
  };
  auto to_f64 = [&]() -> double { return p.const_kind == WG_CONST_FLOAT ? p.const_f64 : (double)p.const_i64; };
  out->col = p.col;
  out->op = p.op;
  out->_pad = 0;
  out->ci = 0;
  out->cf = 0;
  switch (type_id) {
    case WG_TYPE_INT64: case WG_TYPE_TIMESTAMP: case WG_TYPE_DURATION: case WG_TYPE_IPV4: case WG_TYPE_MAC:
      out->cls = WG_CLS_I64; out->ci = to_i64(); return WG_OK;
    case WG_TYPE_INT32: case WG_TYPE_PORT: case WG_TYPE_PROTOCOL:
      out->cls = WG_CLS_I32; out->ci = (int32_t)to_i64(); return WG_OK;
    case WG_TYPE_DATE:
      out->cls = WG_CLS_I32; out->ci = p.const_kind == WG_CONST_FLOAT ? 0 : (int32_t)p.const_i64; return WG_OK;
    case WG_TYPE_FLOAT64:
      out->cls = WG_CLS_F64; out->cf = to_f64(); return WG_OK;
    case WG_TYPE_FLOAT32:
      out->cls = WG_CLS_F32; out->cf = (double)(float)to_f64(); return WG_OK;
    default:
      return fail(WG_E_UNSUPPORTED, "filter on this column type is not on the GPU path");
  }
}

}  // namespace wg

namespace {

using namespace wgd;

constexpr int kBlock = 256;
constexpr int kRows = 8;
constexpr unsigned long long kFlagAgg = 1ULL << 62;
constexpr unsigned long long kFlagInc = 2ULL << 62;
constexpr unsigned long long kValMask = (1ULL << 62) - 1;
// Failed polls of a predecessor's status word before a tile gives up
// (WG_DERR_TIMEOUT). WG_FILTER_SPIN_LIMIT overrides it; 0 makes every tile
// after the first give up at once, which tests the timeout path
// deterministically without a wait that never ends.
constexpr long long kSpinLimit = 1LL << 20;

long long spin_limit() {
  const char* v = std::getenv("WG_FILTER_SPIN_LIMIT");
  return v ? std::max(0LL, std::atoll(v)) : kSpinLimit;
}

struct FilterArgs {
  DCol col;
  Pred p;
  const uint32_t* sel;   // nullptr = rows 0..n-1
  int64_t n;             // items: rows, or selection entries
  uint32_t* out;
  unsigned long long* status;
  int* tile_counter;
  int64_t* out_n;
  int32_t* err;
  int64_t num_tiles;
  long long spin_limit;
};

template <typename T> struct VecOf;
template <> struct VecOf<int32_t> { using type = int4; };
template <> struct VecOf<float> { using type = float4; };
template <> struct VecOf<long long> { using type = longlong2; };
template <> struct VecOf<double> { using type = double2; };

template <int CLS> struct ClsT;
template <> struct ClsT<WG_CLS_I32> { using T = int32_t; };
template <> struct ClsT<WG_CLS_I64> { using T = long long; };
template <> struct ClsT<WG_CLS_F32> { using T = float; };
template <> struct ClsT<WG_CLS_F64> { using T = double; };

template <int CLS, bool VEC, int OP>
__global__ void __launch_bounds__(kBlock) filter_compact_kernel(const FilterArgs a) {
  using T = typename ClsT<CLS>::T;
  constexpr int V = VEC ? (int)(16 / sizeof(T)) : 1;
  constexpr int64_t kTile = (int64_t)kBlock * V * kRows;
  __shared__ int s_tile;
  __shared__ int s_warp[kRows][kBlock / 32];
  __shared__ int s_total;
  __shared__ long long s_prefix;
  __shared__ uint32_t s_out[kTile];

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) s_tile = atomicAdd(a.tile_counter, 1);
  __syncthreads();
  const int64_t tile = s_tile;
  const int64_t tile_base = tile * kTile;
  const T cval = (CLS == WG_CLS_F32 || CLS == WG_CLS_F64) ? (T)a.p.cf : (T)a.p.ci;

  unsigned bits[kRows];
  int excl[kRows];
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    const int64_t i0 = tile_base + ((int64_t)r * kBlock + tid) * V;
    unsigned b = 0;
    if (a.sel == nullptr && VEC && i0 + V <= a.n) {
      typename VecOf<T>::type v = __ldg(reinterpret_cast<const typename VecOf<T>::type*>((const T*)a.col.data + i0));
      const T* e = reinterpret_cast<const T*>(&v);
#pragma unroll
      for (int k = 0; k < V; ++k)
        if (cmp_op<T>(e[k], cval, OP) && !is_null(a.col, i0 + k)) b |= 1u << k;
    } else {
#pragma unroll
      for (int k = 0; k < V; ++k) {
        const int64_t it = i0 + k;
        if (it < a.n) {
          const int64_t row = a.sel ? (int64_t)__ldg(a.sel + it) : it;
          if (!is_null(a.col, row) && cmp_op<T>(__ldg((const T*)a.col.data + row), cval, OP)) b |= 1u << k;
        }
      }
    }
    bits[r] = b;
    // warp inclusive scan of this thread's survivor count
    int c = __popc(b), incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      int y = __shfl_up_sync(WG_FULL_MASK, incl, d);
      if (lane >= d) incl += y;
    }
    excl[r] = incl - c;
    if (lane == 31) s_warp[r][warp] = incl;
  }
  __syncthreads();
  // Decoupled look-back by warp 0: each step reads the status words of the 32
  // closest unread predecessors at once, waits (bounded) until all of them
  // have published, and adds their aggregates up to the closest inclusive one.
  if (warp == 0) {
    int run = 0;
    if (lane == 0) {
      for (int r = 0; r < kRows; ++r)
        for (int w = 0; w < kBlock / 32; ++w) { int t = s_warp[r][w]; s_warp[r][w] = run; run += t; }
      s_total = run;
      atomicExch(a.status + tile, (tile == 0 ? kFlagInc : kFlagAgg) | (unsigned long long)run);
    }
    run = __shfl_sync(WG_FULL_MASK, run, 0);
    long long prefix = 0;
    if (tile > 0) {
      int64_t tail = tile - 1;
      long long spins = 0;
      bool expired = false;
      for (;;) {
        const int64_t idx = tail - lane;
        unsigned long long st = idx >= 0 ? 0ULL : kFlagInc;  // before tile 0: an inclusive 0
        // the tile publishes its (partial) prefix on expiry, so no successor
        // waits forever and every position it writes stays below the true one
        for (;;) {
          if (spins >= a.spin_limit) { expired = true; break; }
          if ((st & ~kValMask) == 0) st = *((volatile unsigned long long*)(a.status + idx));
          if (!__any_sync(WG_FULL_MASK, (st & ~kValMask) == 0)) break;
          ++spins;
          __nanosleep(64);
        }
        if (expired) {
          if (lane == 0) set_error(a.err, WG_DERR_TIMEOUT);
          break;
        }
        const unsigned inc = __ballot_sync(WG_FULL_MASK, (st & ~kValMask) == kFlagInc);
        const int stop = inc ? __ffs(inc) - 1 : 31;  // lanes 0..stop count
        long long v = lane <= stop ? (long long)(st & kValMask) : 0LL;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(WG_FULL_MASK, v, o);
        prefix += v;
        if (inc) break;
        tail -= 32;
      }
      if (lane == 0) atomicExch(a.status + tile, kFlagInc | (unsigned long long)(prefix + run));
    }
    if (lane == 0) {
      s_prefix = prefix;
      if (tile == a.num_tiles - 1) *a.out_n = prefix + run;
    }
  }
  __syncthreads();
  // the tile's survivors gathered in shared memory in order, then written out
  // contiguously (coalesced stores instead of each thread's scattered ones)
  const long long prefix = s_prefix;
#pragma unroll
  for (int r = 0; r < kRows; ++r) {
    unsigned b = bits[r];
    if (!b) continue;
    int pos = s_warp[r][warp] + excl[r];
    const int64_t i0 = tile_base + ((int64_t)r * kBlock + tid) * V;
#pragma unroll
    for (int k = 0; k < V; ++k)
      if (b & (1u << k)) s_out[pos++] = a.sel ? __ldg(a.sel + i0 + k) : (uint32_t)(i0 + k);
  }
  __syncthreads();
  const int total = s_total;
  for (int i = tid; i < total; i += kBlock) a.out[prefix + i] = s_out[i];
}

// One kernel per column class, vector width and comparison (the operator
// compiled in rather than switched on per element).
template <int CLS, int OP>
void launch_op(bool vec, const FilterArgs& a, dim3 grid, cudaStream_t s) {
  if (vec) filter_compact_kernel<CLS, true, OP><<<grid, kBlock, 0, s>>>(a);
  else filter_compact_kernel<CLS, false, OP><<<grid, kBlock, 0, s>>>(a);
}

template <int CLS>
void launch_cls(bool vec, const FilterArgs& a, dim3 grid, cudaStream_t s) {
  switch (a.p.op) {
    case 0: launch_op<CLS, 0>(vec, a, grid, s); break;
    case 1: launch_op<CLS, 1>(vec, a, grid, s); break;
    case 2: launch_op<CLS, 2>(vec, a, grid, s); break;
    case 3: launch_op<CLS, 3>(vec, a, grid, s); break;
    case 4: launch_op<CLS, 4>(vec, a, grid, s); break;
    default: launch_op<CLS, 5>(vec, a, grid, s); break;
  }
}

}  // namespace

struct wg_filter {
  wg::Ctx* ctx;
  wg_predicate pred;
  bool resolved = false;
  int32_t type_id = -1;
  wgd::Pred dp{};
  wg::DevBuf status, counter, out_sel, out_n;
  wg::StagedBatch staged;
};

namespace wg {

// Run the compaction over a device-resident column; *n_out is left on the device.
wg_status filter_launch(Ctx* ctx, const wgd::Pred& p, const wg_column& col, const uint32_t* sel, int64_t n_items,
                        uint32_t* out, int64_t* n_out_dev, DevBuf& status, DevBuf& counter) {
  const int cls = class_of(col.type_id);
  const int64_t es = elem_size(col.type_id);
  const bool vec = sel == nullptr && ((uintptr_t)col.data % 16 == 0);
  const int64_t V = vec ? 16 / es : 1;
  const int64_t tile = (int64_t)kBlock * V * kRows;
  const int64_t tiles = (n_items + tile - 1) / tile;
  if (tiles == 0) {
    WG_CUDA_TRY(cudaMemsetAsync(n_out_dev, 0, sizeof(int64_t), ctx->stream));
    return WG_OK;
  }
  if (tiles > (1LL << 31) - 1) return fail(WG_E_INVALID, "batch too large");
  WG_TRY(status.ensure(ctx, tiles * 8));
  WG_TRY(counter.ensure(ctx, 16));
  WG_CUDA_TRY(cudaMemsetAsync(status.get(), 0, (size_t)(tiles * 8), ctx->stream));
  WG_CUDA_TRY(cudaMemsetAsync(counter.get(), 0, sizeof(int), ctx->stream));
  FilterArgs a;
  a.col = wgd::DCol{col.data, col.valid_words, cls, col.scale};
  a.p = p;
  a.sel = sel;
  a.n = n_items;
  a.out = out;
  a.status = status.as<unsigned long long>();
  a.tile_counter = counter.as<int>();
  a.out_n = n_out_dev;
  a.err = ctx->dev_error;
  a.num_tiles = tiles;
  a.spin_limit = spin_limit();
  dim3 grid((unsigned)tiles);
  switch (cls) {
    case WG_CLS_I32: launch_cls<WG_CLS_I32>(vec, a, grid, ctx->stream); break;
    case WG_CLS_I64: launch_cls<WG_CLS_I64>(vec, a, grid, ctx->stream); break;
    case WG_CLS_F32: launch_cls<WG_CLS_F32>(vec, a, grid, ctx->stream); break;
    case WG_CLS_F64: launch_cls<WG_CLS_F64>(vec, a, grid, ctx->stream); break;
    default: return fail(WG_E_UNSUPPORTED, "filter on this column type is not on the GPU path");
  }
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  return WG_OK;
}

}  // namespace wg

using namespace wg;

static wg_status filter_resolve(wg_filter* f, const wg_batch_desc* in) {
  if (!in) return fail(WG_E_INVALID, "batch is NULL");
  if (f->pred.col < 0 || f->pred.col >= in->ncols)
    return fail(WG_E_INVALID, "filter column " + std::to_string(f->pred.col) + " does not exist in the input schema");
  const int32_t t = in->cols[f->pred.col].type_id;
  if (!f->resolved) {
    WG_TRY(resolve_pred(f->pred, t, &f->dp));
    f->type_id = t;
    f->resolved = true;
  } else if (t != f->type_id) {
    return fail(WG_E_INVALID, "filter column changed type after the kernel was resolved");
  }
  return WG_OK;
}

extern "C" {

wg_status wg_filter_create(wg_ctx* ctx, int32_t col_idx, int32_t op, int32_t const_kind, int64_t const_i64,
                           double const_f64, wg_filter** out) {
  if (!ctx || !out) return fail(WG_E_INVALID, "NULL argument");
  if (op < WG_OP_EQ || op > WG_OP_GE) return fail(WG_E_INVALID, "unknown compare op");
  if (const_kind != WG_CONST_INT && const_kind != WG_CONST_FLOAT) return fail(WG_E_INVALID, "unknown constant kind");
  wg_filter* f = new wg_filter();
  f->ctx = ctx;
  f->pred = wg_predicate{col_idx, op, const_kind, 0, const_i64, const_f64};
  *out = f;
  return WG_OK;
}

wg_status wg_filter_execute_device(wg_filter* f, const wg_batch_desc* in, uint32_t* out_sel_dev, int64_t* out_n) {
  if (!f || !out_n) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(f->ctx));
  WG_TRY(filter_resolve(f, in));
  Ctx* ctx = f->ctx;
  const int64_t n_items = in->sel ? in->sel_len : in->len;
  WG_TRY(f->out_n.ensure(ctx, 16));
  WG_TRY(filter_launch(ctx, f->dp, in->cols[f->pred.col], in->sel, n_items, out_sel_dev, f->out_n.as<int64_t>(),
                       f->status, f->counter));
  WG_TRY(read_back_i64(ctx, f->out_n.as<int64_t>(), out_n, 1));
  return check_device_error(ctx);
}

wg_status wg_filter_execute(wg_filter* f, const wg_batch_desc* in, uint32_t* out_sel, int64_t* out_n) {
  if (!f || !out_n || !out_sel) return fail(WG_E_INVALID, "NULL argument");
  WG_TRY(ensure_device(f->ctx));
  WG_TRY(filter_resolve(f, in));
  Ctx* ctx = f->ctx;
  // stage only the filtered column (and the selection vector)
  wg_column only = in->cols[f->pred.col];
  wg_batch_desc one{1, 0, &only, in->len, in->sel, in->sel_len};
  WG_TRY(stage_batch(ctx, &one, &f->staged));
  const int64_t n_items = in->sel ? in->sel_len : in->len;
  WG_TRY(f->out_sel.ensure(ctx, std::max<int64_t>(n_items * 4, 16)));
  WG_TRY(f->out_n.ensure(ctx, 16));
  wgd::Pred p = f->dp;
  WG_TRY(filter_launch(ctx, p, f->staged.cols[0], f->staged.desc.sel, n_items, f->out_sel.as<uint32_t>(),
                       f->out_n.as<int64_t>(), f->status, f->counter));
  WG_TRY(read_back_i64(ctx, f->out_n.as<int64_t>(), out_n, 1));
  WG_TRY(check_device_error(ctx));
  if (*out_n > 0) {
    WG_CUDA_TRY(cudaMemcpyAsync(out_sel, f->out_sel.get(), (size_t)(*out_n * 4), cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  return WG_OK;
}

wg_status wg_filter_destroy(wg_filter* f) {
  if (!f) return WG_OK;
  ensure_device(f->ctx);
  cudaStreamSynchronize(f->ctx->stream);
  delete f;
  return WG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free variant for callers that cannot call cudaMalloc (see the
// header): the tile-status words, the tile counter, the device error word and
// the survivor count live in one static device array instead of per-handle
// device buffers. Layout: status[65536] | counter (int32) | error (int32) |
// count (int64).
// ---------------------------------------------------------------------------
namespace {

constexpr int64_t kNoAllocTiles = 65536;
static __device__ __align__(256) unsigned char g_noalloc_scratch[WG_NOALLOC_SCRATCH_BYTES];

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};  // per device: the array's device address, looked up once

}  // namespace

extern "C" wg_status wg_filter_execute_device_noalloc(void* stream, const wg_column* col, const uint32_t* sel,
                                                      int64_t n_items, int32_t op, int32_t const_kind,
                                                      int64_t const_i64, double const_f64, uint32_t* out_sel,
                                                      int64_t* out_n) {
  if (!col || !col->data || !out_n || (n_items > 0 && !out_sel) || n_items < 0)
    return fail(WG_E_INVALID, "NULL argument");
  if (n_items > WG_NOALLOC_MAX_ITEMS)
    return fail(WG_E_INVALID, "input of " + std::to_string(n_items) + " rows exceeds the allocation-free limit of " +
                                  std::to_string((long long)WG_NOALLOC_MAX_ITEMS));
  if (op < WG_OP_EQ || op > WG_OP_GE || (const_kind != WG_CONST_INT && const_kind != WG_CONST_FLOAT))
    return fail(WG_E_INVALID, "unknown compare op or constant kind");
  // without a selection vector the items are the column's rows: more would read past it
  if (!sel && n_items > col->len)
    return fail(WG_E_INVALID, "n_items (" + std::to_string(n_items) + ") exceeds the column length (" +
                                  std::to_string(col->len) + ")");
  wgd::Pred p;
  WG_TRY(resolve_pred(wg_predicate{0, op, const_kind, 0, const_i64, const_f64}, col->type_id, &p));
  int dev = -1;
  WG_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(WG_E_INVALID, "device ordinal out of range");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {  // set-up, once per device, with that device current
      void* ptr = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess) return fail(WG_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_noalloc_addr[dev] = ptr;
    }
    base = (unsigned char*)g_noalloc_addr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* status = (unsigned long long*)base;
  int* counter = (int*)(base + kNoAllocTiles * 8);
  int32_t* err = (int32_t*)(base + kNoAllocTiles * 8 + 4);
  int64_t* count = (int64_t*)(base + kNoAllocTiles * 8 + 8);
  const int cls = class_of(col->type_id);
  const int64_t es = elem_size(col->type_id);
  const bool vec = sel == nullptr && ((uintptr_t)col->data % 16 == 0);
  const int64_t V = vec ? 16 / es : 1;
  const int64_t tiles = (n_items + kBlock * V * kRows - 1) / (kBlock * V * kRows);
  // the previous call's words are still there: clear the counter, error, count and the status words in use
  WG_CUDA_TRY(cudaMemsetAsync(counter, 0, 16, st));
  if (tiles > 0) WG_CUDA_TRY(cudaMemsetAsync(status, 0, (size_t)(tiles * 8), st));
  if (tiles > 0) {
    FilterArgs a;
    a.col = wgd::DCol{col->data, col->valid_words, cls, col->scale};
    a.p = p;
    a.sel = sel;
    a.n = n_items;
    a.out = out_sel;
    a.status = status;
    a.tile_counter = counter;
    a.out_n = count;
    a.err = err;
    a.num_tiles = tiles;
    a.spin_limit = spin_limit();
    dim3 grid((unsigned)tiles);
    switch (cls) {
      case WG_CLS_I32: launch_cls<WG_CLS_I32>(vec, a, grid, st); break;
      case WG_CLS_I64: launch_cls<WG_CLS_I64>(vec, a, grid, st); break;
      case WG_CLS_F32: launch_cls<WG_CLS_F32>(vec, a, grid, st); break;
      case WG_CLS_F64: launch_cls<WG_CLS_F64>(vec, a, grid, st); break;
      default: return fail(WG_E_UNSUPPORTED, "filter on this column type is not on the GPU path");
    }
    WG_CUDA_TRY(cudaGetLastError());
  }
  int64_t host[2] = {0, 0};  // count, then the error word
  WG_CUDA_TRY(cudaMemcpyAsync(&host[0], count, 8, cudaMemcpyDeviceToHost, st));
  WG_CUDA_TRY(cudaMemcpyAsync(&host[1], err, 4, cudaMemcpyDeviceToHost, st));
  WG_CUDA_TRY(cudaStreamSynchronize(st));
  if ((int32_t)host[1] != WG_DERR_NONE) return fail(WG_E_TIMEOUT, "bounded device wait expired");
  *out_n = tiles > 0 ? host[0] : 0;
  return WG_OK;
}
