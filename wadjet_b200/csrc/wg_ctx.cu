// wg_ctx.cu — context, HBM ledger, errors, host-batch staging.
#include "wg_internal.h"
#include "wg_device.cuh"

#include <condition_variable>
#include <cstdlib>
#include <cstdio>
#include <thread>

namespace wg {

// ---- host copy threads -------------------------------------------------------
namespace {
struct CopyPool {
  std::mutex mu;
  std::condition_variable cv_job, cv_done;
  std::vector<std::thread> threads;
  // the current job: piece i of n copies [i * per, min(bytes, (i + 1) * per))
  char* dst = nullptr;
  const char* src = nullptr;
  int64_t bytes = 0, per = 0;
  int n = 0, next = 0, left = 0;
  uint64_t gen = 0;
  std::mutex job_mu;  // one job at a time
  explicit CopyPool(int t) {
    for (int i = 0; i < t; ++i) threads.emplace_back([this] { run(); });
  }
  void run() {
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
      cv_job.wait(lk, [&] { return next < n; });
      const int i = next++;
      char* d = dst;
      const char* s = src;
      const int64_t b0 = (int64_t)i * per, b1 = std::min(bytes, b0 + per);
      lk.unlock();
      if (b1 > b0) std::memcpy(d + b0, s + b0, (size_t)(b1 - b0));
      lk.lock();
      if (--left == 0) cv_done.notify_all();
    }
  }
};
CopyPool* copy_pool() {
  // threads live until the process exits (the pool is never destroyed, so no
  // thread is joined from a static destructor)
  static CopyPool* p = new CopyPool([] {
    const char* v = std::getenv("WG_COPY_THREADS");  // default: the host's cores, at most 16
    const int t = v ? std::atoi(v) : (int)std::min(16u, std::thread::hardware_concurrency());
    return std::max(1, std::min(64, t));
  }());
  return p;
}
}  // namespace

void parallel_copy(void* dst, const void* src, int64_t bytes) {
  if (bytes <= 0) return;
  if (bytes < (int64_t(4) << 20)) {
    std::memcpy(dst, src, (size_t)bytes);
    return;
  }
  CopyPool* p = copy_pool();
  std::lock_guard<std::mutex> job(p->job_mu);
  std::unique_lock<std::mutex> lk(p->mu);
  const int t = (int)p->threads.size();
  p->dst = (char*)dst;
  p->src = (const char*)src;
  p->bytes = bytes;
  p->per = ((bytes + t - 1) / t + 4095) & ~int64_t(4095);
  p->n = (int)((bytes + p->per - 1) / p->per);
  p->next = 0;
  p->left = p->n;
  p->cv_job.notify_all();
  p->cv_done.wait(lk, [&] { return p->left == 0; });
  p->n = 0;
  p->next = 0;
}

thread_local std::string t_err;

void set_error(const std::string& msg) { t_err = msg; }
wg_status fail(wg_status code, const std::string& msg) {
  t_err = msg;
  return code;
}

wg_status ensure_device(Ctx* ctx) {
  int cur = -1;
  WG_CUDA_TRY(cudaGetDevice(&cur));
  if (cur != ctx->device) WG_CUDA_TRY(cudaSetDevice(ctx->device));
  return WG_OK;
}

wg_status DevBuf::alloc(Ctx* ctx, int64_t bytes) {
  reset();
  if (bytes <= 0) return WG_OK;
  int64_t rounded = (bytes + 255) & ~int64_t(255);
  if (!ctx->ledger.reserve(rounded))
    return fail(WG_E_NOMEM, "HBM ledger: memory budget exceeded (used=" + std::to_string(ctx->ledger.used()) +
                                ", requested=" + std::to_string(rounded) +
                                ", budget=" + std::to_string(ctx->ledger.budget()) + ")");
  void* p = nullptr;
  cudaError_t e = cudaMalloc(&p, (size_t)rounded);
  if (e != cudaSuccess) {
    ctx->ledger.release(rounded);
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? WG_E_NOMEM : WG_E_CUDA,
                std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  ctx_ = ctx; ptr_ = p; bytes_ = rounded;
  return WG_OK;
}

wg_status DevBuf::ensure(Ctx* ctx, int64_t bytes) {
  if (bytes <= bytes_ && ctx_ == ctx) return WG_OK;
  return alloc(ctx, bytes);
}

void DevBuf::reset() {
  if (ptr_) {
    cudaFree(ptr_);
    ctx_->ledger.release(bytes_);
  }
  ctx_ = nullptr; ptr_ = nullptr; bytes_ = 0;
}

int64_t elem_size(int32_t t) {
  switch (t) {
    case WG_TYPE_INT32: case WG_TYPE_PORT: case WG_TYPE_PROTOCOL: case WG_TYPE_DATE: case WG_TYPE_FLOAT32: return 4;
    case WG_TYPE_INT64: case WG_TYPE_TIMESTAMP: case WG_TYPE_IPV4: case WG_TYPE_MAC: case WG_TYPE_DURATION:
    case WG_TYPE_FLOAT64: return 8;
    case WG_TYPE_DECIMAL: return 16;
    default: return 0;
  }
}

int class_of(int32_t t) {
  switch (t) {
    case WG_TYPE_INT32: case WG_TYPE_PORT: case WG_TYPE_PROTOCOL: case WG_TYPE_DATE: return WG_CLS_I32;
    case WG_TYPE_INT64: case WG_TYPE_TIMESTAMP: case WG_TYPE_IPV4: case WG_TYPE_MAC: case WG_TYPE_DURATION:
      return WG_CLS_I64;
    case WG_TYPE_FLOAT32: return WG_CLS_F32;
    case WG_TYPE_FLOAT64: return WG_CLS_F64;
    case WG_TYPE_DECIMAL: return WG_CLS_DEC;
    default: return WG_CLS_BAD;
  }
}

wg_status read_back_i64(Ctx* ctx, const int64_t* dev, int64_t* out, int n) {
  std::lock_guard<std::mutex> g(ctx->mu);
  WG_CUDA_TRY(cudaMemcpyAsync(ctx->host_scalar, dev, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int i = 0; i < n; ++i) out[i] = ctx->host_scalar[i];
  return WG_OK;
}

static wg_status device_error_status(Ctx* ctx, int32_t h);

wg_status check_device_error(Ctx* ctx) {
  int32_t h = 0;
  WG_CUDA_TRY(cudaMemcpyAsync(&h, ctx->dev_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return device_error_status(ctx, h);
}

wg_status read_back_checked(Ctx* ctx, const int64_t* dev, int64_t* out, int n) {
  int32_t h = 0;
  {
    std::lock_guard<std::mutex> g(ctx->mu);
    if (n > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(ctx->host_scalar, dev, sizeof(int64_t) * n, cudaMemcpyDeviceToHost, ctx->stream));
    int32_t* herr = reinterpret_cast<int32_t*>(ctx->host_scalar + 63);
    WG_CUDA_TRY(cudaMemcpyAsync(herr, ctx->dev_error, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < n; ++i) out[i] = ctx->host_scalar[i];
    h = *herr;
  }
  return device_error_status(ctx, h);
}

static wg_status device_error_status(Ctx* ctx, int32_t h) {
  if (h == WG_DERR_NONE) return WG_OK;
  WG_CUDA_TRY(cudaMemsetAsync(ctx->dev_error, 0, sizeof(int32_t), ctx->stream));
  switch (h) {
    case WG_DERR_TABLE_FULL: return fail(WG_E_NOMEM, "device hash table full");
    case WG_DERR_TIMEOUT: return fail(WG_E_TIMEOUT, "bounded device wait expired");
    case WG_DERR_NULL_PACKED: return fail(WG_E_UNSUPPORTED, "NULL in a composite GROUP BY key");
    case WG_DERR_STACK: return fail(WG_E_INVALID, "malformed expression program");
    case WG_DERR_BAD_PAGE: return fail(WG_E_INVALID, "malformed Parquet page");
    case WG_DERR_HASH_COLLISION: return fail(WG_E_UNSUPPORTED, "two GROUP BY strings share a 128-bit hash");
    default: return fail(WG_E_CUDA, "device error " + std::to_string(h));
  }
}

wg_status stage_batch(Ctx* ctx, const wg_batch_desc* in, StagedBatch* out) {
  if (!in || in->ncols < 0 || (in->ncols > 0 && !in->cols)) return fail(WG_E_INVALID, "bad batch descriptor");
  out->data.clear(); out->valid.clear();
  out->data.resize((size_t)in->ncols);
  out->valid.resize((size_t)in->ncols);
  out->cols.assign(in->cols, in->cols + in->ncols);
  for (int c = 0; c < in->ncols; ++c) {
    const wg_column& src = in->cols[c];
    int64_t es = elem_size(src.type_id);
    if (es == 0 || !src.data) { out->cols[c].data = nullptr; out->cols[c].valid_words = nullptr; continue; }
    int64_t n = in->len;
    WG_TRY(out->data[c].alloc(ctx, std::max<int64_t>(n * es, 16)));
    if (n > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(out->data[c].get(), src.data, (size_t)(n * es), cudaMemcpyHostToDevice, ctx->stream));
    out->cols[c].data = out->data[c].get();
    if (src.valid_words) {
      int64_t words = (n + 63) / 64;
      WG_TRY(out->valid[c].alloc(ctx, std::max<int64_t>(words * 8, 16)));
      if (words > 0)
        WG_CUDA_TRY(cudaMemcpyAsync(out->valid[c].get(), src.valid_words, (size_t)(words * 8), cudaMemcpyHostToDevice,
                                    ctx->stream));
      out->cols[c].valid_words = out->valid[c].as<uint64_t>();
    }
  }
  out->desc = *in;
  out->desc.cols = out->cols.data();
  if (in->sel) {
    WG_TRY(out->sel.alloc(ctx, std::max<int64_t>(in->sel_len * 4, 16)));
    if (in->sel_len > 0)
      WG_CUDA_TRY(cudaMemcpyAsync(out->sel.get(), in->sel, (size_t)(in->sel_len * 4), cudaMemcpyHostToDevice, ctx->stream));
    out->desc.sel = out->sel.as<uint32_t>();
  }
  return WG_OK;
}

}  // namespace wg

using namespace wg;

extern "C" {

const char* wg_last_error(void) { return wg::t_err.c_str(); }

const char* wg_version(void) { return "wadjet-b200 0.1.0 (sm_100a)"; }

static wg_status ctx_make(int32_t device, int64_t budget, wg::Ledger* parent, int64_t pinned_spill_bytes,
                          wg_ctx** out) {
  wg_ctx* c = new wg_ctx(budget, parent);
  c->device = device;
  c->pinned_spill_bytes = pinned_spill_bytes;
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e == cudaSuccess) {
    c->sm_count = prop.multiProcessorCount;
    c->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
    c->smem_per_sm = (int)prop.sharedMemPerMultiprocessor;
  }
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost((void**)&c->host_scalar, 64 * sizeof(int64_t)) != cudaSuccess ||
      cudaMalloc((void**)&c->dev_scalar, 64 * sizeof(int64_t)) != cudaSuccess ||
      cudaMalloc((void**)&c->dev_error, 256) != cudaSuccess) {
    wg_ctx_destroy(c);
    return fail(WG_E_CUDA, "context resources could not be created");
  }
  for (int i = 0; i < 2; ++i) {
    cudaEventCreateWithFlags(&c->staged[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->consumed[i], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&c->h2d_done[i], cudaEventDisableTiming);
  }
  cudaMemset(c->dev_error, 0, 256);
  cudaMemset(c->dev_scalar, 0, 64 * sizeof(int64_t));
  cudaDeviceSynchronize();
  *out = c;
  return WG_OK;
}

wg_status wg_ctx_create(int32_t device, int64_t hbm_budget_bytes, int64_t pinned_spill_bytes, wg_ctx** out) {
  if (!out) return fail(WG_E_INVALID, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  WG_CUDA_TRY(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) return fail(WG_E_INVALID, "no such CUDA device");
  WG_CUDA_TRY(cudaSetDevice(device));
  int64_t budget = hbm_budget_bytes;
  if (budget <= 0) {
    size_t free_b = 0, total_b = 0;
    WG_CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    budget = (int64_t)free_b;
  }
  return ctx_make(device, budget, nullptr, pinned_spill_bytes, out);
}

wg_status wg_ctx_create_child(wg_ctx* parent, wg_ctx** out) {
  if (!parent || !out) return fail(WG_E_INVALID, "NULL argument");
  *out = nullptr;
  WG_TRY(ensure_device(parent));
  return ctx_make(parent->device, parent->ledger.budget(), &parent->ledger, parent->pinned_spill_bytes, out);
}

wg_status wg_ctx_destroy(wg_ctx* c) {
  if (!c) return WG_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->copy_stream) cudaStreamSynchronize(c->copy_stream);
  for (int i = 0; i < 2; ++i) {
    if (c->staged[i]) cudaEventDestroy(c->staged[i]);
    if (c->consumed[i]) cudaEventDestroy(c->consumed[i]);
    if (c->h2d_done[i]) cudaEventDestroy(c->h2d_done[i]);
    c->win[i].reset();
  }
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->host_scalar) cudaFreeHost(c->host_scalar);
  if (c->dev_scalar) cudaFree(c->dev_scalar);
  if (c->dev_error) cudaFree(c->dev_error);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  delete c;
  return WG_OK;
}

wg_status wg_ctx_synchronize(wg_ctx* c) {
  if (!c) return fail(WG_E_INVALID, "ctx is NULL");
  WG_TRY(ensure_device(c));
  WG_CUDA_TRY(cudaStreamSynchronize(c->stream));
  return check_device_error(c);
}

wg_status wg_ledger_stats(wg_ctx* c, int64_t* used, int64_t* peak, int64_t* budget) {
  if (!c) return fail(WG_E_INVALID, "ctx is NULL");
  if (used) *used = c->ledger.used();
  if (peak) *peak = c->ledger.peak();
  if (budget) *budget = c->ledger.budget();
  return WG_OK;
}

wg_status wg_ledger_reserve(wg_ctx* c, int64_t bytes) {
  if (!c || bytes < 0) return fail(WG_E_INVALID, "bad ledger reservation");
  if (!c->ledger.reserve(bytes)) return fail(WG_E_NOMEM, "HBM ledger: memory budget exceeded");
  return WG_OK;
}

wg_status wg_ledger_release(wg_ctx* c, int64_t bytes) {
  if (!c || bytes < 0) return fail(WG_E_INVALID, "bad ledger release");
  c->ledger.release(bytes);
  return WG_OK;
}

void* wg_ctx_stream(wg_ctx* c) { return c ? (void*)c->stream : nullptr; }

int64_t wg_ctx_launch_count(wg_ctx* c) { return c ? c->launches.load() : 0; }

}  // extern "C"
