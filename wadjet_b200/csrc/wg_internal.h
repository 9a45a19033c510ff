// wg_internal.h — host-side internals shared by the libwadjetgpu.so sources:
// the context (device, stream, pinned staging), the HBM ledger, thread-local
// errors and the device-buffer RAII type that charges the ledger.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/wadjet_gpu.h"

namespace wg {

// ---- errors ----------------------------------------------------------------
void set_error(const std::string& msg);
wg_status fail(wg_status code, const std::string& msg);

#define WG_CUDA_TRY(expr)                                                                   \
  do {                                                                                      \
    cudaError_t e__ = (expr);                                                               \
    if (e__ != cudaSuccess)                                                                 \
      return ::wg::fail(WG_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__));    \
  } while (0)

#define WG_TRY(expr)                      \
  do {                                    \
    wg_status s__ = (expr);               \
    if (s__ != WG_OK) return s__;         \
  } while (0)

// ---- HBM ledger (memory.Tracker, internal/engine/memory/tracker.go:19-160) ----
// Lock-free Reserve with rollback; Peak is the high-water mark of Used. A child
// ledger (Tracker.Child, tracker.go:44) shares its parent's budget: a
// reservation must fit both, and releases bubble up.
class Ledger {
 public:
  explicit Ledger(int64_t budget, Ledger* parent = nullptr) : budget_(budget), parent_(parent) {}
  bool reserve(int64_t n) {
    int64_t now = used_.fetch_add(n) + n;
    if (budget_ > 0 && now > budget_) {
      used_.fetch_sub(n);
      return false;
    }
    if (parent_ && !parent_->reserve(n)) {
      used_.fetch_sub(n);
      return false;
    }
    bump_peak(now);
    return true;
  }
  void release(int64_t n) {
    used_.fetch_sub(n);
    if (parent_) parent_->release(n);
  }
  Ledger* parent() const { return parent_; }
  int64_t used() const { return used_.load(); }
  int64_t peak() const { return peak_.load(); }
  int64_t budget() const { return budget_; }

 private:
  void bump_peak(int64_t v) {
    int64_t p = peak_.load();
    while (v > p && !peak_.compare_exchange_weak(p, v)) {}
  }
  int64_t budget_;
  Ledger* parent_;
  std::atomic<int64_t> used_{0};
  std::atomic<int64_t> peak_{0};
};

struct Ctx;

// Device buffer charged to a context's ledger; freed and released on reset.
class DevBuf {
 public:
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept { *this = std::move(o); }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      reset();
      ctx_ = o.ctx_; ptr_ = o.ptr_; bytes_ = o.bytes_;
      o.ctx_ = nullptr; o.ptr_ = nullptr; o.bytes_ = 0;
    }
    return *this;
  }
  ~DevBuf() { reset(); }
  wg_status alloc(Ctx* ctx, int64_t bytes);    // reserve + cudaMalloc (256 B aligned)
  wg_status ensure(Ctx* ctx, int64_t bytes);   // grow (contents discarded) if smaller
  void reset();
  void* get() const { return ptr_; }
  template <typename T> T* as() const { return static_cast<T*>(ptr_); }
  int64_t bytes() const { return bytes_; }

 private:
  Ctx* ctx_ = nullptr;
  void* ptr_ = nullptr;
  int64_t bytes_ = 0;
};

// ---- context ---------------------------------------------------------------
struct Ctx {
  int device = 0;
  int sm_count = 148;
  int max_smem_optin = 227 * 1024;
  int smem_per_sm = 228 * 1024;
  cudaStream_t stream = nullptr;      // compute stream
  cudaStream_t copy_stream = nullptr; // host→device staging stream
  Ledger ledger{0};
  int64_t pinned_spill_bytes = 0;
  std::atomic<int64_t> launches{0};
  // pinned staging ring for host batches (two halves, ping-pong)
  void* pinned = nullptr;
  int64_t pinned_bytes = 0;
  cudaEvent_t staged[2] = {nullptr, nullptr};
  cudaEvent_t consumed[2] = {nullptr, nullptr};
  // small pinned/device scalars for read-backs
  int64_t* host_scalar = nullptr;   // pinned, 64 slots
  int64_t* dev_scalar = nullptr;    // device, 64 slots
  // device-side error word written by bounded waits / invariants
  int32_t* dev_error = nullptr;
  std::mutex mu;                    // serialises scalar read-backs
  // host-input pipeline runs: two device windows and (for pageable sources) two
  // pinned slots the host threads fill, kept for the next run; one run at a time
  std::mutex stage_mu;
  DevBuf win[2];
  cudaEvent_t h2d_done[2] = {nullptr, nullptr};

  explicit Ctx(int64_t budget, Ledger* parent = nullptr) : ledger(budget, parent) {}
  void count_launch(int n = 1) { launches.fetch_add(n); }
};

// Copy `bytes` from src to dst with the library's host threads (a pool shared by
// every context, sized to the host's cores): the pageable-to-pinned leg of
// host-input staging.
void parallel_copy(void* dst, const void* src, int64_t bytes);

wg_status ensure_device(Ctx* ctx);           // cudaSetDevice(ctx->device)
wg_status read_back_i64(Ctx* ctx, const int64_t* dev, int64_t* out, int n);
wg_status check_device_error(Ctx* ctx);      // reads and clears dev_error
// read_back_i64 and check_device_error with one wait: n values (n < 63) and
// the error word, which fails the call when set
wg_status read_back_checked(Ctx* ctx, const int64_t* dev, int64_t* out, int n);

// Copy a host column/bitmap into a device buffer (synchronous on ctx->stream).
int64_t elem_size(int32_t type_id);          // 4 / 8 / 16, or 0 when unsupported
int class_of(int32_t type_id);               // see WG_CLS_* in wg_device.cuh

// Device copy of a host batch: every column staged, selection vector staged.
struct StagedBatch {
  std::vector<DevBuf> data, valid;
  DevBuf sel;
  std::vector<wg_column> cols;
  wg_batch_desc desc{};
};
wg_status stage_batch(Ctx* ctx, const wg_batch_desc* in, StagedBatch* out);

// String GROUP BY keys (wg_strkey.cu): a device dictionary from each distinct
// string to a dense id. strdict_map maps column `col` of `in` (its string
// column in host memory when `host`, else on the device) and sets *out to an
// INT32 column of the ids on the device, with the string column's validity.
struct StrDict;
wg_status strdict_map(Ctx* ctx, StrDict** d, const wg_batch_desc* in, int col, bool host, int64_t hint, wg_column* out);
wg_status strdict_strings(Ctx* ctx, StrDict* d, const int64_t* ids, int64_t n, uint32_t* out_offsets,
                          uint8_t* out_bytes, int64_t bytes_cap, int64_t* need_bytes);
void strdict_reset(StrDict* d, Ctx* ctx);
void strdict_free(StrDict* d);
int64_t strdict_size(const StrDict* d);

}  // namespace wg

// Opaque handle bodies live in their .cu files; only the context is shared.
struct wg_ctx : wg::Ctx {
  explicit wg_ctx(int64_t budget, wg::Ledger* parent = nullptr) : wg::Ctx(budget, parent) {}
};
