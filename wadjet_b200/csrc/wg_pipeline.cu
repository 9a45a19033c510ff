// wg_pipeline.cu — Pipeline.Run (internal/engine/exec/pipeline.go:81) for the
// filter → hash-join probe → project → hash-aggregate chain as one kernel per
// input window.
//
// Device-resident input runs directly. Host input is fed in windows through
// two device buffers kept on the context: the copy of window i+1 (copy stream)
// overlaps the kernel over window i (compute stream), ordered by events — the
// GPU form of the scan source pushing decoded batches down a channel to the
// pipeline workers (planner/physical/plan.go:11096-11115). Pageable sources
// are first copied into pinned slots by host threads, which then overlap both.
#include "wg_internal.h"

#include <cstdlib>

namespace wg {
wg_status agg_run_device(wg_agg* a, const wg_batch_desc* in, int32_t nf, const wg_predicate* f, wg_join* j, int32_t ne,
                         const wg_expr* e, bool defer_check = false, bool str_ids = false);
Ctx* agg_ctx(wg_agg* a);
int agg_str_key_col(wg_agg* a, const wg_batch_desc* in);
wg_status agg_map_str_key(wg_agg* a, const wg_batch_desc* in, int col, bool host, wg_column* out);
}  // namespace wg

using namespace wg;

namespace {

constexpr int64_t kWindowRows = 1LL << 24;


// Which input columns the pipeline reads (others are not copied).
std::vector<bool> referenced(const wg_pipeline_desc* p, int ncols, int npay_base) {
  std::vector<bool> r((size_t)ncols, false);
  auto mark = [&](int c) { if (c >= 0 && c < ncols) r[c] = true; };
  for (int f = 0; f < p->n_filters; ++f) mark(p->filters[f].col);
  for (int e = 0; e < p->n_exprs; ++e)
    for (int k = 0; k < p->exprs[e].n_ops && k < WG_EXPR_MAX_OPS; ++k)
      if (p->exprs[e].ops[k].opcode == WG_EXPR_COL) mark(p->exprs[e].ops[k].arg);
  (void)npay_base;
  return r;
}

}  // namespace

namespace wg {
int32_t join_probe_key_col(wg_join* j);
std::vector<int32_t> agg_input_cols(wg_agg* a);
}  // namespace wg

extern "C" {

wg_status wg_pipeline_run_device(wg_ctx* ctx, const wg_pipeline_desc* p) {
  if (!ctx || !p || !p->input || !p->agg) return fail(WG_E_INVALID, "NULL argument");
  if (agg_ctx(p->agg) != ctx) return fail(WG_E_INVALID, "aggregate belongs to another context");
  WG_TRY(ensure_device(ctx));
  return agg_run_device(p->agg, p->input, p->n_filters, p->filters, p->join, p->n_exprs, p->exprs);
}

wg_status wg_pipeline_run(wg_ctx* ctx, const wg_pipeline_desc* p) {
  if (!ctx || !p || !p->input || !p->agg) return fail(WG_E_INVALID, "NULL argument");
  if (agg_ctx(p->agg) != ctx) return fail(WG_E_INVALID, "aggregate belongs to another context");
  WG_TRY(ensure_device(ctx));
  const wg_batch_desc* in = p->input;
  if (in->ncols < 0 || (in->ncols > 0 && !in->cols)) return fail(WG_E_INVALID, "bad batch descriptor");
  const int sk = agg_str_key_col(p->agg, in);
  if (in->sel || sk >= 0) {
    // a selected host batch is staged whole, and so is one grouped by a string
    // column (its dictionary maps the column before the fused launch)
    StagedBatch sb;
    WG_TRY(stage_batch(ctx, in, &sb));
    if (sk >= 0) WG_TRY(agg_map_str_key(p->agg, in, sk, true, &sb.cols[(size_t)sk]));
    WG_TRY(agg_run_device(p->agg, &sb.desc, p->n_filters, p->filters, p->join, p->n_exprs, p->exprs, false, sk >= 0));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return WG_OK;
  }
  const int ncols = in->ncols;
  std::vector<bool> need = referenced(p, ncols, 0);
  if (p->join) { int pk = join_probe_key_col(p->join); if (pk >= 0 && pk < ncols) need[pk] = true; }
  for (int32_t c : agg_input_cols(p->agg)) if (c >= 0 && c < ncols) need[c] = true;
  const int64_t n = in->len;
  // Pageable source columns (ordinary host memory, as a cgo caller's Go slices
  // are) go through pinned slots the library's host threads fill, so the DMA
  // engine reads pinned memory at full speed while the threads copy the next
  // window; pinned sources are copied by DMA directly.
  bool pageable = false;
  int64_t row_bytes = 0;
  for (int c = 0; c < ncols; ++c) {
    if (!need[c] || elem_size(in->cols[c].type_id) == 0) continue;
    row_bytes += elem_size(in->cols[c].type_id) + (in->cols[c].valid_words ? 1 : 0);
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, in->cols[c].data) != cudaSuccess) { cudaGetLastError(); pageable = true; }
    else if (at.type == cudaMemoryTypeUnregistered) pageable = true;
  }
  // windows of rows: a multiple of 64 (validity words stay whole); pageable
  // sources take smaller windows so the pinned slots stay modest
  const int64_t stage_mb = std::max<int64_t>(1, std::getenv("WG_STAGE_WINDOW_MB") ? std::atoll(std::getenv("WG_STAGE_WINDOW_MB")) : 64);
  const int64_t max_win = pageable ? std::max<int64_t>(1 << 16, ((stage_mb << 20) / std::max<int64_t>(row_bytes, 1)) & ~int64_t(63))
                                   : kWindowRows;
  const int64_t win = std::min<int64_t>(max_win, std::max<int64_t>((n + 63) & ~int64_t(63), 64));
  // one host-input run at a time per context: it owns the context's windows
  std::lock_guard<std::mutex> stage_lock(ctx->stage_mu);
  // per window: each referenced column's data, then its validity words, at
  // 256-byte aligned offsets of one device (and one pinned) slot
  std::vector<int64_t> off_data((size_t)ncols, -1), off_valid((size_t)ncols, -1);
  int64_t slot_bytes = 0;
  for (int c = 0; c < ncols; ++c) {
    const int64_t es = elem_size(in->cols[c].type_id);
    if (!need[c] || es == 0) continue;
    off_data[(size_t)c] = slot_bytes;
    slot_bytes += (win * es + 255) & ~int64_t(255);
    if (in->cols[c].valid_words) {
      off_valid[(size_t)c] = slot_bytes;
      slot_bytes += ((win / 64 + 1) * 8 + 255) & ~int64_t(255);
    }
  }
  slot_bytes = std::max<int64_t>(slot_bytes, 256);
  for (int s = 0; s < 2; ++s) WG_TRY(ctx->win[s].ensure(ctx, slot_bytes));
  if (pageable && ctx->pinned_bytes < 2 * slot_bytes) {
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    WG_CUDA_TRY(cudaHostAlloc(&ctx->pinned, (size_t)(2 * slot_bytes), cudaHostAllocDefault));
    ctx->pinned_bytes = 2 * slot_bytes;
  }
  std::vector<wg_column> cols[2];
  for (int s = 0; s < 2; ++s) {
    cols[s].assign(in->cols, in->cols + ncols);
    for (int c = 0; c < ncols; ++c) {
      if (off_data[(size_t)c] < 0) { cols[s][c].data = nullptr; cols[s][c].valid_words = nullptr; continue; }
      cols[s][c].data = ctx->win[s].as<char>() + off_data[(size_t)c];
      cols[s][c].valid_words = off_valid[(size_t)c] >= 0 ? (const uint64_t*)(ctx->win[s].as<char>() + off_valid[(size_t)c])
                                                        : nullptr;
    }
  }
  const int64_t nwin = (n + win - 1) / win;
  // both streams start after anything already queued on the compute stream;
  // the pinned slots are free
  WG_CUDA_TRY(cudaEventRecord(ctx->consumed[0], ctx->stream));
  WG_CUDA_TRY(cudaEventRecord(ctx->consumed[1], ctx->stream));
  WG_CUDA_TRY(cudaEventRecord(ctx->h2d_done[0], ctx->copy_stream));
  WG_CUDA_TRY(cudaEventRecord(ctx->h2d_done[1], ctx->copy_stream));
  auto issue_copy = [&](int64_t wi) -> wg_status {
    const int s = (int)(wi & 1);
    const int64_t r0 = wi * win;
    const int64_t m = std::min<int64_t>(win, n - r0);
    char* pin = (char*)ctx->pinned + (size_t)s * (size_t)slot_bytes;
    if (pageable) {
      // the slot's previous copy to the device has finished before the threads refill it
      WG_CUDA_TRY(cudaEventSynchronize(ctx->h2d_done[s]));
      for (int c = 0; c < ncols; ++c) {
        if (off_data[(size_t)c] < 0) continue;
        const int64_t es = elem_size(in->cols[c].type_id);
        parallel_copy(pin + off_data[(size_t)c], (const char*)in->cols[c].data + r0 * es, m * es);
        if (off_valid[(size_t)c] >= 0)
          std::memcpy(pin + off_valid[(size_t)c], in->cols[c].valid_words + (r0 >> 6), (size_t)(((m + 63) / 64) * 8));
      }
    }
    WG_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->consumed[s], 0));
    for (int c = 0; c < ncols; ++c) {
      if (off_data[(size_t)c] < 0) continue;
      const int64_t es = elem_size(in->cols[c].type_id);
      const void* src = pageable ? (const void*)(pin + off_data[(size_t)c]) : (const char*)in->cols[c].data + r0 * es;
      WG_CUDA_TRY(cudaMemcpyAsync(ctx->win[s].as<char>() + off_data[(size_t)c], src, (size_t)(m * es),
                                  cudaMemcpyHostToDevice, ctx->copy_stream));
      if (off_valid[(size_t)c] >= 0) {
        const void* vs = pageable ? (const void*)(pin + off_valid[(size_t)c]) : (const void*)(in->cols[c].valid_words + (r0 >> 6));
        WG_CUDA_TRY(cudaMemcpyAsync(ctx->win[s].as<char>() + off_valid[(size_t)c], vs, (size_t)(((m + 63) / 64) * 8),
                                    cudaMemcpyHostToDevice, ctx->copy_stream));
      }
    }
    WG_CUDA_TRY(cudaEventRecord(ctx->staged[s], ctx->copy_stream));
    WG_CUDA_TRY(cudaEventRecord(ctx->h2d_done[s], ctx->copy_stream));
    return WG_OK;
  };
  auto drain = [&]() {
    cudaStreamSynchronize(ctx->copy_stream);
    cudaStreamSynchronize(ctx->stream);
  };
  if (nwin > 0) {
    wg_status st = issue_copy(0);
    if (st != WG_OK) { drain(); return st; }
  }
  for (int64_t wi = 0; wi < nwin; ++wi) {
    const int s = (int)(wi & 1);
    const int64_t r0 = wi * win;
    const int64_t m = std::min<int64_t>(win, n - r0);
    WG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->staged[s], 0));
    wg_batch_desc d{ncols, 0, cols[s].data(), m, nullptr, 0};
    for (int c = 0; c < ncols; ++c) cols[s][c].len = m;
    wg_status st = agg_run_device(p->agg, &d, p->n_filters, p->filters, p->join, p->n_exprs, p->exprs, true);
    if (st != WG_OK) { drain(); return st; }
    WG_CUDA_TRY(cudaEventRecord(ctx->consumed[s], ctx->stream));
    // the next window's host copy overlaps this window's kernel
    if (wi + 1 < nwin) {
      st = issue_copy(wi + 1);
      if (st != WG_OK) { drain(); return st; }
    }
  }
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

}  // extern "C"
