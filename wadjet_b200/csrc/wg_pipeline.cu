// wg_pipeline.cu — Pipeline.Run (internal/engine/exec/pipeline.go:81) for the
// filter → hash-join probe → project → hash-aggregate chain as one kernel per
// input window.
//
// Device-resident input runs directly. Host input is fed in windows of up to
// 2^24 rows through two device buffers: the copy of window i+1 (copy stream)
// overlaps the kernel over window i (compute stream), ordered by events —
// the GPU form of the scan source pushing decoded batches down a channel to
// the pipeline workers (planner/physical/plan.go:11096-11115).
#include "wg_internal.h"

namespace wg {
wg_status agg_run_device(wg_agg* a, const wg_batch_desc* in, int32_t nf, const wg_predicate* f, wg_join* j, int32_t ne,
                         const wg_expr* e);
Ctx* agg_ctx(wg_agg* a);
}  // namespace wg

using namespace wg;

namespace {

constexpr int64_t kWindowRows = 1LL << 24;

struct Window {
  std::vector<DevBuf> data, valid;
  std::vector<wg_column> cols;
};

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
  if (in->sel) {
    // a selected host batch is staged whole
    StagedBatch sb;
    WG_TRY(stage_batch(ctx, in, &sb));
    WG_TRY(agg_run_device(p->agg, &sb.desc, p->n_filters, p->filters, p->join, p->n_exprs, p->exprs));
    WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return WG_OK;
  }
  const int ncols = in->ncols;
  std::vector<bool> need = referenced(p, ncols, 0);
  if (p->join) { int pk = join_probe_key_col(p->join); if (pk >= 0 && pk < ncols) need[pk] = true; }
  for (int32_t c : agg_input_cols(p->agg)) if (c >= 0 && c < ncols) need[c] = true;
  const int64_t n = in->len;
  const int64_t win = std::min<int64_t>(kWindowRows, std::max<int64_t>(n, 64));
  Window w[2];
  for (int s = 0; s < 2; ++s) {
    w[s].data.resize((size_t)ncols);
    w[s].valid.resize((size_t)ncols);
    w[s].cols.assign(in->cols, in->cols + ncols);
    for (int c = 0; c < ncols; ++c) {
      const int64_t es = elem_size(in->cols[c].type_id);
      if (!need[c] || es == 0) { w[s].cols[c].data = nullptr; w[s].cols[c].valid_words = nullptr; continue; }
      WG_TRY(w[s].data[c].alloc(ctx, win * es));
      w[s].cols[c].data = w[s].data[c].get();
      if (in->cols[c].valid_words) {
        WG_TRY(w[s].valid[c].alloc(ctx, ((win + 63) / 64) * 8));
        w[s].cols[c].valid_words = w[s].valid[c].as<uint64_t>();
      }
    }
  }
  const int64_t nwin = (n + win - 1) / win;
  // both streams start after anything already queued on the compute stream
  WG_CUDA_TRY(cudaEventRecord(ctx->consumed[0], ctx->stream));
  WG_CUDA_TRY(cudaEventRecord(ctx->consumed[1], ctx->stream));
  auto issue_copy = [&](int64_t wi) -> wg_status {
    const int s = (int)(wi & 1);
    const int64_t r0 = wi * win;
    const int64_t m = std::min<int64_t>(win, n - r0);
    WG_CUDA_TRY(cudaStreamWaitEvent(ctx->copy_stream, ctx->consumed[s], 0));
    for (int c = 0; c < ncols; ++c) {
      if (!w[s].cols[c].data) continue;
      const int64_t es = elem_size(in->cols[c].type_id);
      WG_CUDA_TRY(cudaMemcpyAsync(w[s].data[c].get(), (const char*)in->cols[c].data + r0 * es, (size_t)(m * es),
                                  cudaMemcpyHostToDevice, ctx->copy_stream));
      if (in->cols[c].valid_words)
        WG_CUDA_TRY(cudaMemcpyAsync(w[s].valid[c].get(), in->cols[c].valid_words + (r0 >> 6),
                                    (size_t)(((m + 63) / 64) * 8), cudaMemcpyHostToDevice, ctx->copy_stream));
    }
    WG_CUDA_TRY(cudaEventRecord(ctx->staged[s], ctx->copy_stream));
    return WG_OK;
  };
  if (nwin > 0) WG_TRY(issue_copy(0));
  for (int64_t wi = 0; wi < nwin; ++wi) {
    const int s = (int)(wi & 1);
    const int64_t r0 = wi * win;
    const int64_t m = std::min<int64_t>(win, n - r0);
    if (wi + 1 < nwin) WG_TRY(issue_copy(wi + 1));
    WG_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, ctx->staged[s], 0));
    wg_batch_desc d{ncols, 0, w[s].cols.data(), m, nullptr, 0};
    wg_status st = agg_run_device(p->agg, &d, p->n_filters, p->filters, p->join, p->n_exprs, p->exprs);
    if (st != WG_OK) {
      cudaStreamSynchronize(ctx->copy_stream);
      cudaStreamSynchronize(ctx->stream);
      return st;
    }
    WG_CUDA_TRY(cudaEventRecord(ctx->consumed[s], ctx->stream));
  }
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->copy_stream));
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return check_device_error(ctx);
}

}  // extern "C"
