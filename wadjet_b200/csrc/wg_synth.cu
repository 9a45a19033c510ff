// wg_synth.cu — the benchmark tables of include/wadjet_synth.h generated in HBM,
// one thread per row, bit-identical to the host generator of the same header.
#include "wg_internal.h"
#include "../../include/wadjet_synth.h"

namespace {

__global__ void starjoin_fact_kernel(uint64_t seed, int64_t row0, int64_t n, const double* cdf, int32_t* fk,
                                     int32_t* qty, wg_int128* price, double* disc) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r = (uint64_t)(row0 + i);
    if (fk) fk[i] = wg_syn_sj_fk(seed, r, cdf, WG_SYN_SJ_DIM_BITS);
    if (qty) qty[i] = wg_syn_sj_qty(seed, r);
    if (price) { wg_int128 p; p.hi = 0; p.lo = (uint64_t)wg_syn_sj_price(seed, r); price[i] = p; }
    if (disc) disc[i] = wg_syn_sj_disc(seed, r);
  }
}

__global__ void starjoin_dim_kernel(uint64_t seed, int64_t n, int32_t* key, int32_t* grp) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (key) key[i] = wg_syn_sj_dim_key((uint64_t)i, WG_SYN_SJ_DIM_BITS);
    if (grp) grp[i] = wg_syn_sj_grp(seed, (uint64_t)i);
  }
}

__global__ void groupby_kernel(uint64_t seed, int64_t row0, int64_t n, int64_t ngroups, int64_t* k, int64_t* v,
                               double* f, int32_t* flag) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r = (uint64_t)(row0 + i);
    if (k) k[i] = wg_syn_gb_k(seed, r, ngroups);
    if (v) v[i] = wg_syn_gb_v(seed, r);
    if (f) f[i] = wg_syn_gb_f(seed, r);
    if (flag) flag[i] = wg_syn_gb_flag(seed, r);
  }
}

__global__ void highcard_kernel(uint64_t seed, int64_t row0, int64_t n, int32_t* a, int64_t* b, wg_int128* amt,
                                double* x) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t r = (uint64_t)(row0 + i);
    const int64_t bv = wg_syn_hc_b(seed, r, WG_SYN_HC_B_BITS);
    if (b) b[i] = bv;
    if (a) a[i] = wg_syn_hc_a(bv);
    if (amt) { const int64_t v = wg_syn_hc_amt(seed, r); wg_int128 d; d.hi = v < 0 ? -1 : 0; d.lo = (uint64_t)v; amt[i] = d; }
    if (x) x[i] = wg_syn_hc_x(seed, r);
  }
}

__global__ void batched_query_kernel(uint64_t seed, int64_t n, int64_t card, int64_t* key, int64_t* vi, double* vf,
                                     int32_t* filt) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (key) key[i] = wg_syn_bq_key(seed, (uint64_t)i, card);
    if (vi) vi[i] = wg_syn_bq_vi(seed, (uint64_t)i);
    if (vf) vf[i] = wg_syn_bq_vf(seed, (uint64_t)i);
    if (filt) filt[i] = wg_syn_bq_filt(seed, (uint64_t)i);
  }
}

unsigned synth_grid(wg::Ctx* ctx, int64_t n) {
  int64_t b = (n + 255) / 256;
  return (unsigned)std::max<int64_t>(1, std::min<int64_t>(b, (int64_t)ctx->sm_count * 32));
}

// The Zipf(1.1) CDF over the 2^22 dimension keys, built once per process on the
// host with the header's function and kept on each device that asks for it.
struct ZipfTable {
  std::mutex mu;
  std::vector<double> host;
  std::vector<std::pair<int, wg::DevBuf*>> dev;
};
ZipfTable g_zipf;

wg_status zipf_cdf_device(wg::Ctx* ctx, const double** out) {
  std::lock_guard<std::mutex> g(g_zipf.mu);
  if (g_zipf.host.empty()) {
    g_zipf.host.resize((size_t)1 << WG_SYN_SJ_DIM_BITS);
    wg_syn_zipf_cdf(g_zipf.host.data(), (int64_t)g_zipf.host.size(), WG_SYN_SJ_ZIPF_S);
  }
  for (auto& e : g_zipf.dev)
    if (e.first == ctx->device) { *out = e.second->as<double>(); return WG_OK; }
  auto* buf = new wg::DevBuf();
  WG_TRY(buf->alloc(ctx, (int64_t)g_zipf.host.size() * 8));
  WG_CUDA_TRY(cudaMemcpy(buf->get(), g_zipf.host.data(), g_zipf.host.size() * 8, cudaMemcpyHostToDevice));
  g_zipf.dev.push_back({ctx->device, buf});  // lives for the process: shared by every context on the device
  *out = buf->as<double>();
  return WG_OK;
}

}  // namespace

using namespace wg;

extern "C" {

wg_status wg_synth_starjoin_fact(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int32_t* fk, int32_t* qty,
                                 wg_int128* price, double* disc) {
  if (!ctx || n < 0) return fail(WG_E_INVALID, "bad generator arguments");
  WG_TRY(ensure_device(ctx));
  const double* cdf = nullptr;
  if (fk) WG_TRY(zipf_cdf_device(ctx, &cdf));
  if (n == 0) return WG_OK;
  starjoin_fact_kernel<<<synth_grid(ctx, n), 256, 0, ctx->stream>>>(seed, row0, n, cdf, fk, qty, price, disc);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

wg_status wg_synth_starjoin_dim(wg_ctx* ctx, uint64_t seed, int64_t n, int32_t* key, int32_t* grp) {
  if (!ctx || n < 0) return fail(WG_E_INVALID, "bad generator arguments");
  WG_TRY(ensure_device(ctx));
  if (n == 0) return WG_OK;
  starjoin_dim_kernel<<<synth_grid(ctx, n), 256, 0, ctx->stream>>>(seed, n, key, grp);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

wg_status wg_synth_groupby(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int64_t ngroups, int64_t* k,
                           int64_t* v, double* f, int32_t* flag) {
  if (!ctx || n < 0 || ngroups < 1) return fail(WG_E_INVALID, "bad generator arguments");
  WG_TRY(ensure_device(ctx));
  if (n == 0) return WG_OK;
  groupby_kernel<<<synth_grid(ctx, n), 256, 0, ctx->stream>>>(seed, row0, n, ngroups, k, v, f, flag);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

wg_status wg_synth_highcard(wg_ctx* ctx, uint64_t seed, int64_t row0, int64_t n, int32_t* a, int64_t* b,
                            wg_int128* amt, double* x) {
  if (!ctx || n < 0) return fail(WG_E_INVALID, "bad generator arguments");
  WG_TRY(ensure_device(ctx));
  if (n == 0) return WG_OK;
  highcard_kernel<<<synth_grid(ctx, n), 256, 0, ctx->stream>>>(seed, row0, n, a, b, amt, x);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

wg_status wg_synth_batched_params(uint64_t seed, int32_t q, int64_t* rows, int64_t* card, int32_t* threshold) {
  if (!rows || !card || !threshold || q < 0) return fail(WG_E_INVALID, "bad generator arguments");
  wg_syn_bq_params(seed, (uint32_t)q, rows, card, threshold);
  return WG_OK;
}

wg_status wg_synth_batched(wg_ctx* ctx, uint64_t seed, int32_t q, int64_t n, int64_t card, int64_t* key, int64_t* vi,
                           double* vf, int32_t* filt) {
  if (!ctx || n < 0 || card < 1 || q < 0) return fail(WG_E_INVALID, "bad generator arguments");
  WG_TRY(ensure_device(ctx));
  if (n == 0) return WG_OK;
  batched_query_kernel<<<synth_grid(ctx, n), 256, 0, ctx->stream>>>(seed + (uint64_t)q, n, card, key, vi, vf, filt);
  ctx->count_launch();
  WG_CUDA_TRY(cudaGetLastError());
  WG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return WG_OK;
}

}  // extern "C"
