// wg_serve.cu — the serving loop: continuous batching of filter → join →
// aggregate requests over device-resident tables.
//
// n_slots worker threads each own a child context (own streams, a child ledger
// sharing the server context's budget). A request is admitted when a slot is
// free, the requests already on the device stream fewer input bytes than the
// work limit (256 MB; WG_SERVE_WORK_LIMIT_MB) together with it, and the shared
// ledger can hold its estimated HBM footprint. A request larger than the limit
// runs alone (one such request already fills the GPU; sharing it only slows
// both); small ones overlap, which is where concurrency pays. Admission is
// first-come first-served, so a large request waits at the head of the queue
// rather than being overtaken forever.
// Results stay on the device until the caller releases them.
#include "wg_internal.h"

#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

using namespace wg;

namespace wg {
void agg_trim(wg_agg* a);  // wg_agg.cu
}  // namespace wg

namespace {

double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Req {
  int64_t ticket = 0;
  wg_batch_desc input{};
  std::vector<wg_column> cols;
  std::vector<wg_predicate> filters;
  std::vector<wg_expr> exprs;
  wg_join* join = nullptr;
  std::vector<int32_t> keys;
  std::vector<wg_agg_spec> aggs;
  int64_t hint = 0;
  int64_t est = 0;
  int64_t work = 0;   // input bytes the request streams
  double t_submit = 0, t_start = 0, t_done = 0;
  wg_agg* agg = nullptr;
  wg_ctx* slot = nullptr;
  int64_t n_groups = 0;
  wg_status status = WG_OK;
  std::string err;
  bool done = false;
  bool held = false;
};

// A finished request's aggregate, kept on its slot for the next request of the
// same shape (its table and buffers stay resident; reuse is a reset).
struct Pooled {
  wg_agg* agg;
  wg_ctx* slot;
  std::vector<int32_t> keys;
  std::vector<wg_agg_spec> aggs;
  int64_t hint;
};

bool same_shape(const Pooled& p, const Req* r, wg_ctx* slot) {
  if (p.slot != slot || p.hint != r->hint || p.keys != r->keys || p.aggs.size() != r->aggs.size()) return false;
  for (size_t i = 0; i < p.aggs.size(); ++i)
    if (p.aggs[i].func != r->aggs[i].func || p.aggs[i].input_col != r->aggs[i].input_col ||
        p.aggs[i].out_type != r->aggs[i].out_type)
      return false;
  return true;
}

}  // namespace

struct wg_server {
  wg_ctx* ctx = nullptr;
  std::vector<wg_ctx*> slots;
  std::vector<Pooled> pool;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Req*> queue;
  std::unordered_map<int64_t, Req*> reqs;
  int64_t next_ticket = 1;
  bool stop = false;
  int64_t submitted = 0, completed = 0, failed = 0, cancelled = 0, running = 0;
  // requests overlap on the device while their input bytes together stay under
  // work_limit; a request at least that large runs alone (it fills the GPU)
  int64_t inflight_work = 0, work_limit = int64_t(256) << 20;
  std::vector<double> lat;
  double queue_sum = 0, service_sum = 0;
  double t_first = -1, t_last = 0;
};

namespace {

void run_request(wg_server* s, wg_ctx* slot, Req* r) {
  r->slot = slot;
  wg_status st = WG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (size_t i = 0; i < s->pool.size(); ++i)
      if (same_shape(s->pool[i], r, slot)) {
        r->agg = s->pool[i].agg;
        s->pool.erase(s->pool.begin() + (long)i);
        break;
      }
  }
  if (r->agg) st = wg_agg_reset(r->agg);
  else st = wg_agg_create(slot, (int32_t)r->keys.size(), r->keys.data(), (int32_t)r->aggs.size(), r->aggs.data(),
                          r->hint, &r->agg);
  if (st == WG_OK) {
    wg_pipeline_desc p{};
    p.input = &r->input;
    p.n_filters = (int32_t)r->filters.size();
    p.filters = r->filters.data();
    p.join = r->join;
    p.n_exprs = (int32_t)r->exprs.size();
    p.exprs = r->exprs.data();
    p.agg = r->agg;
    st = wg_pipeline_run_device(slot, &p);
  }
  if (st == WG_OK) st = wg_agg_finalize(r->agg, &r->n_groups);
  r->status = st;
  if (st != WG_OK) r->err = wg_last_error();
  (void)s;
}

void worker_main(wg_server* s, int slot_idx) {
  wg_ctx* slot = s->slots[(size_t)slot_idx];
  cudaSetDevice(slot->device);
  for (;;) {
    Req* r = nullptr;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      for (;;) {
        if (s->stop) return;
        if (!s->queue.empty()) {
          Req* head = s->queue.front();
          // admission: the device has room for more work (or is idle), and the
          // head request's footprint fits the shared ledger
          const bool room = s->running == 0 || s->inflight_work + head->work <= s->work_limit;
          if (room && s->ctx->ledger.reserve(head->est)) {
            head->held = true;
            s->queue.pop_front();
            r = head;
            ++s->running;
            s->inflight_work += r->work;
            break;
          }
          if (s->running == 0) {  // nothing will free memory: fail the request rather than wait forever
            s->queue.pop_front();
            head->status = WG_E_NOMEM;
            head->err = "request footprint exceeds the HBM budget";
            head->done = true;
            head->t_done = now_s();
            ++s->failed;
            s->cv_done.notify_all();
            continue;
          }
        }
        s->cv_work.wait(lk);
      }
    }
    r->t_start = now_s();
    run_request(s, slot, r);
    {
      std::lock_guard<std::mutex> lk(s->mu);
      r->t_done = now_s();
      r->done = true;
      --s->running;
      s->inflight_work -= r->work;
      if (r->status == WG_OK) {
        ++s->completed;
        s->lat.push_back(r->t_done - r->t_submit);
        s->queue_sum += r->t_start - r->t_submit;
        s->service_sum += r->t_done - r->t_start;
        s->t_last = std::max(s->t_last, r->t_done);
      } else {
        ++s->failed;
        if (r->agg) { wg_agg_destroy(r->agg); r->agg = nullptr; }
        if (r->held) { s->ctx->ledger.release(r->est); r->held = false; }
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
}

double percentile(std::vector<double> v, double p) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double idx = p * (double)(v.size() - 1);
  const size_t lo = (size_t)idx, hi = std::min(v.size() - 1, lo + 1);
  return v[lo] + (v[hi] - v[lo]) * (idx - (double)lo);
}

}  // namespace

extern "C" {

wg_status wg_server_create(wg_ctx* ctx, int32_t n_slots, wg_server** out) {
  if (!ctx || !out || n_slots < 1 || n_slots > 64) return fail(WG_E_INVALID, "bad server arguments");
  WG_TRY(ensure_device(ctx));
  wg_server* s = new wg_server();
  s->ctx = ctx;
  if (const char* w = std::getenv("WG_SERVE_WORK_LIMIT_MB")) s->work_limit = std::max<int64_t>(1, std::atoll(w)) << 20;
  for (int i = 0; i < n_slots; ++i) {
    wg_ctx* c = nullptr;
    wg_status st = wg_ctx_create_child(ctx, &c);
    if (st != WG_OK) {
      wg_server_destroy(s);
      return st;
    }
    s->slots.push_back(c);
  }
  for (int i = 0; i < n_slots; ++i) s->workers.emplace_back(worker_main, s, i);
  *out = s;
  return WG_OK;
}

wg_status wg_server_submit(wg_server* s, const wg_serve_request* q, int64_t* ticket) {
  if (!s || !q || !q->plan || !q->plan->input || !ticket) return fail(WG_E_INVALID, "NULL argument");
  const wg_pipeline_desc* p = q->plan;
  if (p->n_filters < 0 || p->n_exprs < 0 || q->n_keys < 0 || q->n_aggs < 0) return fail(WG_E_INVALID, "bad request");
  Req* r = new Req();
  r->input = *p->input;
  r->cols.assign(p->input->cols, p->input->cols + p->input->ncols);
  r->input.cols = r->cols.data();
  r->filters.assign(p->filters, p->filters + p->n_filters);
  r->exprs.assign(p->exprs, p->exprs + p->n_exprs);
  r->join = p->join;
  r->keys.assign(q->key_cols, q->key_cols + q->n_keys);
  r->aggs.assign(q->aggs, q->aggs + q->n_aggs);
  r->hint = q->ndv_hint;
  for (const wg_column& c : r->cols) r->work += c.len * wg::elem_size(c.type_id);
  r->est = q->est_bytes > 0 ? q->est_bytes : 128 * std::max<int64_t>(q->ndv_hint, 1024) + (16 << 20);
  r->t_submit = now_s();
  const int64_t budget = s->ctx->ledger.budget();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    r->ticket = s->next_ticket++;
    s->reqs[r->ticket] = r;
    ++s->submitted;
    if (s->t_first < 0) s->t_first = r->t_submit;
    if (budget > 0 && r->est > budget) {  // can never be admitted: refuse now
      r->status = WG_E_NOMEM;
      r->err = "request footprint exceeds the HBM budget";
      r->done = true;
      r->t_done = r->t_submit;
      ++s->failed;
    } else {
      s->queue.push_back(r);
    }
  }
  s->cv_work.notify_one();
  *ticket = r->ticket;
  return WG_OK;
}

wg_status wg_server_wait(wg_server* s, int64_t ticket, double timeout_s, int64_t* n_groups, double* latency_s) {
  if (!s) return fail(WG_E_INVALID, "server is NULL");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return fail(WG_E_INVALID, "unknown ticket");
  Req* r = it->second;
  auto ready = [&] { return r->done; };
  if (timeout_s < 0) s->cv_done.wait(lk, ready);
  else if (!s->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
    return fail(WG_E_TIMEOUT, "request not finished before the timeout");
  if (n_groups) *n_groups = r->n_groups;
  if (latency_s) *latency_s = r->t_done - r->t_submit;
  if (r->status != WG_OK) return fail(r->status, r->err);
  return WG_OK;
}

wg_status wg_server_export(wg_server* s, int64_t ticket, const wg_group_export* out) {
  if (!s || !out) return fail(WG_E_INVALID, "NULL argument");
  Req* r = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end() || !it->second->done) return fail(WG_E_STATE, "request unknown or not finished");
    r = it->second;
  }
  if (r->status != WG_OK || !r->agg) return fail(WG_E_STATE, "request failed");
  return wg_agg_export(r->agg, out);
}

wg_status wg_server_release(wg_server* s, int64_t ticket) {
  if (!s) return fail(WG_E_INVALID, "server is NULL");
  Req* r = nullptr;
  bool park = false;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(WG_E_INVALID, "unknown ticket");
    if (!it->second->done) return fail(WG_E_STATE, "request still running");
    r = it->second;
    s->reqs.erase(it);
    // keep enough finished aggregates that a slot rarely has to allocate a new
    // one while the previous result of the same shape is still held
    park = r->agg && r->status == WG_OK && s->pool.size() < 16 * s->slots.size();
  }
  // Trimming frees device memory (a device-wide synchronisation) and switches
  // this thread's current device, so it runs with the server lock released:
  // workers keep taking pooled aggregates and finishing requests meanwhile.
  if (park) {
    int prev_dev = -1;
    cudaGetDevice(&prev_dev);
    agg_trim(r->agg);  // a parked aggregate keeps its table, not its reorder copy
    if (prev_dev >= 0) cudaSetDevice(prev_dev);
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->pool.size() < 16 * s->slots.size()) {
      s->pool.push_back(Pooled{r->agg, r->slot, r->keys, r->aggs, r->hint});
      r->agg = nullptr;
    }
  }
  if (r->agg) wg_agg_destroy(r->agg);
  if (r->held) s->ctx->ledger.release(r->est);
  delete r;
  s->cv_work.notify_all();
  return WG_OK;
}

wg_status wg_server_cancel(wg_server* s, int64_t ticket) {
  if (!s) return fail(WG_E_INVALID, "server is NULL");
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail(WG_E_INVALID, "unknown ticket");
    Req* r = it->second;
    if (r->done) return fail(WG_E_STATE, "request already finished");
    auto q = std::find(s->queue.begin(), s->queue.end(), r);
    if (q == s->queue.end()) return fail(WG_E_STATE, "request already running");
    s->queue.erase(q);
    r->status = WG_E_CANCELLED;
    r->err = "request cancelled before it was admitted";
    r->done = true;
    r->t_done = now_s();
    ++s->cancelled;
  }
  s->cv_done.notify_all();
  s->cv_work.notify_all();
  return WG_OK;
}

wg_status wg_server_stats(wg_server* s, wg_serve_stats* o) {
  if (!s || !o) return fail(WG_E_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  o->submitted = s->submitted;
  o->completed = s->completed;
  o->failed = s->failed;
  o->cancelled = s->cancelled;
  o->in_flight = s->running;
  o->queued = (int64_t)s->queue.size();
  o->p50_s = percentile(s->lat, 0.50);
  o->p99_s = percentile(s->lat, 0.99);
  double sum = 0, mx = 0;
  for (double x : s->lat) { sum += x; mx = std::max(mx, x); }
  o->mean_s = s->lat.empty() ? 0.0 : sum / (double)s->lat.size();
  o->max_s = mx;
  o->qps = (s->completed > 0 && s->t_last > s->t_first) ? (double)s->completed / (s->t_last - s->t_first) : 0.0;
  o->mean_queue_s = s->lat.empty() ? 0.0 : s->queue_sum / (double)s->lat.size();
  o->mean_service_s = s->lat.empty() ? 0.0 : s->service_sum / (double)s->lat.size();
  return WG_OK;
}

wg_status wg_server_reset_stats(wg_server* s) {
  if (!s) return fail(WG_E_INVALID, "server is NULL");
  std::lock_guard<std::mutex> lk(s->mu);
  s->lat.clear();
  s->queue_sum = s->service_sum = 0;
  s->completed = s->failed = s->submitted = s->cancelled = 0;
  s->t_first = -1;
  s->t_last = 0;
  return WG_OK;
}

wg_status wg_server_destroy(wg_server* s) {
  if (!s) return WG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& t : s->workers) t.join();
  for (auto& kv : s->reqs) {
    if (kv.second->agg) wg_agg_destroy(kv.second->agg);
    if (kv.second->held) s->ctx->ledger.release(kv.second->est);
    delete kv.second;
  }
  for (Pooled& p : s->pool) wg_agg_destroy(p.agg);
  for (wg_ctx* c : s->slots) wg_ctx_destroy(c);
  delete s;
  return WG_OK;
}

}  // extern "C"
