// serve.cu — the serving loop: continuous batching of single-query requests over one index.
//
// The reference serves by calling ivf::Index::search from many threads, one query each
// (src/bin/search.rs:272-323). Here requests are queued by sg_server_submit and a dispatcher
// thread forms batches from whatever is pending whenever an execution context frees up:
//   - a context is a CUDA stream with its own device scratch (candidate buffers, work queues,
//     per-query state); `contexts` batches are in flight at once and overlap on the GPU;
//   - a batch takes pending requests with the same search params (each may carry its own
//     filter: the scans read a per-query allow table), as many as fit the context's share of the
//     HBM scratch budget and max_batch;
//   - inputs are staged through pinned host buffers, the pipeline is launched without a host
//     sync, results come back on the same stream, and a host callback on that stream wakes the
//     dispatcher when they land;
//   - a query whose candidate buffer filled up is run again alone with its exact bound, as
//     sg_search does, so every result equals the query's result alone.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "internal.hpp"

namespace {

using sg::fail;
using Clock = std::chrono::steady_clock;

#define SV_CK(call)                                                                    \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess)                                                             \
      return fail(SG_ERR_DEVICE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct Req {
  uint64_t ticket = 0;
  std::vector<float> q768, q256;
  bool have_q256 = false;
  sg_params p;
  const sg_filter* filter = nullptr;
  std::vector<float> sc;
  std::vector<uint32_t> id;
  uint32_t n = 0;
  int status = SG_OK;
  bool done = false;
  uint32_t batch = 0, retried = 0;
  Clock::time_point t_submit, t_launch, t_done;
};

struct Slot {
  sg_server* srv = nullptr;
  sg::Ctx ctx;
  uint32_t cap = 0;  // queries its pinned buffers hold
  float* h_q768 = nullptr;
  float* h_q256 = nullptr;
  float* h_sc = nullptr;
  uint32_t* h_id = nullptr;
  uint32_t* h_n = nullptr;
  uint8_t* h_ovf = nullptr;
  uint32_t* h_status = nullptr;
  const uint64_t** h_allow = nullptr;
  uint64_t* h_allow_w = nullptr;
  std::vector<std::shared_ptr<Req>> batch;
  sg_params p;
  sg::Config cfg;      // the index's tuning when the batch was formed (prepare, launch and retries)
  uint32_t limit = 0;  // largest batch of these params that fits the slot's scratch share
  bool have_q256 = false;
  bool busy = false;
  bool gpu_done = false;
};

}  // namespace

struct sg_server {
  sg_index* h = nullptr;
  sg_server_config cfg;
  std::vector<std::unique_ptr<Slot>> slots;
  std::deque<std::shared_ptr<Req>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<Req>> live;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::thread dispatcher;
  bool stopping = false;
  uint64_t next_ticket = 1;
  sg_server_stats st = {};
  int dispatcher_rc = SG_OK;
};

namespace {

void CUDART_CB on_batch_done(void* arg) {
  Slot* s = static_cast<Slot*>(arg);
  sg_server* srv = s->srv;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    s->gpu_done = true;
  }
  srv->cv_work.notify_all();
}

int slot_alloc(Slot& s, uint32_t cap, uint32_t kmax) {
  SV_CK(cudaMallocHost(&s.h_q768, (size_t)cap * SG_DIM * 4));
  SV_CK(cudaMallocHost(&s.h_q256, (size_t)cap * SG_PDIM * 4));
  SV_CK(cudaMallocHost(&s.h_sc, (size_t)cap * kmax * 4));
  SV_CK(cudaMallocHost(&s.h_id, (size_t)cap * kmax * 4));
  SV_CK(cudaMallocHost(&s.h_n, (size_t)cap * 4));
  SV_CK(cudaMallocHost(&s.h_ovf, (size_t)cap));
  SV_CK(cudaMallocHost(&s.h_status, 16));
  SV_CK(cudaMallocHost(&s.h_allow, (size_t)cap * sizeof(void*)));
  SV_CK(cudaMallocHost(&s.h_allow_w, (size_t)cap * 8));
  SV_CK(cudaStreamCreateWithFlags(&s.ctx.stream, cudaStreamNonBlocking));
  s.cap = cap;
  return SG_OK;
}

void slot_free(Slot& s) {
  sg::free_ctx(s.ctx);
  cudaFreeHost(s.h_q768);
  cudaFreeHost(s.h_q256);
  cudaFreeHost(s.h_sc);
  cudaFreeHost(s.h_id);
  cudaFreeHost(s.h_n);
  cudaFreeHost(s.h_ovf);
  cudaFreeHost(s.h_status);
  cudaFreeHost(s.h_allow);
  cudaFreeHost(s.h_allow_w);
}

// Stages the slot's batch and launches it; results land in the slot's pinned buffers.
int launch_batch(sg_server* srv, Slot& s) {
  sg_index* h = srv->h;
  const uint32_t n = (uint32_t)s.batch.size();
  const sg_params& p = s.p;
  bool any_filter = false;
  for (uint32_t i = 0; i < n; i++) {
    const Req& r = *s.batch[i];
    memcpy(s.h_q768 + (size_t)i * SG_DIM, r.q768.data(), SG_DIM * 4);
    if (s.have_q256) memcpy(s.h_q256 + (size_t)i * SG_PDIM, r.q256.data(), SG_PDIM * 4);
    s.h_allow[i] = r.filter ? r.filter->allow : nullptr;
    s.h_allow_w[i] = r.filter ? r.filter->words : 0;
    any_filter |= r.filter != nullptr;
  }
  int rc;
  // scratch for the largest batch these params may form, so later batches reuse it without
  // reallocating (a cudaFree would wait for the other contexts' batches)
  if ((rc = sg::ctx_prepare(h, s.cfg, s.ctx, std::max(n, s.limit), p))) return rc;
  sg::Workspace& w = s.ctx.ws;
  if (n > w.allow_q_cap) {
    if (w.allow_q) cudaFree(w.allow_q);
    if (w.allow_wq) cudaFree(w.allow_wq);
    w.allow_q = nullptr;
    w.allow_wq = nullptr;
    w.allow_q_cap = 0;
    SV_CK(cudaMalloc(&w.allow_q, (size_t)s.cap * sizeof(void*)));
    SV_CK(cudaMalloc(&w.allow_wq, (size_t)s.cap * 8));
    w.allow_q_cap = s.cap;
  }
  cudaStream_t st = s.ctx.stream;
  SV_CK(cudaMemcpyAsync(w.q768, s.h_q768, (size_t)n * SG_DIM * 4, cudaMemcpyHostToDevice, st));
  if (s.have_q256)
    SV_CK(cudaMemcpyAsync(w.q256, s.h_q256, (size_t)n * SG_PDIM * 4, cudaMemcpyHostToDevice, st));
  if (any_filter) {
    SV_CK(cudaMemcpyAsync(w.allow_q, s.h_allow, (size_t)n * sizeof(void*), cudaMemcpyHostToDevice, st));
    SV_CK(cudaMemcpyAsync(w.allow_wq, s.h_allow_w, (size_t)n * 8, cudaMemcpyHostToDevice, st));
  }
  w.per_query_allow = any_filter;
  rc = sg::ctx_launch(h, s.cfg, s.ctx, n, p, s.have_q256);
  w.per_query_allow = false;
  if (rc) return rc;
  const uint32_t k = p.k;
  if (k) {
    SV_CK(cudaMemcpyAsync(s.h_sc, w.out_sc, (size_t)n * k * 4, cudaMemcpyDeviceToHost, st));
    SV_CK(cudaMemcpyAsync(s.h_id, w.out_id, (size_t)n * k * 4, cudaMemcpyDeviceToHost, st));
  }
  SV_CK(cudaMemcpyAsync(s.h_n, w.out_n, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
  SV_CK(cudaMemcpyAsync(s.h_ovf, w.overflow, n, cudaMemcpyDeviceToHost, st));
  SV_CK(cudaMemcpyAsync(s.h_status, w.counters + 2, 4, cudaMemcpyDeviceToHost, st));
  SV_CK(cudaLaunchHostFunc(st, on_batch_done, &s));
  return SG_OK;
}

// Hands a finished batch's results to its requests (re-running overflowed queries alone).
void complete_batch(sg_server* srv, Slot& s, int launch_rc) {
  const uint32_t n = (uint32_t)s.batch.size();
  const uint32_t k = s.p.k;
  const bool queue_overflow = launch_rc == SG_OK && (*s.h_status & sg::kStatusOverflow);
  uint64_t retried = 0;
  for (uint32_t i = 0; i < n; i++) {
    Req& r = *s.batch[i];
    r.sc.assign(std::max<uint32_t>(k, 1), 0.0f);
    r.id.assign(std::max<uint32_t>(k, 1), 0u);
    r.batch = n;
    if (launch_rc != SG_OK) {
      r.status = launch_rc;
      continue;
    }
    if (queue_overflow) {
      r.status = fail(SG_ERR_INVALID, "work queue overflow");
      continue;
    }
    if (*s.h_status & sg::kStatusTimeout) {
      r.status = fail(SG_ERR_DEVICE, "a tensor-core wait ran out (routing GEMM or scan)");
      continue;
    }
    if (s.h_ovf[i]) {
      r.status = sg::ctx_search_one(srv->h, s.cfg, s.ctx, r.q768.data(),
                                    r.have_q256 ? r.q256.data() : nullptr, s.p,
                                    r.filter ? r.filter->allow : nullptr,
                                    r.filter ? r.filter->words : 0, r.sc.data(), r.id.data(), &r.n);
      r.retried = 1;
      retried++;
      continue;
    }
    r.n = s.h_n[i];
    if (k) {
      memcpy(r.sc.data(), s.h_sc + (size_t)i * k, (size_t)k * 4);
      memcpy(r.id.data(), s.h_id + (size_t)i * k, (size_t)k * 4);
    }
    r.status = SG_OK;
  }
  const auto now = Clock::now();
  {
    std::lock_guard<std::mutex> g(srv->mu);
    for (auto& r : s.batch) {
      r->done = true;
      r->t_done = now;
    }
    srv->st.completed += n;
    srv->st.retried += retried;
    srv->st.in_flight -= n;
    s.batch.clear();
    s.busy = false;
    s.gpu_done = false;
  }
  srv->cv_done.notify_all();
}

// Takes a batch for a free slot from the pending requests (caller holds mu).
void form_batch(sg_server* srv, Slot& s) {
  auto& pend = srv->pending;
  const sg_params p = pend.front()->p;
  const bool hq = pend.front()->have_q256;
  const uint64_t budget = srv->cfg.scratch_bytes / std::max<uint32_t>(srv->cfg.contexts, 1);
  uint32_t limit = std::min<uint32_t>(srv->cfg.max_batch, s.cap);
  s.cfg = sg::index_config(srv->h);
  // the largest batch whose scratch fits this slot's share (one query always goes)
  while (limit > 1 && sg::ctx_bytes(srv->h, s.cfg, p, limit) > budget) limit = (limit + 1) / 2;
  // Requests of these params, oldest first, until the batch is full; the scan stops there (a
  // backlog of many thousands would otherwise be walked once per batch), and requests of other
  // params that it passed go back to the front in their order.
  std::deque<std::shared_ptr<Req>> skipped;
  while (!pend.empty() && s.batch.size() < limit) {
    auto r = pend.front();
    pend.pop_front();
    if (r->have_q256 == hq && memcmp(&r->p, &p, sizeof p) == 0)
      s.batch.push_back(r);
    else
      skipped.push_back(r);
  }
  for (auto it = skipped.rbegin(); it != skipped.rend(); ++it) pend.push_front(*it);
  s.p = p;
  s.limit = limit;
  s.have_q256 = hq;
  s.busy = true;
  s.gpu_done = false;
  const auto now = Clock::now();
  for (auto& r : s.batch) r->t_launch = now;
  srv->st.batches++;
  srv->st.queries_batched += s.batch.size();
  srv->st.in_flight += (uint32_t)s.batch.size();
}

void dispatch_loop(sg_server* srv) {
  cudaSetDevice(srv->h->ix.device);
  std::unique_lock<std::mutex> lk(srv->mu);
  for (;;) {
    srv->cv_work.wait(lk, [&] {
      bool busy = false, free_slot = false;
      for (auto& s : srv->slots) {
        if (s->busy && s->gpu_done) return true;
        busy |= s->busy;
        free_slot |= !s->busy;
      }
      if (!srv->pending.empty() && free_slot) return true;
      return srv->stopping && !busy && srv->pending.empty();
    });
    bool any_busy = false;
    for (auto& sp : srv->slots) {
      Slot& s = *sp;
      if (s.busy && s.gpu_done) {
        lk.unlock();
        complete_batch(srv, s, SG_OK);
        lk.lock();
      }
      any_busy |= s.busy;
    }
    if (srv->stopping && !any_busy && srv->pending.empty()) break;
    for (auto& sp : srv->slots) {
      Slot& s = *sp;
      if (s.busy || srv->pending.empty()) continue;
      form_batch(srv, s);
      lk.unlock();
      const int rc = launch_batch(srv, s);
      if (rc != SG_OK) {
        // nothing is in flight on this stream beyond what ran before the failure
        cudaStreamSynchronize(s.ctx.stream);
        complete_batch(srv, s, rc);
      }
      lk.lock();
    }
  }
}

}  // namespace

extern "C" {

int sg_server_start(sg_index* h, const sg_server_config* cfg, sg_server** out) {
  if (!h || !out) return fail(SG_ERR_INVALID, "null argument");
  *out = nullptr;
  sg_server_config c = {};
  if (cfg) c = *cfg;
  if (c.max_batch == 0) c.max_batch = 1024;
  if (c.contexts == 0) c.contexts = 2;
  if (c.scratch_bytes == 0) c.scratch_bytes = 8ull << 30;
  if (c.max_pending == 0) c.max_pending = 1u << 20;
  if (c.max_batch > 65536 || c.contexts > 16) return fail(SG_ERR_INVALID, "max_batch <= 65536, contexts <= 16");
  std::unique_ptr<sg_server> srv(new sg_server());
  srv->h = h;
  srv->cfg = c;
  if (cudaSetDevice(h->ix.device) != cudaSuccess) return fail(SG_ERR_DEVICE, "cudaSetDevice");
  for (uint32_t i = 0; i < c.contexts; i++) {
    std::unique_ptr<Slot> s(new Slot());
    s->srv = srv.get();
    int rc = slot_alloc(*s, c.max_batch, sg::kMaxCand);
    srv->slots.push_back(std::move(s));
    if (rc) {
      for (auto& x : srv->slots) slot_free(*x);
      return rc;
    }
  }
  srv->dispatcher = std::thread(dispatch_loop, srv.get());
  *out = srv.release();
  return SG_OK;
}

int sg_server_submit(sg_server* srv, const float* q768, const float* q256, const sg_params* params,
                     const sg_filter* filter, uint64_t* ticket) {
  if (!srv || !q768 || !params || !ticket) return fail(SG_ERR_INVALID, "null argument");
  if (filter && filter->h != srv->h) return fail(SG_ERR_INVALID, "the filter belongs to another index");
  int rc;
  if ((rc = sg::index_check_params(srv->h, params))) return rc;
  auto r = std::make_shared<Req>();
  r->q768.assign(q768, q768 + SG_DIM);
  if (q256) {
    r->q256.assign(q256, q256 + SG_PDIM);
    r->have_q256 = true;
  }
  r->p = *params;
  r->filter = filter;
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(srv->mu);
    if (srv->stopping) return fail(SG_ERR_INVALID, "server is stopping");
    const uint64_t budget = srv->cfg.scratch_bytes / std::max<uint32_t>(srv->cfg.contexts, 1);
    if (srv->pending.size() >= srv->cfg.max_pending ||
        sg::ctx_bytes(srv->h, sg::index_config(srv->h), *params, 1) > budget) {
      srv->st.rejected++;
      return fail(SG_ERR_ADMISSION, "no queue slot or scratch for this request");
    }
    r->ticket = srv->next_ticket++;
    srv->pending.push_back(r);
    srv->live[r->ticket] = r;
    srv->st.submitted++;
    *ticket = r->ticket;
  }
  srv->cv_work.notify_all();
  return SG_OK;
}

int sg_server_poll(sg_server* srv, uint64_t ticket, int wait_ms, float* out_scores, uint32_t* out_ids,
                   uint32_t* out_count, sg_request_info* info) {
  if (!srv) return fail(SG_ERR_INVALID, "null server");
  std::unique_lock<std::mutex> lk(srv->mu);
  auto it = srv->live.find(ticket);
  if (it == srv->live.end()) return fail(SG_ERR_INVALID, "unknown ticket");
  std::shared_ptr<Req> r = it->second;
  auto ready = [&] { return r->done; };
  if (!r->done) {
    if (wait_ms < 0) srv->cv_done.wait(lk, ready);
    else if (wait_ms > 0) srv->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  }
  if (!r->done) return fail(SG_ERR_TIMEOUT, "request not finished");
  srv->live.erase(it);
  lk.unlock();
  if (r->status != SG_OK) return r->status;
  const uint32_t k = r->p.k;
  if (out_count) *out_count = r->n;
  if (k && out_scores) memcpy(out_scores, r->sc.data(), (size_t)k * 4);
  if (k && out_ids) memcpy(out_ids, r->id.data(), (size_t)k * 4);
  if (info) {
    using ms = std::chrono::duration<float, std::milli>;
    info->queue_ms = ms(r->t_launch - r->t_submit).count();
    info->service_ms = ms(r->t_done - r->t_launch).count();
    info->batch = r->batch;
    info->retried = r->retried;
  }
  return SG_OK;
}

int sg_server_replay(sg_server* srv, uint32_t nreq, const uint64_t* arrival_ns, const float* q768,
                     const uint32_t* which, const sg_params* params, const sg_filter* const* filters,
                     const int32_t* filter_of, float* out_latency_ms, uint32_t* out_batch,
                     double* out_wall_s) {
  if (!srv || !params || (nreq && (!arrival_ns || !q768 || !which || !out_latency_ms)))
    return fail(SG_ERR_INVALID, "null argument");
  if (nreq == 0) return SG_OK;
  std::vector<uint64_t> tickets(nreq, 0);
  std::vector<std::atomic<uint8_t>> ready(nreq);
  for (auto& r : ready) r.store(0, std::memory_order_relaxed);
  std::atomic<int> collect_rc{SG_OK};
  // the collector waits for each request in submission order; latency is the library's clock
  // from submit to results on the host
  std::thread collector([&] {
    for (uint32_t i = 0; i < nreq; i++) {
      while (!ready[i].load(std::memory_order_acquire)) std::this_thread::yield();
      sg_request_info info;
      const int rc = sg_server_poll(srv, tickets[i], -1, nullptr, nullptr, nullptr, &info);
      if (rc != SG_OK) {
        int expect = SG_OK;
        collect_rc.compare_exchange_strong(expect, rc);
        out_latency_ms[i] = -1.0f;
        if (out_batch) out_batch[i] = 0;
        continue;
      }
      out_latency_ms[i] = info.queue_ms + info.service_ms;
      if (out_batch) out_batch[i] = info.batch;
    }
  });
  // the submitter keeps the open-loop schedule: each request goes at its arrival time, whatever
  // the state of earlier ones
  const auto t0 = Clock::now();
  int rc = SG_OK;
  for (uint32_t i = 0; i < nreq; i++) {
    const auto due = t0 + std::chrono::nanoseconds(arrival_ns[i]);
    while (Clock::now() < due) {
    }
    const sg_filter* f = (filters && filter_of && filter_of[i] >= 0) ? filters[filter_of[i]] : nullptr;
    int r = sg_server_submit(srv, q768 + (size_t)which[i] * SG_DIM, nullptr, params, f, &tickets[i]);
    if (r != SG_OK) {
      if (rc == SG_OK) rc = r;
      // the request is not queued: record it as refused so the collector does not wait on it
      tickets[i] = 0;
    }
    ready[i].store(1, std::memory_order_release);
  }
  collector.join();
  if (out_wall_s) *out_wall_s = std::chrono::duration<double>(Clock::now() - t0).count();
  if (rc != SG_OK) return rc;
  return collect_rc.load();
}

int sg_server_get_stats(sg_server* srv, sg_server_stats* out) {
  if (!srv || !out) return fail(SG_ERR_INVALID, "null argument");
  std::lock_guard<std::mutex> g(srv->mu);
  *out = srv->st;
  out->pending = (uint32_t)srv->pending.size();
  return SG_OK;
}

int sg_server_stop(sg_server* srv) {
  if (!srv) return SG_OK;
  {
    std::lock_guard<std::mutex> g(srv->mu);
    srv->stopping = true;
  }
  srv->cv_work.notify_all();
  if (srv->dispatcher.joinable()) srv->dispatcher.join();
  {
    std::lock_guard<std::mutex> g(srv->mu);
    for (auto& r : srv->pending) {
      r->status = SG_ERR_INVALID;
      r->done = true;
    }
    srv->pending.clear();
  }
  srv->cv_done.notify_all();
  cudaSetDevice(srv->h->ix.device);
  for (auto& s : srv->slots) slot_free(*s);
  delete srv;
  return SG_OK;
}

}  // extern "C"
