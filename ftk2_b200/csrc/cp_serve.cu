// Serving runtime: a request loop over worker slots (no counterpart in the
// reference, whose engine runs one extraction per call).
//
// Each worker thread owns a context (its own device buffers and CUDA stream),
// so the device work of requests running on different workers overlaps.
// Requests wait in one arrival-ordered queue; a free worker takes the first
// request that can start:
//   * a stream push only when no earlier push of the same stream is queued or
//     running (pushes run in order on the stream's own context, which keeps
//     the previous timestep and the union-find state resident);
//   * any request only when its estimated device memory fits the HBM budget
//     next to the requests already running, or when nothing runs at all.
// Later requests may pass one that waits for memory, except once the oldest
// waiting request has waited longer than kMaxBypassMs (no starvation).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <set>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ftk2b.h"
#include <cuda_runtime.h>

namespace {

constexpr double kMaxBypassMs = 250.0;
constexpr uint64_t kExtractOverhead = 64ull << 20;  // feature, candidate and sort buffers
constexpr uint64_t kPushOverhead = 32ull << 20;

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Req {
  uint64_t ticket = 0;
  int pin = -1;       // worker that must run it (-1: any)
  bool warm = false;  // warm-up request: kept out of the statistics
  ftk2b_request r;
  uint64_t est = 0;
  Clock::time_point t_submit, t_start, t_end;
  bool started = false, done = false;
  ftk2b_status status = FTK2B_OK;
  int slot = -1;
  ftk2b_cp_result* res = nullptr;
  uint64_t n_features = 0, n_simplices = 0;
  double phase_ms[4] = {0, 0, 0, 0};
  std::string err;
};

struct StreamRec {
  ftk2b_ctx* ctx = nullptr;
  ftk2b_stream* s = nullptr;
  bool busy = false;
  unsigned queued = 0;
};

uint64_t field_bytes(const ftk2b_field_desc& f) {
  const uint64_t es = f.dtype == FTK2B_F64 ? 8 : 4;
  uint64_t n = 1;
  for (int k = 0; k < f.nd && k < 4; ++k) n *= f.dims[k];
  const uint64_t arrays = f.layout == FTK2B_LAYOUT_MULTICOMPONENT ? 1 : (uint64_t)(f.ncomp > 0 ? f.ncomp : 1);
  const uint64_t per = f.layout == FTK2B_LAYOUT_MULTICOMPONENT ? (uint64_t)f.ncomp : 1;
  return n * per * arrays * es;
}

}  // namespace

struct ftk2b_server {
  int device = 0;
  int n_slots = 0;
  uint64_t budget = 0, reserved = 0, reserved_peak = 0;
  uint64_t reserved_pool = 0;  // bytes mapped into the allocation pool at creation
  int queue_limit = 0;
  int in_flight = 0, max_in_flight = 0;
  std::vector<ftk2b_ctx*> slot_ctx;
  std::deque<Req*> queue;
  std::map<uint64_t, Req*> reqs;
  std::map<uint64_t, StreamRec> streams;
  uint64_t next_ticket = 1, next_stream = 1;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::vector<std::thread> workers;
  bool stop = false;
  // statistics
  uint64_t submitted = 0, completed = 0, failed = 0, rejected = 0, simplices = 0;
  std::vector<double> latencies;
  bool any_submit = false;
  Clock::time_point first_submit, last_done;
  std::string err;
};

namespace {

// First request of the queue that worker `slot` may start now (called with
// the lock held).
Req* pick_locked(ftk2b_server* sv, int slot) {
  std::set<uint64_t> blocked_streams;
  const Clock::time_point now = Clock::now();
  for (auto it = sv->queue.begin(); it != sv->queue.end(); ++it) {
    Req* q = *it;
    if (q->pin >= 0 && q->pin != slot) continue;
    if (q->r.kind == FTK2B_REQ_STREAM_PUSH) {
      auto s = sv->streams.find(q->r.stream);
      if (s == sv->streams.end()) {  // closed under it: fail it right away
        sv->queue.erase(it);
        return q;
      }
      if (s->second.busy || blocked_streams.count(q->r.stream)) {
        blocked_streams.insert(q->r.stream);
        continue;
      }
    }
    const bool fits = sv->in_flight == 0 || sv->reserved + q->est <= sv->budget;
    if (fits) {
      sv->queue.erase(it);
      return q;
    }
    if (q->r.kind == FTK2B_REQ_STREAM_PUSH) blocked_streams.insert(q->r.stream);
    if (ms_between(q->t_submit, now) > kMaxBypassMs) return nullptr;
  }
  return nullptr;
}

void run_request(ftk2b_server* sv, Req* q, int slot) {
  if (q->r.kind == FTK2B_REQ_EXTRACT) {
    ftk2b_ctx* ctx = sv->slot_ctx[slot];
    ftk2b_cp_result* res = nullptr;
    q->status = ftk2b_cp_extract(ctx, &q->r.mesh, &q->r.field, &q->r.params, &res);
    ftk2b_ctx_last_phases(ctx, q->phase_ms);
    if (q->status == FTK2B_OK) {
      q->res = res;
      q->n_features = res->n_features;
      q->n_simplices = res->n_simplices;
    } else {
      q->err = ftk2b_last_error(ctx);
    }
    return;
  }
  ftk2b_stream* s = nullptr;
  ftk2b_ctx* ctx = nullptr;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->streams.find(q->r.stream);
    if (it != sv->streams.end()) {
      s = it->second.s;
      ctx = it->second.ctx;
    }
  }
  if (!s) {
    q->status = FTK2B_INVALID_ARG;
    q->err = "unknown or closed stream";
    return;
  }
  uint64_t n_new = 0;
  q->status = ftk2b_stream_push(s, &q->r.field, &n_new);
  if (q->status == FTK2B_OK) q->n_features = n_new;
  else q->err = ftk2b_last_error(ctx);
}

void worker_main(ftk2b_server* sv, int slot) {
  cudaSetDevice(sv->device);
  for (;;) {
    Req* q = nullptr;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_work.wait(lk, [&] { return sv->stop || (q = pick_locked(sv, slot)) != nullptr; });
      if (!q) return;
      q->started = true;
      q->slot = slot;
      q->t_start = Clock::now();
      sv->reserved += q->est;
      sv->reserved_peak = std::max(sv->reserved_peak, sv->reserved);
      sv->in_flight += 1;
      sv->max_in_flight = std::max(sv->max_in_flight, sv->in_flight);
      if (q->r.kind == FTK2B_REQ_STREAM_PUSH) {
        auto it = sv->streams.find(q->r.stream);
        if (it != sv->streams.end()) {
          it->second.busy = true;
          it->second.queued -= 1;
        }
      }
    }
    run_request(sv, q, slot);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      q->t_end = Clock::now();
      q->done = true;
      sv->reserved -= q->est;
      sv->in_flight -= 1;
      if (q->r.kind == FTK2B_REQ_STREAM_PUSH) {
        auto it = sv->streams.find(q->r.stream);
        if (it != sv->streams.end()) it->second.busy = false;
      }
      if (q->warm) {
        // warm-up requests stay out of the statistics
      } else if (q->status == FTK2B_OK) {
        sv->completed += 1;
        sv->latencies.push_back(ms_between(q->t_submit, q->t_end));
        sv->simplices += q->n_simplices;
        sv->last_done = q->t_end;
      } else {
        sv->failed += 1;
        sv->err = q->err;
        sv->last_done = q->t_end;
      }
    }
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
}

uint64_t estimate_bytes(const ftk2b_request* req) {
  uint64_t est;
  if (req->kind == FTK2B_REQ_EXTRACT) {
    est = kExtractOverhead + (req->field.location == FTK2B_HOST ? field_bytes(req->field) : 0);
    if (req->mesh.kind == FTK2B_MESH_EXTRUDED) {
      const uint64_t nv = req->mesh.n_base_verts * (req->mesh.n_layers + 1);
      est += 4 * nv + 48 * req->mesh.n_base_cells * (uint64_t)(req->mesh.base_cell_dim + 1);
    }
  } else {
    est = kPushOverhead + (req->field.location == FTK2B_HOST ? field_bytes(req->field) : 0);
  }
  return est;
}

ftk2b_status sv_fail(ftk2b_server* sv, ftk2b_status st, const std::string& msg) {
  std::lock_guard<std::mutex> lk(sv->mu);
  sv->err = msg;
  return st;
}

}  // namespace

extern "C" ftk2b_status ftk2b_server_create(int device, int n_slots, uint64_t hbm_budget, int queue_limit,
                                            ftk2b_server** out) {
  if (!out || n_slots < 1 || n_slots > 64 || queue_limit < 0) return FTK2B_INVALID_ARG;
  *out = nullptr;
  ftk2b_server* sv = new ftk2b_server();
  sv->device = device;
  sv->n_slots = n_slots;
  sv->queue_limit = queue_limit;
  for (int i = 0; i < n_slots; ++i) {
    ftk2b_ctx* c = nullptr;
    const ftk2b_status st = ftk2b_ctx_create(device, &c);
    if (st != FTK2B_OK) {
      for (ftk2b_ctx* x : sv->slot_ctx) ftk2b_ctx_destroy(x);
      delete sv;
      return st;
    }
    ftk2b_ctx_set_option(c, FTK2B_OPT_BLOCKING_SYNC, 1);
    sv->slot_ctx.push_back(c);
  }
  if (hbm_budget == 0) {
    size_t fr = 0, tot = 0;
    cudaSetDevice(device);
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
      cudaGetLastError();
      fr = 0;
    }
    hbm_budget = (uint64_t)(0.9 * (double)fr);
  }
  sv->budget = hbm_budget;
  // Growing a buffer maps new device memory into the stream-ordered pool,
  // which holds up the work of every slot while it happens.  Keep freed pool
  // memory mapped and map a reserve up front: min(budget / 2, n_slots GiB).
  {
    cudaSetDevice(device);
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
      uint64_t keep = ~0ull;
      cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      const uint64_t reserve = std::min<uint64_t>(sv->budget / 2, (uint64_t)n_slots << 30);
      void* p = nullptr;
      cudaStream_t st = (cudaStream_t)ftk2b_ctx_stream(sv->slot_ctx[0]);
      if (reserve && cudaMallocAsync(&p, reserve, st) == cudaSuccess) {
        cudaFreeAsync(p, st);
        cudaStreamSynchronize(st);
      }
      sv->reserved_pool = reserve;
    }
    cudaGetLastError();
  }
  for (int i = 0; i < n_slots; ++i) sv->workers.emplace_back(worker_main, sv, i);
  *out = sv;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_server_stream_open(ftk2b_server* sv, const ftk2b_mesh_desc* mesh,
                                                 const ftk2b_field_desc* tmpl, const ftk2b_cp_params* params,
                                                 uint64_t* stream_id) {
  if (!sv || !stream_id) return FTK2B_INVALID_ARG;
  ftk2b_ctx* ctx = nullptr;
  ftk2b_status st = ftk2b_ctx_create(sv->device, &ctx);
  if (st != FTK2B_OK) return sv_fail(sv, st, "context creation failed");
  ftk2b_ctx_set_option(ctx, FTK2B_OPT_BLOCKING_SYNC, 1);
  ftk2b_stream* s = nullptr;
  st = ftk2b_stream_open(ctx, mesh, tmpl, params, &s);
  if (st != FTK2B_OK) {
    std::string e = ftk2b_last_error(ctx);
    ftk2b_ctx_destroy(ctx);
    return sv_fail(sv, st, e);
  }
  std::lock_guard<std::mutex> lk(sv->mu);
  const uint64_t id = sv->next_stream++;
  StreamRec rec;
  rec.ctx = ctx;
  rec.s = s;
  sv->streams[id] = rec;
  *stream_id = id;
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_server_submit(ftk2b_server* sv, const ftk2b_request* req, uint64_t* ticket) {
  if (!sv || !req || !ticket) return FTK2B_INVALID_ARG;
  if (req->kind != FTK2B_REQ_EXTRACT && req->kind != FTK2B_REQ_STREAM_PUSH)
    return sv_fail(sv, FTK2B_INVALID_ARG, "unknown request kind");
  Req* q = new Req();
  q->r = *req;
  q->est = estimate_bytes(req);
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    if (req->kind == FTK2B_REQ_STREAM_PUSH) {
      auto it = sv->streams.find(req->stream);
      if (it == sv->streams.end()) {
        delete q;
        sv->err = "unknown stream id";
        return FTK2B_INVALID_ARG;
      }
      it->second.queued += 1;
    }
    if (sv->queue_limit && (int)sv->queue.size() >= sv->queue_limit) {
      if (req->kind == FTK2B_REQ_STREAM_PUSH) sv->streams[req->stream].queued -= 1;
      sv->rejected += 1;
      delete q;
      sv->err = "queue full";
      return FTK2B_BUSY;
    }
    q->ticket = sv->next_ticket++;
    q->t_submit = Clock::now();
    if (!sv->any_submit) {
      sv->any_submit = true;
      sv->first_submit = q->t_submit;
    }
    sv->submitted += 1;
    sv->queue.push_back(q);
    sv->reqs[q->ticket] = q;
    *ticket = q->ticket;
  }
  sv->cv_work.notify_one();
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_server_warm(ftk2b_server* sv, const ftk2b_request* req) {
  if (!sv || !req) return FTK2B_INVALID_ARG;
  if (req->kind != FTK2B_REQ_EXTRACT) return sv_fail(sv, FTK2B_INVALID_ARG, "only extraction requests warm slots");
  std::vector<Req*> mine;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    for (int w = 0; w < sv->n_slots; ++w) {
      Req* q = new Req();
      q->r = *req;
      q->est = estimate_bytes(req);
      q->pin = w;
      q->warm = true;
      q->ticket = sv->next_ticket++;
      q->t_submit = Clock::now();
      sv->queue.push_back(q);
      mine.push_back(q);
    }
  }
  sv->cv_work.notify_all();
  ftk2b_status worst = FTK2B_OK;
  std::unique_lock<std::mutex> lk(sv->mu);
  for (Req* q : mine) {
    sv->cv_done.wait(lk, [&] { return q->done; });
    if (q->status != FTK2B_OK) {
      worst = q->status;
      sv->err = q->err;
    }
    if (q->res) ftk2b_cp_result_free(q->res);
    delete q;
  }
  return worst;
}

extern "C" ftk2b_status ftk2b_server_wait(ftk2b_server* sv, uint64_t ticket, double timeout_s,
                                          ftk2b_cp_result** out, ftk2b_request_stats* stats) {
  if (!sv) return FTK2B_INVALID_ARG;
  if (out) *out = nullptr;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->reqs.find(ticket);
  if (it == sv->reqs.end()) {
    sv->err = "unknown ticket";
    return FTK2B_INVALID_ARG;
  }
  Req* q = it->second;
  auto ready = [&] { return q->done; };
  if (timeout_s < 0) {
    sv->cv_done.wait(lk, ready);
  } else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready)) {
    return FTK2B_TIMEOUT;
  }
  sv->reqs.erase(it);
  if (stats) {
    stats->status = q->status;
    stats->slot = q->slot;
    stats->queue_ms = ms_between(q->t_submit, q->t_start);
    stats->run_ms = ms_between(q->t_start, q->t_end);
    stats->latency_ms = ms_between(q->t_submit, q->t_end);
    stats->n_features = q->n_features;
    stats->n_simplices = q->n_simplices;
    for (int i = 0; i < 4; ++i) stats->phase_ms[i] = q->phase_ms[i];
  }
  const ftk2b_status st = q->status;
  if (st != FTK2B_OK) sv->err = q->err;
  if (out) *out = q->res;
  else if (q->res) ftk2b_cp_result_free(q->res);
  delete q;
  return st;
}

// Waits (lock held) until a stream has no queued or running push.
static StreamRec* idle_stream_locked(ftk2b_server* sv, std::unique_lock<std::mutex>& lk, uint64_t id) {
  for (;;) {
    auto it = sv->streams.find(id);
    if (it == sv->streams.end()) return nullptr;
    if (!it->second.busy && it->second.queued == 0) return &it->second;
    sv->cv_done.wait(lk);
  }
}

extern "C" ftk2b_status ftk2b_server_stream_result(ftk2b_server* sv, uint64_t stream_id, ftk2b_cp_result** out) {
  if (!sv || !out) return FTK2B_INVALID_ARG;
  *out = nullptr;
  std::unique_lock<std::mutex> lk(sv->mu);
  StreamRec* rec = idle_stream_locked(sv, lk, stream_id);
  if (!rec) {
    sv->err = "unknown stream id";
    return FTK2B_INVALID_ARG;
  }
  rec->busy = true;
  ftk2b_stream* s = rec->s;
  ftk2b_ctx* ctx = rec->ctx;
  lk.unlock();
  const ftk2b_status st = ftk2b_stream_result(s, out);
  lk.lock();
  if (st != FTK2B_OK) sv->err = ftk2b_last_error(ctx);
  auto it = sv->streams.find(stream_id);
  if (it != sv->streams.end()) it->second.busy = false;
  lk.unlock();
  sv->cv_work.notify_all();
  sv->cv_done.notify_all();
  return st;
}

extern "C" ftk2b_status ftk2b_server_stream_close(ftk2b_server* sv, uint64_t stream_id) {
  if (!sv) return FTK2B_INVALID_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  StreamRec* rec = idle_stream_locked(sv, lk, stream_id);
  if (!rec) {
    sv->err = "unknown stream id";
    return FTK2B_INVALID_ARG;
  }
  StreamRec copy = *rec;
  sv->streams.erase(stream_id);
  lk.unlock();
  ftk2b_stream_close(copy.s);
  ftk2b_ctx_destroy(copy.ctx);
  return FTK2B_OK;
}

extern "C" ftk2b_status ftk2b_server_get_stats(ftk2b_server* sv, ftk2b_server_stats* out) {
  if (!sv || !out) return FTK2B_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  memset(out, 0, sizeof(*out));
  out->submitted = sv->submitted;
  out->completed = sv->completed;
  out->failed = sv->failed;
  out->rejected = sv->rejected;
  out->simplices = sv->simplices;
  out->hbm_budget = sv->budget;
  out->hbm_reserved_peak = sv->reserved_peak;
  out->max_in_flight = sv->max_in_flight;
  if (sv->any_submit && sv->completed + sv->failed > 0)
    out->elapsed_s = ms_between(sv->first_submit, sv->last_done) / 1000.0;
  if (!sv->latencies.empty()) {
    std::vector<double> v = sv->latencies;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      // nearest-rank percentile
      size_t k = (size_t)std::ceil(p * (double)v.size());
      if (k < 1) k = 1;
      return v[k - 1];
    };
    out->p50_ms = pct(0.50);
    out->p99_ms = pct(0.99);
    out->max_ms = v.back();
    double s = 0;
    for (double x : v) s += x;
    out->mean_ms = s / (double)v.size();
  }
  return FTK2B_OK;
}

extern "C" const char* ftk2b_server_last_error(ftk2b_server* sv) {
  if (!sv) return "null server";
  std::lock_guard<std::mutex> lk(sv->mu);
  thread_local std::string copy;
  copy = sv->err;
  return copy.c_str();
}

extern "C" void ftk2b_server_destroy(ftk2b_server* sv) {
  if (!sv) return;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->workers) t.join();
  for (auto& kv : sv->reqs) {
    if (kv.second->res) ftk2b_cp_result_free(kv.second->res);
    delete kv.second;
  }
  for (auto& kv : sv->streams) {
    ftk2b_stream_close(kv.second.s);
    ftk2b_ctx_destroy(kv.second.ctx);
  }
  for (ftk2b_ctx* c : sv->slot_ctx) ftk2b_ctx_destroy(c);
  delete sv;
}
