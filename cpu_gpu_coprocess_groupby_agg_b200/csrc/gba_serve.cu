// Serving: a request loop with continuous batching under a device-memory budget.
//
// No counterpart in the reference, which runs one query per process call.
//
// A server owns `lanes` workers.  Each lane is a host thread with its own CUDA
// stream and library context, so lanes run on the device at the same time and
// each context keeps its tables and workspace resident between requests.  Requests (device columns in, device columns out) enter one FIFO
// queue.  A lane that comes free takes work from the head of the queue:
//   * a request of more than batch_rows rows runs alone (gba_groupby);
//   * otherwise the lane takes the head and every following small request
//     (up to max_batch) whose estimated device memory still fits the budget,
//     and runs them as one gba_groupby_batch call.
// Requests that arrive while lanes are busy wait in the queue and join the
// next batch a lane forms, so work is admitted as lanes and memory free up.
// Admission: the sum of the estimated device bytes of all running requests
// stays within memory_budget; a request that alone exceeds it is refused at
// submit with GBA_ERR_BUDGET.  A lane whose resident workspace would push the
// lanes' total past the budget releases it when it finishes a request.
// If a batch call fails, its requests are rerun one by one so that each gets
// its own status.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "gba_context.h"
#include "gba_plan.h"

namespace {
using Clock = std::chrono::steady_clock;

struct Request {
  int64_t ticket;
  gba_query q;
  gba_output out;
  int64_t bytes;  // estimated device memory while it runs
  Clock::time_point t_submit, t_start, t_end;
  gba_request_info info{};
  bool done = false;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}
}  // namespace

struct gba_server {
  gba_server_config cfg{};
  std::vector<gba_context*> ctxs;
  std::vector<cudaStream_t> streams;
  std::vector<std::thread> threads;
  std::vector<int64_t> resident;  // per lane: device bytes its context holds
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> queue;
  std::unordered_map<int64_t, Request*> all;
  std::deque<int64_t> completed;  // tickets finished and not yet collected
  int64_t next_ticket = 1;
  int64_t inflight_bytes = 0;
  int64_t submitted = 0, finished = 0;
  bool stop = false;
  gba_context* admin = nullptr;  // validates queries at submit (under mu)
  std::string last_failure;      // message of the latest failed request (or failed batch)
  int64_t batch_failures = 0;    // batch calls that failed and were rerun request by request
  // where the time goes: lane calls, the longest one, workspace releases
  // (a release synchronises the device) and the longest of them
  int64_t lane_calls = 0, ws_releases = 0, regrows = 0;
  double lane_ms_max = 0.0, release_ms_max = 0.0;
};

static int64_t ctx_resident_bytes(const gba_context* c) {
  return int64_t(c->ws_bytes + c->stage_bytes + c->rp_bytes + c->est_ws_bytes);
}

// Device bytes a request may need while it runs: the larger of the plain-sized
// HBM table (a power of two >= rows / load factor, 8 bytes per key and
// accumulator) and the partition strategy's two row buffers.
static int64_t request_bytes(const QDesc& q, const gba_knobs& k) {
  const double lf = (k.load_factor > 0.05 && k.load_factor < 0.95) ? k.load_factor : 0.5;
  const uint64_t slots = gba_pow2_ceil(uint64_t(double(std::max<int64_t>(q.n, 1)) / lf));
  const int64_t table = int64_t(slots + 1) * gba_gt_stride(q.naccs) * 8;
  const int64_t part = 2 * q.n * int64_t(gba_row_bytes(q)) + (int64_t(1) << 24);
  return std::max(table, part) + (int64_t(1) << 20);
}

static void lane_main(gba_server* sv, int lane) {
  gba_context* ctx = sv->ctxs[lane];
  cudaStream_t s = sv->streams[lane];
  cudaSetDevice(sv->cfg.device);
  std::vector<Request*> take;
  std::vector<gba_query> qs;
  std::vector<gba_output> outs;
  std::vector<int64_t> ng;
  for (;;) {
    take.clear();
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      sv->cv_work.wait(lk, [&] {
        return sv->stop || (!sv->queue.empty() &&
                            sv->inflight_bytes + sv->queue.front()->bytes <= sv->cfg.memory_budget);
      });
      if (sv->stop && sv->queue.empty()) return;
      if (sv->queue.empty()) continue;
      Request* head = sv->queue.front();
      if (sv->inflight_bytes + head->bytes > sv->cfg.memory_budget) continue;
      sv->queue.pop_front();
      take.push_back(head);
      sv->inflight_bytes += head->bytes;
      if (head->q.n_rows <= sv->cfg.batch_rows) {
        for (auto it = sv->queue.begin(); it != sv->queue.end() && int(take.size()) < sv->cfg.max_batch;) {
          Request* r = *it;
          if (r->q.n_rows > sv->cfg.batch_rows) {
            ++it;
            continue;
          }
          if (sv->inflight_bytes + r->bytes > sv->cfg.memory_budget) break;  // keep arrival order
          sv->inflight_bytes += r->bytes;
          take.push_back(r);
          it = sv->queue.erase(it);
        }
      }
      const auto now = Clock::now();
      for (Request* r : take) r->t_start = now;
    }
    // ---- run outside the lock ----
    const int nb = int(take.size());
    gba_status st;
    if (nb == 1) {
      int64_t g = 0;
      st = gba_groupby(ctx, &take[0]->q, &take[0]->out, &sv->cfg.knobs, s, &g);
      take[0]->info.status = st;
      take[0]->info.n_groups = g;
    } else {
      qs.resize(nb);
      outs.resize(nb);
      ng.assign(nb, 0);
      for (int i = 0; i < nb; ++i) {
        qs[i] = take[i]->q;
        outs[i] = take[i]->out;
      }
      st = gba_groupby_batch(ctx, nb, qs.data(), outs.data(), &sv->cfg.knobs, s, ng.data());
      if (st == GBA_OK) {
        for (int i = 0; i < nb; ++i) {
          take[i]->info.status = GBA_OK;
          take[i]->info.n_groups = ng[i];
        }
      } else {
        {
          std::lock_guard<std::mutex> lk(sv->mu);
          ++sv->batch_failures;
          sv->last_failure = "lane " + std::to_string(lane) + ": a batch of " + std::to_string(nb) + " failed (" +
                             gba_status_string(st) + ": " + ctx->err + "); its requests ran one by one";
        }
        for (int i = 0; i < nb; ++i) {  // attribute the failure
          int64_t g = 0;
          take[i]->info.status = gba_groupby(ctx, &take[i]->q, &take[i]->out, &sv->cfg.knobs, s, &g);
          take[i]->info.n_groups = g;
        }
      }
    }
    const auto t_end = Clock::now();
    const double call_ms = nb ? ms_between(take[0]->t_start, t_end) : 0.0;
    // release the workspace if the lanes together hold more than the budget
    int64_t mine = ctx_resident_bytes(ctx);
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      int64_t total = 0;
      for (int64_t b : sv->resident) total += b;
      total += mine - sv->resident[lane];
      ++sv->lane_calls;
      sv->regrows += ctx->stats.regrows;
      sv->lane_ms_max = std::max(sv->lane_ms_max, call_ms);
      if (total > sv->cfg.memory_budget && ctx->ws) {
        const auto t_rel = Clock::now();
        cudaStreamSynchronize(s);
        cudaFree(ctx->ws);
        ctx->ws = nullptr;
        ctx->ws_bytes = 0;
        mine = ctx_resident_bytes(ctx);
        ++sv->ws_releases;
        sv->release_ms_max = std::max(sv->release_ms_max, ms_between(t_rel, Clock::now()));
      }
      sv->resident[lane] = mine;
      for (Request* r : take)
        if (r->info.status != GBA_OK)
          sv->last_failure = "lane " + std::to_string(lane) + ": " + gba_status_string(gba_status(r->info.status)) +
                             ": " + ctx->err;
      for (Request* r : take) {
        r->t_end = t_end;
        r->info.lane = lane;
        r->info.batch_size = nb;
        r->info.queue_ms = ms_between(r->t_submit, r->t_start);
        r->info.service_ms = ms_between(r->t_start, r->t_end);
        r->info.latency_ms = ms_between(r->t_submit, r->t_end);
        r->done = true;
        sv->inflight_bytes -= r->bytes;
        sv->completed.push_back(r->ticket);
        ++sv->finished;
      }
    }
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
}

extern "C" void gba_server_default_config(gba_server_config* c) {
  std::memset(c, 0, sizeof(*c));
  c->device = 0;
  c->lanes = 4;
  c->memory_budget = int64_t(120) << 30;
  c->max_batch = 64;
  c->batch_rows = int64_t(1) << 24;
  gba_default_knobs(&c->knobs);
}

extern "C" gba_status gba_server_create(gba_server** out, const gba_server_config* cfg) {
  if (!out) return GBA_ERR_INVALID_ARG;
  *out = nullptr;
  gba_server_config c;
  if (cfg) c = *cfg;
  else gba_server_default_config(&c);
  if (c.lanes <= 0) c.lanes = 4;
  if (c.lanes > 64) return GBA_ERR_INVALID_ARG;
  if (c.memory_budget <= 0) c.memory_budget = int64_t(120) << 30;
  if (c.max_batch <= 0) c.max_batch = 64;
  if (c.batch_rows <= 0) c.batch_rows = int64_t(1) << 24;
  // Lanes do not capture graphs: each batch a lane forms has a new shape (so a
  // captured graph would rarely be replayed), and a capture on one lane's
  // thread must not meet another lane's workspace growth, whose cudaFree
  // synchronises the device.
  c.knobs.use_graph = 0;
  // Lanes' batch kernels share the GPU: at 3 or 4 CTAs per SM one lane's
  // launch fills every SM and the others queue behind it; at 2 two lanes'
  // launches fit side by side.
  if (c.knobs.blocks_per_sm == 0) c.knobs.blocks_per_sm = 2;
  gba_server* sv = new gba_server();
  sv->cfg = c;
  gba_status st = gba_create(&sv->admin, c.device);
  if (st != GBA_OK) {
    delete sv;
    return st;
  }
  cudaSetDevice(c.device);
  // Each lane reserves 90% of its share of the budget up front as workspace
  // (at most 60% of the device's free memory between the lanes), and learned
  // sizing's sampling scratch and the batch descriptors' pinned staging too,
  // so that serving rarely grows a buffer: a growth frees the old block, and
  // cudaFree synchronises the device, stalling every lane.  (The other 10%
  // covers those smaller buffers, so the lanes together stay within the
  // budget and keep their workspaces.)
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) free_b = 0;
  const size_t share = std::min<size_t>(size_t(c.memory_budget) / size_t(c.lanes) / 10 * 9,
                                        free_b / 10 * 6 / size_t(c.lanes));
  const size_t est_share = std::min<size_t>(size_t(512) << 20, size_t(c.memory_budget) / size_t(c.lanes) / 20);
  for (int i = 0; i < c.lanes; ++i) {
    gba_context* ctx = nullptr;
    cudaStream_t s = nullptr;
    st = gba_create(&ctx, c.device);
    if (st == GBA_OK && cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) st = GBA_ERR_CUDA;
    if (st == GBA_OK && share > 0) st = gba_ws_reserve(ctx, share, s);
    if (st == GBA_OK && c.knobs.sizing == GBA_SIZING_LEARNED && est_share > 0) st = gba_est_reserve(ctx, est_share, s);
    if (st == GBA_OK) st = gba_batch_host_reserve(ctx, size_t(4) << 20);
    if (st != GBA_OK) {
      if (ctx) gba_destroy(ctx);
      for (size_t j = 0; j < sv->ctxs.size(); ++j) {
        cudaStreamDestroy(sv->streams[j]);
        gba_destroy(sv->ctxs[j]);
      }
      gba_destroy(sv->admin);
      delete sv;
      return st;
    }
    sv->ctxs.push_back(ctx);
    sv->streams.push_back(s);
    sv->resident.push_back(ctx_resident_bytes(ctx));
  }
  for (int i = 0; i < c.lanes; ++i) sv->threads.emplace_back(lane_main, sv, i);
  *out = sv;
  return GBA_OK;
}

extern "C" gba_status gba_server_estimator_load(gba_server* sv, const float* params) {
  if (!sv || !params) return GBA_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  if (sv->submitted != sv->finished) return GBA_ERR_INVALID_ARG;  // only while idle
  for (gba_context* c : sv->ctxs) {
    const gba_status st = gba_estimator_load(c, params);
    if (st != GBA_OK) return st;
  }
  return gba_estimator_load(sv->admin, params);
}

extern "C" gba_status gba_server_submit(gba_server* sv, const gba_query* q, const gba_output* out, int64_t* ticket) {
  if (!sv || !q || !out || !ticket) return GBA_ERR_INVALID_ARG;
  Request* r = new Request();
  r->q = *q;
  r->out = *out;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    gba_query qc;
    gba_compact_query(q, &qc);
    QDesc d;
    const gba_status st = gba_build_qdesc(sv->admin, &qc, &d);
    if (st != GBA_OK) {
      delete r;
      return st;
    }
    r->bytes = request_bytes(d, sv->cfg.knobs);
    if (r->bytes > sv->cfg.memory_budget) {
      sv->admin->err = "request needs about " + std::to_string(r->bytes) + " device bytes, budget " +
                       std::to_string(sv->cfg.memory_budget);
      delete r;
      return GBA_ERR_BUDGET;
    }
    r->ticket = sv->next_ticket++;
    r->t_submit = Clock::now();
    sv->all[r->ticket] = r;
    sv->queue.push_back(r);
    ++sv->submitted;
    *ticket = r->ticket;
  }
  sv->cv_work.notify_one();
  return GBA_OK;
}

// Collects a finished request: copies its info and forgets it.
static void collect_locked(gba_server* sv, Request* r, gba_request_info* info) {
  if (info) *info = r->info;
  sv->all.erase(r->ticket);
  auto it = std::find(sv->completed.begin(), sv->completed.end(), r->ticket);
  if (it != sv->completed.end()) sv->completed.erase(it);
  delete r;
}

extern "C" gba_status gba_server_wait(gba_server* sv, int64_t ticket, double timeout_s, gba_request_info* info) {
  if (!sv) return GBA_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  auto it = sv->all.find(ticket);
  if (it == sv->all.end()) return GBA_ERR_INVALID_ARG;
  Request* r = it->second;
  const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(
                                        timeout_s > 0 ? timeout_s : 0.0));
  if (!sv->cv_done.wait_until(lk, until, [&] { return r->done; })) return GBA_ERR_TIMEOUT;
  collect_locked(sv, r, info);
  return GBA_OK;
}

extern "C" gba_status gba_server_next_done(gba_server* sv, double timeout_s, int64_t* ticket,
                                           gba_request_info* info) {
  if (!sv || !ticket) return GBA_ERR_INVALID_ARG;
  std::unique_lock<std::mutex> lk(sv->mu);
  const auto until = Clock::now() + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(
                                        timeout_s > 0 ? timeout_s : 0.0));
  if (!sv->cv_done.wait_until(lk, until, [&] { return !sv->completed.empty(); })) return GBA_ERR_TIMEOUT;
  const int64_t t = sv->completed.front();
  *ticket = t;
  collect_locked(sv, sv->all[t], info);
  return GBA_OK;
}

extern "C" gba_status gba_server_pending(gba_server* sv, int64_t* queued, int64_t* running, int64_t* inflight_bytes) {
  if (!sv) return GBA_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  if (queued) *queued = int64_t(sv->queue.size());
  if (running) *running = sv->submitted - sv->finished - int64_t(sv->queue.size());
  if (inflight_bytes) *inflight_bytes = sv->inflight_bytes;
  return GBA_OK;
}

extern "C" gba_status gba_server_counters(gba_server* sv, int64_t* lane_calls, int64_t* batch_failures,
                                          int64_t* ws_releases, int64_t* regrows, double* lane_ms_max,
                                          double* release_ms_max) {
  if (!sv) return GBA_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> lk(sv->mu);
  if (lane_calls) *lane_calls = sv->lane_calls;
  if (regrows) *regrows = sv->regrows;
  if (batch_failures) *batch_failures = sv->batch_failures;
  if (ws_releases) *ws_releases = sv->ws_releases;
  if (lane_ms_max) *lane_ms_max = sv->lane_ms_max;
  if (release_ms_max) *release_ms_max = sv->release_ms_max;
  return GBA_OK;
}

extern "C" const char* gba_server_last_error(const gba_server* sv) {
  if (!sv || !sv->admin) return "null server";
  return sv->last_failure.empty() ? sv->admin->err.c_str() : sv->last_failure.c_str();
}

extern "C" gba_status gba_server_destroy(gba_server* sv) {
  if (!sv) return GBA_ERR_INVALID_ARG;
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->threads) t.join();
  for (size_t i = 0; i < sv->ctxs.size(); ++i) {
    cudaStreamSynchronize(sv->streams[i]);
    cudaStreamDestroy(sv->streams[i]);
    gba_destroy(sv->ctxs[i]);
  }
  gba_destroy(sv->admin);
  for (auto& kv : sv->all) delete kv.second;
  delete sv;
  return GBA_OK;
}
