// server.cpp — request queue and worker thread (tsi_server_*).
//
// Continuous form (default): the worker admits queued requests into the
// engine's free slots between launch steps (engine.h) and keeps stepping
// while any slot runs; a request that arrives while others are on the GPU
// joins at the next step.  Static form (TSI_SERVER_STATIC_BATCHES): the
// worker takes, in submission order, the pending requests of distinct
// scenes and runs them as one tsi_batch_run, then the next batch.
//
// In both forms a scene's requests run in submission order (a request waits
// while an earlier one of its scene is running), the queue is bounded, and
// a request's frame is admitted against the context's memory budget when it
// is submitted.  Latency is measured on the host from submission to the
// worker seeing the request's frame ready.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "api_internal.h"
#include "api_state.h"
#include "engine.h"
#include "tsi.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Pending {
  uint64_t ticket;
  tsi_request req;
  Clock::time_point submitted;
};

struct Done {
  tsi_status status;
  float latency_ms;
  std::string error;
};

}  // namespace

struct tsi_server {
  tsi_ctx *ctx = nullptr;
  uint32_t max_batch = 1;
  uint32_t max_queue = 4096;
  bool static_batches = false;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> queue;
  std::unordered_map<uint64_t, Done> done;
  std::unordered_set<uint64_t> live;  // submitted and not yet polled to completion
  std::unordered_map<uint64_t, Clock::time_point> running;  // admitted: submission time
  // frame pixels the queued requests need per scene (memory admission)
  std::unordered_map<const tsi_scene *, uint64_t> want_px;
  uint64_t next_ticket = 1;
  bool stop = false;
  std::vector<float> latencies;
  uint64_t batches = 0, batched_requests = 0;
  std::thread worker;

  void finish(uint64_t ticket, tsi_status st, Clock::time_point submitted, const std::string &err) {
    const float ms = std::chrono::duration<float, std::milli>(Clock::now() - submitted).count();
    done[ticket] = Done{st, ms, err};
    if (st == TSI_OK) latencies.push_back(ms);
  }

  // Device bytes the context's scenes would hold once every queued request
  // has its frame buffers (called with mu held).
  uint64_t committed_bytes() const {
    uint64_t b = tsi_host::scenes_bytes(ctx);
    for (const auto &kv : want_px)
      if (kv.second > kv.first->img_cap) b += (kv.second - kv.first->img_cap) * 32u;
    return b;
  }

  void run_static() {
    std::vector<Pending> batch;
    std::vector<tsi_request> reqs;
    for (;;) {
      {
        std::unique_lock<std::mutex> lock(mu);
        cv_work.wait(lock, [&] { return stop || !queue.empty(); });
        if (stop) break;
        batch.clear();
        std::unordered_set<const tsi_scene *> scenes;
        for (auto it = queue.begin(); it != queue.end() && batch.size() < max_batch;) {
          if (scenes.insert(it->req.scene).second) {
            batch.push_back(*it);
            it = queue.erase(it);
          } else {
            ++it;
          }
        }
      }
      reqs.clear();
      for (const Pending &p : batch) reqs.push_back(p.req);
      const tsi_status st = tsi_batch_run(ctx, reqs.data(), (uint32_t)reqs.size());
      const std::string err = st == TSI_OK ? std::string() : std::string(tsi_last_error());
      {
        std::lock_guard<std::mutex> lock(mu);
        for (const Pending &p : batch) {
          // each request reports its own scene's error bits
          tsi_status own = st;
          if (p.req.stats && st != TSI_OK && st != TSI_ERR_CUDA && st != TSI_ERR_INVALID_ARGUMENT)
            own = p.req.stats->error_flags ? st : TSI_OK;
          finish(p.ticket, own, p.submitted, own == TSI_OK ? std::string() : err);
        }
        ++batches;
        batched_requests += batch.size();
      }
      cv_done.notify_all();
    }
  }

  void run_continuous() {
    tsi_host::Engine eng(ctx, max_batch);
    tsi_status est = eng.start();
    std::vector<tsi_host::EngineDone> completed;
    std::vector<std::pair<uint64_t, std::pair<tsi_status, std::string>>> refused;
    for (;;) {
      refused.clear();
      {
        std::unique_lock<std::mutex> lock(mu);
        if (est != TSI_OK) break;  // the engine cannot run: everything fails below
        if (!stop) {
          // admit queued requests, in submission order, into free slots
          for (auto it = queue.begin(); it != queue.end() && eng.free_slots() > 0;) {
            if (eng.scene_busy(it->req.scene)) {
              ++it;
              continue;
            }
            const tsi_status st = eng.admit(it->req, it->ticket);
            if (st == TSI_OK) {
              running[it->ticket] = it->submitted;
            } else {
              finish(it->ticket, st, it->submitted, tsi_last_error());
              refused.push_back({it->ticket, {st, tsi_last_error()}});
            }
            it = queue.erase(it);
          }
        }
        if (!eng.any_busy()) {
          if (!refused.empty()) cv_done.notify_all();
          if (stop) break;
          cv_work.wait(lock, [&] { return stop || !queue.empty(); });
          continue;
        }
      }
      if (!refused.empty()) cv_done.notify_all();
      if (eng.any_inverting()) {
        est = eng.step();
        std::lock_guard<std::mutex> lock(mu);
        ++batches;
        batched_requests += running.size();
      }
      completed.clear();
      eng.reap(completed, false);
      if (!completed.empty()) {
        std::lock_guard<std::mutex> lock(mu);
        for (const auto &d : completed) {
          auto it = running.find(d.ticket);
          if (it == running.end()) continue;
          finish(d.ticket, d.status, it->second, d.status == TSI_OK ? std::string() : tsi_last_error());
          running.erase(it);
        }
        cv_done.notify_all();
      }
      if (!eng.any_inverting() && eng.any_busy()) {
        // only traces on the device: wait a little for them or for a new request
        std::unique_lock<std::mutex> lock(mu);
        cv_work.wait_for(lock, std::chrono::microseconds(20), [&] { return stop || !queue.empty(); });
      }
    }
    // an engine failure fails what runs; requests still queued are cancelled
    std::lock_guard<std::mutex> lock(mu);
    for (const auto &kv : running) finish(kv.first, est != TSI_OK ? est : TSI_ERR_SHUTDOWN, kv.second, "engine failed");
    running.clear();
    if (est != TSI_OK)
      for (const Pending &p : queue) finish(p.ticket, est, p.submitted, "engine failed");
    else
      for (const Pending &p : queue) finish(p.ticket, TSI_ERR_SHUTDOWN, p.submitted, "server stopped");
    queue.clear();
    cv_done.notify_all();
  }

  void run() {
    if (static_batches) {
      run_static();
      std::lock_guard<std::mutex> lock(mu);
      for (const Pending &p : queue) done[p.ticket] = Done{TSI_ERR_SHUTDOWN, 0.0f, "server stopped"};
      queue.clear();
      cv_done.notify_all();
    } else {
      run_continuous();
    }
  }
};

extern "C" {

TSI_API tsi_status tsi_server_create(tsi_ctx *ctx, const tsi_server_opts *opts, tsi_server **out) {
  if (!ctx || !out) {
    tsi_internal_set_error("null argument");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  *out = nullptr;
  tsi_server *s = new tsi_server();
  s->ctx = ctx;
  const uint32_t cap = tsi_internal_max_scenes(ctx);
  s->max_batch = (opts && opts->max_batch) ? std::min(opts->max_batch, cap) : cap;
  if (s->max_batch == 0) s->max_batch = 1;
  s->static_batches = opts && (opts->flags & TSI_SERVER_STATIC_BATCHES);
  s->max_queue = (opts && opts->max_queue) ? opts->max_queue : 4096u;
  s->worker = std::thread([s] { s->run(); });
  *out = s;
  return TSI_OK;
}

TSI_API tsi_status tsi_server_submit(tsi_server *s, const tsi_request *req, uint64_t *ticket) {
  if (!s || !req || !req->scene || !ticket) {
    tsi_internal_set_error("null argument");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  if (tsi_internal_scene_ctx(req->scene) != s->ctx) {
    tsi_internal_set_error("scene belongs to another context");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  {
    std::lock_guard<std::mutex> lock(s->mu);
    if (s->stop) {
      tsi_internal_set_error("server stopped");
      return TSI_ERR_SHUTDOWN;
    }
    if (s->queue.size() >= s->max_queue) {
      tsi_internal_set_error("server queue full");
      return TSI_ERR_BUSY;
    }
    if (req->uniforms && s->ctx->hbm_budget) {
      // the request's frame buffers against the memory budget, counting
      // what the requests already queued will need
      const uint64_t px = (uint64_t)req->uniforms->resolution[0] * req->uniforms->resolution[1];
      const uint64_t have = std::max<uint64_t>(req->scene->img_cap, s->want_px[req->scene]);
      if (px > have && s->committed_bytes() + (px - have) * 32u > s->ctx->hbm_budget) {
        tsi_internal_set_error("the request's frame would exceed the context's HBM budget");
        return TSI_ERR_OOM;
      }
      s->want_px[req->scene] = std::max(have, px);
    }
    *ticket = s->next_ticket++;
    s->queue.push_back(Pending{*ticket, *req, Clock::now()});
    s->live.insert(*ticket);
  }
  s->cv_work.notify_one();
  return TSI_OK;
}

TSI_API tsi_status tsi_server_poll(tsi_server *s, uint64_t ticket, uint32_t wait_ms, float *latency_ms) {
  if (!s) {
    tsi_internal_set_error("null argument");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  std::unique_lock<std::mutex> lock(s->mu);
  if (!s->live.count(ticket)) {
    tsi_internal_set_error("unknown ticket");
    return TSI_ERR_NOT_FOUND;
  }
  auto ready = [&] { return s->done.count(ticket) != 0; };
  if (!ready() && wait_ms) s->cv_done.wait_for(lock, std::chrono::milliseconds(wait_ms), ready);
  auto it = s->done.find(ticket);
  if (it == s->done.end()) {
    tsi_internal_set_error("request still pending");
    return TSI_ERR_BUSY;
  }
  const Done d = it->second;
  s->done.erase(it);
  s->live.erase(ticket);
  if (latency_ms) *latency_ms = d.latency_ms;
  if (d.status != TSI_OK) tsi_internal_set_error(d.error.c_str());
  return d.status;
}

TSI_API tsi_status tsi_server_stats_get(tsi_server *s, tsi_server_stats *out) {
  if (!s || !out) {
    tsi_internal_set_error("null argument");
    return TSI_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(s->mu);
  *out = tsi_server_stats{};
  out->completed = s->latencies.size();
  out->batches = s->batches;
  out->mean_batch = s->batches ? (float)s->batched_requests / (float)s->batches : 0.0f;
  out->queued = (uint32_t)s->queue.size();
  if (!s->latencies.empty()) {
    std::vector<float> v = s->latencies;
    std::sort(v.begin(), v.end());
    auto q = [&](double f) { return v[std::min(v.size() - 1, (size_t)(f * (double)(v.size() - 1) + 0.5))]; };
    out->p50_ms = q(0.50);
    out->p99_ms = q(0.99);
    out->max_ms = v.back();
  }
  return TSI_OK;
}

TSI_API void tsi_server_destroy(tsi_server *s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  delete s;
}

}  // extern "C"
