// server.cpp — request queue and worker thread over tsi_batch_run.
//
// The worker takes, in submission order, the pending requests of distinct
// scenes (at most max_batch) and runs them as one fused launch sequence; a
// request whose scene is already in the batch waits for a later one, so a
// scene's frames run in submission order.  Latency is measured on the host
// from submission to the end of the batch that ran the request.
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
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Pending> queue;
  std::unordered_map<uint64_t, Done> done;
  std::unordered_set<uint64_t> live;  // submitted and not yet polled to completion
  uint64_t next_ticket = 1;
  bool stop = false;
  std::vector<float> latencies;
  uint64_t batches = 0, batched_requests = 0;
  std::thread worker;

  void run() {
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
      const Clock::time_point now = Clock::now();
      {
        std::lock_guard<std::mutex> lock(mu);
        for (const Pending &p : batch) {
          const float ms = std::chrono::duration<float, std::milli>(now - p.submitted).count();
          done[p.ticket] = Done{st, ms, err};
          latencies.push_back(ms);
        }
        ++batches;
        batched_requests += batch.size();
      }
      cv_done.notify_all();
    }
    // cancel what is still queued
    std::lock_guard<std::mutex> lock(mu);
    for (const Pending &p : queue) done[p.ticket] = Done{TSI_ERR_SHUTDOWN, 0.0f, "server stopped"};
    queue.clear();
    cv_done.notify_all();
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
