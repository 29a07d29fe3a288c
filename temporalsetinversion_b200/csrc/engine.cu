// engine.cu — the continuous served form (engine.h).
#include "engine.h"

#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <thread>

namespace tsi_host {

namespace {
constexpr uint32_t kStepRing = 4;  // step events kept; at most two steps run ahead
#define ECK(call)                                        \
  do {                                                   \
    const cudaError_t e_ = (call);                       \
    if (e_ != cudaSuccess) return cuda_err(e_, #call);   \
  } while (0)
}  // namespace

Engine::Engine(tsi_ctx *c, uint32_t slots) : c_(c) {
  const uint32_t n = std::max(1u, std::min({slots, c->max_scenes, (uint32_t)TSI_SEEDS_MAX}));
  slots_.resize(n);
  nfree_ = n;
}

Engine::~Engine() {
  if (c_) {
    cudaSetDevice(c_->device);
    cudaStreamSynchronize(c_->stream);
    cudaStreamSynchronize(c_->trace_stream);
  }
  for (Slot &s : slots_) {
    if (s.start) cudaEventDestroy(s.start);
    if (s.done) cudaEventDestroy(s.done);
  }
  for (cudaEvent_t e : step_ev_) cudaEventDestroy(e);
  cudaFreeHost(h_desc_);
  cudaFreeHost(h_rec_);
  cudaFreeHost(h_err_);
  cudaFreeHost(h_stats_);
  cudaFreeHost(h_ctr_);
}

tsi_status Engine::start() {
  ECK(cudaSetDevice(c_->device));
  ECK(cudaStreamSynchronize(c_->stream));
  ECK(cudaStreamSynchronize(c_->trace_stream));
  const size_t n = slots_.size();
  ECK(cudaMallocHost((void **)&h_desc_, n * sizeof(SceneLaunch)));
  ECK(cudaMallocHost((void **)&h_rec_, n * sizeof(TapeRec)));
  ECK(cudaMallocHost((void **)&h_err_, n * sizeof(uint32_t)));
  ECK(cudaMallocHost((void **)&h_stats_, n * ST_COUNT * sizeof(unsigned long long)));
  ECK(cudaMallocHost((void **)&h_ctr_, n * sizeof(SceneCounters)));
  memset(h_desc_, 0, n * sizeof(SceneLaunch));
  memset(h_rec_, 0, n * sizeof(TapeRec));
  for (Slot &s : slots_) {
    ECK(cudaEventCreate(&s.start));
    ECK(cudaEventCreate(&s.done));
  }
  step_ev_.resize(kStepRing);
  for (cudaEvent_t &e : step_ev_) ECK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  const tsi_status st = replan();
  if (st != TSI_OK) return st;
  // every step's lists and the tape arenas start empty
  const LaunchParams P = make_params(c_, 0, plan_.smem, false);
  ECK(tsi::launch_frame_begin(P, c_->stream));
  ECK(cudaStreamSynchronize(c_->stream));
  ok_ = true;
  return TSI_OK;
}

// Launch geometry over every scene of the context (the plan of a step must
// cover each slot that may run in it); running slots get their descriptors
// again in case a wide working set moved between shared and global memory.
tsi_status Engine::replan() {
  ECK(cudaStreamSynchronize(c_->stream));
  std::vector<tsi_scene *> all(c_->scenes.begin(), c_->scenes.end());
  FramePlan fp;
  if (!all.empty()) {
    const tsi_status st = plan_frame(c_, all.data(), (uint32_t)all.size(), fp);
    if (st != TSI_OK) return st;
  } else {
    tsi_scene *none = nullptr;
    const tsi_status st = plan_frame(c_, &none, 0, fp);
    if (st != TSI_OK) return st;
  }
  plan_ = fp;
  planned_.assign(all.begin(), all.end());
  planned_global_ = fp.global;
  for (uint32_t i = 0; i < slots_.size(); ++i) {
    Slot &s = slots_[i];
    if (!s.inverting) continue;
    const auto it = std::find(planned_.begin(), planned_.end(), s.req.scene);
    const bool g = it != planned_.end() && planned_global_[it - planned_.begin()] != 0;
    h_desc_[i].wide.global = g ? 1u : 0u;
    ECK(cudaMemcpyAsync(c_->d_scenes + i, h_desc_ + i, sizeof(SceneLaunch), cudaMemcpyHostToDevice, c_->stream));
  }
  ECK(cudaStreamSynchronize(c_->stream));
  return TSI_OK;
}

bool Engine::scene_busy(const tsi_scene *sc) const {
  for (const Slot &s : slots_)
    if (s.busy && s.req.scene == sc) return true;
  return false;
}

tsi_status Engine::admit(const tsi_request &r, uint64_t ticket) {
  if (!ok_) return set_err(TSI_ERR_INVALID_ARGUMENT, "engine not started");
  if (!r.scene || r.scene->ctx != c_) return set_err(TSI_ERR_INVALID_ARGUMENT, "request scene of another context");
  if (scene_busy(r.scene)) return set_err(TSI_ERR_BUSY, "the scene has a request running");
  uint32_t i = 0;
  while (i < slots_.size() && slots_[i].busy) ++i;
  if (i == slots_.size()) return set_err(TSI_ERR_BUSY, "no free slot");
  tsi_scene *sc = r.scene;
  if (std::find(planned_.begin(), planned_.end(), sc) == planned_.end()) {
    const tsi_status st = replan();
    if (st != TSI_OK) return st;
  }
  tsi_status st = drain_copy(sc);
  if (st != TSI_OK) return st;
  if (r.uniforms) {
    // the frame buffers are admitted against the context's memory budget
    st = ensure_image(sc, r.uniforms->resolution[0], r.uniforms->resolution[1]);
    if (st != TSI_OK) return st;
    if (r.out && (r.out->width != r.uniforms->resolution[0] || r.out->height != r.uniforms->resolution[1]))
      return set_err(TSI_ERR_BUFFER_TOO_SMALL, "tsi_image size does not match the uniforms' resolution");
  }
  const auto it = std::find(planned_.begin(), planned_.end(), sc);
  const bool g = planned_global_[it - planned_.begin()] != 0;
  fill_launch(sc, i, r.time, r.t0_or_nan, g, h_desc_[i], h_rec_[i]);
  // Under load the narrow path's throughput beats the wide path's latency:
  // a request admitted while others run gets its tape's wide threshold
  // scaled by the number of requests then running (x1 alone, x2 from 2,
  // x4 from 4, x8 from 8).  Results never depend on the threshold.
  const uint32_t running = (uint32_t)slots_.size() - nfree_;
  const uint32_t scale = running >= 8 ? 8u : running >= 4 ? 4u : running >= 2 ? 2u : 1u;
  for (uint32_t *ml : {&h_desc_[i].wide.min_len, &h_desc_[i].wide.deep_min_len})
    *ml = (*ml >= 0xffffffffu / scale) ? 0xffffffffu : *ml * scale;
  Slot &s = slots_[i];
  s.busy = true;
  s.inverting = true;
  s.req = r;
  s.ticket = ticket;
  s.levels = tree_levels(sc->p);
  s.first = step_;
  s.last = step_ + s.levels - 1u;
  joining_.push_back(i);
  --nfree_;
  ++ninv_;
  return TSI_OK;
}

tsi_status Engine::step() {
  if (!ok_) return set_err(TSI_ERR_INVALID_ARGUMENT, "engine not started");
  if (ninv_ == 0) return TSI_OK;
  const uint64_t s = step_;
  // at most two steps queued ahead of the device, so that a request that
  // arrives now joins within about two steps
  if (s >= 2) {
    const cudaEvent_t e = step_ev_[(s - 2) % kStepRing];
    for (uint32_t spin = 0;; ++spin) {
      const cudaError_t q = cudaEventQuery(e);
      if (q == cudaSuccess) break;
      if (q != cudaErrorNotReady) return cuda_err(q, "cudaEventQuery");
      if (spin < 64) std::this_thread::yield();
      else std::this_thread::sleep_for(std::chrono::microseconds(10));
    }
  }
  StepSeeds sd;
  sd.n = (uint32_t)joining_.size();
  uint64_t oldest = s;
  for (uint32_t k = 0; k < sd.n; ++k) {
    const uint32_t i = joining_[k];
    sd.slot[k] = i;
    ECK(cudaEventRecord(slots_[i].start, c_->stream));
    ECK(cudaMemcpyAsync(c_->d_scenes + i, h_desc_ + i, sizeof(SceneLaunch), cudaMemcpyHostToDevice, c_->stream));
    ECK(cudaMemcpyAsync(c_->d_recs + i, h_rec_ + i, sizeof(TapeRec), cudaMemcpyHostToDevice, c_->stream));
  }
  for (const Slot &sl : slots_)
    if (sl.inverting) oldest = std::min(oldest, sl.first);
  sd.oldest = (uint32_t)oldest;
  LaunchParams P = make_params(c_, (uint32_t)slots_.size(), plan_.smem, false);
  P.level_stats = nullptr;
  if (sd.n) ECK(tsi::launch_step_begin(P, (uint32_t)s, sd, c_->stream));
  ECK(tsi::launch_refine(P, (uint32_t)s, plan_.rcap, plan_.grid, kBlock, plan_.smem, c_->stream));
  const cudaEvent_t done = step_ev_[s % kStepRing];
  ECK(cudaEventRecord(done, c_->stream));
  joining_.clear();
  for (uint32_t i = 0; i < slots_.size(); ++i)
    if (slots_[i].inverting && slots_[i].last == s) {
      const tsi_status st = finish_slot(i, done);
      if (st != TSI_OK) return st;
    }
  ++step_;
  return TSI_OK;
}

// After the slot's last level: its frame end (freed bricks become
// allocatable), trace, frame copy and counters, on the trace stream.
tsi_status Engine::finish_slot(uint32_t i, cudaEvent_t after) {
  Slot &s = slots_[i];
  tsi_scene *sc = s.req.scene;
  const cudaStream_t ts = c_->trace_stream;
  ECK(cudaStreamWaitEvent(ts, after, 0));
  const LaunchParams P = make_params(c_, (uint32_t)slots_.size(), plan_.smem, false);
  ECK(tsi::launch_frame_end(P, i, 1, ts));
  s.inverting = false;
  --ninv_;
  if (s.req.uniforms) {
    tsi_status st = enqueue_trace(sc, s.req.uniforms, ts);
    if (st == TSI_OK && s.req.out) st = copy_image_out(sc, s.req.out, ts);
    if (st != TSI_OK) return st;
  }
  ECK(cudaMemcpyAsync(h_err_ + i, c_->d_error + i, sizeof(uint32_t), cudaMemcpyDeviceToHost, ts));
  ECK(cudaMemcpyAsync(h_stats_ + (size_t)i * ST_COUNT, c_->d_stats + (size_t)i * ST_COUNT,
                      ST_COUNT * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ts));
  ECK(cudaMemcpyAsync(h_ctr_ + i, sc->d_ctr, sizeof(SceneCounters), cudaMemcpyDeviceToHost, ts));
  ECK(cudaEventRecord(s.done, ts));
  return TSI_OK;
}

void Engine::reap(std::vector<EngineDone> &out, bool wait) {
  for (;;) {
    bool tracing = false;
    for (uint32_t i = 0; i < slots_.size(); ++i) {
      Slot &s = slots_[i];
      if (!s.busy || s.inverting) continue;
      const cudaError_t q = cudaEventQuery(s.done);
      if (q == cudaErrorNotReady) {
        tracing = true;
        continue;
      }
      EngineDone d{s.ticket, TSI_OK, 0.0f};
      if (q != cudaSuccess) {
        d.status = cuda_err(q, "request completion");
      } else {
        d.status = status_from_error_bits(h_err_[i]);
        cudaEventElapsedTime(&d.device_ms, s.start, s.done);
        if (s.req.stats) {
          fill_stats_row(h_stats_ + (size_t)i * ST_COUNT, h_err_[i], s.req.scene, s.req.stats,
                         (uint64_t)h_ctr_[i].live_bricks * 8u);
          s.req.stats->levels = s.levels;
          s.req.stats->device_ms = d.device_ms;
        }
      }
      out.push_back(d);
      s.busy = false;
      s.req = tsi_request{};
      ++nfree_;
    }
    if (!wait || !out.empty() || !tracing) return;
    std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

}  // namespace tsi_host
