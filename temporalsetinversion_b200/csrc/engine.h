// engine.h — the continuous form of serving: requests join a running
// inversion at the next launch step.
//
// The reference re-seeds its one octree and dispatches `main` once per frame
// from the window's event loop (main.rs:1056-1075), and inside the dispatch
// its persistent workgroups keep dequeuing work until the queue drains
// (compute.wgsl:3525-3556).  Here the device work lists are indexed by
// launch step instead of octree level, so scenes at different levels share
// one launch: every step is one refinement launch over every running slot;
// a request admitted between two steps is seeded into the next step's lists
// and runs one octree level per step, while the others continue.  When a
// slot's last level is done its frame end, trace and read-back run on a
// low-priority stream, overlapping the next steps of the other slots (the
// inversion stream has the highest priority, so its latency-bound launches
// get SMs ahead of queued trace blocks).
//
// One engine drives one context; the server's worker thread is its only
// user.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "api_state.h"

namespace tsi_host {

struct EngineDone {
  uint64_t ticket;
  tsi_status status;
  float device_ms;
};

class Engine {
 public:
  explicit Engine(tsi_ctx *c, uint32_t slots);
  ~Engine();
  // Clears the work lists and arenas (the context's plain calls must not
  // run while an engine exists).
  tsi_status start();
  uint32_t free_slots() const { return nfree_; }
  bool scene_busy(const tsi_scene *s) const;
  bool any_inverting() const { return ninv_ > 0; }
  bool any_busy() const { return nfree_ < (uint32_t)slots_.size(); }
  // Takes a free slot for the request; it joins at the next step.  Fails
  // (nothing admitted) when the request's frame would exceed the context's
  // memory budget or its scene has another request running.
  tsi_status admit(const tsi_request &r, uint64_t ticket);
  // One launch step: the joining slots' roots, one refinement launch over
  // all running slots, and the traces of the slots whose last level it is.
  // Keeps at most two steps queued ahead of the device.
  tsi_status step();
  // Requests whose frame is ready (their stats filled in); wait: block
  // until at least one is, when any slot is busy.
  void reap(std::vector<EngineDone> &out, bool wait);
  uint64_t steps() const { return step_; }

 private:
  struct Slot {
    bool busy = false, inverting = false;
    tsi_request req{};
    uint64_t ticket = 0;
    uint64_t first = 0, last = 0;  // launch steps of its inversion
    uint32_t levels = 0;
    cudaEvent_t start = nullptr, done = nullptr;
  };
  tsi_status replan();
  tsi_status finish_slot(uint32_t i, cudaEvent_t after);

  tsi_ctx *c_;
  std::vector<Slot> slots_;
  uint32_t nfree_ = 0, ninv_ = 0;
  uint64_t step_ = 0;
  std::vector<cudaEvent_t> step_ev_;  // ring: end of each step's launch
  std::vector<uint32_t> joining_;     // slots seeded at the next step
  FramePlan plan_;
  std::vector<const tsi_scene *> planned_;  // scenes the plan covers
  std::vector<uint8_t> planned_global_;
  // pinned: descriptors and root records staged per slot, read-back rows
  SceneLaunch *h_desc_ = nullptr;
  TapeRec *h_rec_ = nullptr;
  uint32_t *h_err_ = nullptr;
  unsigned long long *h_stats_ = nullptr;
  SceneCounters *h_ctr_ = nullptr;
  bool ok_ = false;
};

}  // namespace tsi_host
