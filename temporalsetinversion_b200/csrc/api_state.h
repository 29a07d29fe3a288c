// api_state.h — host-side state behind the C ABI handles (tsi_tape,
// tsi_scene, tsi_ctx) and the helpers the runtime's translation units share
// (api.cu: plain and batched forms; engine.cu: the continuous served form).
// Internal: not installed, not part of include/tsi.h.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <set>
#include <string>
#include <vector>

#include "device_types.h"
#include "trace_params.h"
#include "tsi.h"

namespace tsi {
// overlap: launched as a programmatic dependent of the stream's previous
// kernel (refinement steps, the frame's begin and end kernels)
cudaError_t launch_refine(const LaunchParams &P, uint32_t step, uint32_t rcap, int grid, int block, size_t smem,
                          cudaStream_t st, bool overlap = false);
cudaError_t launch_frame_begin(const LaunchParams &P, cudaStream_t st);
cudaError_t launch_step_begin(const LaunchParams &P, uint32_t step, const StepSeeds &sd, cudaStream_t st);
cudaError_t launch_frame_end(const LaunchParams &P, uint32_t first, uint32_t count, cudaStream_t st,
                             bool overlap = false);
cudaError_t refine_set_smem(size_t bytes);
cudaError_t refine_occupancy(int block, size_t smem, int *blocks_per_sm);
cudaError_t refine_static_smem(size_t *bytes);
}  // namespace tsi

// Host mirror of what one launch sequence leaves on the device: the
// per-step list sizes and the tracer's visit counter.
struct TsiReadback {
  uint32_t item_count[TSI_STEP_RING];
  unsigned long long visits;
};

struct tsi_tape {
  tsi_ctx *ctx = nullptr;
  uint2 *d_code = nullptr;
  uint32_t len = 0;  // instructions after the 4 ARG slots
  uint32_t count = 0, nregs = 0, out_reg = 0, n_minmax = 0;
  uint64_t fwd_cost = 0, rev_cost = 0;
  // bundled form for the wide path (absent when the tape is short)
  uint4 *d_wslots = nullptr;
  uint2 *d_wbundles = nullptr;
  uint32_t *d_wmm = nullptr;
  uint32_t wslots = 0, wbundles = 0, wvalues = 0, wmin_len = 0xffffffffu, wcontrib = 0;
  uint32_t wdeep_level = 0xffffffffu, wdeep_min_len = 0xffffffffu;  // level-dependent threshold (off by default)
  uint32_t narrow_parents = 1;  // parents per narrow item above the leaf level
  uint32_t wprune_level = 0xffffffffu;  // first level whose wide groups prune (0xffffffff: half the levels)
  uint32_t warg_gbase[4] = {TSI_NONE, TSI_NONE, TSI_NONE, TSI_NONE}, warg_gcount[4] = {0, 0, 0, 0};
};

struct tsi_scene {
  tsi_ctx *ctx = nullptr;
  const tsi_tape *tape = nullptr;
  tsi_params p{};
  uint32_t cap_bricks = 0;
  VoxelPoolDev pool{};
  SceneCounters *d_ctr = nullptr;
  uint32_t img_w = 0, img_h = 0;
  uint64_t img_cap = 0;  // pixels the frame buffers hold (frames of any size up to it reuse them)
  float4 *d_rgba = nullptr;
  float *d_depth = nullptr;
  float *d_normal = nullptr;
  // the tracer's arguments: written on the host, uploaded before each trace
  // (a captured upload reads the pinned copy when the graph replays)
  tsi::TraceParams *h_trace = nullptr, *d_trace = nullptr;
  // asynchronous frame read-back (tsi_scene_trace_async): the trace's end,
  // the copy's end on the context's copy stream, and the upload of h_trace
  cudaEvent_t traced = nullptr, copy_done = nullptr, trace_up = nullptr;
  bool copy_pending = false, trace_up_pending = false;
  uint64_t bytes = 0;
};

struct tsi_ctx {
  int device = 0;
  int sm_count = 0;
  size_t smem_per_sm = 0, smem_reserved = 0;  // shared memory of an SM, reserved per block
  cudaStream_t stream = nullptr;        // inversions (highest priority) and plain traces
  cudaStream_t trace_stream = nullptr;  // traces of the batched form (lowest priority)
  cudaStream_t copy_stream = nullptr;   // frame read-back of tsi_scene_trace_async
  uint32_t max_scenes = 64;
  SceneLaunch *d_scenes = nullptr, *h_scenes = nullptr;
  TapeRec *d_recs = nullptr, *h_recs = nullptr;
  uint32_t rec_cap = 0;
  unsigned long long *d_rec_count = nullptr, *d_rec_low = nullptr;
  uint2 *d_code = nullptr;
  unsigned long long *d_code_count = nullptr, *d_code_low = nullptr;
  unsigned long long *d_step_code_start = nullptr, *d_step_rec_start = nullptr;
  uint64_t code_cap = 0;
  WorkItem *d_items[2] = {nullptr, nullptr};
  uint32_t item_cap = 0;
  uint32_t *d_item_count = nullptr, *d_item_cursor = nullptr;
  WorkItem *d_witems[2] = {nullptr, nullptr};
  uint32_t *d_witem_count = nullptr, *d_witem_cursor = nullptr;
  // wide path: per-cell hand-over to the group (per step parity) and, for
  // tapes whose working set exceeds shared memory, per-block scratch
  CellInfo *d_cell_info[2] = {nullptr, nullptr};
  uint32_t *d_cell_bits[2] = {nullptr, nullptr};
  size_t cell_arena_bytes = 0;  // of each parity's info + bits
  uint32_t witem_cap = 0, bm_words = 0;
  unsigned char *d_wscratch = nullptr;
  size_t wscratch_bytes = 0, wscratch_stride = 0;
  size_t wide_smem_bytes = 0;  // shared-memory budget of a wide cell (0: keep the narrow occupancy)
  uint64_t hbm_budget = 0;     // bytes the scenes may hold together (0: no limit)

  uint2 *d_dealloc[2] = {nullptr, nullptr};
  uint32_t dealloc_cap = 0;
  uint32_t *d_dealloc_count = nullptr, *d_dealloc_cursor = nullptr;
  float4 *d_log = nullptr;
  uint2 *d_dec = nullptr;
  uint32_t slice_len = 0;
  uint32_t max_warps = 0;
  float4 *d_log_overflow = nullptr;
  unsigned long long *d_log_used = nullptr;
  uint64_t log_overflow_cap = 0;
  uint32_t *d_error = nullptr;         // [max_scenes] error bits per scene slot
  uint32_t *d_error_sticky = nullptr;  // error words of asynchronous inversions since the last wait
  // the upload of h_scenes/h_recs of the last launch sequence: the host may
  // rewrite them only after it ran (inversions queued without waiting)
  cudaEvent_t launch_up = nullptr;
  bool launch_up_pending = false;
  unsigned long long *d_stats = nullptr;        // [max_scenes][ST_COUNT]
  unsigned long long *d_level_stats = nullptr;  // [TSI_STEP_RING][ST_COUNT]
  unsigned long long *d_visits = nullptr;
  TsiReadback *h_rb = nullptr;
  // per-scene rows read back after a launch sequence (pinned, rb_rows rows)
  uint32_t *h_err = nullptr;
  unsigned long long *h_stats = nullptr;
  uint32_t rb_rows = 0;
  // per-level profile of the last inversion (events when profiling is on)
  bool profile_levels = false;
  std::vector<cudaEvent_t> level_events;
  uint32_t last_levels = 0;
  // end of each level's refinement launch, for the traces of the batched
  // form (a scene's trace starts when its own last level is done)
  std::vector<cudaEvent_t> fork_events;
  cudaEvent_t join_event = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr, ev2 = nullptr;
  // scratch for tsi_tape_eval_boxes
  void *d_scratch = nullptr;
  size_t scratch_bytes = 0;
  uint32_t watchdog = 0;
  // objects created on this context, released by tsi_destroy if still alive
  std::set<tsi_tape *> tapes;
  std::set<tsi_scene *> scenes;
};

namespace tsi_host {

constexpr int kBlock = 256;
constexpr int kWarpsPerBlock = kBlock / 32;

tsi_status set_err(tsi_status s, const std::string &msg);
tsi_status cuda_err(cudaError_t e, const char *what);
tsi_status status_from_error_bits(uint32_t e);
uint32_t tree_levels(const tsi_params &p);
void fill_launch(tsi_scene *s, uint32_t slot, float time, float t0_or_nan, bool wide_global, SceneLaunch &L,
                 TapeRec &R);
LaunchParams make_params(tsi_ctx *c, uint32_t n_scenes, size_t dyn_smem, bool sticky);

// Launch geometry of one step (or frame) for a set of scenes.
struct FramePlan {
  uint32_t lmax = 0, rcap = 4;
  size_t smem = 0;
  int grid = 0;
  std::vector<uint8_t> global;  // per scene: wide cells in the global scratch
};
tsi_status plan_frame(tsi_ctx *c, tsi_scene *const *scenes, uint32_t n, FramePlan &fp);

bool capturing(tsi_ctx *c);
tsi_status drain_copy(tsi_scene *s);
uint64_t scenes_bytes(const tsi_ctx *c);
tsi_status ensure_image(tsi_scene *s, uint32_t w, uint32_t h);
// The tracer's launch for these uniforms on stream st (the scene's frame
// buffers, its pinned TraceParams uploaded on st first).
tsi_status enqueue_trace(tsi_scene *s, const tsi_uniforms *u, cudaStream_t st);
tsi_status copy_image_out(tsi_scene *s, tsi_image *out, cudaStream_t st);
// Grows the pinned per-scene readback rows to at least n.
tsi_status ensure_readback_rows(tsi_ctx *c, uint32_t n);
// tsi_stats of one scene from its readback row (and the launch's list sizes).
void fill_stats(const tsi_ctx *c, uint32_t row, const tsi_scene *s, tsi_stats *st, uint64_t voxels_live);
// tsi_stats of one scene from a stats row (ST_COUNT counters) and error word.
void fill_stats_row(const unsigned long long *row, uint32_t err, const tsi_scene *s, tsi_stats *st,
                    uint64_t voxels_live);

}  // namespace tsi_host
