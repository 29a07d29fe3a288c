// api.cu — host runtime behind include/tsi.h.
//
// Replaces the reference's host side of the hot path: State::new buffer
// setup (src/main.rs:97-303), State::compute (main.rs:724-820: first_eval
// reseed, one `main` dispatch, blocking timestamp readback) and
// State::render's rt_main dispatch (main.rs:639-656).  All device state of a
// scene (voxel pool, counters, frame buffers) stays resident in HBM between
// calls; only the per-frame launch descriptor goes up and the counters come
// back.
#include <cuda_runtime.h>
#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "api_internal.h"
#include "api_state.h"
#include "composite.h"
#include "device_types.h"
#include "ir_lower.h"
#include "tape_compile.h"
#include "trace_params.h"
#include "tsi.h"

namespace tsi {
cudaError_t launch_evalbox(bool directed, const uint2 *code, uint32_t len, uint32_t nregs, uint32_t out_reg,
                           uint32_t n, const float *boxes, int reverse, float *out, float2 *regs, float4 *log,
                           cudaStream_t st);
cudaError_t launch_math(int which, uint32_t n, const float *a, const float *b, float *out, cudaStream_t st);
}  // namespace tsi

using namespace tsi;
using namespace tsi_host;

namespace {

thread_local std::string g_last_error;

#define CK(call)                                                                     \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) {                                                         \
      g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);             \
      cudaGetLastError(); /* clear it, or the next launch check reports it again */  \
      return TSI_ERR_CUDA;                                                           \
    }                                                                                \
  } while (0)

template <typename T>
cudaError_t dalloc(T **p, size_t count) {
  *p = nullptr;
  if (count == 0) return cudaSuccess;
  return cudaMalloc((void **)p, count * sizeof(T));
}

}  // namespace

struct tsi_batch_graph {
  tsi_ctx *ctx = nullptr;
  const tsi_request *user = nullptr;  // the caller's requests, re-read at every replay
  std::vector<tsi_request> reqs;      // as captured
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  bool launched = false;
  std::vector<uint8_t> global;  // per request: wide cells in the global scratch
};

namespace tsi_host {

tsi_status set_err(tsi_status s, const std::string &msg) {
  g_last_error = msg;
  return s;
}

tsi_status cuda_err(cudaError_t e, const char *what) {
  if (e == cudaSuccess) return TSI_OK;
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return TSI_ERR_CUDA;
}

LaunchParams make_params(tsi_ctx *c, uint32_t n_scenes, size_t dyn_smem, bool sticky) {
  LaunchParams P{};
  P.scenes = c->d_scenes;
  P.n_scenes = n_scenes;
  P.rec_cap = c->rec_cap;
  P.recs = c->d_recs;
  P.rec_count = c->d_rec_count;
  P.rec_low = c->d_rec_low;
  P.rec_base = c->max_scenes;
  P.code_arena = c->d_code;
  P.code_count = c->d_code_count;
  P.code_low = c->d_code_low;
  P.code_cap = c->code_cap;
  P.step_code_start = c->d_step_code_start;
  P.step_rec_start = c->d_step_rec_start;
  P.items[0] = c->d_items[0];
  P.items[1] = c->d_items[1];
  P.item_count = c->d_item_count;
  P.item_cursor = c->d_item_cursor;
  P.item_cap = c->item_cap;
  P.witems[0] = c->d_witems[0];
  P.witems[1] = c->d_witems[1];
  P.witem_count = c->d_witem_count;
  P.witem_cursor = c->d_witem_cursor;
  P.witem_cap = c->witem_cap;
  P.bm_words = c->bm_words;
  P.wscratch = c->d_wscratch;
  P.wscratch_stride = c->wscratch_stride;
  P.dyn_smem = (uint32_t)dyn_smem;
  P.error_sticky = sticky ? c->d_error_sticky : nullptr;
  for (int q = 0; q < 2; ++q) {
    P.cell_info[q] = c->d_cell_info[q];
    P.cell_bits[q] = c->d_cell_bits[q];
  }

  P.dealloc_cap = c->dealloc_cap;
  P.dealloc[0] = c->d_dealloc[0];
  P.dealloc[1] = c->d_dealloc[1];
  P.dealloc_count = c->d_dealloc_count;
  P.dealloc_cursor = c->d_dealloc_cursor;
  P.log_slices = c->d_log;
  P.dec_slices = c->d_dec;
  P.slice_len = c->slice_len;
  P.log_overflow = c->d_log_overflow;
  P.log_overflow_used = c->d_log_used;
  P.log_overflow_cap = c->log_overflow_cap;
  P.error = c->d_error;
  P.stats = c->d_stats;
  P.level_stats = c->d_level_stats;
  return P;
}

tsi_status status_from_error_bits(uint32_t e) {
  if (e & EB_OOM) return set_err(TSI_ERR_OOM, "voxel pool exhausted");
  if (e & EB_LOG_OOM) return set_err(TSI_ERR_OOM, "reverse-AD log arena exhausted");
  if (e & EB_QUEUE_FULL) return set_err(TSI_ERR_QUEUE_FULL, "work list capacity exceeded");
  if (e & EB_WATCHDOG) return set_err(TSI_ERR_WATCHDOG, "bounded device wait expired");
  if (e & EB_SMEM) return set_err(TSI_ERR_TAPE_TOO_WIDE, "wide cell larger than the launch's shared memory");
  return TSI_OK;
}

// Levels of parents a frame expands: the root, then every level whose cells
// are wider than epsilon (localsubdiv for the default root box, fewer for a
// subtree's root).  Capped at TSI_MAX_LEVELS, which scene creation checks.
uint32_t tree_levels(const tsi_params &p) {
  const float eps = 10.0f * ldexpf(1.0f, -p.localsubdiv);
  float w = 0.0f;
  for (int a = 0; a < 3; ++a) w = std::max(w, p.root_hi[a] - p.root_lo[a]);
  uint32_t l = 0;
  while (w > eps && l < TSI_MAX_LEVELS) {
    w = w / 2.0f;
    ++l;
  }
  return std::max(1u, l);
}

void fill_launch(tsi_scene *s, uint32_t slot, float time, float t0_or_nan, bool wide_global, SceneLaunch &L,
                 TapeRec &R) {
  const tsi_params &p = s->p;
  L.pool = s->pool;
  L.ctr = s->d_ctr;
  L.eps = 10.0f * ldexpf(1.0f, -p.localsubdiv);  // compute.wgsl:3521 (exact power of two)
  L.delta = p.delta;
  L.fast_thresh = p.delta * p.fast_multiplier;
  L.time = time;
  L.t0 = (t0_or_nan != t0_or_nan) ? time - p.swept_dt : t0_or_nan;
  uint32_t f = 0;
  if (p.pointsample) f |= SF_POINTSAMPLE;
  if (p.fastenabled) f |= SF_FASTENABLED;
  if (p.lipschitz_corrected) f |= SF_LIPSCHITZ;
  if (p.swept_volume) f |= SF_SWEPT;
  if (!p.fast_normals && p.normal_viz) f |= SF_ALWAYS_DERIV;
  if (p.pruning) f |= SF_PRUNING;
  if (p.rounding_mode == TSI_ROUND_DIRECTED) f |= SF_DIRECTED;
  L.flags = f;
  L.root_rec = slot;
  L.levels = tree_levels(p);
  L.full_len = s->tape->len;
  L.narrow_parents = s->tape->narrow_parents;
  L.wide.slots = s->tape->d_wslots;
  L.wide.bundles = s->tape->d_wbundles;
  L.wide.narrow_mm = s->tape->d_wmm;
  L.wide.nslots = s->tape->wslots;
  L.wide.nbundles = s->tape->wbundles;
  L.wide.nvalues = s->tape->wvalues;
  // a tape without a bundled form never sends a cell to the wide path,
  // whatever thresholds were set on it
  const bool has_wide = s->tape->d_wslots != nullptr && s->tape->wbundles > 0;
  L.wide.min_len = has_wide ? s->tape->wmin_len : 0xffffffffu;
  L.wide.deep_level = s->tape->wdeep_level;
  L.wide.deep_min_len = has_wide ? s->tape->wdeep_min_len : 0xffffffffu;
  L.wide.ncontrib = s->tape->wcontrib;
  L.wide.prune_level = s->tape->wprune_level != 0xffffffffu ? s->tape->wprune_level : tree_levels(p) / 2u;
  L.wide.global = wide_global ? 1u : 0u;
  for (int q = 0; q < 4; ++q) {
    L.wide.arg_gbase[q] = s->tape->warg_gbase[q];
    L.wide.arg_gcount[q] = s->tape->warg_gcount[q];
  }
  R.code = s->tape->d_code;
  R.len = s->tape->len;
  R.nregs = s->tape->nregs;
  R.out_reg = s->tape->out_reg;
  R.n_minmax = s->tape->n_minmax;
  R.t_lo = -INFINITY;
  R.t_hi = INFINITY;
  R.parent = TSI_NONE;
  R.fwd_cost = (uint32_t)std::min<uint64_t>(s->tape->fwd_cost, 0xffffffffull);
  R.rev_cost = (uint32_t)std::min<uint64_t>(s->tape->rev_cost, 0xffffffffull);
  R.c_lo = -INFINITY;
  R.c_hi = INFINITY;
  R.c_level = TSI_NONE;
}

// Shared-memory working set of one wide cell (the device's cell_layout):
// values and sensitivities (8 bytes per SSA value each), contribution
// records, decision bits, liveness flags.
size_t wide_cell_bytes(size_t nvalues, size_t ncontrib, size_t bm_words) {
  return 16 * nvalues + ((ncontrib * 8 + 15) & ~size_t(15)) + ((bm_words * 4 + 15) & ~size_t(15)) +
         ((nvalues + 15) & ~size_t(15));
}
// Tapes whose cell working set exceeds this stay on the narrow path (the
// block also needs its static shared memory and room for a second block's
// decision bits is kept).
constexpr size_t kWideCellMaxBytes = 192u << 10;
// Beyond this a tape has no wide form (global scratch per block of the grid).
constexpr size_t kWideCellMaxGlobalBytes = 8u << 20;


// Sizes the launch for these scenes and grows the wide path's arenas (no
// allocation when they are large enough, so a plan made once before stream
// capture holds inside it).
tsi_status plan_frame(tsi_ctx *c, tsi_scene *const *scenes, uint32_t n, FramePlan &fp) {
  uint32_t rmax = 4, mm_max = 0, bm_words = 1;
  size_t cell_bytes = 0;
  fp.lmax = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const tsi_tape *t = scenes[i]->tape;
    fp.lmax = std::max(fp.lmax, tree_levels(scenes[i]->p));
    rmax = std::max(rmax, t->nregs);
    if (t->d_wslots) mm_max = std::max(mm_max, t->n_minmax);
  }
  bm_words = std::max(1u, (mm_max + 15u) / 16u);
  fp.rcap = (rmax + 3u) & ~3u;
  const size_t regfile = (size_t)kWarpsPerBlock * fp.rcap * 32u * sizeof(float2);
  // A wide cell keeps its working set in shared memory when it fits the
  // budget: by default what leaves the narrow path's blocks per SM as the
  // register files alone allow; larger working sets use the global scratch.
  size_t budget = c->wide_smem_bytes;
  if (budget == 0) {
    CK(refine_set_smem(regfile));
    int bps0 = 0;
    CK(refine_occupancy(kBlock, regfile, &bps0));
    if (bps0 < 1) return set_err(TSI_ERR_TAPE_TOO_WIDE, "register file does not fit in shared memory");
    size_t stat = 0;
    CK(refine_static_smem(&stat));
    const size_t per_block = c->smem_per_sm / (size_t)bps0;
    budget = per_block > stat + c->smem_reserved ? ((per_block - stat - c->smem_reserved) & ~size_t(127)) : 0;
  }
  budget = std::min(budget, kWideCellMaxBytes);
  size_t gm_bytes = 0;  // largest working set kept in the global scratch
  fp.global.assign(n, 0);
  for (uint32_t i = 0; i < n; ++i) {
    const tsi_tape *t = scenes[i]->tape;
    if (!t->d_wslots) continue;
    const size_t b = wide_cell_bytes(t->wvalues, t->wcontrib, bm_words);
    if (b > budget) {
      fp.global[i] = 1;
      gm_bytes = std::max(gm_bytes, b);
    } else {
      cell_bytes = std::max(cell_bytes, b);
    }
  }
  // the wide cell's working set and the narrow register files share the
  // dynamic shared memory (the phases run one after the other)
  fp.smem = std::max(regfile, cell_bytes);
  CK(refine_set_smem(fp.smem));
  int bps = 0;
  CK(refine_occupancy(kBlock, fp.smem, &bps));
  if (bps < 1) return set_err(TSI_ERR_TAPE_TOO_WIDE, "register file does not fit in shared memory");
  fp.grid = std::min<int>(bps * c->sm_count, (int)(c->max_warps / kWarpsPerBlock));
  // one working-set slice per block of the persistent grid
  if (gm_bytes) {
    const size_t stride = (gm_bytes + 255) & ~size_t(255);
    const size_t need = stride * (size_t)fp.grid;
    if (need > c->wscratch_bytes) {
      cudaFree(c->d_wscratch);
      c->d_wscratch = nullptr;
      c->wscratch_bytes = 0;
      CK(dalloc(&c->d_wscratch, need));
      c->wscratch_bytes = need;
    }
    c->wscratch_stride = stride;
  }
  // hand-over arenas: 64 MB per level parity, as many wide items as fit
  const size_t per_item = 8 * (sizeof(CellInfo) + (size_t)bm_words * 4);
  const size_t arena = std::max<size_t>(64u << 20, c->cell_arena_bytes);
  if (arena > c->cell_arena_bytes || !c->d_cell_info[0]) {
    for (int q = 0; q < 2; ++q) {
      cudaFree(c->d_cell_info[q]);
      c->d_cell_info[q] = nullptr;
    }
    c->cell_arena_bytes = 0;
    for (int q = 0; q < 2; ++q) CK(dalloc((unsigned char **)&c->d_cell_info[q], arena));
    c->cell_arena_bytes = arena;
  }
  c->bm_words = bm_words;
  c->witem_cap = (uint32_t)std::min<size_t>(c->item_cap, c->cell_arena_bytes / per_item);
  for (int q = 0; q < 2; ++q)
    c->d_cell_bits[q] = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(c->d_cell_info[q]) +
                                                     (size_t)c->witem_cap * 8 * sizeof(CellInfo));
  return TSI_OK;
}

// One frame of set inversion for n scenes, all levels in one launch sequence.
bool capturing(tsi_ctx *c);

// With fork = true the end of every level's launch is recorded in
// c->fork_events[level] (the batched form starts each scene's trace there).
tsi_status enqueue_invert(tsi_ctx *c, tsi_scene *const *scenes, const float *times, const float *t0s, uint32_t n,
                          bool sticky = false, bool fork = false) {
  if (n == 0) return TSI_OK;
  if (n > c->max_scenes) return set_err(TSI_ERR_INVALID_ARGUMENT, "too many scenes in one launch");
  FramePlan fp;
  tsi_status pst = plan_frame(c, scenes, n, fp);
  if (pst != TSI_OK) return pst;
  const bool cap = capturing(c);
  if (c->launch_up_pending && !cap) {
    CK(cudaEventSynchronize(c->launch_up));
    c->launch_up_pending = false;
  }
  for (uint32_t i = 0; i < n; ++i)
    fill_launch(scenes[i], i, times[i], t0s[i], fp.global[i] != 0, c->h_scenes[i], c->h_recs[i]);
  const uint32_t lmax = fp.lmax, rcap = fp.rcap;
  const size_t smem = fp.smem;
  const int grid = fp.grid;
  CK(cudaMemcpyAsync(c->d_scenes, c->h_scenes, n * sizeof(SceneLaunch), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_recs, c->h_recs, n * sizeof(TapeRec), cudaMemcpyHostToDevice, c->stream));
  if (!cap) {
    CK(cudaEventRecord(c->launch_up, c->stream));
    c->launch_up_pending = true;
  }
  CK(cudaMemsetAsync(c->d_error, 0, n * sizeof(uint32_t), c->stream));
  CK(cudaMemsetAsync(c->d_stats, 0, (size_t)n * ST_COUNT * sizeof(unsigned long long), c->stream));
  CK(cudaMemsetAsync(c->d_level_stats, 0, TSI_STEP_RING * ST_COUNT * sizeof(unsigned long long), c->stream));
  const LaunchParams P = make_params(c, n, fp.smem, sticky);
  CK(launch_frame_begin(P, c->stream));
  const bool prof = c->profile_levels && c->level_events.size() >= lmax + 1;
  // Each level's launch overlaps the end of the one before (programmatic
  // dependent launch: its blocks take the SMs the last level's blocks leave
  // and wait for it on the device), unless events sit between the levels
  // (per-level timing, the batched form's trace forks) or a graph is being
  // captured.
  const bool overlap = !cap && !prof && !fork;
  for (uint32_t level = 0; level < lmax; ++level) {
    if (prof) CK(cudaEventRecord(c->level_events[level], c->stream));
    CK(launch_refine(P, level, rcap, grid, kBlock, smem, c->stream, overlap));
    if (fork) CK(cudaEventRecord(c->fork_events[level], c->stream));
  }
  if (prof) CK(cudaEventRecord(c->level_events[lmax], c->stream));
  c->last_levels = lmax;
  CK(launch_frame_end(P, 0, n, c->stream, overlap));
  return TSI_OK;
}

tsi_status ensure_readback_rows(tsi_ctx *c, uint32_t n) {
  if (n <= c->rb_rows) return TSI_OK;
  if (capturing(c)) return set_err(TSI_ERR_BUSY, "readback rows grown during graph capture");
  CK(cudaStreamSynchronize(c->stream));
  cudaFreeHost(c->h_err);
  cudaFreeHost(c->h_stats);
  c->h_err = nullptr;
  c->h_stats = nullptr;
  c->rb_rows = 0;
  const uint32_t rows = std::max(n, 64u);
  CK(cudaMallocHost((void **)&c->h_err, rows * sizeof(uint32_t)));
  CK(cudaMallocHost((void **)&c->h_stats, (size_t)rows * ST_COUNT * sizeof(unsigned long long)));
  memset(c->h_err, 0, rows * sizeof(uint32_t));
  memset(c->h_stats, 0, (size_t)rows * ST_COUNT * sizeof(unsigned long long));
  c->rb_rows = rows;
  return TSI_OK;
}

// Error words and stats rows of the launch's n scenes into readback rows
// row0 .. row0 + n - 1, and the list sizes of its steps.
tsi_status enqueue_readback(tsi_ctx *c, uint32_t n, uint32_t row0 = 0) {
  if (row0 + n > c->rb_rows) return set_err(TSI_ERR_INVALID_ARGUMENT, "readback rows not reserved");
  CK(cudaMemcpyAsync(c->h_err + row0, c->d_error, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_stats + (size_t)row0 * ST_COUNT, c->d_stats, (size_t)n * ST_COUNT * sizeof(unsigned long long),
                     cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(c->h_rb->item_count, c->d_item_count, sizeof(c->h_rb->item_count), cudaMemcpyDeviceToHost,
                     c->stream));
  return TSI_OK;
}

void fill_stats(const tsi_ctx *c, uint32_t row, const tsi_scene *s, tsi_stats *st, uint64_t voxels_live) {
  if (!st) return;
  fill_stats_row(c->h_stats + (size_t)row * ST_COUNT, c->h_err[row], s, st, voxels_live);
  uint64_t hw = 0;
  uint32_t levels = 0;
  for (uint32_t l = 0; l < TSI_STEP_RING; ++l) {
    hw = std::max<uint64_t>(hw, c->h_rb->item_count[l]);
    if (c->h_rb->item_count[l]) levels = l + 1;
  }
  st->items_high_water = hw;
  st->levels = levels;
}

void fill_stats_row(const unsigned long long *r, uint32_t err, const tsi_scene *s, tsi_stats *st,
                    uint64_t voxels_live) {
  if (!st) return;
  memset(st, 0, sizeof(*st));
  st->parents_expanded = r[ST_PARENTS];
  st->cells_evaluated = r[ST_EVAL];
  st->cells_reverse = r[ST_REVERSE];
  st->cells_skipped = r[ST_SKIPPED];
  st->cells_ambiguous = r[ST_AMBIG];
  st->cells_empty = r[ST_EMPTY];
  st->cells_full = r[ST_FULL];
  st->cells_enqueued = r[ST_ENQUEUED];
  st->cells_reused = r[ST_REUSED];
  st->instr_forward = r[ST_INSTR_FWD];
  st->instr_reverse = r[ST_INSTR_REV];
  st->instr_full_equiv = r[ST_INSTR_FULL];
  st->fp32_ops = r[ST_FP32];
  st->bricks_allocated = r[ST_BRICK_ALLOC];
  st->bricks_freed = r[ST_BRICK_FREE];
  st->tape_words = r[ST_TAPE_WORDS];
  st->prune_fallbacks = r[ST_PRUNE_FALLBACK];
  if (s) {
    st->fp32_ops_full_fwd = r[ST_EVAL] * s->tape->fwd_cost;
    st->fp32_ops_full_rev = r[ST_REVERSE] * s->tape->rev_cost;
    if (s->p.pruning && s->tape->nregs > TSI_PRUNE_MAX_REGS) st->cells_unpruned_regs = r[ST_EVAL];
  }
  st->voxels_live = voxels_live;
  st->error_flags = err;
}

// tsi_stats summed over readback rows 0 .. n-1 (a batch or graph replay as
// a whole); the error word is the or of the rows'.
void fill_stats_sum(const tsi_ctx *c, tsi_scene *const *scenes, uint32_t n, tsi_stats *st) {
  if (!st) return;
  tsi_stats acc;
  memset(&acc, 0, sizeof(acc));
  for (uint32_t i = 0; i < n; ++i) {
    tsi_stats one;
    fill_stats(c, i, scenes ? scenes[i] : nullptr, &one, 0);
    uint64_t *a = &acc.parents_expanded;
    const uint64_t *b = &one.parents_expanded;
    for (size_t k = 0; k < (offsetof(tsi_stats, levels) - offsetof(tsi_stats, parents_expanded)) / sizeof(uint64_t); ++k)
      a[k] += b[k];
    acc.items_high_water = one.items_high_water;
    acc.levels = one.levels;
    acc.error_flags |= one.error_flags;
  }
  *st = acc;
}

uint32_t readback_error_or(const tsi_ctx *c, uint32_t n) {
  uint32_t e = 0;
  for (uint32_t i = 0; i < n; ++i) e |= c->h_err[i];
  return e;
}

// camera of rt_main (compute.wgsl:4651-4685), computed once per frame
void rotation_matrix(const float axis_in[3], float angle, float out[16]) {
  float l = sqrtf((axis_in[0] * axis_in[0] + axis_in[1] * axis_in[1]) + axis_in[2] * axis_in[2]);
  const float ax = axis_in[0] / l, ay = axis_in[1] / l, az = axis_in[2] / l;
  const float s = sinf(angle), cc = cosf(angle), oc = 1.0f - cc;
  const float m[16] = {oc * ax * ax + cc, oc * ax * ay - az * s, oc * az * ax + ay * s, 0.0f,
                       oc * ax * ay + az * s, oc * ay * ay + cc, oc * ay * az - ax * s, 0.0f,
                       oc * az * ax - ay * s, oc * ay * az + ax * s, oc * az * az + cc, 0.0f,
                       0.0f, 0.0f, 0.0f, 1.0f};
  memcpy(out, m, sizeof(m));
}

void matmul4(const float a[16], const float b[16], float out[16]) {
  float r[16];
  for (int col = 0; col < 4; ++col)
    for (int row = 0; row < 4; ++row) {
      float s = a[0 * 4 + row] * b[col * 4 + 0];
      s = s + a[1 * 4 + row] * b[col * 4 + 1];
      s = s + a[2 * 4 + row] * b[col * 4 + 2];
      s = s + a[3 * 4 + row] * b[col * 4 + 3];
      r[col * 4 + row] = s;
    }
  memcpy(out, r, sizeof(r));
}

void make_camera(const tsi_params &p, const tsi_uniforms &u, TraceParams &T) {
  float view[16];
  memcpy(view, u.view_matrix, sizeof(view));
  float eye[3] = {view[12], view[13], view[14]};
  const float PI = 3.1415927410125732f;
  if (p.scene_id == 3) {
    eye[0] = eye[0] + 7.7f;
    eye[1] = eye[1] + -2.21f;
    eye[2] = eye[2] + 7.7f;
    const float ax[3] = {0.0f, 1.0f, 0.0f};
    float r[16];
    rotation_matrix(ax, (PI / 4.0f) * 3.0f, r);
    matmul4(r, view, view);
  } else if (p.scene_id == 4) {
    eye[0] = eye[0] + 0.0f;
    eye[1] = eye[1] + -0.78f;
    eye[2] = eye[2] + -7.0f;
  } else if (p.scene_id == 5) {
    eye[0] = eye[0] + 7.13f;
    eye[1] = eye[1] + 2.14f;
    eye[2] = eye[2] + -5.6f;
    float r[16];
    const float ax1[3] = {0.0f, 1.0f, 0.0f};
    rotation_matrix(ax1, PI / 4.0f, r);
    matmul4(r, view, view);
    const float ax2[3] = {-1.0f, 0.0f, -1.0f};
    rotation_matrix(ax2, (PI / 4.0f) * 0.45f, r);
    matmul4(r, view, view);
  }
  memcpy(T.eye, eye, sizeof(eye));
  memcpy(T.m, view, sizeof(view));
  const float fov = 90.0f;
  const float rad = fov * 0.017453292519943295474f;
  T.zdist = (float)u.resolution[1] / tanf(rad / 2.0f);
  T.yshift = (p.scene_id == 0) ? (float)u.resolution[1] * 0.32f : 0.0f;
  T.W = u.resolution[0];
  T.H = u.resolution[1];
  T.time = u.time;
  T.rendermode = u.rendermode;
  T.normal_viz = p.normal_viz ? 1u : 0u;
  T.darken = p.octree_darken_factor;
}

// Whether the context's stream is being captured into a graph (no host
// waits and no outside events then).
bool capturing(tsi_ctx *c) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(c->stream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

// Host wait for the scene's pending asynchronous frame copy.
tsi_status drain_copy(tsi_scene *s) {
  if (s->copy_pending) {
    CK(cudaEventSynchronize(s->copy_done));
    s->copy_pending = false;
  }
  return TSI_OK;
}

// Device bytes of all scenes of the context (pools and frame buffers).
uint64_t scenes_bytes(const tsi_ctx *c) {
  uint64_t b = 0;
  for (const tsi_scene *s : c->scenes) b += s->bytes;
  return b;
}

tsi_status ensure_image(tsi_scene *s, uint32_t w, uint32_t h) {
  if (s->d_rgba && (uint64_t)w * h <= s->img_cap) {  // no reallocation while a request mix varies sizes
    s->img_w = w;
    s->img_h = h;
    return TSI_OK;
  }
  const uint64_t old_img = s->img_cap * 32u, new_img = (uint64_t)w * h * 32u;
  if (s->ctx->hbm_budget && new_img > old_img && scenes_bytes(s->ctx) + (new_img - old_img) > s->ctx->hbm_budget)
    return set_err(TSI_ERR_OOM, "frame buffers would exceed the context's HBM budget");
  if (s->copy_pending) {
    const tsi_status st = drain_copy(s);
    if (st != TSI_OK) return st;
  }
  cudaFree(s->d_rgba);
  cudaFree(s->d_depth);
  cudaFree(s->d_normal);
  s->d_rgba = nullptr;
  s->d_depth = nullptr;
  s->d_normal = nullptr;
  const size_t np = (size_t)w * h;
  CK(dalloc(&s->d_rgba, np));
  CK(dalloc(&s->d_depth, np));
  CK(dalloc(&s->d_normal, np * 3));
  s->img_w = w;
  s->img_h = h;
  s->img_cap = np;
  s->bytes = s->bytes - old_img + new_img;
  return TSI_OK;
}

// The tracer's arguments for these uniforms, into the scene's pinned copy.
tsi_status fill_trace(tsi_scene *s, const tsi_uniforms *u) {
  tsi_ctx *c = s->ctx;
  // the previous upload of the pinned descriptor has been read
  if (s->trace_up_pending && !capturing(c)) {
    CK(cudaEventSynchronize(s->trace_up));
    s->trace_up_pending = false;
  }
  const tsi_status st = ensure_image(s, u->resolution[0], u->resolution[1]);
  if (st != TSI_OK) return st;
  TraceParams &T = *s->h_trace;
  T = TraceParams{};
  make_camera(s->p, *u, T);
  T.pool = s->pool;
  T.rgba = s->d_rgba;
  T.depth = s->d_depth;
  T.normal = s->d_normal;
  T.visits = c->d_visits;
  T.swept = s->p.swept_volume ? 1u : 0u;
  T.cinematic = s->p.cinematic ? 1u : 0u;
  T.samples = s->p.samples > 0 ? (uint32_t)s->p.samples : 1u;
  T.see_background = s->p.see_background ? 1u : 0u;
  T.scene_id = s->p.scene_id;
  if (s->p.fast_normals) {  // normals by finite differences of the full tape
    if (s->tape->nregs > 96u)
      return set_err(TSI_ERR_TAPE_TOO_WIDE, "fast normals need a tape of at most 96 interval registers");
    T.code = s->tape->d_code;
    T.len = s->tape->len;
    T.nregs = s->tape->nregs;
    T.out_reg = s->tape->out_reg;
  }
  (void)c;
  return TSI_OK;
}

tsi_status enqueue_trace(tsi_scene *s, const tsi_uniforms *u, cudaStream_t st_) {
  tsi_ctx *c = s->ctx;
  tsi_status st = fill_trace(s, u);
  if (st != TSI_OK) return st;
  const TraceParams &T = *s->h_trace;
  if (T.W == 0 || T.H == 0) return TSI_OK;
  const bool cap = capturing(c);
  CK(cudaMemcpyAsync(s->d_trace, s->h_trace, sizeof(TraceParams), cudaMemcpyHostToDevice, st_));
  if (!cap) {
    CK(cudaEventRecord(s->trace_up, st_));
    s->trace_up_pending = true;
    // the frame buffers are free once the last asynchronous copy read them
    if (s->copy_pending) CK(cudaStreamWaitEvent(st_, s->copy_done, 0));
  }
  CK(launch_trace(T, s->d_trace, st_));
  return TSI_OK;
}
tsi_status enqueue_trace(tsi_scene *s, const tsi_uniforms *u) { return enqueue_trace(s, u, s->ctx->stream); }

tsi_status copy_image_out(tsi_scene *s, tsi_image *out, cudaStream_t st) {
  if (!out) return TSI_OK;
  if (out->width != s->img_w || out->height != s->img_h)
    return set_err(TSI_ERR_BUFFER_TOO_SMALL, "tsi_image size does not match the uniforms' resolution");
  const size_t np = (size_t)s->img_w * s->img_h;
  if (out->rgba) CK(cudaMemcpyAsync(out->rgba, s->d_rgba, np * 16, cudaMemcpyDeviceToHost, st));
  if (out->depth) CK(cudaMemcpyAsync(out->depth, s->d_depth, np * 4, cudaMemcpyDeviceToHost, st));
  if (out->normal) CK(cudaMemcpyAsync(out->normal, s->d_normal, np * 12, cudaMemcpyDeviceToHost, st));
  return TSI_OK;
}
tsi_status copy_image_out(tsi_scene *s, tsi_image *out) { return copy_image_out(s, out, s->ctx->stream); }

tsi_status reset_scene(tsi_scene *s) {
  tsi_ctx *c = s->ctx;
  // main.rs:749-766: root voxel 0 = root box, t 0, no children, f 0
  const float4 xy = make_float4(s->p.root_lo[0], s->p.root_hi[0], s->p.root_lo[1], s->p.root_hi[1]);
  const float2 z = make_float2(s->p.root_lo[2], s->p.root_hi[2]);
  const float zero = 0.0f;
  const uint32_t none = TSI_NONE;
  const float4 n0 = make_float4(0, 0, 0, 0);
  CK(cudaMemcpyAsync(s->pool.box_xy, &xy, sizeof(xy), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.box_z, &z, sizeof(z), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.t, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.time_err, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.f, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.fast, &zero, 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.child, &none, 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(s->pool.normal, &n0, sizeof(n0), cudaMemcpyHostToDevice, c->stream));
  SceneCounters ctr{0, 1u, 0u, 1u};
  CK(cudaMemcpyAsync(s->d_ctr, &ctr, sizeof(ctr), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

tsi_status read_counters(tsi_scene *s, SceneCounters &ctr) {
  CK(cudaMemcpy(&ctr, s->d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost));
  return TSI_OK;
}

}  // namespace tsi_host

extern "C" {

TSI_API uint32_t tsi_version(void) { return TSI_ABI_VERSION; }

TSI_API const char *tsi_status_string(tsi_status s) {
  switch (s) {
    case TSI_OK: return "ok";
    case TSI_ERR_INVALID_ARGUMENT: return "invalid argument";
    case TSI_ERR_PARSE: return "cannot parse LLVM IR";
    case TSI_ERR_CUDA: return "CUDA error";
    case TSI_ERR_OOM: return "out of device memory or pool capacity";
    case TSI_ERR_QUEUE_FULL: return "device work list full";
    case TSI_ERR_WATCHDOG: return "bounded device wait expired";
    case TSI_ERR_BAD_OPCODE: return "bad opcode";
    case TSI_ERR_TAPE_TOO_WIDE: return "tape needs more than 256 registers";
    case TSI_ERR_NO_DEVICE: return "no sm_100 CUDA device";
    case TSI_ERR_BUFFER_TOO_SMALL: return "buffer too small";
    case TSI_ERR_BUSY: return "busy";
    case TSI_ERR_NOT_FOUND: return "not found";
    case TSI_ERR_SHUTDOWN: return "shut down";
  }
  return "unknown status";
}

TSI_API const char *tsi_last_error(void) { return g_last_error.c_str(); }

TSI_API void tsi_rgba8_from_frame(const float *rgba, uint64_t n_pixels, uint8_t *out) {
  if (!rgba || !out) return;
  for (uint64_t i = 0; i < n_pixels * 4; ++i) {
    const float v = rgba[i];
    const float c = v > 0.0f ? (v < 1.0f ? v : 1.0f) : 0.0f;  // NaN compares false: 0
    out[i] = (uint8_t)roundf(c * 255.0f);
  }
}

TSI_API void tsi_default_params(tsi_params *p) {  // compute.wgsl:3494-3511, ir.rs:343-347
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->localsubdiv = 8;
  p->delta = 0.01f;
  p->pointsample = 1;
  p->fastenabled = 1;
  p->lipschitz_corrected = 0;
  p->swept_volume = 0;
  p->fast_normals = 0;
  p->normal_viz = 0;
  p->rounding_mode = TSI_ROUND_NEAREST;
  p->fast_multiplier = 1.0f;
  p->scene_id = 1;
  p->octree_darken_factor = 0.98f;
  for (int i = 0; i < 3; ++i) {
    p->root_lo[i] = -5.0f;
    p->root_hi[i] = 5.0f;
  }
  p->pruning = 1;
  p->swept_dt = 1.0f / 60.0f;
  p->cinematic = 0;
  p->samples = 8;
  p->see_background = 0;
}

TSI_API tsi_status tsi_ir_lower(const char *text, size_t len, float time, tsi_gpu_instruction *out, uint32_t cap,
                                uint32_t *n) {
  if (!text || !n) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  IrError err;
  const float lo[3] = {-5.0f, -5.0f, -5.0f}, hi[3] = {5.0f, 5.0f, 5.0f};
  if (!ir_new(std::string(text, len), time, lo, hi, ins, err))
    return set_err(TSI_ERR_PARSE, "line " + std::to_string(err.line) + ": " + err.message);
  *n = (uint32_t)ins.size();
  if (out)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap, *n); ++i) out[i] = ir_to_gpu(ins[i]);
  return (out && cap < *n) ? TSI_ERR_BUFFER_TOO_SMALL : TSI_OK;
}

// host-only: register allocation summary of an LLVM IR scene (no device)
TSI_API tsi_status tsi_ir_tape_info(const char *text, size_t len, tsi_tape_info *info, uint32_t *slot_reg,
                                    uint32_t cap) {
  if (!text || !info) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  IrError err;
  const float lo[3] = {-5.0f, -5.0f, -5.0f}, hi[3] = {5.0f, 5.0f, 5.0f};
  if (!ir_new(std::string(text, len), 0.0f, lo, hi, ins, err))
    return set_err(TSI_ERR_PARSE, "line " + std::to_string(err.line) + ": " + err.message);
  PackedTape pt;
  tsi_status st = TSI_OK;
  std::string why;
  if (!compile_tape(ins, pt, st, why)) return set_err(st, why);
  info->instruction_count = pt.count;
  info->registers = pt.nregs;
  info->minmax_count = pt.n_minmax;
  info->reserved = pt.out_reg;
  if (slot_reg)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap, pt.count); ++i) slot_reg[i] = pt.slot_reg[i];
  return TSI_OK;
}

// host-only: the packed device tape words of an uploaded-format tape (tests)
TSI_API tsi_status tsi_compile_gpu_instructions(const tsi_gpu_instruction *instr, uint32_t n, uint32_t *words,
                                                uint32_t cap_words, tsi_tape_info *info) {
  if (!instr || !info) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  tsi_status st = TSI_OK;
  std::string why;
  if (!ir_from_gpu(instr, n, ins, st, why)) return set_err(st, why);
  PackedTape pt;
  if (!compile_tape(ins, pt, st, why)) return set_err(st, why);
  info->instruction_count = pt.count;
  info->registers = pt.nregs;
  info->minmax_count = pt.n_minmax;
  info->reserved = pt.out_reg;
  if (words)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap_words, (uint32_t)pt.code.size()); ++i) words[i] = pt.code[i];
  return TSI_OK;
}

// host-only: the bundled form of a tape given in the ir.rs layout (tests)
TSI_API tsi_status tsi_compile_wide_gpu_instructions(const tsi_gpu_instruction *instr, uint32_t n, uint32_t *slots,
                                                     uint32_t cap_slot_words, uint32_t *bundles,
                                                     uint32_t cap_bundle_words, tsi_tape_info *info,
                                                     uint32_t *n_bundles) {
  if (!instr || !info || !n_bundles) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  tsi_status st = TSI_OK;
  std::string why;
  if (!ir_from_gpu(instr, n, ins, st, why)) return set_err(st, why);
  PackedTape pt;
  if (!compile_tape(ins, pt, st, why)) return set_err(st, why);
  WideTape wt;
  if (!compile_wide(ins, pt, wt, st, why)) return set_err(st, why);
  info->instruction_count = pt.count;
  info->registers = wt.nvalues;
  info->minmax_count = pt.n_minmax;
  info->reserved = wt.ncontrib;
  *n_bundles = wt.nbundles;
  if (slots)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap_slot_words, (uint32_t)wt.slots.size()); ++i) slots[i] = wt.slots[i];
  if (bundles)
    for (uint32_t i = 0; i < std::min<uint32_t>(cap_bundle_words, (uint32_t)wt.bundles.size()); ++i)
      bundles[i] = wt.bundles[i];
  return TSI_OK;
}

TSI_API tsi_status tsi_create(const tsi_device_opts *opts, tsi_ctx **out) {
  if (!out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return set_err(TSI_ERR_NO_DEVICE, "no CUDA device");
  }
  const int dev = opts ? opts->device : 0;
  if (dev < 0 || dev >= ndev) return set_err(TSI_ERR_NO_DEVICE, "device ordinal out of range");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, dev));
  if (prop.major != 10) return set_err(TSI_ERR_NO_DEVICE, std::string("not an sm_100 device: ") + prop.name);
  CK(cudaSetDevice(dev));
  tsi_ctx *c = new tsi_ctx();
  c->device = dev;
  c->sm_count = prop.multiProcessorCount;
  c->smem_per_sm = prop.sharedMemPerMultiprocessor;
  c->smem_reserved = prop.reservedSharedMemPerBlock;
  auto fail = [&](tsi_status s) {
    tsi_destroy(c);
    return s;
  };
#define CKC(call)                                                          \
  do {                                                                     \
    cudaError_t e_ = (call);                                               \
    if (e_ != cudaSuccess) {                                               \
      g_last_error = std::string(#call) + ": " + cudaGetErrorString(e_);   \
      return fail(TSI_ERR_CUDA);                                           \
    }                                                                      \
  } while (0)
  // inversions run on the highest-priority stream, so that their
  // latency-bound launches get SMs ahead of queued trace blocks; traces of
  // the batched form run on the lowest-priority one
  int prio_low = 0, prio_high = 0;
  CKC(cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high));
  CKC(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_high));
  CKC(cudaStreamCreateWithPriority(&c->trace_stream, cudaStreamNonBlocking, prio_low));
  CKC(cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking));
  c->max_scenes = (opts && opts->max_scenes_per_launch) ? opts->max_scenes_per_launch : 64u;
  c->wide_smem_bytes = opts ? opts->wide_smem_bytes : 0u;
  c->hbm_budget = opts ? opts->hbm_budget_bytes : 0u;
  c->item_cap = (opts && opts->work_item_capacity) ? (uint32_t)opts->work_item_capacity : (4u << 20);
  c->dealloc_cap = c->item_cap * 2u;
  // pruned records form a ring of a power-of-two size above the scene
  // slots' root records (ring indices are masked, not divided)
  {
    uint32_t ring = 1u;
    while (ring < c->item_cap * 2u && ring < (1u << 30)) ring <<= 1;
    c->rec_cap = c->max_scenes + ring;
  }
  // defaults sized for fused launches of many scenes (the pruned-tape arena
  // and the operand log of long narrow tapes fill per level and frame)
  c->code_cap = (opts && opts->tape_arena_words) ? opts->tape_arena_words : (256ull << 20);
  {  // the code arena is a ring of a power-of-two size (rounded down)
    uint64_t pw = 1;
    while (pw * 2 <= c->code_cap) pw *= 2;
    c->code_cap = pw;
  }
  c->log_overflow_cap = (opts && opts->log_arena_bytes) ? opts->log_arena_bytes / 16 : ((4ull << 30) / 16);
  c->watchdog = (opts && opts->watchdog_iters) ? opts->watchdog_iters : (1u << 22);
  c->slice_len = 1024;
  // resident warps at the smallest register file
  {
    const size_t smem_min = (size_t)kWarpsPerBlock * 4u * 32u * sizeof(float2);
    CKC(refine_set_smem(smem_min));
    int bps = 0;
    CKC(refine_occupancy(kBlock, smem_min, &bps));
    c->max_warps = (uint32_t)std::max(1, bps) * (uint32_t)c->sm_count * kWarpsPerBlock;
  }
  CKC(dalloc(&c->d_scenes, c->max_scenes));
  CKC(cudaMallocHost((void **)&c->h_scenes, c->max_scenes * sizeof(SceneLaunch)));
  CKC(dalloc(&c->d_recs, c->rec_cap));
  CKC(cudaMallocHost((void **)&c->h_recs, c->max_scenes * sizeof(TapeRec)));
  CKC(dalloc(&c->d_rec_count, 1));
  CKC(dalloc(&c->d_rec_low, 1));
  CKC(dalloc(&c->d_code, c->code_cap));
  CKC(dalloc(&c->d_code_count, 1));
  CKC(dalloc(&c->d_code_low, 1));
  CKC(dalloc(&c->d_step_code_start, TSI_STEP_RING));
  CKC(dalloc(&c->d_step_rec_start, TSI_STEP_RING));
  CKC(dalloc(&c->d_items[0], c->item_cap));
  CKC(dalloc(&c->d_items[1], c->item_cap));
  CKC(dalloc(&c->d_item_count, TSI_STEP_RING));
  CKC(dalloc(&c->d_item_cursor, TSI_STEP_RING));
  CKC(dalloc(&c->d_witems[0], c->item_cap));
  CKC(dalloc(&c->d_witems[1], c->item_cap));
  CKC(dalloc(&c->d_witem_count, TSI_STEP_RING));
  CKC(dalloc(&c->d_witem_cursor, TSI_STEP_RING));
  CKC(dalloc(&c->d_dealloc[0], c->dealloc_cap));
  CKC(dalloc(&c->d_dealloc[1], c->dealloc_cap));
  CKC(dalloc(&c->d_dealloc_count, TSI_STEP_RING));
  CKC(dalloc(&c->d_dealloc_cursor, TSI_STEP_RING));
  CKC(dalloc(&c->d_log, (size_t)c->max_warps * c->slice_len * 32u));
  CKC(dalloc(&c->d_dec, (size_t)c->max_warps * c->slice_len));
  CKC(dalloc(&c->d_log_overflow, c->log_overflow_cap));
  CKC(dalloc(&c->d_log_used, TSI_STEP_RING));
  CKC(dalloc(&c->d_error, c->max_scenes));
  CKC(dalloc(&c->d_error_sticky, 1));
  CKC(cudaMemset(c->d_error_sticky, 0, sizeof(uint32_t)));
  CKC(dalloc(&c->d_stats, (size_t)c->max_scenes * ST_COUNT));
  CKC(dalloc(&c->d_level_stats, (size_t)TSI_STEP_RING * ST_COUNT));
  c->fork_events.resize(TSI_STEP_RING);
  for (auto &ev : c->fork_events) CKC(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
  CKC(cudaEventCreateWithFlags(&c->join_event, cudaEventDisableTiming));
  if (getenv("TSI_PROFILE_LEVELS")) {
    c->profile_levels = true;
    c->level_events.resize(TSI_MAX_LEVELS + 1);
    for (auto &ev : c->level_events) CKC(cudaEventCreate(&ev));
  }
  CKC(dalloc(&c->d_visits, 1));
  CKC(cudaMallocHost((void **)&c->h_rb, sizeof(TsiReadback)));
  memset(c->h_rb, 0, sizeof(TsiReadback));
  if (ensure_readback_rows(c, c->max_scenes) != TSI_OK) return fail(TSI_ERR_CUDA);
  CKC(cudaEventCreate(&c->ev0));
  CKC(cudaEventCreateWithFlags(&c->launch_up, cudaEventDisableTiming));
  CKC(cudaEventCreate(&c->ev1));
  CKC(cudaEventCreate(&c->ev2));
  CKC(cudaMemsetAsync(c->d_item_count, 0, TSI_STEP_RING * sizeof(uint32_t), c->stream));
  CKC(cudaStreamSynchronize(c->stream));
#undef CKC
  *out = c;
  return TSI_OK;
}

TSI_API void tsi_destroy(tsi_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  if (c->trace_stream) cudaStreamSynchronize(c->trace_stream);
  while (!c->scenes.empty()) tsi_scene_destroy(*c->scenes.begin());
  while (!c->tapes.empty()) tsi_tape_destroy(*c->tapes.begin());
  cudaFree(c->d_scenes);
  cudaFreeHost(c->h_scenes);
  cudaFree(c->d_recs);
  cudaFreeHost(c->h_recs);
  cudaFree(c->d_rec_count);
  cudaFree(c->d_rec_low);
  cudaFree(c->d_code);
  cudaFree(c->d_code_count);
  cudaFree(c->d_code_low);
  cudaFree(c->d_step_code_start);
  cudaFree(c->d_step_rec_start);
  cudaFree(c->d_items[0]);
  cudaFree(c->d_items[1]);
  cudaFree(c->d_item_count);
  cudaFree(c->d_item_cursor);
  cudaFree(c->d_witems[0]);
  cudaFree(c->d_witems[1]);
  cudaFree(c->d_witem_count);
  cudaFree(c->d_witem_cursor);
  for (int q = 0; q < 2; ++q) cudaFree(c->d_cell_info[q]);
  cudaFree(c->d_wscratch);
  cudaFree(c->d_dealloc[0]);
  cudaFree(c->d_dealloc[1]);
  cudaFree(c->d_dealloc_count);
  cudaFree(c->d_dealloc_cursor);
  cudaFree(c->d_log);
  cudaFree(c->d_dec);
  cudaFree(c->d_log_overflow);
  cudaFree(c->d_log_used);
  cudaFree(c->d_error);
  cudaFree(c->d_error_sticky);
  cudaFree(c->d_stats);
  cudaFree(c->d_level_stats);
  for (auto &ev : c->level_events) cudaEventDestroy(ev);
  for (auto &ev : c->fork_events) cudaEventDestroy(ev);
  if (c->join_event) cudaEventDestroy(c->join_event);
  cudaFree(c->d_visits);
  cudaFree(c->d_scratch);
  cudaFreeHost(c->h_rb);
  cudaFreeHost(c->h_err);
  cudaFreeHost(c->h_stats);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->launch_up) cudaEventDestroy(c->launch_up);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->ev2) cudaEventDestroy(c->ev2);
  if (c->stream) cudaStreamDestroy(c->stream);
  if (c->trace_stream) cudaStreamDestroy(c->trace_stream);
  if (c->copy_stream) cudaStreamDestroy(c->copy_stream);
  delete c;
}

TSI_API tsi_status tsi_synchronize(tsi_ctx *c) {
  if (!c) return set_err(TSI_ERR_INVALID_ARGUMENT, "null ctx");
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

static tsi_status upload_ir(tsi_ctx *c, const std::vector<IrInstr> &ins, tsi_tape **out) {
  PackedTape pt;
  tsi_status st = TSI_OK;
  std::string why;
  if (!compile_tape(ins, pt, st, why)) return set_err(st, why);
  tsi_tape *t = new tsi_tape();
  t->ctx = c;
  t->len = pt.count - 4u;
  t->count = pt.count;
  t->nregs = pt.nregs;
  t->out_reg = pt.out_reg;
  t->n_minmax = pt.n_minmax;
  t->fwd_cost = pt.fwd_cost;
  t->rev_cost = pt.rev_cost;
  c->tapes.insert(t);
  if (t->len) {
    cudaError_t e = dalloc(&t->d_code, t->len);
    if (e == cudaSuccess)
      e = cudaMemcpy(t->d_code, pt.code.data(), (size_t)t->len * sizeof(uint2), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      g_last_error = cudaGetErrorString(e);
      tsi_tape_destroy(t);
      return TSI_ERR_CUDA;
    }
  }
  // bundled form for long tapes (the wide path pays off once a tape has
  // several times more instructions than bundles); a working set beyond
  // shared memory lives in the per-block global scratch
  if (t->len >= 256) {
    WideTape wt;
    if (compile_wide(ins, pt, wt, st, why) && wt.nbundles > 0 &&
        wide_cell_bytes(wt.nvalues, wt.ncontrib, (pt.n_minmax + 15) / 16) <= kWideCellMaxGlobalBytes) {
      // device layout: the three uint4 of every slot in three arrays
      const size_t nsl = wt.slots.size() / 12;
      std::vector<uint32_t> soa(wt.slots.size());
      for (size_t i = 0; i < nsl; ++i)
        for (size_t q = 0; q < 3; ++q)
          for (size_t w = 0; w < 4; ++w) soa[(q * nsl + i) * 4 + w] = wt.slots[i * 12 + q * 4 + w];
      cudaError_t e = dalloc(&t->d_wslots, wt.slots.size() / 4);
      if (e == cudaSuccess) e = dalloc(&t->d_wbundles, wt.bundles.size() / 2);
      if (e == cudaSuccess) e = dalloc(&t->d_wmm, wt.narrow_mm.size());
      if (e == cudaSuccess)
        e = cudaMemcpy(t->d_wslots, soa.data(), soa.size() * 4, cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(t->d_wbundles, wt.bundles.data(), wt.bundles.size() * 4, cudaMemcpyHostToDevice);
      if (e == cudaSuccess)
        e = cudaMemcpy(t->d_wmm, wt.narrow_mm.data(), wt.narrow_mm.size() * 4, cudaMemcpyHostToDevice);
      if (e != cudaSuccess) {
        g_last_error = cudaGetErrorString(e);
        tsi_tape_destroy(t);
        return TSI_ERR_CUDA;
      }
      t->wslots = (uint32_t)nsl;
      t->wbundles = wt.nbundles;
      t->wvalues = wt.nvalues;
      // four bundle steps' worth of instructions: near the fastest of the
      // thresholds tsi_scene_autotune tries on the tapes measured (CSG scenes
      // of 16 to 1123 primitives, rotating swept scenes)
      t->wmin_len = std::max<uint32_t>(64u, 4u * wt.nbundles);
      t->wcontrib = wt.ncontrib;
      for (int q = 0; q < 4; ++q) {
        t->warg_gbase[q] = wt.arg_gbase[q];
        t->warg_gcount[q] = wt.arg_gcount[q];
      }
    }
  }
  *out = t;
  return TSI_OK;
}

TSI_API tsi_status tsi_tape_upload(tsi_ctx *c, const tsi_gpu_instruction *instr, uint32_t n, tsi_tape **out) {
  if (!c || !instr || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  tsi_status st = TSI_OK;
  std::string why;
  if (!ir_from_gpu(instr, n, ins, st, why)) return set_err(st, why);
  CK(cudaSetDevice(c->device));
  return upload_ir(c, ins, out);
}

TSI_API tsi_status tsi_tape_from_llvm_ir(tsi_ctx *c, const char *text, size_t len, tsi_tape **out) {
  if (!c || !text || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  std::vector<IrInstr> ins;
  IrError err;
  const float lo[3] = {-5.0f, -5.0f, -5.0f}, hi[3] = {5.0f, 5.0f, 5.0f};
  if (!ir_new(std::string(text, len), 0.0f, lo, hi, ins, err))
    return set_err(TSI_ERR_PARSE, "line " + std::to_string(err.line) + ": " + err.message);
  CK(cudaSetDevice(c->device));
  return upload_ir(c, ins, out);
}

TSI_API tsi_status tsi_tape_info_get(const tsi_tape *t, tsi_tape_info *info) {
  if (!t || !info) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  info->instruction_count = t->count;
  info->registers = t->nregs;
  info->minmax_count = t->n_minmax;
  info->reserved = t->out_reg;
  return TSI_OK;
}

TSI_API void tsi_tape_destroy(tsi_tape *t) {
  if (!t) return;
  if (t->ctx) t->ctx->tapes.erase(t);
  cudaFree(t->d_code);
  cudaFree(t->d_wslots);
  cudaFree(t->d_wbundles);
  cudaFree(t->d_wmm);
  delete t;
}

TSI_API tsi_status tsi_tape_eval_boxes(tsi_ctx *c, const tsi_tape *t, uint32_t n, const float *boxes,
                                       int32_t rounding_mode, int32_t reverse, float *out) {
  if (!c || !t || (!boxes && n) || (!out && n)) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) return TSI_OK;
  CK(cudaSetDevice(c->device));
  const size_t nb = (size_t)n * 8 * 4, no = (size_t)n * 10 * 4;
  const size_t nr = (size_t)n * t->nregs * 8, nl = (size_t)n * std::max<uint32_t>(t->len, 1u) * 16;
  const size_t need = nb + no + nr + nl + 1024;
  if (need > c->scratch_bytes) {
    cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    c->scratch_bytes = 0;
    CK(cudaMalloc(&c->d_scratch, need));
    c->scratch_bytes = need;
  }
  char *base = (char *)c->d_scratch;
  float *d_boxes = (float *)base;
  float *d_out = (float *)(base + ((nb + 255) & ~(size_t)255));
  float2 *d_regs = (float2 *)(base + ((nb + 255) & ~(size_t)255) + ((no + 255) & ~(size_t)255));
  float4 *d_log = (float4 *)((char *)d_regs + ((nr + 255) & ~(size_t)255));
  CK(cudaMemcpyAsync(d_boxes, boxes, nb, cudaMemcpyHostToDevice, c->stream));
  CK(launch_evalbox(rounding_mode == TSI_ROUND_DIRECTED, t->d_code, t->len, t->nregs, t->out_reg, n, d_boxes, reverse,
                    d_out, d_regs, d_log, c->stream));
  CK(cudaMemcpyAsync(out, d_out, no, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

}  // extern "C"

// Internal view of a tape for the library's other translation units.
tsi_status tsi_internal_tape_view(const tsi_tape *t, TsiTapeView *v) {
  if (!t || !v || !t->ctx) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  v->code = t->d_code;
  v->len = t->len;
  v->nregs = t->nregs;
  v->out_reg = t->out_reg;
  v->device = t->ctx->device;
  v->stream = t->ctx->stream;
  return TSI_OK;
}
void tsi_internal_set_error(const char *msg) { g_last_error = msg; }
tsi_ctx *tsi_internal_scene_ctx(const tsi_scene *s) { return s ? s->ctx : nullptr; }
uint32_t tsi_internal_max_scenes(const tsi_ctx *c) { return c ? c->max_scenes : 0u; }

extern "C" {

// device f32 math on host arrays (GPU math tests)
TSI_API tsi_status tsi_debug_math(tsi_ctx *c, int32_t which, uint32_t n, const float *a, const float *b, float *out) {
  if (!c || !a || !b || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0) return TSI_OK;
  CK(cudaSetDevice(c->device));
  const size_t need = (size_t)n * 12 + 1024;
  if (need > c->scratch_bytes) {
    cudaFree(c->d_scratch);
    c->d_scratch = nullptr;
    c->scratch_bytes = 0;
    CK(cudaMalloc(&c->d_scratch, need));
    c->scratch_bytes = need;
  }
  float *da = (float *)c->d_scratch, *db = da + n, *dout = db + n;
  CK(cudaMemcpyAsync(da, a, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(db, b, (size_t)n * 4, cudaMemcpyHostToDevice, c->stream));
  CK(launch_math(which, n, da, db, dout, c->stream));
  CK(cudaMemcpyAsync(out, dout, (size_t)n * 4, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

static_assert(ST_COUNT == TSI_LEVEL_COUNTERS, "level counters of tsi.h");
TSI_API tsi_status tsi_debug_level_profile(tsi_ctx *c, uint32_t max_levels, float *ms, uint64_t *counters,
                                           uint32_t *n_levels) {
  if (!c || !n_levels) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  const uint32_t L = std::min(c->last_levels, max_levels);
  *n_levels = c->last_levels;
  if (counters) {
    std::vector<unsigned long long> h((size_t)(TSI_MAX_LEVELS + 1) * ST_COUNT);
    CK(cudaMemcpy(h.data(), c->d_level_stats, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    for (uint32_t l = 0; l < L; ++l)
      for (int i = 0; i < ST_COUNT; ++i) counters[(size_t)l * ST_COUNT + i] = h[(size_t)l * ST_COUNT + i];
  }
  if (ms) {
    for (uint32_t l = 0; l < L; ++l) {
      ms[l] = -1.0f;
      if (c->profile_levels && c->level_events.size() > l + 1)
        CK(cudaEventElapsedTime(&ms[l], c->level_events[l], c->level_events[l + 1]));
    }
  }
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_create(tsi_ctx *c, const tsi_tape *tape, const tsi_params *params,
                                    uint64_t voxel_capacity, tsi_scene **out) {
  if (!c || !tape || !params || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  if (params->localsubdiv < 1 || params->localsubdiv > TSI_MAX_LEVELS - 1)
    return set_err(TSI_ERR_INVALID_ARGUMENT, "localsubdiv out of range");
  for (int a = 0; a < 3; ++a)
    if (!(params->root_lo[a] < params->root_hi[a]) || !isfinite(params->root_hi[a] - params->root_lo[a]))
      return set_err(TSI_ERR_INVALID_ARGUMENT, "root box must have lo < hi, finite");
  if (tree_levels(*params) > TSI_MAX_LEVELS - 1)
    return set_err(TSI_ERR_INVALID_ARGUMENT, "root box too wide for localsubdiv (too many levels)");
  if (tape->ctx != c) return set_err(TSI_ERR_INVALID_ARGUMENT, "tape belongs to another context");
  CK(cudaSetDevice(c->device));
  if (voxel_capacity == 0) voxel_capacity = 4ull << 20;
  uint64_t bricks = (voxel_capacity + 7) / 8;
  if (bricks < 2) bricks = 2;
  if (bricks > 0x1fffffffull) return set_err(TSI_ERR_INVALID_ARGUMENT, "voxel capacity too large");
  {
    const uint64_t nv = (uint64_t)bricks * 8;
    const uint64_t need = nv * (16 + 8 + 4 * 5 + 16) + (uint64_t)bricks * 8 + sizeof(SceneCounters);
    if (c->hbm_budget && scenes_bytes(c) + need > c->hbm_budget)
      return set_err(TSI_ERR_OOM, "scene would exceed the context's HBM budget");
  }
  tsi_scene *s = new tsi_scene();
  s->ctx = c;
  c->scenes.insert(s);
  s->tape = tape;
  s->p = *params;
  s->cap_bricks = (uint32_t)bricks;
  const size_t nv = (size_t)bricks * 8;
  cudaError_t e = cudaSuccess;
  auto A = [&](cudaError_t r) {
    if (e == cudaSuccess) e = r;
  };
  A(dalloc(&s->pool.box_xy, nv));
  A(dalloc(&s->pool.box_z, nv));
  A(dalloc(&s->pool.t, nv));
  A(dalloc(&s->pool.time_err, nv));
  A(dalloc(&s->pool.f, nv));
  A(dalloc(&s->pool.fast, nv));
  A(dalloc(&s->pool.child, nv));
  A(dalloc(&s->pool.normal, nv));
  A(dalloc(&s->pool.free_list, bricks));
  A(dalloc(&s->pool.pending, bricks));
  A(dalloc(&s->d_ctr, 1));
  A(dalloc(&s->d_trace, 1));
  A(cudaMallocHost((void **)&s->h_trace, sizeof(TraceParams)));
  A(cudaEventCreateWithFlags(&s->traced, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&s->copy_done, cudaEventDisableTiming));
  A(cudaEventCreateWithFlags(&s->trace_up, cudaEventDisableTiming));
  s->pool.cap_bricks = s->cap_bricks;
  s->bytes = nv * (16 + 8 + 4 * 5 + 16) + bricks * 8 + sizeof(SceneCounters);
  if (e != cudaSuccess) {
    g_last_error = cudaGetErrorString(e);
    tsi_scene_destroy(s);
    return e == cudaErrorMemoryAllocation ? TSI_ERR_OOM : TSI_ERR_CUDA;
  }
  tsi_status st = reset_scene(s);
  if (st != TSI_OK) {
    tsi_scene_destroy(s);
    return st;
  }
  *out = s;
  return TSI_OK;
}

TSI_API void tsi_scene_destroy(tsi_scene *s) {
  if (!s) return;
  if (s->ctx) {
    cudaSetDevice(s->ctx->device);
    cudaStreamSynchronize(s->ctx->stream);
    if (s->copy_pending) cudaEventSynchronize(s->copy_done);
    s->ctx->scenes.erase(s);
  }
  if (s->traced) cudaEventDestroy(s->traced);
  if (s->copy_done) cudaEventDestroy(s->copy_done);
  if (s->trace_up) cudaEventDestroy(s->trace_up);
  cudaFree(s->pool.box_xy);
  cudaFree(s->pool.box_z);
  cudaFree(s->pool.t);
  cudaFree(s->pool.time_err);
  cudaFree(s->pool.f);
  cudaFree(s->pool.fast);
  cudaFree(s->pool.child);
  cudaFree(s->pool.normal);
  cudaFree(s->pool.free_list);
  cudaFree(s->pool.pending);
  cudaFreeHost(s->h_trace);
  cudaFree(s->d_trace);
  cudaFree(s->d_ctr);
  cudaFree(s->d_rgba);
  cudaFree(s->d_depth);
  cudaFree(s->d_normal);
  delete s;
}

TSI_API tsi_status tsi_scene_reset(tsi_scene *s) {
  if (!s) return set_err(TSI_ERR_INVALID_ARGUMENT, "null scene");
  CK(cudaSetDevice(s->ctx->device));
  return reset_scene(s);
}

TSI_API tsi_status tsi_scene_invert(tsi_scene *s, float time, float t0_or_nan, tsi_stats *stats) {
  if (!s) return set_err(TSI_ERR_INVALID_ARGUMENT, "null scene");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaEventRecord(c->ev0, c->stream));
  tsi_status st = enqueue_invert(c, &s, &time, &t0_or_nan, 1);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(c->ev1, c->stream));
  st = enqueue_readback(c, 1);
  if (st != TSI_OK) return st;
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  if (stats) {
    SceneCounters ctr;
    st = read_counters(s, ctr);
    if (st != TSI_OK) return st;
    fill_stats(c, 0, s, stats, (uint64_t)ctr.live_bricks * 8u);
    stats->device_ms = ms;
  }
  return status_from_error_bits(c->h_err[0]);
}

TSI_API tsi_status tsi_scene_invert_async(tsi_scene *s, float time, float t0_or_nan) {
  if (!s) return set_err(TSI_ERR_INVALID_ARGUMENT, "null scene");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaEventRecord(c->ev0, c->stream));
  tsi_status st = enqueue_invert(c, &s, &time, &t0_or_nan, 1, true);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(c->ev1, c->stream));
  return enqueue_readback(c, 1);
}

TSI_API tsi_status tsi_scene_invert_wait(tsi_scene *s, tsi_stats *stats) {
  if (!s) return set_err(TSI_ERR_INVALID_ARGUMENT, "null scene");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  uint32_t sticky = 0;
  CK(cudaMemcpy(&sticky, c->d_error_sticky, sizeof(uint32_t), cudaMemcpyDeviceToHost));
  CK(cudaMemset(c->d_error_sticky, 0, sizeof(uint32_t)));
  if (stats) {
    SceneCounters ctr;
    const tsi_status st = read_counters(s, ctr);
    if (st != TSI_OK) return st;
    fill_stats(c, 0, s, stats, (uint64_t)ctr.live_bricks * 8u);
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    stats->device_ms = ms;
  }
  return status_from_error_bits(sticky);
}

TSI_API tsi_status tsi_scene_trace(tsi_scene *s, const tsi_uniforms *u, tsi_image *out, tsi_stats *stats) {
  if (!s || !u) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaMemsetAsync(c->d_visits, 0, sizeof(unsigned long long), c->stream));
  CK(cudaEventRecord(c->ev0, c->stream));
  tsi_status st = enqueue_trace(s, u);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(c->ev1, c->stream));
  st = copy_image_out(s, out);
  if (st != TSI_OK) return st;
  CK(cudaMemcpyAsync(&c->h_rb->visits, c->d_visits, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (stats) {
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    memset(stats, 0, sizeof(*stats));
    stats->device_ms = ms;
    stats->reserved = (float)c->h_rb->visits;
  }
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_trace_async(tsi_scene *s, const tsi_uniforms *u, tsi_image *out) {
  if (!s || !u || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (out->width != u->resolution[0] || out->height != u->resolution[1])
    return set_err(TSI_ERR_BUFFER_TOO_SMALL, "tsi_image size does not match the uniforms' resolution");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  tsi_status st = enqueue_trace(s, u);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(s->traced, c->stream));
  CK(cudaStreamWaitEvent(c->copy_stream, s->traced, 0));
  st = copy_image_out(s, out, c->copy_stream);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(s->copy_done, c->copy_stream));
  s->copy_pending = true;
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_trace_wait(tsi_scene *s) {
  if (!s) return set_err(TSI_ERR_INVALID_ARGUMENT, "null scene");
  CK(cudaSetDevice(s->ctx->device));
  return drain_copy(s);
}

TSI_API tsi_status tsi_scene_image_copy(tsi_scene *s, tsi_image *out) {
  if (!s || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaStreamSynchronize(s->ctx->stream));
  const tsi_status st = copy_image_out(s, out);
  if (st != TSI_OK) return st;
  CK(cudaStreamSynchronize(s->ctx->stream));
  return TSI_OK;
}

TSI_API uint32_t tsi_tape_wide_threshold(const tsi_tape *t) { return t ? t->wmin_len : 0xffffffffu; }

TSI_API tsi_status tsi_tape_set_wide_threshold(tsi_tape *t, uint32_t min_len) {
  if (!t) return set_err(TSI_ERR_INVALID_ARGUMENT, "null tape");
  if (t->d_wslots) t->wmin_len = min_len;
  return TSI_OK;
}

TSI_API tsi_status tsi_tape_set_wide_threshold_deep(tsi_tape *t, uint32_t level, uint32_t min_len) {
  if (!t) return set_err(TSI_ERR_INVALID_ARGUMENT, "null tape");
  if (!t->d_wslots) return TSI_OK;  // no bundled form: every cell stays on the narrow path
  t->wdeep_level = level;
  t->wdeep_min_len = min_len;
  return TSI_OK;
}

TSI_API tsi_status tsi_tape_set_narrow_parents(tsi_tape *t, uint32_t parents) {
  if (!t) return set_err(TSI_ERR_INVALID_ARGUMENT, "null tape");
  if (parents != 1 && parents != 2 && parents != 4) return set_err(TSI_ERR_INVALID_ARGUMENT, "parents must be 1, 2 or 4");
  t->narrow_parents = parents;
  return TSI_OK;
}

TSI_API uint32_t tsi_tape_narrow_parents(const tsi_tape *t) { return t ? t->narrow_parents : 0u; }

TSI_API tsi_status tsi_tape_set_wide_prune_level(tsi_tape *t, uint32_t level) {
  if (!t) return set_err(TSI_ERR_INVALID_ARGUMENT, "null tape");
  t->wprune_level = level;
  return TSI_OK;
}

TSI_API uint32_t tsi_tape_wide_prune_level(const tsi_tape *t) { return t ? t->wprune_level : 0xffffffffu; }

TSI_API tsi_status tsi_tape_wide_threshold_deep(const tsi_tape *t, uint32_t *level, uint32_t *min_len) {
  if (!t || !level || !min_len) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  *level = t->wdeep_level;
  *min_len = t->wdeep_min_len;
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_autotune(tsi_scene *s, const float *times, uint32_t ntimes, uint32_t reps,
                                      tsi_autotune_result *out) {
  if (!s || !times || ntimes == 0 || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  memset(out, 0, sizeof(*out));
  // the tape belongs to the caller's context; its threshold is the tunable
  tsi_tape *t = const_cast<tsi_tape *>(s->tape);
  if (!t->d_wslots) {
    out->wide_threshold = t->wmin_len;
    return tsi_scene_reset(s);
  }
  const uint32_t nb = t->wbundles, keep = t->wmin_len;
  std::vector<uint32_t> cand = {std::max(128u, nb), std::max(128u, 2 * nb), 3 * nb, 4 * nb, 6 * nb,
                                256u, 512u, 1024u, 2048u, keep};
  cand.erase(std::remove_if(cand.begin(), cand.end(), [&](uint32_t v) { return v > t->len; }), cand.end());
  cand.push_back(0xffffffffu);  // narrow only
  std::sort(cand.begin(), cand.end());
  cand.erase(std::unique(cand.begin(), cand.end()), cand.end());
  if (cand.size() > TSI_AUTOTUNE_MAX) cand.erase(cand.begin(), cand.end() - TSI_AUTOTUNE_MAX);
  if (reps == 0) reps = 1;
  float best = INFINITY;
  uint32_t pick = keep;
  for (size_t k = 0; k < cand.size(); ++k) {
    t->wmin_len = cand[k];
    float bk = INFINITY;
    for (uint32_t r = 0; r < reps; ++r) {
      tsi_status st = tsi_scene_reset(s);
      float ms = 0.0f;
      for (uint32_t i = 0; i < ntimes && st == TSI_OK; ++i) {
        tsi_stats fs;
        st = tsi_scene_invert(s, times[i], NAN, &fs);
        ms += fs.device_ms;
      }
      if (st == TSI_ERR_QUEUE_FULL || st == TSI_ERR_OOM) {  // this threshold does not fit the arenas
        bk = INFINITY;
        break;
      }
      if (st != TSI_OK) {
        t->wmin_len = keep;
        tsi_scene_reset(s);
        return st;
      }
      bk = std::min(bk, ms);
    }
    out->threshold[k] = cand[k];
    out->ms[k] = bk;
    if (bk < best) {
      best = bk;
      pick = cand[k];
    }
  }
  out->candidates = (uint32_t)cand.size();
  out->wide_threshold = pick;
  t->wmin_len = pick;
  // then a higher threshold for the deepest levels, where many cells make
  // the narrow path's throughput pay (kept only when it is faster)
  const uint32_t keep_level = t->wdeep_level, keep_deep = t->wdeep_min_len;
  uint32_t dl = 0xffffffffu, dm = 0xffffffffu;
  const uint32_t levels = tree_levels(s->p);
  if (pick != 0xffffffffu && levels >= 4) {
    for (uint32_t back = 2; back <= 3; ++back)
      for (uint32_t mul : {4u, 8u}) {
        t->wdeep_level = levels - back;
        t->wdeep_min_len = pick >= 0xffffffffu / mul ? 0xffffffffu : pick * mul;
        float bk = INFINITY;
        for (uint32_t r = 0; r < reps; ++r) {
          tsi_status st = tsi_scene_reset(s);
          float ms = 0.0f;
          for (uint32_t i = 0; i < ntimes && st == TSI_OK; ++i) {
            tsi_stats fs;
            st = tsi_scene_invert(s, times[i], NAN, &fs);
            ms += fs.device_ms;
          }
          if (st == TSI_ERR_QUEUE_FULL || st == TSI_ERR_OOM) {
            bk = INFINITY;
            break;
          }
          if (st != TSI_OK) {
            t->wdeep_level = keep_level;
            t->wdeep_min_len = keep_deep;
            tsi_scene_reset(s);
            return st;
          }
          bk = std::min(bk, ms);
        }
        if (bk < best * 0.99f) {
          best = bk;
          dl = t->wdeep_level;
          dm = t->wdeep_min_len;
        }
      }
  }
  t->wdeep_level = dl;
  t->wdeep_min_len = dm;
  out->deep_level = dl;
  out->deep_threshold = dm;
  // then the parents per narrow item above the leaf level
  const uint32_t keep_parents = t->narrow_parents;
  uint32_t pp = keep_parents;
  for (uint32_t cand_p : {1u, 2u, 4u}) {
    if (cand_p == keep_parents) continue;
    t->narrow_parents = cand_p;
    float bk = INFINITY;
    for (uint32_t r = 0; r < reps; ++r) {
      tsi_status st = tsi_scene_reset(s);
      float ms = 0.0f;
      for (uint32_t i = 0; i < ntimes && st == TSI_OK; ++i) {
        tsi_stats fs;
        st = tsi_scene_invert(s, times[i], NAN, &fs);
        ms += fs.device_ms;
      }
      if (st == TSI_ERR_QUEUE_FULL || st == TSI_ERR_OOM) {
        bk = INFINITY;
        break;
      }
      if (st != TSI_OK) {
        t->narrow_parents = keep_parents;
        tsi_scene_reset(s);
        return st;
      }
      bk = std::min(bk, ms);
    }
    if (bk < best * 0.99f) {
      best = bk;
      pp = cand_p;
    }
  }
  t->narrow_parents = pp;
  out->narrow_parents = pp;
  // then the first level whose wide groups prune their tape (automatic:
  // half the scene's levels; `levels`: the wide path never prunes)
  const uint32_t keep_prune = t->wprune_level;
  const uint32_t auto_level = levels / 2u;
  const uint32_t current = keep_prune == 0xffffffffu ? auto_level : keep_prune;
  uint32_t pl = keep_prune;
  for (uint32_t cand_l : {auto_level >= 2u ? auto_level - 2u : 0u, auto_level >= 1u ? auto_level - 1u : 0u,
                          auto_level, auto_level + 1u, levels}) {
    if (cand_l == current) continue;
    t->wprune_level = cand_l;
    float bk = INFINITY;
    for (uint32_t r = 0; r < reps; ++r) {
      tsi_status st = tsi_scene_reset(s);
      float ms = 0.0f;
      for (uint32_t i = 0; i < ntimes && st == TSI_OK; ++i) {
        tsi_stats fs;
        st = tsi_scene_invert(s, times[i], NAN, &fs);
        ms += fs.device_ms;
      }
      if (st == TSI_ERR_QUEUE_FULL || st == TSI_ERR_OOM) {
        bk = INFINITY;
        break;
      }
      if (st != TSI_OK) {
        t->wprune_level = keep_prune;
        tsi_scene_reset(s);
        return st;
      }
      bk = std::min(bk, ms);
    }
    if (bk < best * 0.99f) {
      best = bk;
      pl = cand_l;
    }
  }
  t->wprune_level = pl;
  out->wide_prune_level = pl;
  return tsi_scene_reset(s);
}

TSI_API tsi_status tsi_scene_image_device(tsi_scene *s, tsi_image_device *out) {
  if (!s || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  out->width = s->img_w;
  out->height = s->img_h;
  out->rgba = (const float *)s->d_rgba;
  out->depth = s->d_depth;
  out->normal = s->d_normal;
  return TSI_OK;
}

TSI_API tsi_status tsi_params_subtree(const tsi_params *full, uint32_t level, uint32_t index, tsi_params *out) {
  if (!full || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (level > 10u || (int32_t)level >= full->localsubdiv)
    return set_err(TSI_ERR_INVALID_ARGUMENT, "subtree level must be below localsubdiv and at most 10");
  const uint64_t n = 1ull << level;
  if ((uint64_t)index >= n * n * n) return set_err(TSI_ERR_INVALID_ARGUMENT, "subtree index out of range");
  const uint32_t ix = (uint32_t)(index % n), iy = (uint32_t)((index / n) % n), iz = (uint32_t)(index / (n * n));
  tsi_params p = *full;
  for (uint32_t j = 0; j < level; ++j) {  // one child step per level (compute.wgsl:3582-3589)
    const uint32_t sh = level - 1u - j;
    const uint32_t b[3] = {(ix >> sh) & 1u, (iy >> sh) & 1u, (iz >> sh) & 1u};
    for (int a = 0; a < 3; ++a) {
      const float lo = p.root_lo[a], d = (p.root_hi[a] - p.root_lo[a]) / 2.0f;
      p.root_lo[a] = lo + d * (float)b[a];
      p.root_hi[a] = lo + d * (float)(1u + b[a]);
    }
  }
  *out = p;
  return TSI_OK;
}

namespace {
tsi_status check_frame(const tsi_frame_device *f) {
  if (!f->rgba || !f->depth || !f->normal || !f->key) return set_err(TSI_ERR_INVALID_ARGUMENT, "null frame buffer");
  if (((uintptr_t)f->rgba & 15u) || ((uintptr_t)f->key & 7u) || ((uintptr_t)f->depth & 3u) ||
      ((uintptr_t)f->normal & 3u))
    return set_err(TSI_ERR_INVALID_ARGUMENT, "frame buffers misaligned (rgba 16, key 8, depth/normal 4 bytes)");
  return TSI_OK;
}
}  // namespace

TSI_API tsi_status tsi_frames_composite(tsi_ctx *c, tsi_scene *const *scenes, const uint32_t *ids, uint32_t n,
                                        tsi_frame_device *out) {
  if (!c || !scenes || !ids || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (n == 0 || n > TSI_COMPOSITE_MAX) return set_err(TSI_ERR_INVALID_ARGUMENT, "1 to TSI_COMPOSITE_MAX parts");
  tsi_status st = check_frame(out);
  if (st != TSI_OK) return st;
  if (capturing(c)) return set_err(TSI_ERR_BUSY, "composite during graph capture");
  tsi::CompositeParts P{};
  for (uint32_t i = 0; i < n; ++i) {
    const tsi_scene *s = scenes[i];
    if (!s || s->ctx != c) return set_err(TSI_ERR_INVALID_ARGUMENT, "part is not a scene of this context");
    if (!s->d_rgba || s->img_w != out->width || s->img_h != out->height)
      return set_err(TSI_ERR_BUFFER_TOO_SMALL, "a part's last frame differs in size from the composite");
    for (uint32_t j = 0; j < i; ++j)
      if (ids[j] == ids[i]) return set_err(TSI_ERR_INVALID_ARGUMENT, "subtree indices must differ");
    P.rgba[i] = s->d_rgba;
    P.depth[i] = s->d_depth;
    P.normal[i] = s->d_normal;
    P.id[i] = ids[i];
  }
  P.n = n;
  CK(cudaSetDevice(c->device));
  const uint64_t npix = (uint64_t)out->width * out->height;
  CK(tsi::launch_composite(P, npix, reinterpret_cast<float4 *>(out->rgba), out->depth, out->normal,
                           reinterpret_cast<unsigned long long *>(out->key), c->sm_count * 8, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

TSI_API tsi_status tsi_frame_keep_nearest(tsi_ctx *c, const uint64_t *global_key, tsi_frame_device *frame) {
  if (!c || !global_key || !frame) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  tsi_status st = check_frame(frame);
  if (st != TSI_OK) return st;
  if ((uintptr_t)global_key & 7u) return set_err(TSI_ERR_INVALID_ARGUMENT, "global key misaligned");
  if (capturing(c)) return set_err(TSI_ERR_BUSY, "keep-nearest during graph capture");
  CK(cudaSetDevice(c->device));
  const uint64_t npix = (uint64_t)frame->width * frame->height;
  CK(tsi::launch_keep_nearest(reinterpret_cast<const unsigned long long *>(frame->key),
                              reinterpret_cast<const unsigned long long *>(global_key), npix,
                              reinterpret_cast<float4 *>(frame->rgba), frame->depth, frame->normal,
                              c->sm_count * 8, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_readback_cells(tsi_scene *s, tsi_cell *out, uint64_t cap, uint64_t *n) {
  if (!s || !n) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  tsi_ctx *c = s->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  SceneCounters ctr;
  tsi_status st = read_counters(s, ctr);
  if (st != TSI_OK) return st;
  const size_t nv = (size_t)std::min(ctr.bump, s->cap_bricks) * 8;
  std::vector<float4> xy(nv), nrm(nv);
  std::vector<float2> z(nv);
  std::vector<float> t(nv), te(nv), f(nv), fast(nv);
  std::vector<uint32_t> child(nv);
  CK(cudaMemcpy(xy.data(), s->pool.box_xy, nv * sizeof(float4), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(z.data(), s->pool.box_z, nv * sizeof(float2), cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(t.data(), s->pool.t, nv * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(te.data(), s->pool.time_err, nv * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(f.data(), s->pool.f, nv * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(fast.data(), s->pool.fast, nv * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(child.data(), s->pool.child, nv * 4, cudaMemcpyDeviceToHost));
  CK(cudaMemcpy(nrm.data(), s->pool.normal, nv * sizeof(float4), cudaMemcpyDeviceToHost));
  struct E {
    uint32_t v, level, ix, iy, iz;
  };
  std::vector<E> stack{{0, 0, 0, 0, 0}};
  uint64_t cnt = 0;
  while (!stack.empty()) {
    const E e = stack.back();
    stack.pop_back();
    if (e.v >= nv) return set_err(TSI_ERR_INVALID_ARGUMENT, "corrupt octree (child index out of range)");
    if (out && cnt < cap) {
      tsi_cell &o = out[cnt];
      o.level = e.level;
      o.ix = e.ix;
      o.iy = e.iy;
      o.iz = e.iz;
      o.f = f[e.v];
      o.t = t[e.v];
      o.time_err = te[e.v];
      o.fast = fast[e.v];
      o.dx = nrm[e.v].x;
      o.dy = nrm[e.v].y;
      o.dz = nrm[e.v].z;
      o.has_children = child[e.v] != TSI_NONE;
      o.x[0] = xy[e.v].x;
      o.x[1] = xy[e.v].y;
      o.y[0] = xy[e.v].z;
      o.y[1] = xy[e.v].w;
      o.z[0] = z[e.v].x;
      o.z[1] = z[e.v].y;
    }
    ++cnt;
    if (child[e.v] != TSI_NONE) {
      if (e.level >= 32) return set_err(TSI_ERR_INVALID_ARGUMENT, "corrupt octree (too deep)");
      for (int k = 7; k >= 0; --k)
        stack.push_back(E{child[e.v] + (uint32_t)k, e.level + 1, 2 * e.ix + (k & 1), 2 * e.iy + ((k >> 1) & 1),
                          2 * e.iz + (k >> 2)});
    }
  }
  *n = cnt;
  return (out && cap < cnt) ? TSI_ERR_BUFFER_TOO_SMALL : TSI_OK;
}

}  // extern "C"

// Snapshot blob: header, then the pool arrays over [0, bump * 8) voxels
// in VoxelPoolDev order, then the free list [0, free_count).
namespace {
struct SnapshotHeader {
  uint32_t magic, version;
  uint32_t bump, free_count, live_bricks, tape_len;
  uint64_t params_hash;
};
constexpr uint32_t kSnapMagic = 0x54534931u;  // "TSI1"
constexpr size_t kVoxelBytes = sizeof(float4) + sizeof(float2) + 4 * sizeof(float) + sizeof(uint32_t) + sizeof(float4);

uint64_t params_hash(const tsi_params &p) {  // FNV-1a over the bytes of the parameters
  const unsigned char *b = reinterpret_cast<const unsigned char *>(&p);
  uint64_t h = 1469598103934665603ull;
  for (size_t i = 0; i < sizeof(p); ++i) h = (h ^ b[i]) * 1099511628211ull;
  return h;
}

template <typename T>
tsi_status copy_part(T *dev, unsigned char *&host, size_t n, bool to_host) {
  const size_t bytes = n * sizeof(T);
  const cudaError_t e = to_host ? cudaMemcpy(host, dev, bytes, cudaMemcpyDeviceToHost)
                                : cudaMemcpy(dev, host, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return set_err(TSI_ERR_CUDA, cudaGetErrorString(e));
  host += bytes;
  return TSI_OK;
}

tsi_status snapshot_io(tsi_scene *s, unsigned char *p, uint32_t bump, uint32_t free_count, bool to_host) {
  const size_t nv = (size_t)bump * 8;
  tsi_status st = TSI_OK;
  if ((st = copy_part(s->pool.box_xy, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.box_z, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.t, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.time_err, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.f, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.fast, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.child, p, nv, to_host)) != TSI_OK) return st;
  if ((st = copy_part(s->pool.normal, p, nv, to_host)) != TSI_OK) return st;
  return copy_part(s->pool.free_list, p, free_count, to_host);
}
}  // namespace

extern "C" {

TSI_API tsi_status tsi_scene_snapshot_size(tsi_scene *s, uint64_t *bytes) {
  if (!s || !bytes) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaStreamSynchronize(s->ctx->stream));
  SceneCounters ctr;
  tsi_status st = read_counters(s, ctr);
  if (st != TSI_OK) return st;
  const uint32_t bump = std::min(ctr.bump, s->cap_bricks);
  *bytes = sizeof(SnapshotHeader) + (uint64_t)bump * 8 * kVoxelBytes + (uint64_t)std::max(ctr.free_count, 0) * 4;
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_snapshot(tsi_scene *s, void *host, uint64_t cap, uint64_t *bytes) {
  if (!s || !host || !bytes) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  uint64_t need = 0;
  tsi_status st = tsi_scene_snapshot_size(s, &need);
  if (st != TSI_OK) return st;
  *bytes = need;
  if (cap < need) return set_err(TSI_ERR_BUFFER_TOO_SMALL, "snapshot buffer too small");
  SceneCounters ctr;
  if ((st = read_counters(s, ctr)) != TSI_OK) return st;
  if (ctr.pending_count != 0) return set_err(TSI_ERR_BUSY, "snapshot taken inside a frame");
  SnapshotHeader h{kSnapMagic, 1u, std::min(ctr.bump, s->cap_bricks), (uint32_t)std::max(ctr.free_count, 0),
                   ctr.live_bricks, s->tape->len, params_hash(s->p)};
  unsigned char *p = static_cast<unsigned char *>(host);
  memcpy(p, &h, sizeof(h));
  return snapshot_io(s, p + sizeof(h), h.bump, h.free_count, true);
}

TSI_API tsi_status tsi_scene_restore(tsi_scene *s, const void *host, uint64_t bytes) {
  if (!s || !host) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (bytes < sizeof(SnapshotHeader)) return set_err(TSI_ERR_INVALID_ARGUMENT, "snapshot too short");
  SnapshotHeader h;
  memcpy(&h, host, sizeof(h));
  if (h.magic != kSnapMagic || h.version != 1u) return set_err(TSI_ERR_INVALID_ARGUMENT, "not a scene snapshot");
  if (h.tape_len != s->tape->len || h.params_hash != params_hash(s->p))
    return set_err(TSI_ERR_INVALID_ARGUMENT, "snapshot of a scene with another tape or other parameters");
  if (h.bump > s->cap_bricks) return set_err(TSI_ERR_BUFFER_TOO_SMALL, "voxel pool smaller than the snapshot's");
  if (bytes != sizeof(h) + (uint64_t)h.bump * 8 * kVoxelBytes + (uint64_t)h.free_count * 4)
    return set_err(TSI_ERR_INVALID_ARGUMENT, "snapshot size does not match its header");
  CK(cudaSetDevice(s->ctx->device));
  CK(cudaStreamSynchronize(s->ctx->stream));
  unsigned char *p = const_cast<unsigned char *>(static_cast<const unsigned char *>(host)) + sizeof(h);
  tsi_status st = snapshot_io(s, p, h.bump, h.free_count, false);
  if (st != TSI_OK) return st;
  SceneCounters ctr{(int32_t)h.free_count, h.bump, 0u, h.live_bricks};
  CK(cudaMemcpy(s->d_ctr, &ctr, sizeof(ctr), cudaMemcpyHostToDevice));
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_readback_leaves(tsi_scene *s, tsi_leaf *out, uint64_t cap, uint64_t *n) {
  if (!s || !n) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  uint64_t nc = 0;
  tsi_status st = tsi_scene_readback_cells(s, nullptr, 0, &nc);
  if (st != TSI_OK) return st;
  std::vector<tsi_cell> cells(nc);
  st = tsi_scene_readback_cells(s, cells.data(), nc, &nc);
  if (st != TSI_OK) return st;
  uint64_t cnt = 0;
  for (const tsi_cell &c : cells) {
    if (c.has_children || !(c.f <= 0.0f)) continue;
    if (out && cnt < cap) out[cnt] = tsi_leaf{c.level, c.ix, c.iy, c.iz};
    ++cnt;
  }
  *n = cnt;
  return TSI_OK;
}

TSI_API tsi_status tsi_scene_get_params(const tsi_scene *s, tsi_params *out) {
  if (!s || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  *out = s->p;
  return TSI_OK;
}

TSI_API uint64_t tsi_scene_device_bytes(const tsi_scene *s) { return s ? s->bytes : 0; }

TSI_API uint64_t tsi_scenes_device_bytes(const tsi_ctx *c) { return c ? scenes_bytes(c) : 0; }

static tsi_status batch_enqueue(tsi_ctx *c, tsi_request *reqs, uint32_t n) {
  std::vector<tsi_scene *> sc(n);
  std::vector<float> times(n), t0s(n);
  for (uint32_t i = 0; i < n; ++i) {
    if (!reqs[i].scene || reqs[i].scene->ctx != c) return set_err(TSI_ERR_INVALID_ARGUMENT, "bad request scene");
    for (uint32_t j = 0; j < i; ++j)
      if (reqs[j].scene == reqs[i].scene) return set_err(TSI_ERR_INVALID_ARGUMENT, "scenes in a batch must differ");
    sc[i] = reqs[i].scene;
    times[i] = reqs[i].time;
    t0s[i] = reqs[i].t0_or_nan;
  }
  tsi_status st = ensure_readback_rows(c, n);
  if (st != TSI_OK) return st;
  // Batches wider than one launch run as consecutive launch sequences; each
  // one's error words and counters go to its own readback rows, so nothing
  // of an earlier chunk is lost.  Every scene's trace starts on the trace
  // stream as soon as its own last level is done, overlapping the deeper
  // levels of the other scenes (and the next chunk's inversion).
  bool forked = false;  // traces queued on the trace stream (joined back below)
  for (uint32_t i0 = 0; i0 < n; i0 += c->max_scenes) {
    const uint32_t m = std::min(c->max_scenes, n - i0);
    st = enqueue_invert(c, sc.data() + i0, times.data() + i0, t0s.data() + i0, m, false, true);
    if (st != TSI_OK) return st;
    for (uint32_t i = i0; i < i0 + m; ++i) {
      if (!reqs[i].uniforms) continue;
      const uint32_t last = tree_levels(sc[i]->p) - 1u;
      CK(cudaStreamWaitEvent(c->trace_stream, c->fork_events[last], 0));
      forked = true;
      st = enqueue_trace(reqs[i].scene, reqs[i].uniforms, c->trace_stream);
      if (st != TSI_OK) return st;
    }
    st = enqueue_readback(c, m, i0);
    if (st != TSI_OK) return st;
  }
  if (forked) {
    CK(cudaEventRecord(c->join_event, c->trace_stream));
    CK(cudaStreamWaitEvent(c->stream, c->join_event, 0));
  }
  return TSI_OK;
}

TSI_API tsi_status tsi_batch_run(tsi_ctx *c, tsi_request *reqs, uint32_t n) {
  if (!c || (!reqs && n)) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  CK(cudaSetDevice(c->device));
  CK(cudaEventRecord(c->ev0, c->stream));
  tsi_status st = batch_enqueue(c, reqs, n);
  if (st != TSI_OK) return st;
  CK(cudaEventRecord(c->ev1, c->stream));
  for (uint32_t i = 0; i < n; ++i) {
    if (reqs[i].uniforms && reqs[i].out) {
      st = copy_image_out(reqs[i].scene, reqs[i].out);
      if (st != TSI_OK) return st;
    }
  }
  CK(cudaStreamSynchronize(c->stream));
  float ms = 0.0f;
  CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
  uint32_t err = 0;
  for (uint32_t i = 0; i < n; ++i) {
    err |= c->h_err[i];
    if (reqs[i].stats) {
      SceneCounters ctr;
      st = read_counters(reqs[i].scene, ctr);
      if (st != TSI_OK) return st;
      fill_stats(c, i, reqs[i].scene, reqs[i].stats, (uint64_t)ctr.live_bricks * 8u);
      reqs[i].stats->device_ms = ms;
    }
  }
  return status_from_error_bits(err);
}

TSI_API tsi_status tsi_batch_autotune(tsi_ctx *c, const tsi_request *reqs, uint32_t n, uint32_t frames,
                                      tsi_autotune_result *out) {
  if (!c || !reqs || n == 0 || frames == 0 || !out) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  memset(out, 0, sizeof(*out));
  CK(cudaSetDevice(c->device));
  // the distinct tapes with a bundled form, and their thresholds now
  std::vector<tsi_tape *> tapes;
  std::vector<uint32_t> base, base_deep;
  for (uint32_t i = 0; i < n; ++i) {
    if (!reqs[i].scene || reqs[i].scene->ctx != c) return set_err(TSI_ERR_INVALID_ARGUMENT, "bad request scene");
    tsi_tape *t = const_cast<tsi_tape *>(reqs[i].scene->tape);
    if (t->d_wslots && std::find(tapes.begin(), tapes.end(), t) == tapes.end()) {
      tapes.push_back(t);
      base.push_back(t->wmin_len);
      base_deep.push_back(t->wdeep_min_len);
    }
  }
  auto reset_all = [&]() -> tsi_status {
    for (uint32_t i = 0; i < n; ++i) {
      const tsi_status st = tsi_scene_reset(reqs[i].scene);
      if (st != TSI_OK) return st;
    }
    return TSI_OK;
  };
  auto apply = [&](uint32_t scale) {
    for (size_t q = 0; q < tapes.size(); ++q) {
      tapes[q]->wmin_len = base[q] >= 0xffffffffu / scale ? 0xffffffffu : base[q] * scale;
      tapes[q]->wdeep_min_len = base_deep[q] >= 0xffffffffu / scale ? 0xffffffffu : base_deep[q] * scale;
    }
  };
  const uint32_t scales[] = {1u, 2u, 4u, 8u};
  const uint32_t ncand = tapes.empty() ? 1u : 4u;
  std::vector<tsi_request> rq(n);
  std::vector<tsi_stats> st(n);
  float best = INFINITY;
  uint32_t pick = 1u;
  for (uint32_t k = 0; k < ncand; ++k) {
    apply(scales[k]);
    tsi_status s = reset_all();
    float ms = 0.0f;
    for (uint32_t f = 0; f < frames && s == TSI_OK; ++f) {
      for (uint32_t i = 0; i < n; ++i) {
        rq[i] = tsi_request{reqs[i].scene, reqs[i].time + (float)f / 60.0f, NAN, nullptr, nullptr, &st[i]};
      }
      s = tsi_batch_run(c, rq.data(), n);
      if (s == TSI_OK) ms += st[0].device_ms;
    }
    if (s == TSI_ERR_QUEUE_FULL || s == TSI_ERR_OOM) {
      ms = INFINITY;  // this scale does not fit the arenas
    } else if (s != TSI_OK) {
      apply(1u);
      reset_all();
      return s;
    }
    out->threshold[k] = scales[k];
    out->ms[k] = ms;
    if (ms < best) {
      best = ms;
      pick = scales[k];
    }
  }
  out->candidates = ncand;
  out->wide_threshold = pick;
  apply(pick);
  return reset_all();
}

TSI_API tsi_status tsi_batch_graph_create(tsi_ctx *c, tsi_request *reqs, uint32_t n, tsi_batch_graph **out) {
  if (!c || !reqs || !out || n == 0) return set_err(TSI_ERR_INVALID_ARGUMENT, "null argument");
  if (n > c->max_scenes) return set_err(TSI_ERR_INVALID_ARGUMENT, "graph batch wider than one launch");
  CK(cudaSetDevice(c->device));
  tsi_batch_graph *g = new tsi_batch_graph();
  g->ctx = c;
  g->user = reqs;
  g->reqs.assign(reqs, reqs + n);
  CK(cudaStreamSynchronize(c->stream));
  // grow the shared-memory attribute, the wide path's arenas and the frame
  // buffers before capture
  {
    std::vector<tsi_scene *> sc(n);
    for (uint32_t i = 0; i < n; ++i) sc[i] = reqs[i].scene;
    FramePlan fp;
    const tsi_status pst = plan_frame(c, sc.data(), n, fp);
    if (pst != TSI_OK) {
      delete g;
      return pst;
    }
    g->global = fp.global;  // the captured launches' choice, re-applied at every replay
  }
  for (uint32_t i = 0; i < n; ++i) {
    const tsi_status dst = drain_copy(reqs[i].scene);  // no outside event inside the capture
    if (dst != TSI_OK) {
      delete g;
      return dst;
    }
  }
  for (uint32_t i = 0; i < n; ++i)
    if (reqs[i].uniforms) {
      tsi_status st = ensure_image(reqs[i].scene, reqs[i].uniforms->resolution[0], reqs[i].uniforms->resolution[1]);
      if (st != TSI_OK) {
        delete g;
        return st;
      }
    }
  CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
  // the replay records its own timing events and reads back its error word
  // and counters (tsi_batch_graph_wait reports them)
  tsi_status st = TSI_OK;
  if (cudaEventRecordWithFlags(c->ev0, c->stream, cudaEventRecordExternal) != cudaSuccess)
    st = set_err(TSI_ERR_CUDA, "event record in capture");
  if (st == TSI_OK) st = batch_enqueue(c, g->reqs.data(), n);
  if (st == TSI_OK && cudaEventRecordWithFlags(c->ev1, c->stream, cudaEventRecordExternal) != cudaSuccess)
    st = set_err(TSI_ERR_CUDA, "event record in capture");
  cudaGraph_t graph = nullptr;
  cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
  if (st != TSI_OK || e != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();  // a failed capture leaves an error behind
    delete g;
    if (st != TSI_OK) return st;
    return set_err(TSI_ERR_CUDA, cudaGetErrorString(e));
  }
  g->graph = graph;
  e = cudaGraphInstantiate(&g->exec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    delete g;
    return set_err(TSI_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = g;
  return TSI_OK;
}

TSI_API tsi_status tsi_batch_graph_launch(tsi_batch_graph *g) {
  if (!g) return set_err(TSI_ERR_INVALID_ARGUMENT, "null graph");
  tsi_ctx *c = g->ctx;
  CK(cudaSetDevice(c->device));
  // the previous replay has read the pinned descriptors before they change
  CK(cudaStreamSynchronize(c->stream));
  // the captured uploads read the pinned descriptors: refresh them from the
  // caller's requests (same scenes, same image sizes as captured)
  const uint32_t n = (uint32_t)g->reqs.size();
  for (uint32_t i = 0; i < n; ++i) {
    const tsi_request &r = g->user[i], &cap = g->reqs[i];
    if (r.scene != cap.scene || (r.uniforms == nullptr) != (cap.uniforms == nullptr) ||
        (r.uniforms && (r.uniforms->resolution[0] != r.scene->img_w || r.uniforms->resolution[1] != r.scene->img_h)))
      return set_err(TSI_ERR_INVALID_ARGUMENT, "requests differ from the captured ones (scene or image size)");
    fill_launch(r.scene, i, r.time, r.t0_or_nan, g->global[i] != 0, c->h_scenes[i], c->h_recs[i]);
    const tsi_status dst = drain_copy(r.scene);  // the replay's traces rewrite the frame buffers
    if (dst != TSI_OK) return dst;
    if (r.uniforms) {
      const tsi_status st = fill_trace(r.scene, r.uniforms);
      if (st != TSI_OK) return st;
    }
  }
  CK(cudaGraphLaunch(g->exec, c->stream));
  g->launched = true;
  return TSI_OK;
}

TSI_API tsi_status tsi_batch_graph_wait(tsi_batch_graph *g, tsi_stats *stats) {
  if (!g) return set_err(TSI_ERR_INVALID_ARGUMENT, "null graph");
  tsi_ctx *c = g->ctx;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->stream));
  if (!g->launched) return set_err(TSI_ERR_INVALID_ARGUMENT, "graph not launched");
  const uint32_t n = (uint32_t)g->reqs.size();
  if (stats) {
    std::vector<tsi_scene *> sc(n);
    for (uint32_t i = 0; i < n; ++i) sc[i] = g->reqs[i].scene;
    fill_stats_sum(c, sc.data(), n, stats);
    float ms = 0.0f;
    CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    stats->device_ms = ms;
  }
  return status_from_error_bits(readback_error_or(c, n));
}

TSI_API void tsi_batch_graph_destroy(tsi_batch_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
}

}  // extern "C"
