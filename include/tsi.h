/*
 * tsi.h — C ABI of the B200 (sm_100a) temporal set inversion library.
 *
 * The library replaces the device hot path of TemporalSetInversion
 * (src/compute.wgsl entry points `main`, `rt_main`, `buf_main`) and the
 * host contract around it (src/main.rs `State::compute` / `State::render`,
 * src/ir.rs tape lowering, src/uniforms.rs, src/camera.rs).  The reference
 * binds its path through a wgpu bind group (main.rs:305-427,
 * compute.wgsl:3066-3087,3431-3435); this header is the FFI that replaces
 * it.  Every entry point names the reference interface it stands in for.
 *
 * Conventions
 *  - Every function returns tsi_status (0 = TSI_OK).  Device-side failures
 *    (pool exhausted, work list full, bounded wait expired) are reported as
 *    error words read back by the host, never as traps.
 *  - The caller owns host memory; the library owns device memory.
 *  - Handles are not thread safe.  One CUDA stream per tsi_ctx; a server
 *    owns its own worker thread and stream.
 *  - No CPU fallback: when no sm_100 device is present, tsi_create returns
 *    TSI_ERR_NO_DEVICE.  Only tsi_ir_lower, tsi_status_string and
 *    tsi_version work without a device.
 */
#ifndef TSI_H
#define TSI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TSI_ABI_VERSION 1u

#if defined(_WIN32)
#define TSI_API __declspec(dllexport)
#else
#define TSI_API __attribute__((visibility("default")))
#endif

typedef enum tsi_status {
  TSI_OK = 0,
  TSI_ERR_INVALID_ARGUMENT = 1,
  TSI_ERR_PARSE = 2,          /* LLVM IR text the lowering cannot read (ir.rs panics there) */
  TSI_ERR_CUDA = 3,           /* a CUDA runtime call failed */
  TSI_ERR_OOM = 4,            /* voxel pool or device arena exhausted */
  TSI_ERR_QUEUE_FULL = 5,     /* a device work list overflowed (compute.wgsl:3159 drops silently) */
  TSI_ERR_WATCHDOG = 6,       /* a bounded device wait gave up */
  TSI_ERR_BAD_OPCODE = 7,     /* opcode outside ir.rs:8-43 in an uploaded tape */
  TSI_ERR_TAPE_TOO_WIDE = 8,  /* tape needs more than 256 interval registers */
  TSI_ERR_NO_DEVICE = 9,      /* no sm_100 CUDA device */
  TSI_ERR_BUFFER_TOO_SMALL = 10,
  TSI_ERR_BUSY = 11,
  TSI_ERR_NOT_FOUND = 12,
  TSI_ERR_SHUTDOWN = 13
} tsi_status;

/* ---------------------------------------------------------------------
 * Tape instruction in the reference's own 32-byte layout.
 * Mirrors ir.rs:88-97 (GPUInstruction) and compute.wgsl:2989-2996.
 *   opcode_uses = ((op | op_top << 14) << 16) | uses      (ir.rs:171-175)
 *   larg_rarg   = larg << 16 | rarg                        (ir.rs:176)
 *   op_top: 0 reg,reg  1 reg,literal (and unary)  2 literal,reg  3 none
 * ------------------------------------------------------------------- */
typedef struct tsi_gpu_instruction {
  uint32_t index_;
  uint32_t opcode_uses;
  uint32_t larg_rarg;
  float literal;
  float val[2];
  float sens[2];
} tsi_gpu_instruction;

/* Opcode numbers, ir.rs:9-41. */
enum {
  TSI_OP_NOP = 0, TSI_OP_ARGX = 1, TSI_OP_ARGY = 2, TSI_OP_ARGZ = 3, TSI_OP_ARGW = 4,
  TSI_OP_ADD = 5, TSI_OP_SUB = 6, TSI_OP_MUL = 7, TSI_OP_DIV = 8, TSI_OP_EXP = 9,
  TSI_OP_LOG = 10, TSI_OP_SQR = 11, TSI_OP_SQRT = 12, TSI_OP_POW = 13, TSI_OP_SIN = 14,
  TSI_OP_COS = 15, TSI_OP_NEG = 16, TSI_OP_MIN = 17, TSI_OP_MAX = 18, TSI_OP_ABS = 19,
  TSI_OP_CUP = 20, TSI_OP_CAP = 21, TSI_OP_BR = 22, TSI_OP_PHI = 23, TSI_OP_TRUNC = 24,
  TSI_OP_FLOOR = 25, TSI_OP_CEIL = 26, TSI_OP_SIGN = 27, TSI_OP_RET = 28, TSI_OP_MOD = 29,
  TSI_OP_ATAN2 = 30
};

typedef enum tsi_rounding {
  TSI_ROUND_NEAREST = 0,   /* plain f32 as compute.wgsl:2539-2975 (parity mode) */
  TSI_ROUND_DIRECTED = 1   /* outward rounded, rigorous enclosures */
} tsi_rounding;

/* Runtime form of the compile-time PARAMETERS block, compute.wgsl:3494-3511. */
typedef struct tsi_params {
  int32_t localsubdiv;          /* epsilon = 10 * 2^-localsubdiv (compute.wgsl:3521) */
  float delta;                  /* temporal error tolerance */
  int32_t pointsample;          /* point_sample */
  int32_t fastenabled;
  int32_t lipschitz_corrected;
  int32_t swept_volume;         /* sweptvolume */
  int32_t fast_normals;         /* per-pixel finite-difference normals in the tracer */
  int32_t normal_viz;
  int32_t rounding_mode;        /* tsi_rounding */
  float fast_multiplier;        /* 1.0 in the reference */
  int32_t scene_id;             /* `scene`: camera offsets of rt_main (compute.wgsl:4670-4683) */
  float octree_darken_factor;   /* 0.98 */
  float root_lo[3];             /* root box, ir.rs:343-347: [-5,5]^3 */
  float root_hi[3];
  int32_t pruning;              /* per-cell tape pruning (1 = on); never changes results */
  float swept_dt;               /* swept interval length when t0 is NaN (1/60, compute.wgsl:3605) */
  int32_t cinematic;            /* path tracing with sun light, shadow rays and sky (`cinematic`,
                                 * compute.wgsl:3499, get_color_single 4444-4523) */
  int32_t samples;              /* cinematic samples per pixel (`totalsamples`, 3507) */
  int32_t see_background;       /* cinematic: primary misses see the sky (3506) */
} tsi_params;

/* Uniforms, uniforms.rs:8-17 / compute.wgsl:3419-3428 (96 bytes).
 * view_matrix is camera-to-world, column major (camera.rs:78-80). */
typedef struct tsi_uniforms {
  float view_matrix[16];
  uint32_t resolution[2];
  float time;
  float lasttime;
  float rendermode;
  float _padding[3];
} tsi_uniforms;

/* Per-call counters (there are none in the reference; Memory at
 * compute.wgsl:3041-3048 only tracks allocated voxels and work_left). */
typedef struct tsi_stats {
  uint64_t parents_expanded;    /* work items dequeued (compute.wgsl:3528) */
  uint64_t cells_evaluated;     /* child cells whose tape ran forward (3633) */
  uint64_t cells_reverse;       /* of which ran reverse AD (3785) */
  uint64_t cells_skipped;       /* swept interior cells not evaluated (3629) */
  uint64_t cells_ambiguous;
  uint64_t cells_empty;
  uint64_t cells_full;
  uint64_t cells_enqueued;      /* re-enqueued for subdivision (4024) */
  uint64_t cells_reused;        /* ambiguous internal cells kept with their subtree */
  uint64_t instr_forward;       /* interval instructions executed forward */
  uint64_t instr_reverse;       /* interval instructions executed in reverse */
  uint64_t instr_full_equiv;    /* cells_evaluated x full tape length */
  uint64_t fp32_ops;            /* algorithmic FP32 ops of the executed instructions (opcost.h) */
  uint64_t bricks_allocated;    /* 8-voxel bricks taken from the pool */
  uint64_t bricks_freed;
  uint64_t voxels_live;
  uint64_t items_high_water;    /* largest per-level work list */
  uint64_t tape_words;          /* pruned tape instructions written */
  uint64_t prune_fallbacks;     /* warps that re-ran on the full tape */
  /* Algorithmic FP32 work (opcost.h table) of the frame on the FULL tape,
   * whatever pruning saved: cells_evaluated x the full tape's forward cost
   * (fix included), and cells_reverse x its reverse cost (every instruction,
   * the zero-sensitivity skip of compute.wgsl:3802-3805 not subtracted). */
  uint64_t fp32_ops_full_fwd;
  uint64_t fp32_ops_full_rev;
  /* Cells evaluated without tape pruning although pruning was requested:
   * pruning tracks liveness in a 64-bit mask, so tapes of more than 64
   * interval registers run unpruned (same results, more work). */
  uint64_t cells_unpruned_regs;
  uint32_t levels;
  uint32_t error_flags;
  float device_ms;              /* device time of the call (CUDA events) */
  float reserved;
} tsi_stats;

/* A cell of the resident octree, keyed by (level, ix, iy, iz). */
typedef struct tsi_cell {
  uint32_t level, ix, iy, iz;
  float f;          /* -1 full, 0 ambiguous, +1 empty (compute.wgsl:4012-4033) */
  float t;          /* time of last evaluation */
  float time_err;
  float fast;
  float dx, dy, dz; /* interval-gradient midpoints (compute.wgsl:3967-3969) */
  uint32_t has_children;
  float x[2], y[2], z[2];
} tsi_cell;

/* Rendered frame.  Pointers are HOST pointers owned by the caller; any may
 * be NULL to skip that output.  rgba is compute.wgsl:4687 `pixels[]`. */
typedef struct tsi_image {
  uint32_t width, height;
  float *rgba;      /* width*height*4 */
  float *depth;     /* width*height, -1 on miss (compute.wgsl:4398-4401) */
  float *normal;    /* width*height*3, normal at hit */
} tsi_image;

/* Device pointers to a scene's last rendered frame (library owned). */
typedef struct tsi_image_device {
  uint32_t width, height;
  const float *rgba, *depth, *normal;
} tsi_image_device;

typedef struct tsi_device_opts {
  int32_t device;               /* CUDA ordinal */
  uint64_t work_item_capacity;  /* per-level work list capacity (0 = default) */
  uint64_t tape_arena_words;    /* pruned tape arena, 8-byte words (0 = default, 256 Mi words) */
  uint64_t log_arena_bytes;     /* reverse-AD operand log of long narrow tapes (0 = default, 4 GiB) */
  uint32_t watchdog_iters;      /* bound on every device wait (0 = default) */
  uint32_t max_scenes_per_launch; /* batch width (0 = default 64) */
  uint32_t wide_smem_bytes;     /* shared memory a wide cell's working set may take; larger ones run
                                 * from global scratch (0 = what keeps the narrow path's occupancy) */
  uint64_t hbm_budget_bytes;    /* device bytes the context's scenes may hold together (voxel pools
                                 * and frame buffers); a scene or frame size beyond it is refused
                                 * with TSI_ERR_OOM (0 = no limit) */
} tsi_device_opts;

typedef struct tsi_ctx tsi_ctx;
typedef struct tsi_tape tsi_tape;
typedef struct tsi_scene tsi_scene;

typedef struct tsi_tape_info {
  uint32_t instruction_count;   /* including the 4 ARG slots (main.rs:744) */
  uint32_t registers;           /* interval registers after allocation */
  uint32_t minmax_count;
  uint32_t reserved;
} tsi_tape_info;

/* ---------------- library ---------------- */
TSI_API uint32_t tsi_version(void);
TSI_API const char *tsi_status_string(tsi_status s);
TSI_API void tsi_default_params(tsi_params *p);

/* Replaces State::new's adapter/device setup (main.rs:97-122) and the
 * buffer allocations of main.rs:208-303 (now lazily sized, HBM resident). */
TSI_API tsi_status tsi_create(const tsi_device_opts *opts, tsi_ctx **out);
/* Releases the context and every tape and scene still alive on it; their
 * handles become invalid. */
TSI_API void tsi_destroy(tsi_ctx *ctx);
TSI_API tsi_status tsi_synchronize(tsi_ctx *ctx);

/* ---------------- tapes ---------------- */
/* Host-only restatement of ir.rs:190-366 (parseLLVMIR + IR::new + to_gpu):
 * lowers the `@_Z1fffff` function of `text` into the 32-byte layout, with
 * the four ARG slots first (values = root box, time).  Writes at most `cap`
 * instructions and stores the full count in *n (no 4096 cap). */
TSI_API tsi_status tsi_ir_lower(const char *text, size_t len, float time,
                                tsi_gpu_instruction *out, uint32_t cap, uint32_t *n);

/* Uploads a tape in the ir.rs layout (main.rs:743-746 writes it into
 * tapes[0]); the library repacks it into the packed device tape. */
TSI_API tsi_status tsi_tape_upload(tsi_ctx *ctx, const tsi_gpu_instruction *instr, uint32_t n,
                                   tsi_tape **out);
/* tsi_ir_lower + tsi_tape_upload without the 16-bit limits of ir.rs:99-101. */
TSI_API tsi_status tsi_tape_from_llvm_ir(tsi_ctx *ctx, const char *text, size_t len,
                                         tsi_tape **out);
TSI_API tsi_status tsi_tape_info_get(const tsi_tape *tape, tsi_tape_info *info);
TSI_API void tsi_tape_destroy(tsi_tape *tape);

/* Interval evaluation of a tape on n space-time boxes (the body of
 * compute.wgsl:3632-3970 without the octree).  boxes: n x 8 floats
 * (x.lo,x.hi,y.lo,y.hi,z.lo,z.hi,t.lo,t.hi), host memory.  out: n x 10
 * floats: field (lo,hi) then sens of x,y,z,t (lo,hi each); sens are written
 * when `reverse` is nonzero, else zero. */
TSI_API tsi_status tsi_tape_eval_boxes(tsi_ctx *ctx, const tsi_tape *tape, uint32_t n,
                                       const float *boxes, int32_t rounding_mode,
                                       int32_t reverse, float *out);

/* ---------------- scenes (plain path) ---------------- */
TSI_API tsi_status tsi_scene_create(tsi_ctx *ctx, const tsi_tape *tape, const tsi_params *params,
                                    uint64_t voxel_capacity, tsi_scene **out);
TSI_API void tsi_scene_destroy(tsi_scene *scene);
/* first_eval of main.rs:730-766: empty pool, root voxel 0 = root box. */
TSI_API tsi_status tsi_scene_reset(tsi_scene *scene);
/* One dispatch of `main` (main.rs:776-783) preceded by buf_main's
 * re-seeding of the root (compute.wgsl:4706).  time = uniforms.time;
 * t0_or_nan: start of the swept interval (NaN = time - swept_dt). */
TSI_API tsi_status tsi_scene_invert(tsi_scene *scene, float time, float t0_or_nan,
                                    tsi_stats *stats);
/* tsi_scene_invert (one `main` dispatch, main.rs:776-783) without waiting
 * for it, which the reference's event loop never does: the frame is queued on the context's
 * stream and the call returns at once, so the host can queue the frame's
 * trace (tsi_scene_trace_async) and the next frames while the GPU works.
 * tsi_scene_invert_wait waits for everything queued and returns an error
 * status if any inversion queued this way since the last wait hit a device
 * limit (voxel pool, work list, log arena), and, when stats is not NULL,
 * the counters and device time of the last inversion queued.  Plain
 * inversions in between report their own errors. */
TSI_API tsi_status tsi_scene_invert_async(tsi_scene *scene, float time, float t0_or_nan);
TSI_API tsi_status tsi_scene_invert_wait(tsi_scene *scene, tsi_stats *stats);
/* One dispatch of `rt_main` (main.rs:649-656).  `out` may be NULL to keep
 * the frame on the device only (see tsi_scene_image_device). */
TSI_API tsi_status tsi_scene_trace(tsi_scene *scene, const tsi_uniforms *u, tsi_image *out,
                                   tsi_stats *stats);
TSI_API tsi_status tsi_scene_image_device(tsi_scene *scene, tsi_image_device *out);
/* tsi_scene_trace (one `rt_main` dispatch, main.rs:649-656) into host
 * buffers without waiting for the frame: the
 * trace is queued behind the scene's earlier work and the frame's copy to
 * `out` runs on the context's copy stream, overlapping the caller's next
 * device work (the next tsi_scene_invert, say).  `out`'s buffers should be
 * pinned host memory (else the copy is not asynchronous) and must stay
 * valid and unread until tsi_scene_trace_wait returns; the scene's next
 * trace waits on the device for this copy to finish. */
TSI_API tsi_status tsi_scene_trace_async(tsi_scene *scene, const tsi_uniforms *u, tsi_image *out);
/* Waits until the frame of the scene's last tsi_scene_trace_async is in
 * host memory. */
TSI_API tsi_status tsi_scene_trace_wait(tsi_scene *scene);

/* No counterpart in the reference (its workgroup shape is fixed at
 * compute.wgsl:3513).  Child cells whose pruned tape is at least the tape's
 * wide threshold are evaluated one cell per 256-thread block from the
 * tape's bundled SSA form; shorter ones one warp per 8-cell group.  Results
 * are identical for every threshold; only the speed changes.  Tapes shorter
 * than 256 instructions, or whose wide working set would exceed 8 MiB per
 * cell, have no bundled form: they report UINT32_MAX (narrow only) and
 * ignore a new value. */
TSI_API uint32_t tsi_tape_wide_threshold(const tsi_tape *tape);
TSI_API tsi_status tsi_tape_set_wide_threshold(tsi_tape *tape, uint32_t min_len);
// A second wide threshold for children at octree level `level` or deeper
// (levels counted from the root's children at 0): deep levels hold many
// cells, where the narrow path's throughput beats the wide path's latency.
// level = 0xffffffff (the default) turns it off.  Results never depend on
// the thresholds.
TSI_API tsi_status tsi_tape_set_wide_threshold_deep(tsi_tape *tape, uint32_t level, uint32_t min_len);
TSI_API tsi_status tsi_tape_wide_threshold_deep(const tsi_tape *tape, uint32_t *level, uint32_t *min_len);
// Parents per narrow work item above the leaf level (1, 2 or 4; default 1):
// a narrow item evaluates the 8 children of each of its parents with one
// warp, so fewer parents per item put more warps in flight (latency) and
// more fill the lanes (throughput).  Leaves always take 4.  Results never
// depend on it.
TSI_API tsi_status tsi_tape_set_narrow_parents(tsi_tape *tape, uint32_t parents);
TSI_API uint32_t tsi_tape_narrow_parents(const tsi_tape *tape);
// First octree level (of the parents) from which a wide item's group prunes
// its tape for the children (a liveness pass over the bundled tape after the
// eight cells are done).  Above it the children take the wide path, which
// evaluates the full tape anyway, so the pass and the second decision
// interval of the forward pass are skipped.  0xffffffff (the default):
// half the scene's levels; a level past the last: the wide path never
// prunes.  Results never depend on it.
TSI_API tsi_status tsi_tape_set_wide_prune_level(tsi_tape *tape, uint32_t level);
TSI_API uint32_t tsi_tape_wide_prune_level(const tsi_tape *tape);

#define TSI_AUTOTUNE_MAX 16
typedef struct tsi_autotune_result {
  uint32_t wide_threshold;          /* chosen, now set on the scene's tape */
  uint32_t candidates;              /* thresholds tried (0: narrow-only tape) */
  uint32_t threshold[TSI_AUTOTUNE_MAX];
  float ms[TSI_AUTOTUNE_MAX];       /* best of `reps` runs over `times`, device ms */
  uint32_t deep_level;              /* chosen deep-level threshold (tsi_tape_set_wide_threshold_deep); */
  uint32_t deep_threshold;          /* deep_level 0xffffffff: none beat the single threshold */
  uint32_t narrow_parents;          /* chosen parents per narrow item (tsi_tape_set_narrow_parents) */
  uint32_t wide_prune_level;        /* chosen prune level (tsi_tape_set_wide_prune_level) */
} tsi_autotune_result;
/* Times the scene's inversion over the frames `times` (the first from a
 * reset octree, the rest carried over) for each candidate wide threshold,
 * best of `reps`, and keeps the fastest on the scene's tape (shared by every
 * scene of that tape); then, one knob at a time, a deep-level threshold, the
 * parents per narrow item and the wide path's prune level, each kept only
 * when it is faster.  The scene is left reset. */
TSI_API tsi_status tsi_scene_autotune(tsi_scene *scene, const float *times, uint32_t ntimes, uint32_t reps,
                                      tsi_autotune_result *out);
/* Copies the scene's last rendered frame (e.g. from a graph replay or the
 * server, which keep frames on the device) into host buffers; out's size
 * must match the frame. */
TSI_API tsi_status tsi_scene_image_copy(tsi_scene *scene, tsi_image *out);
/* Octree as cells keyed by (level, ix, iy, iz), depth-first order.
 * With out == NULL only the count is returned. */
TSI_API tsi_status tsi_scene_readback_cells(tsi_scene *scene, tsi_cell *out, uint64_t cap,
                                            uint64_t *n);
/* Keys of the leaves the tracer can hit (compute.wgsl:4302, 4313): cells
 * with f <= 0 and no children, depth-first order.  With out == NULL only
 * the count is returned. */
typedef struct tsi_leaf {
  uint32_t level, ix, iy, iz;
} tsi_leaf;
TSI_API tsi_status tsi_scene_readback_leaves(tsi_scene *scene, tsi_leaf *out, uint64_t cap, uint64_t *n);
/* Resident-octree snapshot for eviction and restore (no counterpart in the
 * reference, whose octree lives in one wgpu buffer for the process): the
 * voxel pool up to its high-water mark, the free list and the allocation
 * counters, as one host blob.  Taken between frames.  Restore needs a scene
 * with the same tape and parameters and a pool at least as large; the
 * scene then continues exactly where the snapshot's scene was. */
TSI_API tsi_status tsi_scene_snapshot_size(tsi_scene *scene, uint64_t *bytes);
TSI_API tsi_status tsi_scene_snapshot(tsi_scene *scene, void *host, uint64_t cap, uint64_t *bytes);
TSI_API tsi_status tsi_scene_restore(tsi_scene *scene, const void *host, uint64_t bytes);
TSI_API tsi_status tsi_scene_get_params(const tsi_scene *scene, tsi_params *out);
TSI_API uint64_t tsi_scene_device_bytes(const tsi_scene *scene);
/* No counterpart in the reference: the device bytes all scenes of the
 * context hold, the figure tsi_device_opts.hbm_budget_bytes admits
 * against.  A server under a memory budget evicts an idle scene with
 * tsi_scene_snapshot + tsi_scene_destroy and readmits it with
 * tsi_scene_create + tsi_scene_restore. */
TSI_API uint64_t tsi_scenes_device_bytes(const tsi_ctx *ctx);

/* ---------------- batched form ---------------- */
typedef struct tsi_request {
  tsi_scene *scene;
  float time;
  float t0_or_nan;
  const tsi_uniforms *uniforms;  /* NULL: invert only */
  tsi_image *out;                /* NULL: keep the frame on the device */
  tsi_stats *stats;              /* may be NULL */
} tsi_request;

/* Inverts all requests' scenes in one fused launch sequence (every level
 * of every scene shares each launch); each scene's trace starts on a
 * low-priority stream as soon as its own last level is done.  Scenes must be
 * distinct.  More requests than one launch takes (max_scenes_per_launch) run
 * as consecutive launch sequences.  Each request's stats are its own
 * scene's counters and error bits (voxels_live included); device_ms is the
 * whole call's device time.  The return status reports the error bits of
 * every request. */
TSI_API tsi_status tsi_batch_run(tsi_ctx *ctx, tsi_request *reqs, uint32_t n);

/* No counterpart in the reference.  Tunes the wide thresholds of the
 * requests' tapes for running them together: multiplies every tape's
 * threshold by 1, 2, 4 and 8 in turn, times `frames` fused inversions of the
 * requests (each request's time advancing by 1/60 per frame, from reset
 * octrees), and keeps the fastest multiplier on the tapes.  A full GPU
 * favours the narrow path's throughput over the wide path's latency, so a
 * batch often runs faster with larger thresholds than each scene alone.
 * out->wide_threshold is the multiplier kept, out->threshold[k] and
 * out->ms[k] the multipliers tried and their device times.  The scenes are
 * left reset. */
TSI_API tsi_status tsi_batch_autotune(tsi_ctx *ctx, const tsi_request *reqs, uint32_t n, uint32_t frames,
                                      tsi_autotune_result *out);

/* Captures tsi_batch_run for a fixed request set into a CUDA graph and
 * replays it.  The request array must stay valid while the graph exists:
 * every launch waits for the previous replay, then re-reads each request's
 * time, t0 and uniforms (camera, time) from it; scenes and image sizes must
 * stay as captured.  Images stay on the device (tsi_scene_image_device). */
typedef struct tsi_batch_graph tsi_batch_graph;
TSI_API tsi_status tsi_batch_graph_create(tsi_ctx *ctx, tsi_request *reqs, uint32_t n,
                                          tsi_batch_graph **out);
TSI_API tsi_status tsi_batch_graph_launch(tsi_batch_graph *g);
/* Waits for the last replay and reports it: the status from its scenes'
 * error words (voxel pool, work list, log arena, watchdog) and, when stats
 * is not NULL, its counters summed over the batch with device_ms = the
 * replay's device time.  Plain calls on the same context between the launch and the
 * wait overwrite what it reads. */
TSI_API tsi_status tsi_batch_graph_wait(tsi_batch_graph *g, tsi_stats *stats);
TSI_API void tsi_batch_graph_destroy(tsi_batch_graph *g);

/* ---------------- one animation split at the root ----------------
 * No counterpart in the reference, which keeps one octree per device.  The
 * root's subtrees are independent for inversion, so one animation can be
 * cut at `level` into 8^level subtrees, each inverted as a scene of its own
 * (on this GPU or spread over GPUs), each traced over the whole image, and
 * the frames composited by nearest depth. */

/* `full` with its root box replaced by the box of cell (level, ix, iy, iz)
 * of the full octree, index = ix + n (iy + n iz), n = 2^level: the child
 * bounds of compute.wgsl:3582-3589 applied `level` times, so the subtree's
 * cells have the full octree's bounds bit for bit, and its leaves the full
 * octree's epsilon (which depends on localsubdiv only, 3521).  The subtree
 * root is expanded every frame, like the reference's root (buf_main,
 * 4690-4708): on a fresh octree its cells equal the full octree's cells of
 * that subtree; on later frames its top cells are refreshed every frame
 * where the full octree may carry them over. */
TSI_API tsi_status tsi_params_subtree(const tsi_params *full, uint32_t level, uint32_t index, tsi_params *out);

/* A composited frame in device memory (caller owned, e.g. tensors of a
 * framework): rgba 4, depth 1, normal 3 floats and one key per pixel.
 * key = (bits of depth) << 32 | subtree index for a hit, 0x7fffffff << 32 |
 * subtree index for a miss, so the nearest hit has the least key (ties and
 * all-miss pixels go to the lowest subtree index) and keys are positive as
 * signed 64-bit integers (a collective's MIN over int64 orders them). */
typedef struct tsi_frame_device {
  uint32_t width, height;
  float *rgba, *depth, *normal;
  uint64_t *key;
} tsi_frame_device;
#define TSI_COMPOSITE_MAX 64
/* Per pixel, the last traced frame of the scene with the least key among
 * `scenes` (subtree indices `ids`, n <= TSI_COMPOSITE_MAX, all frames of
 * out's size) into `out`.  Returns when `out` is written. */
TSI_API tsi_status tsi_frames_composite(tsi_ctx *ctx, tsi_scene *const *scenes, const uint32_t *ids, uint32_t n,
                                        tsi_frame_device *out);
/* Zeroes (all bits) every pixel of `frame` whose key differs from
 * `global_key` (device, the MIN of all parts' keys): after it, the parts'
 * frames summed as 32-bit integers give the composite of all parts bit for
 * bit.  Returns when `frame` is written. */
TSI_API tsi_status tsi_frame_keep_nearest(tsi_ctx *ctx, const uint64_t *global_key, tsi_frame_device *frame);

/* ---------------- serving ---------------- */
/* No counterpart in the reference (its frames are driven by the window's
 * event loop, main.rs:978-1063, and each `main` dispatch's persistent
 * workgroups dequeue until the queue drains, compute.wgsl:3525-3556).
 * A server owns a worker thread that runs requests on one context with
 * continuous batching: a request joins the running inversion at the next
 * launch step as soon as a slot is free and its scene has no other request
 * running (a scene's requests run in submission order), runs one octree
 * level per step alongside the other slots, and is traced on a
 * low-priority stream while the others go on.  A request's frame buffers
 * are admitted against the context's memory budget at submission (and
 * again when it starts); one that would exceed it completes with
 * TSI_ERR_OOM.  With TSI_SERVER_STATIC_BATCHES the worker instead fuses the
 * queued requests of distinct scenes into one tsi_batch_run at a time (the
 * earlier form, kept for comparison).  While a server exists only the
 * server uses its context.  A request's uniforms, image and stats pointers
 * must stay valid until its ticket completes; its stats are its own scene's
 * counters, with device_ms from its start to its frame being ready. */
typedef struct tsi_server tsi_server;
#define TSI_SERVER_STATIC_BATCHES 1u
typedef struct tsi_server_opts {
  uint32_t max_batch;       /* requests running at once (0: the context's maximum) */
  uint32_t flags;           /* TSI_SERVER_STATIC_BATCHES */
  uint32_t max_queue;       /* queued requests beyond which submit returns TSI_ERR_BUSY (0: 4096) */
  uint32_t reserved;
} tsi_server_opts;
typedef struct tsi_server_stats {
  uint64_t completed;       /* requests finished */
  uint64_t batches;         /* launch steps (fused launches with TSI_SERVER_STATIC_BATCHES) */
  float mean_batch;         /* requests finished per step or launch */
  float p50_ms, p99_ms;     /* submit-to-completion latency of finished requests */
  float max_ms;
  uint32_t queued;          /* requests waiting to start */
} tsi_server_stats;
TSI_API tsi_status tsi_server_create(tsi_ctx *ctx, const tsi_server_opts *opts, tsi_server **out);
/* Queues one request; *ticket identifies it for tsi_server_poll.
 * TSI_ERR_BUSY when the queue is full, TSI_ERR_OOM when the request's frame
 * cannot fit the context's memory budget. */
TSI_API tsi_status tsi_server_submit(tsi_server *s, const tsi_request *req, uint64_t *ticket);
/* The request's status once it has completed (its stats are filled in and
 * the ticket is released); TSI_ERR_BUSY if it is still pending after
 * waiting up to wait_ms milliseconds; TSI_ERR_NOT_FOUND for an unknown
 * ticket.  latency_ms (may be NULL) receives its submit-to-completion time. */
TSI_API tsi_status tsi_server_poll(tsi_server *s, uint64_t ticket, uint32_t wait_ms, float *latency_ms);
TSI_API tsi_status tsi_server_stats_get(tsi_server *s, tsi_server_stats *out);
/* Stops the worker after the running requests; requests still queued
 * complete with TSI_ERR_SHUTDOWN. */
TSI_API void tsi_server_destroy(tsi_server *s);

/* ---------------- allocation-free evaluation ---------------- */
/* No counterpart in the reference.  tsi_tape_eval_boxes allocates device
 * scratch with cudaMalloc; callers that cannot allocate at call time (a
 * loop recorded into a CUDA graph, a host with a memory budget fixed at
 * start-up, a runtime that forbids allocation on its request path) use this
 * variant instead.  It evaluates `tape` on n boxes already in device memory
 * (n x 8 floats as in tsi_tape_eval_boxes) and writes n x 10 floats to
 * out_dev, on cuda_stream (NULL: the tape context's stream), and returns
 * after enqueueing.  It calls no cudaMalloc, cudaFree or other allocating
 * routine: its scratch is a static device array of TSI_STATIC_SCRATCH_BYTES
 * per device (held by every GPU that loads the library until the process
 * exits), and n x (8 x registers + 16 x tape length) bytes must fit in it,
 * else TSI_ERR_BUFFER_TOO_SMALL (split the call).  Nothing in the array needs
 * to start at zero: each launch writes every register and log entry before
 * reading it.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and loads the evaluation kernel, so make it
 * before any stream capture.  The call makes the tape's device current and
 * puts the caller's current device back before it returns.  All calls share
 * the one array per device: calls that can overlap on the GPU (different
 * streams, or different contexts on the same device) race on it and must be
 * ordered by the caller. */
#define TSI_STATIC_SCRATCH_BYTES (16u << 20)
TSI_API tsi_status tsi_tape_eval_boxes_static(const tsi_tape *tape, uint32_t n, const float *boxes_dev,
                                              int32_t rounding_mode, int32_t reverse, float *out_dev,
                                              void *cuda_stream);
TSI_API uint64_t tsi_static_scratch_bytes(void);

/* Host only.  The frame dump of main.rs:692-715 (save_frames_to_disk):
 * rt_main's f32 RGBA pixels converted to 8-bit RGBA as its image crate does
 * (each channel clamped to [0, 1], times 255, rounded to nearest, halves
 * away from zero; NaN gives 0), ready for a PNG encoder. */
TSI_API void tsi_rgba8_from_frame(const float *rgba, uint64_t n_pixels, uint8_t *out);

/* ---------------- diagnostics (tests and tools) ---------------- */
/* Message of the last failing call on this thread. */
TSI_API const char *tsi_last_error(void);
/* Host-only: lower `text` and report the register allocation (no device).
 * slot_reg, if not NULL, receives the register of each SSA slot. */
TSI_API tsi_status tsi_ir_tape_info(const char *text, size_t len, tsi_tape_info *info, uint32_t *slot_reg,
                                    uint32_t cap);
/* Host-only: packed device words (2 per instruction after the ARG slots) of
 * a tape given in the ir.rs layout. */
TSI_API tsi_status tsi_compile_gpu_instructions(const tsi_gpu_instruction *instr, uint32_t n, uint32_t *words,
                                                uint32_t cap_words, tsi_tape_info *info);
/* Host-only: the bundled (wide) form of a tape given in the ir.rs layout:
 * 12 words per slot after the ARG slots ({handler | fa << 6 | fb << 7,
 * dst | a << 16, b, literal bits, ssa dst, ssa a, ssa b, min/max index,
 * contribution record of a, of b, first record of dst, record count of
 * dst}, TSI_NONE for absent operands and records), 2 words per bundle
 * (first slot, count); info->registers = registers of the bundled form,
 * info->reserved = its output register. */
TSI_API tsi_status tsi_compile_wide_gpu_instructions(const tsi_gpu_instruction *instr, uint32_t n, uint32_t *slots,
                                                     uint32_t cap_slot_words, uint32_t *bundles,
                                                     uint32_t cap_bundle_words, tsi_tape_info *info,
                                                     uint32_t *n_bundles);
/* Elementwise device f32 math, for the math tests: which = 0 sin(a),
 * 1 exp(a), 2 log(a), 3 atan2(a, b), 4 powi(a, (int)b), 5 min(a, b),
 * 6 max(a, b) (minimumNumber / maximumNumber), 7 fminf, 8 fmaxf. */
TSI_API tsi_status tsi_debug_math(tsi_ctx *ctx, int32_t which, uint32_t n, const float *a, const float *b,
                                  float *out);
/* Per-level profile of the context's last inversion: device ms of each
 * level's refinement launch (-1 unless TSI_PROFILE_LEVELS is set in the
 * environment when the context is created) and TSI_LEVEL_COUNTERS counters
 * per level: the tsi_stats fields from parents_expanded to prune_fallbacks
 * (without voxels_live and items_high_water), then wide cells processed
 * and SM clock cycles: wide cells (sum, max), their forward and reverse
 * passes (sums), narrow items (sum, max); then narrow
 * items on a tape at least the wide path's threshold long, and the longest
 * tape a narrow item ran; then narrow items' cycles in the first forward
 * pass, the reverse pass and the pruning scan, and the instructions of the
 * first forward pass; then wide items' group finishes (count) and their
 * cycles in the liveness pass, up to the end of compaction, and in
 * enqueueing the children; then wide cells that ran the forward pass again
 * over their children's wider time range, and its cycles. */
#define TSI_LEVEL_COUNTERS 36
TSI_API tsi_status tsi_debug_level_profile(tsi_ctx *ctx, uint32_t max_levels, float *ms, uint64_t *counters,
                                           uint32_t *n_levels);

#ifdef __cplusplus
}
#endif
#endif /* TSI_H */
