// device_types.h — HBM data layout shared by the host runtime and kernels.
//
// The reference stores each voxel as one 88-byte struct (compute.wgsl:
// 3003-3016) allocated one at a time from a free-list queue (3437-3460), and
// gives every thread a private 128 KB copy of the tape (3562).  Here:
//  - voxels live in structure-of-arrays form, allocated in bricks of 8
//    siblings, so a parent stores one child index (the first voxel of its
//    brick) instead of children[8];
//  - tapes are shared, read-only, 8 bytes per instruction (tape_format.h);
//    per-sibling-group pruned tapes are appended to a per-frame arena and
//    chained to the tape they were derived from.
#pragma once
#include <stdint.h>
#include <vector_types.h>

#include "tape_format.h"

#define TSI_MAX_LEVELS 24
// Work lists are indexed by launch step, not by octree level: in the plain
// and batched forms step = level, in the continuous (served) form scenes
// join at any step and run one level per step.  Per-step counters live in a
// ring of TSI_STEP_RING entries; the item lists are double-buffered by the
// step's parity.
#define TSI_STEP_RING 32u
#define TSI_STEP_MASK (TSI_STEP_RING - 1u)
#define TSI_PRUNE_MAX_REGS 64u  // pruning tracks liveness in one 64-bit mask
#define TSI_PRUNE_MIN_LEN 8u    // shorter tapes are not worth pruning

enum tsi_scene_flags {
  SF_POINTSAMPLE = 1u << 0,
  SF_FASTENABLED = 1u << 1,
  SF_LIPSCHITZ = 1u << 2,
  SF_SWEPT = 1u << 3,
  SF_ALWAYS_DERIV = 1u << 4,  // !fast_normals && normal_viz (compute.wgsl:3780)
  SF_PRUNING = 1u << 5,
  SF_DIRECTED = 1u << 6,  // outward rounding (tsi_rounding TSI_ROUND_DIRECTED)
};

enum tsi_error_bits {
  EB_OOM = 1u << 0,
  EB_QUEUE_FULL = 1u << 1,
  EB_WATCHDOG = 1u << 2,
  EB_LOG_OOM = 1u << 3,
  EB_SMEM = 1u << 4,  // a wide cell's working set did not fit the launch's dynamic shared memory
};

struct VoxelPoolDev {
  float4 *box_xy;    // x.lo, x.hi, y.lo, y.hi
  float2 *box_z;     // z.lo, z.hi
  float *t;          // time of last evaluation
  float *time_err;
  float *f;          // -1 full, 0 ambiguous, +1 empty
  float *fast;
  uint32_t *child;   // first voxel of the child brick, TSI_NONE = no children
  float4 *normal;    // dx, dy, dz, 0
  uint32_t *free_list;  // brick ids free since earlier frames
  uint32_t *pending;    // brick ids freed during the current frame
  uint32_t cap_bricks;
  uint32_t pad;
};

struct SceneCounters {
  int32_t free_count;      // may dip below 0 while popping; fixed at frame end
  uint32_t bump;           // next never-used brick (brick 0 holds the root)
  uint32_t pending_count;
  uint32_t live_bricks;
};

// Bundled form of a scene's full tape (tape_compile.h WideTape), evaluated
// with one block per cell for items whose tape is long.
struct WideDev {
  const uint4 *slots;         // [3][nslots]: words 0-3, 4-7, 8-11 of each slot (tape_compile.h)
  const uint2 *bundles;       // first slot, slot count (padding included)
  const uint32_t *narrow_mm;  // min/max ordinal per narrow instruction
  uint32_t nslots;
  uint32_t nbundles;
  uint32_t nvalues;           // SSA values (nslots + 4); the field is the last
  uint32_t min_len;           // tapes at least this long go to the wide path
  uint32_t deep_level;        // children at this level or deeper use deep_min_len (TSI_NONE: never)
  uint32_t deep_min_len;
  uint32_t ncontrib;          // reverse contribution records per cell
  uint32_t prune_level;       // wide items at this octree level or deeper prune their group's tape
  uint32_t global;            // 1: the cell working set lives in the block's slice of
                              // LaunchParams::wscratch (too large for shared memory)
  uint32_t arg_gbase[4];      // records of x, y, z, t (TSI_NONE: one user)
  uint32_t arg_gcount[4];
};

struct SceneLaunch {
  WideDev wide;
  VoxelPoolDev pool;
  SceneCounters *ctr;
  float eps;          // 10 * 2^-localsubdiv
  float delta;
  float fast_thresh;  // delta * fast_multiplier
  float time;
  float t0;           // start of the swept interval
  uint32_t flags;
  uint32_t root_rec;
  uint32_t levels;          // octree levels of a frame (the leaves are level levels - 1)
  uint32_t full_len;        // full tape length (instr_full_equiv counter)
  uint32_t narrow_parents;  // parents per narrow item above the leaf level (1, 2 or 4)
};

struct TapeRec {
  const uint2 *code;
  uint32_t len;
  uint32_t nregs;
  uint32_t out_reg;
  uint32_t n_minmax;
  float t_lo, t_hi;   // valid for any cell inside the group's boxes with time in [t_lo, t_hi]
  uint32_t parent;    // record it was pruned from (TSI_NONE for a full tape)
  uint32_t fwd_cost;  // opcost.h forward ops of one cell (fix included)
  uint32_t rev_cost;  // opcost.h reverse ops of one cell
  // A work item of level c_level built from this group holds children of the
  // group's enqueued cells, and each child's time range lies inside its own
  // parent's decision interval, for which that parent's decisions hold.
  // [c_lo, c_hi] is the hull of those intervals: such an item may use the
  // record for any time inside it.  Deeper items (which inherit the record
  // when their group prunes nothing) check [t_lo, t_hi] instead.
  float c_lo, c_hi;
  uint32_t c_level;
};

// A narrow item: up to four sibling parents evaluated by one warp.  A wide
// item: one parent, its eight children evaluated by eight blocks; parent[1]
// is the children's brick (allocated when the item was enqueued, TSI_NONE if
// the pool was exhausted), parent[2] is 1 if that brick is new, parent[3]
// counts the children done in its low byte (the last one finishes the group)
// and collects the enqueued ones in bits 8-15.
struct WorkItem {
  uint32_t scene;
  uint32_t rec;
  uint32_t n;         // valid parents (1..4; 1 for a wide item)
  uint32_t level;     // level of the parents
  uint32_t parent[4];
};

// What a wide item's child cell leaves for the block that finishes the group.
struct CellInfo {
  float nl, nh;       // time range its children will be evaluated over
  uint32_t enq;       // 1: enqueued for subdivision
  uint32_t pad;
};

enum tsi_stat_index {
  ST_PARENTS = 0, ST_EVAL, ST_REVERSE, ST_SKIPPED, ST_AMBIG, ST_EMPTY, ST_FULL, ST_ENQUEUED,
  ST_REUSED, ST_INSTR_FWD, ST_INSTR_REV, ST_INSTR_FULL, ST_FP32, ST_BRICK_ALLOC, ST_BRICK_FREE,
  ST_TAPE_WORDS, ST_PRUNE_FALLBACK,
  // SM clock cycles (clock64): wide cells (count, sum, max, and their
  // forward and reverse passes) and narrow items (sum, max)
  ST_WIDE_ITEMS, ST_CYC_WIDE, ST_CYC_WIDE_MAX, ST_CYC_WIDE_FWD, ST_CYC_WIDE_REV, ST_CYC_NARROW,
  ST_CYC_NARROW_MAX,
  // narrow items: on a tape at least the wide threshold long, longest tape
  ST_NARROW_LONG, ST_NARROW_LEN_MAX,
  // narrow items: SM cycles of the first forward pass, the reverse pass and
  // the pruning scan, and the instructions of the first forward pass
  ST_CYC_N_FWD, ST_CYC_N_REV, ST_CYC_N_PRUNE, ST_N_FWD_INSTR,
  // wide items' group finishes: count, SM cycles of the liveness pass, of
  // liveness + compaction + record, and of enqueueing the children
  ST_WIDE_FIN, ST_CYC_FIN_LIVE, ST_CYC_FIN_COMPACT, ST_CYC_FIN_PUSH,
  // wide cells that ran the forward pass again over their children's wider
  // time range (count, SM cycles)
  ST_WIDE_REFWD, ST_CYC_WIDE_REFWD, ST_COUNT
};

// Ring and buffer indices of one launch step.
struct StepIdx {
  uint32_t cur, next;  // counters of this step's lists and of the next step's
  uint32_t buf, nbuf;  // item buffers (step parity)
};

struct LaunchParams {
  SceneLaunch *scenes;
  uint32_t n_scenes;
  uint32_t rec_cap;
  // Tape records: [0, rec_base) are the scenes' root records (one per scene
  // slot); pruned records are taken from a ring over [rec_base, rec_cap) by a
  // 64-bit counter, and the code arena is a ring over code_cap words.  An
  // allocation may not pass the low-water marks (counter values below which
  // records and code may still be read) by a whole ring: the plain form
  // resets counters and marks to 0 per frame; the continuous form moves the
  // marks to the oldest running scene's first step.
  TapeRec *recs;
  unsigned long long *rec_count;
  unsigned long long *rec_low;
  uint32_t rec_base;
  uint32_t pad1;
  uint2 *code_arena;
  unsigned long long *code_count;
  unsigned long long *code_low;
  unsigned long long code_cap;
  // counters at the start of each step (continuous form's low-water marks)
  unsigned long long *step_code_start;  // [TSI_STEP_RING]
  unsigned long long *step_rec_start;   // [TSI_STEP_RING]
  WorkItem *items[2];
  uint32_t *item_count;    // [TSI_STEP_RING]
  uint32_t *item_cursor;   // [TSI_STEP_RING]
  WorkItem *witems[2];     // wide items: one parent each, one block per child cell
  uint32_t *witem_count;   // [TSI_STEP_RING]
  uint32_t *witem_cursor;  // [TSI_STEP_RING], in child cells
  uint32_t witem_cap;      // wide items per level; more go to the narrow list
  uint32_t bm_words;       // branch-decision words per wide cell (2 bits per min/max)
  CellInfo *cell_info[2];  // [witem_cap * 8] per level parity
  unsigned char *wscratch;               // [grid][wscratch_stride]: wide cell working sets
  unsigned long long wscratch_stride;    // of tapes with WideDev::global set
  uint32_t dyn_smem;                     // dynamic shared memory of the launch, bytes
  uint32_t *error_sticky;                // or-ed with the frame's error word at frame end
                                         // (asynchronous inversions), or null
  uint32_t *cell_bits[2];  // [witem_cap * 8][bm_words] per level parity
  uint32_t item_cap;
  uint32_t dealloc_cap;
  uint2 *dealloc[2];       // (scene, brick)
  uint32_t *dealloc_count; // [TSI_STEP_RING]
  uint32_t *dealloc_cursor;
  // per-warp scratch: operand log [slice_len][32] float4, then decisions [slice_len] uint2
  float4 *log_slices;
  uint2 *dec_slices;
  uint32_t slice_len;
  uint32_t pad0;
  float4 *log_overflow;
  // [TSI_STEP_RING], in float4 units: a step's logs are dead once the
  // next step starts, so every step fills the arena from its start
  unsigned long long *log_overflow_used;
  unsigned long long log_overflow_cap;
  uint32_t *error;                  // [n_scenes]: error bits of each scene
  unsigned long long *stats;        // [n_scenes][ST_COUNT]: counters of each scene
  unsigned long long *level_stats;  // [TSI_STEP_RING][ST_COUNT], per refine launch, or null
};

// Slots that join the continuous form at one step (step_begin_kernel's
// parameter).
#define TSI_SEEDS_MAX 256u
struct StepSeeds {
  uint32_t n;       // slots joining at this step
  uint32_t oldest;  // first step of the oldest running slot (low-water marks)
  uint32_t slot[TSI_SEEDS_MAX];
};

static_assert(TSI_MAX_LEVELS + 1 <= TSI_STEP_RING, "a frame's levels fit the step ring");
