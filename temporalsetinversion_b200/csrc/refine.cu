// refine.cu — octree refinement step kernel (compute.wgsl `main`, 3513-4056).
//
// One launch per octree level, over every scene of the launch.  A warp takes
// one work item: up to four sibling parents (children of one grandparent,
// sharing one tape record) x 8 octants, one child cell per lane.  The tape is
// warp-uniform, so instruction fetch is a broadcast and the handler switch
// never diverges.  Interval registers live in shared memory as
// regs[register][lane] (one column per lane, conflict free).
//
// Per child cell the lane runs, as in the reference:
//   cell setup and temporal interval         compute.wgsl:3582-3626
//   forward interval tape                    3632-3774
//   reverse interval AD (operand log replay) 3776-3970
//   temporal error bound, fast flag          3971-4009
//   classify, re-enqueue or deallocate       4011-4045
// then, per sibling group that re-enqueues cells, prunes the tape: min/max
// instructions whose branch is decided for every enqueued sibling become
// copies (or constants), instructions that no longer reach the output are
// dropped.  Pruning never changes a result: a decided MIN/MAX returns its
// chosen operand bit for bit, and the reverse pass falls back to the full
// tape when a sensitivity overflows (the only case where the dead branch of
// the full tape would contribute, through 0 * inf).
//
// A pruned tape is valid for cells inside its group's boxes whose time
// interval lies inside the interval the decisions were taken on.  The
// children of a re-enqueued cell are evaluated over [child.t, time]; when
// that reaches further back than the cell's own evaluation interval (the
// cell was evaluated at a point in time), the branch decisions are taken
// again by a second forward pass over the widened interval, so the children
// can use the pruned tape instead of an ancestor's.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "device_types.h"
#include "interp.cuh"
#include "wide_interp.cuh"
#include "interval.cuh"
#include "opcost.h"

namespace tsi {

__constant__ uint32_t c_cost_fwd[H_COUNT] = TSI_OPCOST_FWD_INIT;
__constant__ uint32_t c_cost_rr[H_COUNT] = TSI_OPCOST_RR_INIT;

constexpr int kWarps = 8;  // warps per block (block of 256)

// Dynamic shared memory of refine_kernel: the narrow path's register files,
// or the working set of the wide path's cell.
extern __shared__ __align__(16) unsigned char tsi_dyn_smem[];

// Programmatic dependent launch (PTX griddepcontrol, sm_90 and later): the
// wait returns once the grids this launch depends on have completed and
// their writes are visible (at once for a launch without that dependency);
// the trigger lets the stream's next launch begin once every block of this
// one has issued it.
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void grid_dependents_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// Backward liveness scan of one sibling group, run by the whole warp with the
// group leaders (lane 8g, `active`) doing the work: decided min/max become
// copies/constants, dead instructions vanish.  The kept instructions are
// written in reverse order to `tmp`; returns their count.  The tape and the
// branch ballots arrive 32 per coalesced load.
__device__ uint32_t prune_scan(const uint2 *__restrict__ code, uint32_t len, uint32_t n_minmax, uint32_t out_reg,
                               const uint2 *dg, uint32_t g, uint32_t E, uint2 *tmp, bool active, uint32_t lane,
                               uint32_t &mm_kept, uint32_t &fwd_cost, uint32_t &rev_cost) {
  unsigned long long live = 1ull << out_reg;
  uint32_t cnt = 0;
  mm_kept = 0;
  fwd_cost = 0;
  rev_cost = 0;
  const int nch = (int)((len + 31u) / 32u);
  uint2 cur = load_chunk(code, len, nch - 1, lane), nxt = load_chunk(code, len, nch - 2, lane);
  // ballots: chunk km holds min/max ordinals [32 km, 32 km + 32)
  int m = (int)n_minmax;
  int km = (m - 1) / 32;
  uint2 dcur = load_chunk(dg, n_minmax, m > 0 ? km : -1, lane);
  for (int k = nch - 1; k >= 0; --k) {
    const int c0 = 32 * k;
    for (int j = min(32, (int)len - c0) - 1; j >= 0; --j) {
      const uint2 w = chunk_word(cur, (uint32_t)j);
      const uint32_t h = TSI_W0_H(w.x);
      const uint32_t d = TSI_W0_DST(w.x), a = TSI_W0_A(w.x), b = w.y & 255u;
      const bool mmx = TSI_H_IS_MINMAX(h);
      uint2 dd = make_uint2(0u, 0u);
      if (mmx) {  // uniform across the warp
        --m;
        if (m < 32 * km) {
          km = m / 32;
          dcur = load_chunk(dg, n_minmax, km, lane);
        }
        dd = chunk_word(dcur, (uint32_t)(m - 32 * km));
      }
      if (!active || !((live >> d) & 1ull)) continue;
      live &= ~(1ull << d);
      uint2 out = w;
      uint32_t hk = h;
      if (mmx) {
        const uint32_t ga = (dd.x >> (g * 8u)) & 0xffu, gb = (dd.y >> (g * 8u)) & 0xffu;
        if ((ga & E) == E) {
          out = make_uint2(TSI_W0(H_COPY, TSI_W0_FA(w.x), 0u, d, a), 0u);
          hk = H_COPY;
          live |= 1ull << a;
        } else if ((gb & E) == E) {
          if (TSI_H_IS_II(h)) {
            out = make_uint2(TSI_W0(H_COPY, TSI_W0_FB(w.x), 0u, d, b), 0u);
            hk = H_COPY;
            live |= 1ull << b;
          } else {
            out = make_uint2(TSI_W0(H_CONST, 0u, 0u, d, 0u), w.y);
            hk = H_CONST;
          }
        } else {
          live |= 1ull << a;
          if (TSI_H_IS_II(h)) live |= 1ull << b;
          ++mm_kept;
        }
      } else {
        if (h != H_CONST) live |= 1ull << a;
        if (TSI_H_IS_II(h)) live |= 1ull << b;
      }
      fwd_cost += c_cost_fwd[hk] + TSI_FIX_COST;
      rev_cost += c_cost_rr[hk] + TSI_REV_OPERAND_COST * TSI_H_NREG(hk);
      tmp[cnt++] = out;
    }
    cur = nxt;
    nxt = load_chunk(code, len, k - 2, lane);
  }
  return cnt;
}

// mallocV (compute.wgsl:3437-3450) for a whole brick of 8 siblings.
__device__ uint32_t alloc_brick(const SceneLaunch &S, uint32_t *error) {
  SceneCounters *c = S.ctr;
  int32_t fc = atomicSub(&c->free_count, 1);
  uint32_t b;
  if (fc > 0) {
    b = S.pool.free_list[fc - 1];
  } else {
    b = atomicAdd(&c->bump, 1u);
    if (b >= S.pool.cap_bricks) {
      atomicOr(error, EB_OOM);
      return TSI_NONE;
    }
  }
  return b * 8u;
}

// The wide threshold for children at `level`: deep levels hold many cells,
// where the narrow path's throughput beats the wide path's latency.
__device__ __forceinline__ uint32_t wide_min_len(const WideDev &W, uint32_t level) {
  return level >= W.deep_level ? W.deep_min_len : W.min_len;
}

__device__ __forceinline__ StepIdx step_idx(uint32_t step) {
  StepIdx si;
  si.cur = step & TSI_STEP_MASK;
  si.next = (step + 1u) & TSI_STEP_MASK;
  si.buf = step & 1u;
  si.nbuf = (step + 1u) & 1u;
  return si;
}

// Reserves n words of the code arena (a ring of code_cap words, a power of
// two); returns the word offset, or ~0 when the ring has no room left above
// the low-water mark (the tape then stays unpruned).  A tape never wraps
// around the ring's end.
__device__ __forceinline__ unsigned long long code_alloc(const LaunchParams &P, uint32_t n) {
  const unsigned long long c = atomicAdd(P.code_count, (unsigned long long)n);
  if (c + n > *P.code_low + P.code_cap) return ~0ull;
  const unsigned long long off = c & (P.code_cap - 1ull);
  return off + n <= P.code_cap ? off : ~0ull;
}

// Takes a tape record from the ring [rec_base, rec_cap) (a power-of-two
// size); TSI_NONE when the ring has no room left above the low-water mark.
__device__ __forceinline__ uint32_t rec_alloc(const LaunchParams &P) {
  const unsigned long long r = atomicAdd(P.rec_count, 1ull);
  const uint32_t ring = P.rec_cap - P.rec_base;
  if (r >= *P.rec_low + ring) return TSI_NONE;
  return P.rec_base + ((uint32_t)r & (ring - 1u));
}

__device__ __forceinline__ void find_valid(const LaunchParams &P, uint32_t &rec, TapeRec &TR, float tl, float th) {
  TR = P.recs[rec];
  while (TR.parent != TSI_NONE && !(TR.t_lo <= tl && th <= TR.t_hi)) {
    rec = TR.parent;
    TR = P.recs[rec];
  }
}

// Next-level work for the enqueued children (mask E) of one parent, whose
// cells are cells[0..7]; one thread.  `wide`: one wide item per child, its
// own children's brick allocated here; children beyond the wide list's
// capacity, or all of them when not `wide`, go to the narrow list in items
// of up to four.  Every reserved list slot below the capacity is written
// (readers take min(count, capacity) entries); narrow-list overflow is
// dropped and reported.
__device__ void push_children(const LaunchParams &P, const SceneLaunch &S, uint32_t scene, uint32_t rec,
                              uint32_t step, uint32_t plevel, uint32_t E, const uint32_t *cells, bool wide,
                              unsigned long long *ws) {
  const StepIdx si = step_idx(step);
  // a scene's items end at its last level: the launch steps of its frame
  // stop there, and in the continuous form later steps belong to others
  if (plevel + 1u >= S.levels) return;
  uint32_t rest = E;
  uint32_t *err = P.error + scene;
  if (wide) {
    const uint32_t n = __popc(E);
    const uint32_t pos = atomicAdd(&P.witem_count[si.next], n);
    uint32_t j = 0;
    while (rest && pos + j < P.witem_cap) {
      const uint32_t bit = __ffs(rest) - 1u;
      rest &= rest - 1u;
      const uint32_t c = cells[bit];
      uint32_t b = S.pool.child[c], fresh = 0;
      if (b == TSI_NONE) {
        b = alloc_brick(S, err);
        if (b != TSI_NONE) {
          S.pool.child[c] = b;
          fresh = 1;
          atomicAdd(&ws[ST_BRICK_ALLOC], 1ull);
        }
      }
      WorkItem wi;
      wi.scene = scene;
      wi.rec = rec;
      wi.n = 1;
      wi.level = plevel + 1;
      wi.parent[0] = c;
      wi.parent[1] = b;
      wi.parent[2] = fresh;
      wi.parent[3] = 0;
      P.witems[si.nbuf][pos + j++] = wi;
    }
  }
  if (rest == 0) return;
  // a narrow item takes up to 4 parents (32 cells, one per lane) at the leaf
  // level, where many short evaluations make throughput count, and fewer
  // above it, where more items in flight hide the interpreter's latency
  const uint32_t per = (plevel + 2u >= S.levels) ? 4u : max(1u, min(4u, S.narrow_parents));
  const uint32_t nitems = (__popc(rest) + per - 1u) / per;
  const uint32_t pos = atomicAdd(&P.item_count[si.next], nitems);
  if (pos + nitems > P.item_cap) atomicOr(err, EB_QUEUE_FULL);
  WorkItem *dst = P.items[si.nbuf];
  for (uint32_t j = 0; j < nitems && pos + j < P.item_cap; ++j) {
    WorkItem wi;
    wi.scene = scene;
    wi.rec = rec;
    wi.level = plevel + 1;
    uint32_t c = 0;
    while (rest && c < per) {
      const uint32_t bit = __ffs(rest) - 1u;
      rest &= rest - 1u;
      wi.parent[c++] = cells[bit];
    }
    wi.n = c;
    for (uint32_t q = c; q < 4u; ++q) wi.parent[q] = wi.parent[0];
    dst[pos + j] = wi;
  }
}

// push_children for the eight children of one wide item (cells base..base+7),
// by one warp: lanes 0-7 take a child each, so the wide list's entries and
// the brick allocations proceed in parallel; the first wide-list slots go
// to the lowest enqueued octants, as in push_children.  `fresh`: the cells'
// brick is new this step (no cell has children yet), so their child fields
// are not read: they are known to be empty.
__device__ __forceinline__ void push_children_warp(const LaunchParams &P, const SceneLaunch &S, uint32_t scene,
                                                   uint32_t rec, uint32_t step, uint32_t plevel, uint32_t E,
                                                   uint32_t base, bool fresh, bool wide, unsigned long long *ws,
                                                   uint32_t lane) {
  const StepIdx si = step_idx(step);
  if (plevel + 1u >= S.levels) return;  // the scene's last level (push_children)
  uint32_t rest = E;
  if (wide && E) {
    // the enqueued children's bricks are read before the list reservation
    // (the two round trips overlap)
    const bool cand = lane < 8u && ((E >> lane) & 1u);
    const uint32_t b0 = (cand && !fresh) ? S.pool.child[base + lane] : TSI_NONE;
    uint32_t pos = 0;
    if (lane == 0) pos = atomicAdd(&P.witem_count[si.next], (uint32_t)__popc(E));
    pos = __shfl_sync(FULL_MASK, pos, 0);
    const uint32_t avail = pos < P.witem_cap ? P.witem_cap - pos : 0u;
    const uint32_t j = __popc(E & ((1u << lane) - 1u));
    const bool take = cand && j < avail;
    if (take) {
      const uint32_t c = base + lane;
      uint32_t b = b0, fresh = 0;
      if (b == TSI_NONE) {
        b = alloc_brick(S, P.error + scene);
        if (b != TSI_NONE) {
          S.pool.child[c] = b;
          fresh = 1;
          atomicAdd(&ws[ST_BRICK_ALLOC], 1ull);
        }
      }
      WorkItem wi;
      wi.scene = scene;
      wi.rec = rec;
      wi.n = 1;
      wi.level = plevel + 1;
      wi.parent[0] = c;
      wi.parent[1] = b;
      wi.parent[2] = fresh;
      wi.parent[3] = 0;
      P.witems[si.nbuf][pos + j] = wi;
    }
    rest = E & ~__ballot_sync(FULL_MASK, take);
  }
  if (lane == 0 && rest) {
    uint32_t cells[8];
    for (int q = 0; q < 8; ++q) cells[q] = base + q;
    push_children(P, S, scene, rec, step, plevel, rest, cells, false, ws);
  }
}

__device__ __forceinline__ float warp_min(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(FULL_MASK, v, o));
  return v;
}
__device__ __forceinline__ float warp_max(float v) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(FULL_MASK, v, o));
  return v;
}

// scratch for one item: operand log + decisions, in the warp's slice or the
// shared overflow arena (long tapes)
__device__ __forceinline__ bool item_scratch(const LaunchParams &P, uint32_t step, uint32_t scene, uint32_t len,
                                             uint32_t lane, float4 *slice_log, uint2 *slice_dec, float4 *&lg,
                                             uint2 *&dg) {
  const StepIdx si = step_idx(step);
  if (len <= P.slice_len) {
    lg = slice_log;
    dg = slice_dec;
    return true;
  }
  const unsigned long long need = (unsigned long long)len * 32ull + ((unsigned long long)len + 1ull) / 2ull;
  unsigned long long off = 0;
  if (lane == 0) off = atomicAdd(P.log_overflow_used + si.cur, need);
  off = __shfl_sync(FULL_MASK, off, 0);
  if (off + need > P.log_overflow_cap) {
    if (lane == 0) atomicOr(P.error + scene, EB_LOG_OOM);
    return false;
  }
  lg = P.log_overflow + off;
  dg = reinterpret_cast<uint2 *>(P.log_overflow + off + (unsigned long long)len * 32ull);
  return true;
}

template <bool D>
__device__ __noinline__ void process_item(const LaunchParams &P, const WorkItem &it, uint32_t step,
                                          uint32_t rf_off, float4 *slice_log, uint2 *slice_dec,
                                          unsigned long long *ws) {
  const StepIdx si = step_idx(step);
  float2 *rf = reinterpret_cast<float2 *>(tsi_dyn_smem) + rf_off;  // this warp's register file
  using A = IA<D>;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t g = lane >> 3, k = lane & 7u;
  const SceneLaunch &S = P.scenes[it.scene];
  const VoxelPoolDev &pool = S.pool;
  const uint32_t flags = S.flags;
  const bool swept = (flags & SF_SWEPT) != 0;

  bool active = g < it.n;
  const uint32_t Pv = it.parent[active ? g : 0];
  const float4 pxy = pool.box_xy[Pv];
  const float2 pz = pool.box_z[Pv];
  const uint32_t pchild = pool.child[Pv];
  const float pfast = pool.fast[Pv];
  const bool new_voxel = (pchild == TSI_NONE);

  // ---- allocate or reuse the 8 children (3564-3580)
  uint32_t base = pchild;
  if (active && new_voxel && k == 0) {
    base = alloc_brick(S, P.error + it.scene);
    if (base != TSI_NONE) atomicAdd(&ws[ST_BRICK_ALLOC], 1ull);
  }
  base = __shfl_sync(FULL_MASK, base, lane & ~7u);
  if (base == TSI_NONE) active = false;
  const uint32_t C = active ? base + k : 0u;
  float c_t = 0.0f, c_f = 1.0f, c_te = 0.0f, c_fast = 0.0f;
  uint32_t c_child = TSI_NONE;
  if (active) {
    if (new_voxel) {
      pool.child[C] = TSI_NONE;
      pool.normal[C] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
      if (k == 0) pool.child[Pv] = base;
    } else {
      c_t = pool.t[C];
      c_f = pool.f[C];
      c_te = pool.time_err[C];
      c_fast = pool.fast[C];
      c_child = pool.child[C];
    }
  }

  // ---- cell setup (3582-3626)
  const float dx = __fdiv_rn(__fsub_rn(pxy.y, pxy.x), 2.0f);
  const float dy = __fdiv_rn(__fsub_rn(pxy.w, pxy.z), 2.0f);
  const float dz = __fdiv_rn(__fsub_rn(pz.y, pz.x), 2.0f);
  float width = fm_max(dx, fm_max(dy, dz));
  const float kx = (float)(k & 1u), ky = (float)((k >> 1) & 1u), kz = (float)(k >> 2);
  Iv cx = Iv{__fadd_rn(pxy.x, __fmul_rn(dx, kx)), __fadd_rn(pxy.x, __fmul_rn(dx, 1.0f + kx))};
  Iv cy = Iv{__fadd_rn(pxy.z, __fmul_rn(dy, ky)), __fadd_rn(pxy.z, __fmul_rn(dy, 1.0f + ky))};
  Iv cz = Iv{__fadd_rn(pz.x, __fmul_rn(dz, kz)), __fadd_rn(pz.x, __fmul_rn(dz, 1.0f + kz))};
  // half extent of this cell's children, as they will compute it
  const float child_width =
      fm_max(__fdiv_rn(__fsub_rn(cx.hi, cx.lo), 2.0f),
             fm_max(__fdiv_rn(__fsub_rn(cy.hi, cy.lo), 2.0f), __fdiv_rn(__fsub_rn(cz.hi, cz.lo), 2.0f)));
  const bool point_branch = new_voxel || pfast == 1.0f || width <= S.eps;
  Iv cur_t;
  if (point_branch) {
    cur_t = swept ? Iv{S.t0, S.time} : iv(S.time);
    c_fast = 0.0f;
  } else {
    cur_t = Iv{c_t, S.time};
  }
  if (active) {
    pool.box_xy[C] = make_float4(cx.lo, cx.hi, cy.lo, cy.hi);
    pool.box_z[C] = make_float2(cz.lo, cz.hi);
    pool.t[C] = S.time;
  }
  if ((flags & SF_POINTSAMPLE) && width <= S.eps) {
    cx = iv(__fdiv_rn(__fadd_rn(cx.lo, cx.hi), 2.0f));
    cy = iv(__fdiv_rn(__fadd_rn(cy.lo, cy.hi), 2.0f));
    cz = iv(__fdiv_rn(__fadd_rn(cz.lo, cz.hi), 2.0f));
    width = 0.0f;
  }
  const Iv targ = Iv{fm_min(cur_t.lo, cur_t.hi), fm_max(cur_t.lo, cur_t.hi)};
  const bool evaluate = active && (new_voxel || c_f >= 0.0f || c_child == TSI_NONE);
  const bool take_deriv = evaluate && ((cur_t.lo != cur_t.hi) || (flags & SF_ALWAYS_DERIV));

  Iv field = iv(0.0f);
  Iv sens[4] = {iv(0.0f), iv(0.0f), iv(0.0f), iv(0.0f)};
  uint32_t rec = it.rec;
  TapeRec TR;
  const uint32_t b_eval = __ballot_sync(FULL_MASK, evaluate);
  const uint32_t b_rev = __ballot_sync(FULL_MASK, take_deriv);
  const bool any_deriv = b_rev != 0;
  bool want_prune = false;
  float4 *lg = nullptr;
  uint2 *dg = nullptr;

  if (b_eval) {
    // ---- the most pruned tape valid for every evaluated cell
    const float tl = warp_min(evaluate ? targ.lo : fm_inf());
    const float th = warp_max(evaluate ? targ.hi : -fm_inf());
    TR = P.recs[rec];
    if (!(TR.c_level == it.level && TR.c_lo <= tl && th <= TR.c_hi)) find_valid(P, rec, TR, tl, th);
    for (int attempt = 0; attempt < 2; ++attempt) {
      want_prune = (flags & SF_PRUNING) && TR.len >= TSI_PRUNE_MIN_LEN && TR.nregs <= TSI_PRUNE_MAX_REGS;
      if (lane == 0 && attempt == 0) {
        if (TR.len >= S.wide.min_len) ws[ST_NARROW_LONG] += 1;
        ws[ST_NARROW_LEN_MAX] = max(ws[ST_NARROW_LEN_MAX], (unsigned long long)TR.len);
      }
      lg = nullptr;
      dg = nullptr;
      if (any_deriv || want_prune) {
        float4 *lgs = nullptr;
        uint2 *dgs = nullptr;
        if (!item_scratch(P, step, it.scene, TR.len, lane, slice_log, slice_dec, lgs, dgs)) return;
        lg = lgs;
        dg = want_prune ? dgs : nullptr;
      }
      const long long q0 = clock64();
      field = forward_pass<D>(TR.code, TR.len, TR.out_reg, rf, lane, cx, cy, cz, targ, any_deriv ? lg : nullptr, dg);
      const long long q1 = clock64();
      bool bad = false;
      if (any_deriv) reverse_pass<D>(TR.code, TR.len, TR.nregs, TR.out_reg, rf, lane, lg, take_deriv, sens, bad);
      if (lane == 0 && attempt == 0) {
        ws[ST_CYC_N_FWD] += (unsigned long long)(q1 - q0);
        ws[ST_N_FWD_INSTR] += TR.len;
        ws[ST_CYC_N_REV] += (unsigned long long)(clock64() - q1);
      }
      // a pruned tape whose sensitivities overflowed: redo on the full tape
      const bool redo = __any_sync(FULL_MASK, bad) && TR.parent != TSI_NONE;
      if (!redo) break;
      rec = S.root_rec;
      TR = P.recs[rec];
      if (lane == 0) ws[ST_PRUNE_FALLBACK]++;
    }
    if (lane == 0) {
      const uint32_t ne = __popc(b_eval), nr = __popc(b_rev);
      ws[ST_INSTR_FWD] += (unsigned long long)TR.len * ne;
      ws[ST_INSTR_REV] += (unsigned long long)TR.len * nr;
      ws[ST_INSTR_FULL] += (unsigned long long)S.full_len * ne;
      ws[ST_FP32] += (unsigned long long)TR.fwd_cost * ne + (unsigned long long)TR.rev_cost * nr;
    }
  }

  // ---- temporal error bound (3966-3997)
  Iv df = iv(0.0f), df_dt = iv(0.0f);
  const float delta = S.delta;
  if (take_deriv) {
    const float nx = __fdiv_rn(__fadd_rn(sens[0].lo, sens[0].hi), 2.0f);
    const float ny = __fdiv_rn(__fadd_rn(sens[1].lo, sens[1].hi), 2.0f);
    const float nz = __fdiv_rn(__fadd_rn(sens[2].lo, sens[2].hi), 2.0f);
    pool.normal[C] = make_float4(nx, ny, nz, 0.0f);
    df_dt = sens[3];
    const float dt = __fsub_rn(targ.hi, targ.lo);
    df = A::mul_f(df_dt, dt);
    const Iv W = A::mul_f(Iv{-1.0f, 1.0f}, __fsub_rn(field.hi, field.lo));
    df = A::cap(df, W);
    if ((flags & SF_LIPSCHITZ) && A::abs_(df).hi != 0.0f) {
      const float lb =
          A::abs_(A::sqrt_(A::add(A::sqr(sens[0]), A::add(A::sqr(sens[1]), A::sqr(sens[2]))))).lo;
      if (!is_nan_f(lb)) df = A::div(df, iv(lb));
    }
    if (df.lo == -fm_inf() || df.hi == fm_inf() || is_nan_f(df.lo) || is_nan_f(df.hi)) df = iv(delta);
    c_te = __fadd_rn(c_te, fm_min(fm_max(A::abs_(df).hi, 0.0f), delta));
  }
  // ---- fast flag (4003-4009)
  if (evaluate && !swept && (flags & SF_FASTENABLED)) c_fast = (A::abs_(df).hi >= S.fast_thresh) ? 1.0f : 0.0f;

  // ---- classification (4011-4045)
  bool enq = false, dealloc = false, reused = false;
  int cls = 3;
  uint32_t dealloc_brick = 0;
  if (evaluate) {
    if (field.lo <= 0.0f && 0.0f <= field.hi) {
      c_f = 0.0f;
      cls = 0;
      if (width > S.eps) {
        if (new_voxel || is_nan_f(df_dt.lo) || is_nan_f(df_dt.hi) || fabsf(df_dt.lo) == fm_inf() ||
            fabsf(df_dt.hi) == fm_inf() || pfast == 1.0f || cur_t.lo == cur_t.hi || c_te >= delta ||
            c_child == TSI_NONE) {
          c_te = 0.0f;
          enq = true;
        } else {
          reused = true;
        }
      }
    } else {
      if (field.hi <= 0.0f) {
        c_f = -1.0f;
        cls = 2;
      } else {
        cls = 1;
        if (!swept) c_f = 1.0f;
      }
      if (!swept && c_child != TSI_NONE) {
        dealloc = true;
        dealloc_brick = c_child >> 3;
      }
    }
  }
  const uint32_t old_child = c_child;
  if (dealloc) c_child = TSI_NONE;
  if (active) {
    pool.f[C] = c_f;
    pool.time_err[C] = c_te;
    pool.fast[C] = c_fast;
    if (dealloc || new_voxel) pool.child[C] = c_child;
  }

  // ---- deallocation of dropped subtrees (4036-4044)
  {
    const uint32_t m = __ballot_sync(FULL_MASK, dealloc);
    if (m) {
      uint32_t basei = 0;
      if (lane == 0) basei = atomicAdd(&P.dealloc_count[si.next], (uint32_t)__popc(m));
      basei = __shfl_sync(FULL_MASK, basei, 0);
      if (dealloc) {
        const uint32_t pos = basei + __popc(m & ((1u << lane) - 1u));
        if (pos < P.dealloc_cap) P.dealloc[si.nbuf][pos] = make_uint2(it.scene, dealloc_brick);
        else atomicOr(P.error + it.scene, EB_QUEUE_FULL);
      }
    }
  }

  // ---- re-enqueue: one sibling group per parent, pruned tape per group
  const uint32_t em = __ballot_sync(FULL_MASK, enq);
  const uint32_t E = (em >> (g * 8u)) & 0xffu;
  uint32_t new_rec = rec;
  if (em) {
    // time range the children will be evaluated over: [child.t, time], or
    // the point branch's range for children at most eps wide or of a fast
    // cell
    const bool child_point = child_width <= S.eps || c_fast == 1.0f;
    float nl = targ.lo, nh = targ.hi;
    if (enq && old_child != TSI_NONE && !child_point) {
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const float ct = pool.t[old_child + q];
        nl = fm_min(nl, fm_min(ct, S.time));
        nh = fm_max(nh, fm_max(ct, S.time));
      }
    }
    if (enq && swept) {  // swept children start their point-branch interval at t0
      nl = fm_min(nl, fm_min(S.t0, S.time));
      nh = fm_max(nh, fm_max(S.t0, S.time));
    }
    if (!enq) {
      nl = fm_inf();
      nh = -fm_inf();
    }
    const bool widen = enq && (nl < targ.lo || nh > targ.hi);
    const uint32_t wb = __ballot_sync(FULL_MASK, widen);
    uint32_t prec = rec;  // record the group tapes are pruned from
    TapeRec PR = TR;
    bool handed = false;  // the group's children go to the wide path unpruned
    if (want_prune && wb) {
      // decisions over the widened interval, from a tape valid there
      const float wl = warp_min(nl), wh = warp_max(nh);
      uint32_t wrec = rec;
      TapeRec WR;
      find_valid(P, wrec, WR, wl, wh);
      if (WR.len >= wide_min_len(S.wide, it.level + 1u)) {
        // A long tape: no pass over it on one warp.  A group with a widened
        // child hands its children, with that tape's record, to the wide
        // path; the other groups prune from the first pass's decisions.
        if ((wb >> (g * 8u)) & 0xffu) {
          prec = wrec;
          PR = WR;
          handed = true;
        }
      } else {
        prec = wrec;
        PR = WR;
        want_prune = (flags & SF_PRUNING) && PR.len >= TSI_PRUNE_MIN_LEN && PR.nregs <= TSI_PRUNE_MAX_REGS;
      }
      if (want_prune && WR.len < wide_min_len(S.wide, it.level + 1u)) {
        float4 *lgs;
        uint2 *dgs;
        if (!item_scratch(P, step, it.scene, PR.len, lane, slice_log, slice_dec, lgs, dgs)) return;
        lg = lgs;
        dg = dgs;
        const Iv tw = enq ? Iv{nl, nh} : targ;
        (void)forward_pass<D>(PR.code, PR.len, PR.out_reg, rf, lane, cx, cy, cz, tw, nullptr, dg);
        if (lane == 0) ws[ST_FP32] += (unsigned long long)PR.fwd_cost * __popc(em);
      }
    }
    // validity of the group's pruned tape: intersection of the enqueued
    // siblings' decision intervals (any cell), and their hull (the group's
    // own children, each covered by its parent's decisions)
    float gl = enq ? nl : -fm_inf();
    float gh = enq ? nh : fm_inf();
    float hl = enq ? nl : fm_inf();
    float hh = enq ? nh : -fm_inf();
    for (int o = 1; o < 8; o <<= 1) {
      gl = fmaxf(gl, __shfl_xor_sync(FULL_MASK, gl, o));
      gh = fminf(gh, __shfl_xor_sync(FULL_MASK, gh, o));
      hl = fminf(hl, __shfl_xor_sync(FULL_MASK, hl, o));
      hh = fmaxf(hh, __shfl_xor_sync(FULL_MASK, hh, o));
    }
    uint32_t cnt = 0, mmk = 0, fcost = 0, rcost = 0;
    bool pruned = false;
    uint2 *tmp =
        (want_prune && !handed && lg != nullptr) ? reinterpret_cast<uint2 *>(lg) + (size_t)g * PR.len : nullptr;
    const uint32_t actm = __ballot_sync(FULL_MASK, k == 0 && E != 0 && tmp != nullptr);
    if (actm) {
      // every pruning group scans the same tape; lanes of other groups (a
      // group handed to the wide path holds another record) follow the
      // scan on that tape, so the warp's shuffles stay uniform
      const int src = __ffs(actm) - 1;
      const uint2 *pcode = reinterpret_cast<const uint2 *>(
          __shfl_sync(FULL_MASK, reinterpret_cast<unsigned long long>(PR.code), src));
      const uint32_t plen = __shfl_sync(FULL_MASK, PR.len, src);
      const uint32_t pmm = __shfl_sync(FULL_MASK, PR.n_minmax, src);
      const uint32_t pout = __shfl_sync(FULL_MASK, PR.out_reg, src);
      const bool act = (actm >> lane) & 1u;
      const long long q0 = clock64();
      cnt = prune_scan(pcode, plen, pmm, pout, dg, g, E, tmp, act, lane, mmk, fcost, rcost);
      if (lane == 0) ws[ST_CYC_N_PRUNE] += (unsigned long long)(clock64() - q0);
      pruned = act && cnt < PR.len;
      if (!act) cnt = 0;
    }
    // reserve arena space and a record (lane 8g), then copy with the group
    unsigned long long off = 0;
    uint32_t ri = TSI_NONE;
    if (k == 0 && pruned) {
      off = code_alloc(P, cnt);
      if (off != ~0ull) ri = rec_alloc(P);
    }
    const uint32_t gl0 = lane & ~7u;
    cnt = __shfl_sync(FULL_MASK, cnt, gl0);
    off = __shfl_sync(FULL_MASK, off, gl0);
    ri = __shfl_sync(FULL_MASK, ri, gl0);
    if (ri != TSI_NONE) {
      for (uint32_t j = k; j < cnt; j += 8u) P.code_arena[off + j] = tmp[cnt - 1u - j];
      if (k == 0) {
        TapeRec nr;
        nr.code = P.code_arena + off;
        nr.len = cnt;
        nr.nregs = PR.nregs;
        nr.out_reg = PR.out_reg;
        nr.n_minmax = mmk;
        nr.t_lo = gl;
        nr.t_hi = gh;
        nr.parent = prec;
        nr.fwd_cost = fcost;
        nr.rev_cost = rcost;
        nr.c_lo = hl;
        nr.c_hi = hh;
        nr.c_level = it.level + 1u;
        P.recs[ri] = nr;
        atomicAdd(&ws[ST_TAPE_WORDS], (unsigned long long)cnt);
      }
      new_rec = ri;
    } else if (E != 0 && want_prune) {
      new_rec = prec;  // not pruned (or no arena room): the widened-valid tape
    }
    // next-level work: wide items for a long tape, else narrow items
    uint32_t cb[8];
#pragma unroll
    for (int b2 = 0; b2 < 8; ++b2) cb[b2] = __shfl_sync(FULL_MASK, C, gl0 + b2);
    const uint32_t next_len = (new_rec == prec) ? PR.len : ((new_rec == rec) ? TR.len : cnt);
    if (k == 0 && E != 0)
      push_children(P, S, it.scene, new_rec, step, it.level, E, cb, next_len >= wide_min_len(S.wide, it.level + 1u),
                    ws);
  }

  // ---- counters
  const uint32_t b_skip = __ballot_sync(FULL_MASK, active && !evaluate);
  const uint32_t b_amb = __ballot_sync(FULL_MASK, cls == 0);
  const uint32_t b_emp = __ballot_sync(FULL_MASK, cls == 1);
  const uint32_t b_full = __ballot_sync(FULL_MASK, cls == 2);
  const uint32_t b_reu = __ballot_sync(FULL_MASK, reused);
  if (lane == 0) {
    ws[ST_PARENTS] += it.n;
    ws[ST_EVAL] += __popc(b_eval);
    ws[ST_REVERSE] += __popc(b_rev);
    ws[ST_SKIPPED] += __popc(b_skip);
    ws[ST_AMBIG] += __popc(b_amb);
    ws[ST_EMPTY] += __popc(b_emp);
    ws[ST_FULL] += __popc(b_full);
    ws[ST_ENQUEUED] += __popc(em);
    ws[ST_REUSED] += __popc(b_reu);
  }
}

// Recursive free of a dropped subtree (compute.wgsl:3533-3543, freeV
// 3452-3460): 8 lanes per brick; children bricks go to the next level's list.
__device__ void dealloc_brick(const LaunchParams &P, uint2 item, uint32_t step, bool valid) {
  const StepIdx si = step_idx(step);
  const uint32_t lane = threadIdx.x & 31u, k = lane & 7u;
  const SceneLaunch &S = P.scenes[valid ? item.x : 0];
  const VoxelPoolDev &pool = S.pool;
  const uint32_t v = item.y * 8u + k;
  uint32_t ch = TSI_NONE;
  if (valid) {
    ch = pool.child[v];
    pool.child[v] = TSI_NONE;
    pool.f[v] = 0.0f;
    pool.t[v] = 0.0f;
    pool.time_err[v] = 0.0f;
    pool.fast[v] = 0.0f;
  }
  const bool push = valid && ch != TSI_NONE;
  const uint32_t m = __ballot_sync(FULL_MASK, push);
  if (m) {
    uint32_t basei = 0;
    if (lane == 0) basei = atomicAdd(&P.dealloc_count[si.next], (uint32_t)__popc(m));
    basei = __shfl_sync(FULL_MASK, basei, 0);
    if (push) {
      const uint32_t pos = basei + __popc(m & ((1u << lane) - 1u));
      if (pos < P.dealloc_cap) P.dealloc[si.nbuf][pos] = make_uint2(item.x, ch >> 3);
      else atomicOr(P.error + item.x, EB_QUEUE_FULL);
    }
  }
  if (valid && k == 0) {
    const uint32_t pos = atomicAdd(&S.ctr->pending_count, 1u);
    if (pos < pool.cap_bricks) pool.pending[pos] = item.y;
    atomicAdd(&P.stats[(size_t)item.x * ST_COUNT + ST_BRICK_FREE], 1ull);  // the brick's own scene
    if (P.level_stats) atomicAdd(&P.level_stats[(size_t)si.cur * ST_COUNT + ST_BRICK_FREE], 1ull);
  }
}

// ======================================================================
// Wide path: one block per child cell of a wide item, one thread per
// instruction of a bundle (tape_compile.h WideTape).  Long tapes at the top
// of the octree leave the narrow path latency bound (few items, thousands of
// dependent instructions each); here a cell takes one block-wide step per
// bundle.  Every SSA value has its own slot in the cell's working set, so
// the reverse pass reads operands where the forward pass left them; values
// with several users sum per-use contribution records in the sequential
// order, so the results are those of the narrow path bit for bit.  The eight
// cells of an item run on eight blocks; the last to finish prunes the
// group's tape and enqueues its children.

// Byte offsets of a cell's working set (values, sensitivities, contribution
// records, decision bits, liveness flags); the host sizes it the same way.
struct CellLayout {
  uint32_t sens, rec, bits, flags;
};
__device__ __forceinline__ CellLayout cell_layout(const WideDev &W, uint32_t bm_words) {
  CellLayout L;
  L.sens = W.nvalues * 8u;
  L.rec = L.sens + W.nvalues * 8u;
  L.bits = L.rec + ((W.ncontrib * 8u + 15u) & ~15u);
  L.flags = L.bits + ((bm_words * 4u + 15u) & ~15u);
  return L;
}

constexpr uint32_t kSmemBundles = 512;  // bundle descriptors held in shared memory

// Base of the block's cell working set: dynamic shared memory, or for tapes
// too large for it the block's slice of the global scratch (each block of
// the persistent grid owns one slice; L2 keeps the active slices).
template <bool GM>
__device__ __forceinline__ unsigned char *cell_base(const LaunchParams &P) {
  if constexpr (GM) return P.wscratch + (size_t)blockIdx.x * P.wscratch_stride;
  else return tsi_dyn_smem;
}

struct WideShared {
  uint32_t last, E, cnt, mmk, fcost, rcost, ri;
  unsigned long long off;
  float gl, gh, hl, hh;
  uint32_t scan[kWarps];
  float2 sens[4];
  uint2 bt[kSmemBundles];  // the tape's bundle descriptors when they fit
};

// Bundle descriptors: the shared copy when the tape has few enough bundles.
__device__ __forceinline__ const uint2 *bundle_table(const WideDev &W, const WideShared &sh) {
  return W.nbundles <= kSmemBundles ? sh.bt : W.bundles;
}

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t *scratch, uint32_t &total) {
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(FULL_MASK, x, o);
    if (lane >= (uint32_t)o) x += y;
  }
  if (lane == 31) scratch[wib] = x;
  __syncthreads();
  uint32_t base = 0, tot = 0;
  for (uint32_t w = 0; w < (blockDim.x >> 5); ++w) {
    if (w < wib) base += scratch[w];
    tot += scratch[w];
  }
  __syncthreads();
  total = tot;
  return base + x - v;
}



// The last cell of a wide item to finish: prunes the full tape with the
// branch decisions shared by all enqueued siblings and enqueues them.
template <bool GM>
__device__ __forceinline__ void finish_group(const LaunchParams &P, const WorkItem &it, uint32_t step,
                                             uint32_t unit0, WideShared &sh, unsigned long long *ws) {
  const StepIdx si = step_idx(step);
  unsigned char *cell = cell_base<GM>(P);
  const uint32_t tid = threadIdx.x;
  const SceneLaunch &S = P.scenes[it.scene];
  const WideDev &W = S.wide;
  const TapeRec root = P.recs[S.root_rec];
  const uint32_t n_narrow = root.len;
  const CellInfo *info = P.cell_info[si.buf] + unit0;
  const long long f0 = clock64();
  // groups above the tape's prune level skip the liveness pass: their
  // children go to the wide path, which evaluates the full tape anyway
  const bool want_prune = (S.flags & SF_PRUNING) && root.nregs <= TSI_PRUNE_MAX_REGS && it.level >= W.prune_level;
  if (tid == 0) {
    ws[ST_PARENTS] += 1;
    ws[ST_WIDE_FIN] += 1;
    // sh.E: the enqueued siblings, from the count-in
    float gl = -fm_inf(), gh = fm_inf(), hl = fm_inf(), hh = -fm_inf();
    for (int q = 0; q < 8 && want_prune; ++q) {
      const CellInfo ci = info[q];
      gl = fmaxf(gl, ci.nl);
      gh = fminf(gh, ci.nh);
      if (ci.enq) {
        hl = fminf(hl, ci.nl);
        hh = fmaxf(hh, ci.nh);
      }
    }
    sh.gl = gl;
    sh.gh = gh;
    sh.hl = hl;
    sh.hh = hh;
  }
  __syncthreads();
  const uint32_t E = sh.E;
  if (E == 0) return;
  uint32_t new_rec = S.root_rec;
  if (want_prune) {
    const CellLayout L = cell_layout(W, P.bm_words);
    uint32_t *cb = reinterpret_cast<uint32_t *>(cell + L.bits);  // decisions shared by the enqueued cells
    uint8_t *flags = cell + L.flags;
    const uint32_t words = (root.n_minmax + 15u) >> 4;
    const uint32_t *gbits = P.cell_bits[si.buf] + (size_t)unit0 * P.bm_words;
    for (uint32_t w = tid; w < words; w += blockDim.x) {
      uint32_t acc = 0xffffffffu;
      for (int q = 0; q < 8; ++q)
        if ((E >> q) & 1u) acc &= gbits[(size_t)q * P.bm_words + w];
      cb[w] = acc;
    }
    for (uint32_t i = tid; i < W.nvalues; i += blockDim.x) flags[i] = 0;
    __syncthreads();
    // liveness from the field backwards, bundle by bundle
    {
      const uint2 *bt_tab = bundle_table(W, sh);
      const uint4 *__restrict__ slots = W.slots;
      const uint32_t ns = W.nslots;
      const uint4 zero4 = make_uint4(0u, 0u, 0u, 0u);
      auto fetch = [&](int kk) -> uint4 {
        if (kk < 0) return zero4;
        const uint2 b = bt_tab[kk];
        return tid < b.y ? slots[ns + b.x + tid] : zero4;
      };
      if (tid == 0) flags[W.nvalues - 1u] = 1;
      int kb = (int)W.nbundles - 1;
      uint4 q0 = fetch(kb), q1 = fetch(kb - 1);
      __syncthreads();
      for (; kb >= 0; --kb) {
        const uint2 bt = bt_tab[kb];
        const uint4 s1 = q0;
        q0 = q1;
        q1 = fetch(kb - 2);
        if (tid < bt.y && flags[s1.x]) {
          bool la = s1.z != TSI_NONE, lb = s1.w != TSI_NONE;
          if (s1.y != TSI_NONE) {  // a min/max: its ordinal
            const uint32_t d = (cb[s1.y >> 4] >> (2u * (s1.y & 15u))) & 3u;
            if (d & 1u) lb = false;
            else if (d & 2u) la = false;
          }
          if (la) flags[s1.z] = 1;
          if (lb) flags[s1.w] = 1;
        }
        __syncthreads();
      }
    }
    const long long f1 = clock64();
    if (tid == 0) ws[ST_CYC_FIN_LIVE] += (unsigned long long)(f1 - f0);
    // compaction of the narrow full tape in program order, one instruction
    // per thread a step: live instructions by ballot, output positions from
    // the warps' counts (coalesced reads of the tape)
    uint32_t mine = 0;
    for (uint32_t i = tid; i < n_narrow; i += blockDim.x) mine += flags[i + 4u];
    uint32_t total = 0;
    (void)block_exclusive_scan(mine, sh.scan, total);
    if (tid == 0) {
      sh.ri = TSI_NONE;
      sh.off = 0;
      sh.cnt = total;
      sh.mmk = 0;
      sh.fcost = 0;
      sh.rcost = 0;
      // a pruned record only for children that go to the narrow path (the
      // wide path evaluates the full tape), or may: children the full wide
      // list turns away run narrow on this record
      const bool wide_room = *(const volatile uint32_t *)&P.witem_count[si.next] + 8u <= P.witem_cap;
      if (total < n_narrow && (total < wide_min_len(W, it.level + 1u) || !wide_room)) {
        const unsigned long long off = code_alloc(P, total);
        if (off != ~0ull) {
          const uint32_t ri = rec_alloc(P);
          if (ri != TSI_NONE) {
            sh.ri = ri;
            sh.off = off;
          }
        }
      }
    }
    __syncthreads();
    if (sh.ri != TSI_NONE) {
      const uint32_t lane = tid & 31u, wib = tid >> 5, nw = blockDim.x >> 5;
      const unsigned long long off = sh.off;
      uint32_t base = 0, mmk = 0, fc = 0, rc = 0;
      // this thread's instruction of a step, read one step ahead
      auto fetch = [&](uint32_t i, uint2 &w, uint32_t &mm) {
        w = make_uint2(0u, 0u);
        mm = TSI_NONE;
        if (i < n_narrow) {
          w = root.code[i];
          mm = W.narrow_mm[i];
        }
      };
      uint2 wn;
      uint32_t mmn;
      fetch(tid, wn, mmn);
      for (uint32_t c0 = 0; c0 < n_narrow; c0 += blockDim.x) {
        const uint32_t i = c0 + tid;
        const uint2 w = wn;
        const uint32_t mm = mmn;
        fetch(i + blockDim.x, wn, mmn);
        const bool live = i < n_narrow && flags[i + 4u];
        const uint32_t bal = __ballot_sync(FULL_MASK, live);
        if (lane == 0) sh.scan[wib] = __popc(bal);
        __syncthreads();
        uint32_t woff = 0, ctot = 0;
        for (uint32_t q = 0; q < nw; ++q) {
          const uint32_t v = sh.scan[q];
          if (q < wib) woff += v;
          ctot += v;
        }
        __syncthreads();  // the counts are read before the next step writes them
        if (live) {
          const uint32_t p = base + woff + __popc(bal & ((1u << lane) - 1u));
          const uint32_t h = TSI_W0_H(w.x);
          uint2 out = w;
          uint32_t hk = h;
          if (TSI_H_IS_MINMAX(h)) {
            const uint32_t d = (cb[mm >> 4] >> (2u * (mm & 15u))) & 3u;
            const uint32_t dd = TSI_W0_DST(w.x);
            if (d & 1u) {
              out = make_uint2(TSI_W0(H_COPY, TSI_W0_FA(w.x), 0u, dd, TSI_W0_A(w.x)), 0u);
              hk = H_COPY;
            } else if (d & 2u) {
              if (TSI_H_IS_II(h)) {
                out = make_uint2(TSI_W0(H_COPY, TSI_W0_FB(w.x), 0u, dd, w.y & 255u), 0u);
                hk = H_COPY;
              } else {
                out = make_uint2(TSI_W0(H_CONST, 0u, 0u, dd, 0u), w.y);
                hk = H_CONST;
              }
            } else {
              ++mmk;
            }
          }
          fc += c_cost_fwd[hk] + TSI_FIX_COST;
          rc += c_cost_rr[hk] + TSI_REV_OPERAND_COST * TSI_H_NREG(hk);
          P.code_arena[off + p] = out;
        }
        base += ctot;
      }
      atomicAdd(&sh.mmk, mmk);
      atomicAdd(&sh.fcost, fc);
      atomicAdd(&sh.rcost, rc);
    }
    __syncthreads();
    if (sh.ri != TSI_NONE) {
      if (tid == 0) {
        TapeRec nr;
        nr.code = P.code_arena + sh.off;
        nr.len = sh.cnt;
        nr.nregs = root.nregs;
        nr.out_reg = root.out_reg;
        nr.n_minmax = sh.mmk;
        nr.t_lo = sh.gl;
        nr.t_hi = sh.gh;
        nr.parent = S.root_rec;
        nr.fwd_cost = sh.fcost;
        nr.rev_cost = sh.rcost;
        nr.c_lo = sh.hl;
        nr.c_hi = sh.hh;
        nr.c_level = it.level + 1u;
        P.recs[sh.ri] = nr;
        ws[ST_TAPE_WORDS] += sh.cnt;
      }
      new_rec = sh.ri;
    }
  }
  const long long f2 = clock64();
  if (tid < 32u) {
    const uint32_t len = (new_rec == S.root_rec) ? root.len : sh.cnt;
    push_children_warp(P, S, it.scene, new_rec, step, it.level, E, it.parent[1], it.parent[2] != 0u,
                       len >= wide_min_len(W, it.level + 1u), ws, tid);
  }
  if (tid == 0) {
    const long long f3 = clock64();
    ws[ST_CYC_FIN_COMPACT] += (unsigned long long)(f2 - f0);
    ws[ST_CYC_FIN_PUSH] += (unsigned long long)(f3 - f2);
  }
}

// One child cell (octant k) of a wide item.  unit = item * 8 + k.
template <bool D, bool GM>
__device__ __noinline__ void process_cell(const LaunchParams &P, WorkItem *itp, uint32_t k, uint32_t unit,
                                          uint32_t step, WideShared &sh, unsigned long long *ws) {
  const StepIdx si = step_idx(step);
  unsigned char *cell = cell_base<GM>(P);  // the cell's working set
  using A = IA<D>;
  const uint32_t tid = threadIdx.x;
  const WorkItem &it = *itp;
  const SceneLaunch &S = P.scenes[it.scene];
  const VoxelPoolDev &pool = S.pool;
  const WideDev &W = S.wide;
  const uint32_t flg = S.flags;
  const bool swept = (flg & SF_SWEPT) != 0;
  const uint32_t Pv = it.parent[0];
  const uint32_t base = it.parent[1];
  const bool new_voxel = it.parent[2] != 0;
  if (base == TSI_NONE) return;  // pool exhausted when the item was enqueued (error bit set)
  const TapeRec root = P.recs[S.root_rec];
  const uint32_t n_narrow = root.len;
  const uint32_t C = base + k;
  const CellLayout L = cell_layout(W, P.bm_words);
  if constexpr (!GM) {  // the host sized the launch for this cell; never write past it
    if (L.flags + ((W.nvalues + 15u) & ~15u) > P.dyn_smem) {
      if (tid == 0) atomicOr(P.error + it.scene, EB_SMEM);
      return;
    }
  }
  float2 *V = reinterpret_cast<float2 *>(cell);
  float2 *G = reinterpret_cast<float2 *>(cell + L.sens);
  float2 *R = reinterpret_cast<float2 *>(cell + L.rec);
  uint32_t *bits = reinterpret_cast<uint32_t *>(cell + L.bits);
  // the cell's and its parent's state, loaded before the bundle table's
  // copy and barrier so that the loads overlap
  const float4 pxy = pool.box_xy[Pv];
  const float2 pz = pool.box_z[Pv];
  const float pfast = pool.fast[Pv];
  float c_t = 0.0f, c_f = 1.0f, c_te = 0.0f, c_fast = 0.0f;
  uint32_t c_child = TSI_NONE;
  if (!new_voxel) {
    c_t = pool.t[C];
    c_f = pool.f[C];
    c_te = pool.time_err[C];
    c_fast = pool.fast[C];
    c_child = pool.child[C];
  }
  if (W.nbundles <= kSmemBundles)
    for (uint32_t i = tid; i < W.nbundles; i += blockDim.x) sh.bt[i] = W.bundles[i];
  const uint2 *bt_tab = bundle_table(W, sh);
  __syncthreads();

  // ---- cell setup (compute.wgsl:3582-3626), uniform across the block
  const float dx = __fdiv_rn(__fsub_rn(pxy.y, pxy.x), 2.0f);
  const float dy = __fdiv_rn(__fsub_rn(pxy.w, pxy.z), 2.0f);
  const float dz = __fdiv_rn(__fsub_rn(pz.y, pz.x), 2.0f);
  float width = fm_max(dx, fm_max(dy, dz));
  const float kx = (float)(k & 1u), ky = (float)((k >> 1) & 1u), kz = (float)(k >> 2);
  Iv cx = Iv{__fadd_rn(pxy.x, __fmul_rn(dx, kx)), __fadd_rn(pxy.x, __fmul_rn(dx, 1.0f + kx))};
  Iv cy = Iv{__fadd_rn(pxy.z, __fmul_rn(dy, ky)), __fadd_rn(pxy.z, __fmul_rn(dy, 1.0f + ky))};
  Iv cz = Iv{__fadd_rn(pz.x, __fmul_rn(dz, kz)), __fadd_rn(pz.x, __fmul_rn(dz, 1.0f + kz))};
  // half extent of this cell's children, as they will compute it
  const float child_width =
      fm_max(__fdiv_rn(__fsub_rn(cx.hi, cx.lo), 2.0f),
             fm_max(__fdiv_rn(__fsub_rn(cy.hi, cy.lo), 2.0f), __fdiv_rn(__fsub_rn(cz.hi, cz.lo), 2.0f)));
  const bool point_branch = new_voxel || pfast == 1.0f || width <= S.eps;
  Iv cur_t;
  if (point_branch) {
    cur_t = swept ? Iv{S.t0, S.time} : iv(S.time);
    c_fast = 0.0f;
  } else {
    cur_t = Iv{c_t, S.time};
  }
  if ((flg & SF_POINTSAMPLE) && width <= S.eps) {
    const Iv ox = cx, oy = cy, oz = cz;
    cx = iv(__fdiv_rn(__fadd_rn(ox.lo, ox.hi), 2.0f));
    cy = iv(__fdiv_rn(__fadd_rn(oy.lo, oy.hi), 2.0f));
    cz = iv(__fdiv_rn(__fadd_rn(oz.lo, oz.hi), 2.0f));
    width = 0.0f;
    if (tid == 0) {
      pool.box_xy[C] = make_float4(ox.lo, ox.hi, oy.lo, oy.hi);
      pool.box_z[C] = make_float2(oz.lo, oz.hi);
    }
  } else if (tid == 0) {
    pool.box_xy[C] = make_float4(cx.lo, cx.hi, cy.lo, cy.hi);
    pool.box_z[C] = make_float2(cz.lo, cz.hi);
  }
  if (tid == 0) {
    pool.t[C] = S.time;
    if (new_voxel) {
      pool.child[C] = TSI_NONE;
      pool.normal[C] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
  }
  const Iv targ = Iv{fm_min(cur_t.lo, cur_t.hi), fm_max(cur_t.lo, cur_t.hi)};
  const bool evaluate = new_voxel || c_f >= 0.0f || c_child == TSI_NONE;
  const bool take_deriv = evaluate && ((cur_t.lo != cur_t.hi) || (flg & SF_ALWAYS_DERIV));
  const bool want_prune = (flg & SF_PRUNING) && root.nregs <= TSI_PRUNE_MAX_REGS
                          && it.level >= W.prune_level;  // finish_group's rule
  const uint32_t words = (root.n_minmax + 15u) >> 4;

  // The time range this cell's children would be evaluated over if it is
  // re-enqueued and they do not take the point branch: when it is wider
  // than the cell's own, the decisions for pruning are taken over it in the
  // same forward pass (values over it in the sensitivity array, unused until
  // the reverse pass; decision bits in the liveness flags, unused until the
  // group finishes).  The range is the one computed after classification
  // below, step for step.
  float wl = targ.lo, wh = targ.hi;
  if (evaluate && want_prune) {
    if (c_child != TSI_NONE && !(child_width <= S.eps)) {
      for (int q = 0; q < 8; ++q) {
        const float ct = pool.t[c_child + q];
        wl = fm_min(wl, fm_min(ct, S.time));
        wh = fm_max(wh, fm_max(ct, S.time));
      }
    }
    if (swept) {
      wl = fm_min(wl, fm_min(S.t0, S.time));
      wh = fm_max(wh, fm_max(S.t0, S.time));
    }
  }
  const bool dual = evaluate && want_prune && (wl < targ.lo || wh > targ.hi);
  uint32_t *bits2 = reinterpret_cast<uint32_t *>(cell + L.flags);

  // ---- forward and reverse over the full tape, bundle by bundle
  Iv field = iv(0.0f);
  Iv sens[4] = {iv(0.0f), iv(0.0f), iv(0.0f), iv(0.0f)};
  if (evaluate) {
    if (want_prune)
      for (uint32_t w = tid; w < words; w += blockDim.x) {
        bits[w] = 0u;
        if (dual) bits2[w] = 0u;
      }
    const long long c0 = clock64();
    if (dual)
      field = cell_forward2<D>(W, bt_tab, V, G, bits, bits2, cx, cy, cz, targ, Iv{wl, wh});
    else
      field = cell_forward<D>(W, bt_tab, V, want_prune ? bits : nullptr, cx, cy, cz, targ);
    const long long c1 = clock64();
    if (take_deriv) {
      cell_reverse<D>(W, bt_tab, V, G, R, sh.sens);
      for (int q = 0; q < 4; ++q) sens[q] = ldv(sh.sens, q);
    }
    if (tid == 0) {
      ws[ST_CYC_WIDE_FWD] += (unsigned long long)(c1 - c0);
      ws[ST_CYC_WIDE_REV] += (unsigned long long)(clock64() - c1);
    }
  }

  // ---- temporal error bound, fast flag, classification (3966-4045)
  Iv df = iv(0.0f), df_dt = iv(0.0f);
  const float delta = S.delta;
  if (take_deriv) {
    const float nx = __fdiv_rn(__fadd_rn(sens[0].lo, sens[0].hi), 2.0f);
    const float ny = __fdiv_rn(__fadd_rn(sens[1].lo, sens[1].hi), 2.0f);
    const float nz = __fdiv_rn(__fadd_rn(sens[2].lo, sens[2].hi), 2.0f);
    if (tid == 0) pool.normal[C] = make_float4(nx, ny, nz, 0.0f);
    df_dt = sens[3];
    const float dt = __fsub_rn(targ.hi, targ.lo);
    df = A::mul_f(df_dt, dt);
    const Iv Wd = A::mul_f(Iv{-1.0f, 1.0f}, __fsub_rn(field.hi, field.lo));
    df = A::cap(df, Wd);
    if ((flg & SF_LIPSCHITZ) && A::abs_(df).hi != 0.0f) {
      const float lb =
          A::abs_(A::sqrt_(A::add(A::sqr(sens[0]), A::add(A::sqr(sens[1]), A::sqr(sens[2]))))).lo;
      if (!is_nan_f(lb)) df = A::div(df, iv(lb));
    }
    if (df.lo == -fm_inf() || df.hi == fm_inf() || is_nan_f(df.lo) || is_nan_f(df.hi)) df = iv(delta);
    c_te = __fadd_rn(c_te, fm_min(fm_max(A::abs_(df).hi, 0.0f), delta));
  }
  if (evaluate && !swept && (flg & SF_FASTENABLED)) c_fast = (A::abs_(df).hi >= S.fast_thresh) ? 1.0f : 0.0f;
  bool enq = false, dealloc = false, reused = false;
  int cls = 3;
  if (evaluate) {
    if (field.lo <= 0.0f && 0.0f <= field.hi) {
      c_f = 0.0f;
      cls = 0;
      if (width > S.eps) {
        if (new_voxel || is_nan_f(df_dt.lo) || is_nan_f(df_dt.hi) || fabsf(df_dt.lo) == fm_inf() ||
            fabsf(df_dt.hi) == fm_inf() || pfast == 1.0f || cur_t.lo == cur_t.hi || c_te >= delta ||
            c_child == TSI_NONE) {
          c_te = 0.0f;
          enq = true;
        } else {
          reused = true;
        }
      }
    } else {
      if (field.hi <= 0.0f) {
        c_f = -1.0f;
        cls = 2;
      } else {
        cls = 1;
        if (!swept) c_f = 1.0f;
      }
      if (!swept && c_child != TSI_NONE) dealloc = true;
    }
  }
  const uint32_t old_child = c_child;
  if (dealloc) c_child = TSI_NONE;
  if (tid == 0) {
    pool.f[C] = c_f;
    pool.time_err[C] = c_te;
    pool.fast[C] = c_fast;
    if (dealloc || new_voxel) pool.child[C] = c_child;
    if (dealloc) {
      const uint32_t pos = atomicAdd(&P.dealloc_count[si.next], 1u);
      if (pos < P.dealloc_cap) P.dealloc[si.nbuf][pos] = make_uint2(it.scene, old_child >> 3);
      else atomicOr(P.error + it.scene, EB_QUEUE_FULL);
    }
    ws[ST_EVAL] += evaluate ? 1ull : 0ull;
    ws[ST_REVERSE] += take_deriv ? 1ull : 0ull;
    ws[ST_SKIPPED] += evaluate ? 0ull : 1ull;
    if (cls == 0) ws[ST_AMBIG] += 1ull;
    if (cls == 1) ws[ST_EMPTY] += 1ull;
    if (cls == 2) ws[ST_FULL] += 1ull;
    if (enq) ws[ST_ENQUEUED] += 1ull;
    if (reused) ws[ST_REUSED] += 1ull;
    if (evaluate) {
      ws[ST_INSTR_FWD] += (unsigned long long)n_narrow;
      ws[ST_INSTR_FULL] += (unsigned long long)S.full_len;
      ws[ST_FP32] += (unsigned long long)root.fwd_cost + (take_deriv ? root.rev_cost : 0u);
    }
    if (take_deriv) ws[ST_INSTR_REV] += (unsigned long long)n_narrow;
  }
  // time range the children will be evaluated over: [child.t, time], or
  // the point branch's range for children at most eps wide or of a fast cell
  const bool child_point = child_width <= S.eps || c_fast == 1.0f;
  float nl = targ.lo, nh = targ.hi;
  if (want_prune && enq && old_child != TSI_NONE && !child_point) {
    for (int q = 0; q < 8; ++q) {
      const float ct = pool.t[old_child + q];
      nl = fm_min(nl, fm_min(ct, S.time));
      nh = fm_max(nh, fm_max(ct, S.time));
    }
  }
  if (want_prune && enq && swept) {
    nl = fm_min(nl, fm_min(S.t0, S.time));
    nh = fm_max(nh, fm_max(S.t0, S.time));
  }
  if (want_prune && enq && (nl < targ.lo || nh > targ.hi)) {
    // decisions over the children's (wider) time range
    __syncthreads();
    if (tid == 0) ws[ST_FP32] += (unsigned long long)root.fwd_cost;
    if (dual && nl == wl && nh == wh) {  // taken in the forward pass
      for (uint32_t w = tid; w < words; w += blockDim.x) bits[w] = bits2[w];
    } else {
      const long long r0 = clock64();
      for (uint32_t w = tid; w < words; w += blockDim.x) bits[w] = 0u;
      (void)cell_forward<D>(W, bt_tab, V, bits, cx, cy, cz, Iv{nl, nh});
      if (tid == 0) {
        ws[ST_WIDE_REFWD] += 1ull;
        ws[ST_CYC_WIDE_REFWD] += (unsigned long long)(clock64() - r0);
      }
    }
  }
  // ---- hand over to the group: decision bits and time range, then count in
  __syncthreads();
  if (want_prune && enq) {
    uint32_t *dst = P.cell_bits[si.buf] + (size_t)unit * P.bm_words;
    for (uint32_t w = tid; w < words; w += blockDim.x) dst[w] = bits[w];
  }
  if (tid == 0 && want_prune) {  // the time ranges matter only to a pruning finish
    CellInfo ci;
    ci.nl = enq ? nl : -fm_inf();
    ci.nh = enq ? nh : fm_inf();
    ci.enq = enq ? 1u : 0u;
    ci.pad = 0;
    P.cell_info[si.buf][unit] = ci;
  }
  // A pruning finish reads the decision bits and time ranges written above.
  // In a fresh brick this block wrote its cell's child field (empty), which
  // the finish overwrites with a brick for an enqueued cell: that write must
  // be ordered before the finish's.  Otherwise the finish reads nothing this
  // step's blocks wrote (the enqueued siblings come with the count; an
  // enqueued cell of an older brick keeps its child field) and writes
  // nothing they wrote, so no fence is needed.
  const bool fence = want_prune || new_voxel;  // new_voxel: the item's brick is fresh (all 8 cells)
  if (fence) __threadfence();
  __syncthreads();
  // the count (low byte) and the enqueued siblings (bits 8-15) in one atomic
  if (tid == 0) {
    const uint32_t mine = enq ? (1u << k) : 0u;
    const uint32_t old = atomicAdd(&itp->parent[3], 1u + (mine << 8));
    sh.last = (old & 255u) == 7u ? 1u : 0u;
    sh.E = ((old >> 8) | mine) & 255u;
  }
  __syncthreads();
  if (!sh.last) return;
  if (fence) __threadfence();
  finish_group<GM>(P, it, step, unit & ~7u, sh, ws);
}

// Clears the lists and counters of ring entry c.
__device__ __forceinline__ void clear_step(const LaunchParams &P, uint32_t c) {
  P.item_count[c] = 0;
  P.item_cursor[c] = 0;
  P.witem_count[c] = 0;
  P.witem_cursor[c] = 0;
  P.dealloc_count[c] = 0;
  P.dealloc_cursor[c] = 0;
  P.log_overflow_used[c] = 0;
}

// A warp's counters belong to the scene whose items it counted: they are
// added to that scene's stats row (and the launch's level row) when the warp
// moves on to another scene's item and at the end of the launch.
__device__ __forceinline__ void flush_stats(const LaunchParams &P, unsigned long long *ws, uint32_t scene,
                                            uint32_t cur, uint32_t lane) {
  __syncwarp();
  unsigned long long *row = P.stats + (size_t)scene * ST_COUNT;
  unsigned long long *lv = P.level_stats ? P.level_stats + (size_t)cur * ST_COUNT : nullptr;
  for (uint32_t i = lane; i < ST_COUNT; i += 32u) {
    const unsigned long long v = ws[i];
    if (!v) continue;
    ws[i] = 0;
    if (i == ST_CYC_WIDE_MAX || i == ST_CYC_NARROW_MAX || i == ST_NARROW_LEN_MAX) {
      atomicMax(row + i, v);
      if (lv) atomicMax(lv + i, v);
    } else {
      atomicAdd(row + i, v);
      if (lv) atomicAdd(lv + i, v);
    }
  }
  __syncwarp();
}

// One launch step over every scene of the launch: the wide items, the narrow
// items and the deallocation items of the step's lists.
__global__ void __launch_bounds__(256) refine_kernel(const __grid_constant__ LaunchParams P, uint32_t step,
                                                     uint32_t rcap) {
  StepIdx si;
  si.cur = step & TSI_STEP_MASK;
  si.next = (step + 1u) & TSI_STEP_MASK;
  si.buf = step & 1u;
  si.nbuf = (step + 1u) & 1u;
  __shared__ unsigned long long s_stats[kWarps][ST_COUNT];
  const uint32_t lane = threadIdx.x & 31u, wib = threadIdx.x >> 5;
  // Launched as a programmatic dependent of the previous step, the blocks
  // may be resident before that step has ended: nothing of it is read
  // before it has completed.  Then the next step's launch may begin (its
  // blocks take the SMs this launch's blocks leave).
  grid_dependency_wait();
  grid_dependents_launch();
  // the lists of the step after next start empty (no launch of this step
  // touches them; the next step fills them)
  if (blockIdx.x == 0 && threadIdx.x == 0) clear_step(P, (step + 2u) & TSI_STEP_MASK);
  const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + wib;
  const uint32_t rf_off = wib * rcap * 32u;  // this warp's register file in tsi_dyn_smem (float2 units)
  float4 *slice_log = P.log_slices + (size_t)gw * P.slice_len * 32u;
  uint2 *slice_dec = P.dec_slices + (size_t)gw * P.slice_len;
  unsigned long long *ws = s_stats[wib];
  for (uint32_t i = lane; i < ST_COUNT; i += 32u) ws[i] = 0;
  __syncwarp();
  uint32_t wscene = TSI_NONE;  // the scene whose counters ws holds (warp uniform)
  auto take = [&](uint32_t sc) {
    if (sc != wscene) {
      if (wscene != TSI_NONE) flush_stats(P, ws, wscene, si.cur, lane);
      wscene = sc;
    }
  };

  __shared__ WideShared sh;
  __shared__ uint32_t s_idx;
  // wide items: one block per child cell (thread 0 and warp 0 count into
  // s_stats[0], warp 0's counters)
  auto wide_phase = [&]() {
    const uint32_t n_units = min(P.witem_count[si.cur], P.witem_cap) * 8u;
    while (true) {
      if (threadIdx.x == 0) s_idx = atomicAdd(&P.witem_cursor[si.cur], 1u);
      __syncthreads();
      const uint32_t u = s_idx;
      __syncthreads();
      if (u >= n_units) break;
      WorkItem *itp = P.witems[si.buf] + (u >> 3);
      const uint32_t sc = itp->scene;
      if (wib == 0) take(sc);
      const long long c0 = clock64();
      const SceneLaunch &S = P.scenes[sc];
      const bool directed = (S.flags & SF_DIRECTED) != 0;
      if (S.wide.global) {
        if (directed) process_cell<true, true>(P, itp, u & 7u, u, step, sh, s_stats[0]);
        else process_cell<false, true>(P, itp, u & 7u, u, step, sh, s_stats[0]);
      } else {
        if (directed) process_cell<true, false>(P, itp, u & 7u, u, step, sh, s_stats[0]);
        else process_cell<false, false>(P, itp, u & 7u, u, step, sh, s_stats[0]);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        const unsigned long long c = (unsigned long long)(clock64() - c0);
        s_stats[0][ST_WIDE_ITEMS] += 1;
        s_stats[0][ST_CYC_WIDE] += c;
        s_stats[0][ST_CYC_WIDE_MAX] = max(s_stats[0][ST_CYC_WIDE_MAX], c);
      }
    }
  };
  // narrow items: one warp per item
  auto narrow_phase = [&]() {
    const uint32_t n_items = min(P.item_count[si.cur], P.item_cap);
    const WorkItem *items = P.items[si.buf];
    while (true) {
      uint32_t idx = 0;
      if (lane == 0) idx = atomicAdd(&P.item_cursor[si.cur], 1u);
      idx = __shfl_sync(FULL_MASK, idx, 0);
      if (idx >= n_items) break;
      const WorkItem &it = items[idx];
      take(it.scene);
      const long long c0 = clock64();
      if (P.scenes[it.scene].flags & SF_DIRECTED) process_item<true>(P, it, step, rf_off, slice_log, slice_dec, ws);
      else process_item<false>(P, it, step, rf_off, slice_log, slice_dec, ws);
      __syncwarp();
      if (lane == 0) {
        const unsigned long long c = (unsigned long long)(clock64() - c0);
        ws[ST_CYC_NARROW] += c;
        ws[ST_CYC_NARROW_MAX] = max(ws[ST_CYC_NARROW_MAX], c);
      }
    }
  };
  // three blocks in four drain the narrow list first, so both lists start
  // draining at once (half of them measured 0.8% slower, all wide first 6%)
  if ((blockIdx.x & 3u) != 0u) {
    narrow_phase();
    wide_phase();
  } else {
    wide_phase();
    narrow_phase();
  }
  // deallocation items: 4 bricks per warp
  const uint32_t n_dealloc = min(P.dealloc_count[si.cur], P.dealloc_cap);
  const uint2 *dl = P.dealloc[si.buf];
  while (true) {
    uint32_t idx = 0;
    if (lane == 0) idx = atomicAdd(&P.dealloc_cursor[si.cur], 4u);
    idx = __shfl_sync(FULL_MASK, idx, 0);
    if (idx >= n_dealloc) break;
    const uint32_t j = idx + (lane >> 3);
    const bool valid = j < n_dealloc;
    const uint2 item = valid ? dl[j] : make_uint2(0u, 0u);
    dealloc_brick(P, item, step, valid);
  }
  if (wscene != TSI_NONE) flush_stats(P, ws, wscene, si.cur, lane);
}

// buf_main's enqueue(0) (compute.wgsl:4706) for scene s: its root as a work
// item of the step (a wide item, with the root's children brick, when the
// root tape is long enough).
__device__ void seed_root(const LaunchParams &P, uint32_t s, uint32_t step) {
  const StepIdx si = step_idx(step);
  WorkItem w;
  w.scene = s;
  w.rec = P.scenes[s].root_rec;
  w.n = 1;
  w.level = 0;
  w.parent[0] = w.parent[1] = w.parent[2] = w.parent[3] = 0u;
  const SceneLaunch &S = P.scenes[s];
  const uint32_t len = P.recs[S.root_rec].len;
  if (len >= S.wide.min_len) {
    const uint32_t pos = atomicAdd(&P.witem_count[si.cur], 1u);
    if (pos < P.witem_cap) {
      uint32_t b = S.pool.child[0], fresh = 0;
      if (b == TSI_NONE) {
        b = alloc_brick(S, P.error + s);
        if (b != TSI_NONE) {
          S.pool.child[0] = b;
          fresh = 1;
          atomicAdd(&P.stats[(size_t)s * ST_COUNT + ST_BRICK_ALLOC], 1ull);
          if (P.level_stats) atomicAdd(&P.level_stats[(size_t)si.cur * ST_COUNT + ST_BRICK_ALLOC], 1ull);
        }
      }
      w.parent[1] = b;
      w.parent[2] = fresh;
      w.parent[3] = 0;
      P.witems[si.buf][pos] = w;
      return;
    }
  }
  const uint32_t pos = atomicAdd(&P.item_count[si.cur], 1u);
  if (pos < P.item_cap) P.items[si.buf][pos] = w;
  else atomicOr(P.error + s, EB_QUEUE_FULL);
}


// Per frame of the plain and batched forms (steps 0, 1, ... are the levels):
// clear every step's lists and the tape arenas, seed the root of every scene
// at step 0.  With n_scenes = 0 it only clears (the continuous form's start).
__global__ void frame_begin_kernel(const __grid_constant__ LaunchParams P) {
  const uint32_t t = threadIdx.x;
  grid_dependents_launch();  // the first level's launch may begin
  for (uint32_t l = t; l < TSI_STEP_RING; l += blockDim.x) clear_step(P, l);
  if (t == 0) {
    *P.rec_count = 0;
    *P.code_count = 0;
    *P.rec_low = 0;
    *P.code_low = 0;
  }
  __syncthreads();
  for (uint32_t s = t; s < P.n_scenes; s += blockDim.x) seed_root(P, s, 0u);
}

// Start of a step of the continuous form at which slots join: record the
// arena counters at the step's start, move the low-water marks to the oldest
// running slot's first step (always a step at which slots joined), clear
// the stats rows and error words of the joining slots and seed their roots.
// (Each refinement launch clears the lists of the step after its next.)
__global__ void step_begin_kernel(const __grid_constant__ LaunchParams P, uint32_t step,
                                  const __grid_constant__ StepSeeds sd) {
  StepIdx si;
  si.cur = step & TSI_STEP_MASK;
  si.next = (step + 1u) & TSI_STEP_MASK;
  si.buf = step & 1u;
  si.nbuf = (step + 1u) & 1u;
  const uint32_t t = threadIdx.x;
  if (t == 0) {
    P.step_code_start[si.cur] = *P.code_count;
    P.step_rec_start[si.cur] = *P.rec_count;
    *P.code_low = P.step_code_start[sd.oldest & TSI_STEP_MASK];
    *P.rec_low = P.step_rec_start[sd.oldest & TSI_STEP_MASK];
    clear_step(P, si.next);
  }
  const uint32_t n = min(sd.n, (uint32_t)TSI_SEEDS_MAX);
  for (uint32_t i = t; i < n * ST_COUNT; i += blockDim.x) P.stats[(size_t)sd.slot[i / ST_COUNT] * ST_COUNT + i % ST_COUNT] = 0;
  for (uint32_t i = t; i < n; i += blockDim.x) P.error[sd.slot[i]] = 0;
  __syncthreads();
  for (uint32_t i = t; i < n; i += blockDim.x) seed_root(P, sd.slot[i], step);
}

// Per frame end of scenes first .. first + gridDim.x - 1: bricks freed during
// the frame become allocatable; the scene's error word is or-ed into the
// sticky word (asynchronous inversions).
__global__ void frame_end_kernel(const __grid_constant__ LaunchParams P, uint32_t first) {
  grid_dependency_wait();  // the last level has completed
  const uint32_t s = first + blockIdx.x;
  if (s >= P.n_scenes) return;
  const SceneLaunch &S = P.scenes[s];
  SceneCounters *c = S.ctr;
  __shared__ int32_t fc0;
  __shared__ uint32_t np;
  if (threadIdx.x == 0 && P.error_sticky) atomicOr(P.error_sticky, P.error[s]);
  if (threadIdx.x == 0) {
    fc0 = max(c->free_count, 0);
    np = min(c->pending_count, S.pool.cap_bricks);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < np; i += blockDim.x) S.pool.free_list[fc0 + i] = S.pool.pending[i];
  __syncthreads();
  if (threadIdx.x == 0) {
    c->free_count = fc0 + (int32_t)np;
    c->pending_count = 0;
    uint32_t used = min(c->bump, S.pool.cap_bricks);
    c->live_bricks = used - (uint32_t)(fc0 + (int32_t)np);
  }
}

// host-side launch helpers
namespace {
// Launch configuration; `overlap`: a programmatic dependent of the stream's
// previous kernel (its launch overlaps that kernel's last blocks; the
// kernel waits for it to complete before reading what it wrote).
struct LaunchCfg {
  cudaLaunchConfig_t cfg{};
  cudaLaunchAttribute attr[1];
  LaunchCfg(int grid, int block, size_t smem, cudaStream_t st, bool overlap) {
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = overlap ? attr : nullptr;
    cfg.numAttrs = overlap ? 1u : 0u;
  }
};
}  // namespace

cudaError_t launch_refine(const LaunchParams &P, uint32_t step, uint32_t rcap, int grid, int block, size_t smem,
                          cudaStream_t st, bool overlap) {
  LaunchCfg lc(grid, block, smem, st, overlap);
  return cudaLaunchKernelEx(&lc.cfg, refine_kernel, P, step, rcap);
}
cudaError_t launch_frame_begin(const LaunchParams &P, cudaStream_t st) {
  frame_begin_kernel<<<1, 64, 0, st>>>(P);
  return cudaGetLastError();
}
cudaError_t launch_step_begin(const LaunchParams &P, uint32_t step, const StepSeeds &sd, cudaStream_t st) {
  step_begin_kernel<<<1, 256, 0, st>>>(P, step, sd);
  return cudaGetLastError();
}
cudaError_t launch_frame_end(const LaunchParams &P, uint32_t first, uint32_t count, cudaStream_t st, bool overlap) {
  if (count == 0) return cudaSuccess;
  LaunchCfg lc((int)count, 256, 0, st, overlap);
  return cudaLaunchKernelEx(&lc.cfg, frame_end_kernel, P, first);
}
// The attribute belongs to the kernel on the current device, shared by every
// context of the process: only ever raise it.
cudaError_t refine_set_smem(size_t bytes) {
  static std::mutex mu;
  static size_t set_bytes[64] = {0};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && bytes <= set_bytes[dev]) return cudaSuccess;
  e = cudaFuncSetAttribute(refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess && dev >= 0 && dev < 64) set_bytes[dev] = bytes;
  return e;
}
cudaError_t refine_occupancy(int block, size_t smem, int *blocks_per_sm) {
  return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, refine_kernel, block, smem);
}
cudaError_t refine_static_smem(size_t *bytes) {
  cudaFuncAttributes fa;
  const cudaError_t e = cudaFuncGetAttributes(&fa, refine_kernel);
  *bytes = e == cudaSuccess ? fa.sharedSizeBytes : 0;
  return e;
}

}  // namespace tsi
