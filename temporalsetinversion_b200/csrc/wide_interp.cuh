// wide_interp.cuh — the block-wide interpreter of the bundled tape
// (tape_compile.h WideTape): one cell per block, one thread per slot of a
// bundle, every SSA value in its own shared-memory slot.
//
// cell_forward follows compute.wgsl:3633-3772, cell_reverse
// compute.wgsl:3786-3900 with per-use contribution records for values with
// several users (their sensitivities are summed in the sequential order).
//
// A bundle step is a block barrier apart from the next, and its cost is
// mostly fixed (the barrier, the dependent shared-memory loads, the
// handler dispatch), so the schedule packs groups of different handlers
// into one step, one handler per warp.  Each thread reads its handler from
// its slot; min/max slots (which also record their decisions) have bodies
// of their own, every other handler shares one generic body, which keeps
// the loops small enough for the instruction cache (bodies specialised per
// handler measured no faster, and slower in the reverse pass).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "device_types.h"
#include "interp.cuh"

namespace tsi {

__device__ __forceinline__ Iv ldv(const float2 *a, uint32_t i) {
  const float2 v = a[i];
  return Iv{v.x, v.y};
}
__device__ __forceinline__ void stv(float2 *a, uint32_t i, Iv v) { a[i] = make_float2(v.lo, v.hi); }

// A thread's slot of bundle kk and the bundle's slot count, or a padding
// slot past the bundle (or past the tape).
struct WideFetch {
  const uint2 *bt;
  const uint4 *__restrict__ slots;
  uint32_t nb, tid;
  __device__ __forceinline__ uint4 operator()(int kk, uint32_t word_group, uint32_t ns) const {
    if (kk < 0 || (uint32_t)kk >= nb) return make_uint4(TSI_H_PAD, 0u, TSI_NONE, TSI_NONE);
    const uint2 b = bt[kk];
    return tid < b.y ? slots[word_group * ns + b.x + tid] : make_uint4(TSI_H_PAD, 0u, TSI_NONE, TSI_NONE);
  }
};

// 2-bit decision of a min/max over A and B (compute.wgsl:3660-3700): bit 0
// the A operand is always chosen, bit 1 the B operand is.
__device__ __forceinline__ uint32_t minmax_decision(bool amax, Iv A, Iv B) {
  const bool a_below = A.hi < B.lo, b_below = B.hi < A.lo;
  return ((amax ? b_below : a_below) ? 1u : 0u) | ((amax ? a_below : b_below) ? 2u : 0u);
}

// ---------------------------------------------------------------- forward
template <bool D, uint32_t H>
__device__ __forceinline__ void fwd_slot(float2 *V, uint32_t *bits, const uint4 &sl) {
  const float lit = __uint_as_float(sl.w);
  const Iv A = ldv(V, sl.y);
  const Iv B = TSI_H_IS_II(H) ? ldv(V, sl.z) : iv(lit);
  stv(V, sl.x >> 8, op_forward<D>(H, A, B, lit));
  if (TSI_H_IS_MINMAX(H) && bits) {
    const uint32_t mm = TSI_H_IS_II(H) ? sl.w : sl.z;
    const uint32_t d = minmax_decision(H == H_MAX_II || H == H_MAX_IF, A, B);
    if (d) atomicOr(&bits[mm >> 4], d << (2u * (mm & 15u)));
  }
}
template <bool D>
__device__ __forceinline__ void fwd_slot_any(uint32_t h, float2 *V, const uint4 &sl) {
  const float lit = __uint_as_float(sl.w);
  const Iv A = ldv(V, sl.y);
  const Iv B = TSI_H_IS_II(h) ? ldv(V, sl.z) : iv(lit);
  stv(V, sl.x >> 8, op_forward<D>(h, A, B, lit));
}

// Forward pass over the bundles (compute.wgsl:3633-3772); returns the field.
// `bits`: 2 bits per min/max of this cell (A always chosen, B always chosen).
template <bool D>
__device__ __forceinline__ Iv cell_forward(const WideDev &W, const uint2 *bt_tab, float2 *V, uint32_t *bits, Iv x, Iv y, Iv z,
                           Iv t) {
  const uint32_t tid = threadIdx.x;
  const int nb = (int)W.nbundles;
  const WideFetch fetch{bt_tab, W.slots, (uint32_t)nb, tid};
  if (tid == 0) {
    stv(V, 0, x);
    stv(V, 1, y);
    stv(V, 2, z);
    stv(V, 3, t);
  }
  // slots fetched three bundles ahead of their use
  uint4 q0 = fetch(0, 0, 0), q1 = fetch(1, 0, 0), q2 = fetch(2, 0, 0);
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const uint4 sl = q0;
    q0 = q1;
    q1 = q2;
    q2 = fetch(k + 3, 0, 0);
    const uint32_t h = sl.x & 63u;
    if (TSI_H_IS_MINMAX(h)) {
      switch (h) {
        case H_MIN_II: fwd_slot<D, H_MIN_II>(V, bits, sl); break;
        case H_MAX_II: fwd_slot<D, H_MAX_II>(V, bits, sl); break;
        case H_MIN_IF: fwd_slot<D, H_MIN_IF>(V, bits, sl); break;
        default: fwd_slot<D, H_MAX_IF>(V, bits, sl); break;
      }
    } else if (h != TSI_H_PAD) {
      fwd_slot_any<D>(h, V, sl);
    }
    __syncthreads();
  }
  return ldv(V, W.nvalues - 1u);
}

// cell_forward over two time intervals at once: V holds the values over
// `t` (the field and the reverse pass use them), V2 those over `t2`, whose
// min/max decisions go to bits2 (those over `t` to bits).  The second
// evaluation is independent of the first, so a bundle step runs both.
template <bool D, uint32_t H>
__device__ __forceinline__ void fwd2_slot(float2 *V, float2 *V2, uint32_t *bits, uint32_t *bits2, const uint4 &sl) {
  const float lit = __uint_as_float(sl.w);
  const Iv A = ldv(V, sl.y), A2 = ldv(V2, sl.y);
  const Iv B = TSI_H_IS_II(H) ? ldv(V, sl.z) : iv(lit);
  const Iv B2 = TSI_H_IS_II(H) ? ldv(V2, sl.z) : iv(lit);
  stv(V, sl.x >> 8, op_forward<D>(H, A, B, lit));
  stv(V2, sl.x >> 8, op_forward<D>(H, A2, B2, lit));
  if (TSI_H_IS_MINMAX(H)) {
    const uint32_t mm = TSI_H_IS_II(H) ? sl.w : sl.z;
    const uint32_t sh = 2u * (mm & 15u);
    constexpr bool amax = (H == H_MAX_II || H == H_MAX_IF);
    const uint32_t d = minmax_decision(amax, A, B), d2 = minmax_decision(amax, A2, B2);
    if (d) atomicOr(&bits[mm >> 4], d << sh);
    if (d2) atomicOr(&bits2[mm >> 4], d2 << sh);
  }
}
template <bool D>
__device__ __forceinline__ void fwd2_slot_any(uint32_t h, float2 *V, float2 *V2, const uint4 &sl) {
  const float lit = __uint_as_float(sl.w);
  const bool II = TSI_H_IS_II(h);
  const Iv A = ldv(V, sl.y), A2 = ldv(V2, sl.y);
  const Iv B = II ? ldv(V, sl.z) : iv(lit);
  const Iv B2 = II ? ldv(V2, sl.z) : iv(lit);
  stv(V, sl.x >> 8, op_forward<D>(h, A, B, lit));
  stv(V2, sl.x >> 8, op_forward<D>(h, A2, B2, lit));
}

template <bool D>
__device__ __forceinline__ Iv cell_forward2(const WideDev &W, const uint2 *bt_tab, float2 *V, float2 *V2,
                                            uint32_t *bits, uint32_t *bits2, Iv x, Iv y, Iv z, Iv t, Iv t2) {
  const uint32_t tid = threadIdx.x;
  const int nb = (int)W.nbundles;
  const WideFetch fetch{bt_tab, W.slots, (uint32_t)nb, tid};
  if (tid == 0) {
    stv(V, 0, x);
    stv(V, 1, y);
    stv(V, 2, z);
    stv(V, 3, t);
    stv(V2, 0, x);
    stv(V2, 1, y);
    stv(V2, 2, z);
    stv(V2, 3, t2);
  }
  uint4 q0 = fetch(0, 0, 0), q1 = fetch(1, 0, 0), q2 = fetch(2, 0, 0);
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    const uint4 sl = q0;
    q0 = q1;
    q1 = q2;
    q2 = fetch(k + 3, 0, 0);
    const uint32_t h = sl.x & 63u;
    if (TSI_H_IS_MINMAX(h)) {
      switch (h) {
        case H_MIN_II: fwd2_slot<D, H_MIN_II>(V, V2, bits, bits2, sl); break;
        case H_MAX_II: fwd2_slot<D, H_MAX_II>(V, V2, bits, bits2, sl); break;
        case H_MIN_IF: fwd2_slot<D, H_MIN_IF>(V, V2, bits, bits2, sl); break;
        default: fwd2_slot<D, H_MAX_IF>(V, V2, bits, bits2, sl); break;
      }
    } else if (h != TSI_H_PAD) {
      fwd2_slot_any<D>(h, V, V2, sl);
    }
    __syncthreads();
  }
  return ldv(V, W.nvalues - 1u);
}

// Sum of a value's contribution records, last user first, onto +0: the
// accumulation order of the sequential reverse pass.
template <bool D>
__device__ __forceinline__ Iv gather_sens(const float2 *R, uint32_t base, uint32_t count) {
  Iv S = iv(0.0f);
  uint32_t i = 0;
  for (; i + 4u <= count; i += 4u) {  // loads ahead of the dependent adds
    const float2 c0 = R[base + i], c1 = R[base + i + 1u], c2 = R[base + i + 2u], c3 = R[base + i + 3u];
    S = IA<D>::add(Iv{c0.x, c0.y}, S);
    S = IA<D>::add(Iv{c1.x, c1.y}, S);
    S = IA<D>::add(Iv{c2.x, c2.y}, S);
    S = IA<D>::add(Iv{c3.x, c3.y}, S);
  }
  for (; i < count; ++i) S = IA<D>::add(ldv(R, base + i), S);
  return S;
}

// ---------------------------------------------------------------- reverse
// One slot of the reverse pass: its sensitivity (its own value's, or the sum
// of its contribution records), the handler's reverse rule and the
// operands' sensitivities (a record per use for an operand with several
// users, else written directly; the skip rule of compute.wgsl:3800-3806).
template <bool D>
__device__ __forceinline__ void rev_slot_body(uint32_t h, const float2 *V, float2 *G, float2 *R, const uint4 &sl,
                                              const uint4 &s2) {
  using I = IA<D>;
  const bool II = TSI_H_IS_II(h);
  const uint32_t fa = (sl.x >> 6) & 1u, fb = (sl.x >> 7) & 1u;
  const uint32_t a = sl.y, b = sl.z;
  const float lit = __uint_as_float(sl.w);
  const Iv A = ldv(V, a);
  const Iv B = II ? ldv(V, b) : iv(lit);
  const Iv s = s2.w ? gather_sens<D>(R, s2.z, s2.w) : ldv(G, sl.x >> 8);
  const bool s0 = (s.lo == 0.0f && s.hi == 0.0f);
  const bool skip = II ? (s0 && fa && fb) : (s0 && fa);
  Iv c0 = iv(0.0f), c1 = iv(0.0f);
  if (!skip) {
    Iv r0, r1;
    op_reverse_rule<D>(h, A, B, lit, r0, r1);
    c0 = I::mul(I::fix(r0), s);
    if (II) c1 = I::mul(I::fix(r1), s);
  }
  // both operands read before either is written (an instruction whose
  // operands are one value keeps the second write)
  const Iv pa = (s2.x == TSI_NONE && !skip) ? ldv(G, a) : iv(0.0f);
  const Iv pb = (II && s2.y == TSI_NONE && !skip) ? ldv(G, b) : iv(0.0f);
  if (s2.x != TSI_NONE) stv(R, s2.x, c0);
  else stv(G, a, skip ? iv(0.0f) : I::add(c0, pa));
  if (II) {
    if (s2.y != TSI_NONE) stv(R, s2.y, c1);
    else stv(G, b, skip ? iv(0.0f) : I::add(c1, pb));
  }
}

// Reverse interval AD over the bundles (compute.wgsl:3786-3900).  A
// single-use operand's sensitivity is written by its one user; an operand
// with several users gets a contribution record per user (R), summed when
// the reverse pass reaches the value.  sens_out: 4 floats x 2 in shared
// memory for the arguments' sensitivities.
template <bool D>
__device__ __forceinline__ void cell_reverse(const WideDev &W, const uint2 *bt_tab, const float2 *V, float2 *G, float2 *R,
                             float2 *sens_out) {
  const uint32_t tid = threadIdx.x;
  const uint32_t ns = W.nslots, nv = W.nvalues;
  const int nb = (int)W.nbundles;
  const WideFetch fetch{bt_tab, W.slots, (uint32_t)nb, tid};
  for (uint32_t v = tid; v < nv; v += blockDim.x) G[v] = make_float2(0.0f, 0.0f);
  // words 0-3 and 8-11 of this thread's slot, two bundles ahead
  uint4 a0 = fetch(nb - 1, 0, ns), a2 = fetch(nb - 1, 2, ns);
  uint4 b0 = fetch(nb - 2, 0, ns), b2 = fetch(nb - 2, 2, ns);
  __syncthreads();
  if (tid == 0) G[nv - 1u] = make_float2(1.0f, 1.0f);
  __syncthreads();
  for (int k = nb - 1; k >= 0; --k) {
    const uint4 sl = a0, s2 = a2;
    a0 = b0;
    a2 = b2;
    b0 = fetch(k - 2, 0, ns);
    b2 = fetch(k - 2, 2, ns);
    const uint32_t h = sl.x & 63u;
    if (h != TSI_H_PAD && h != H_CONST) rev_slot_body<D>(h, V, G, R, sl, s2);
    __syncthreads();
  }
  if (tid < 4u) {
    const uint32_t gc = W.arg_gcount[tid];
    stv(sens_out, tid, gc ? gather_sens<D>(R, W.arg_gbase[tid], gc) : ldv(G, tid));
  }
  __syncthreads();
}

}  // namespace tsi
