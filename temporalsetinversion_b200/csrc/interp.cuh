// interp.cuh — the one-warp tape interpreter: 32 cells per warp (one per
// lane), one tape instruction at a time on the packed register tape
// (tape_format.h), interval registers in shared memory.
//
// forward_pass follows compute.wgsl:3633-3772 (with the operand log and the
// min/max branch ballots the reverse pass and the pruning need);
// reverse_pass follows compute.wgsl:3785-3964.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "interval.cuh"
#include "tape_format.h"

namespace tsi {

#define FULL_MASK 0xffffffffu

// Instruction j of a 32-instruction chunk held one per lane.
__device__ __forceinline__ uint2 chunk_word(uint2 c, uint32_t j) {
  return make_uint2(__shfl_sync(0xffffffffu, c.x, j), __shfl_sync(0xffffffffu, c.y, j));
}
// Chunk k of a tape: instruction 32k + lane (zero past the end).
__device__ __forceinline__ uint2 load_chunk(const uint2 *__restrict__ code, uint32_t len, int k, uint32_t lane) {
  const int i = 32 * k + (int)lane;
  return (k >= 0 && i < (int)len) ? code[i] : make_uint2(0u, 0u);
}

__device__ __forceinline__ bool finite2(Iv a) { return isfinite(a.lo) && isfinite(a.hi); }

__device__ __forceinline__ Iv ld_reg(const float2 *rf, uint32_t r, uint32_t lane) {
  const float2 v = rf[r * 32u + lane];
  return Iv{v.x, v.y};
}
__device__ __forceinline__ void st_reg(float2 *rf, uint32_t r, uint32_t lane, Iv v) {
  rf[r * 32u + lane] = make_float2(v.lo, v.hi);
}

// ---------------------------------------------------------------- handlers
// Rare handlers live out of line so the interpreter loop stays small.
template <bool D>
__device__ __noinline__ Iv cold_forward(uint32_t h, Iv A, Iv B, float lit) {
  return IA<D>::forward(h, A, B, lit);
}

template <bool D>
__device__ __forceinline__ Iv op_forward(uint32_t h, Iv A, Iv B, float lit) {
  using I = IA<D>;
  Iv v;
  switch (h) {
    case H_CONST: v = iv(lit); break;
    case H_COPY: v = A; break;
    case H_ADD_II: v = I::add(A, B); break;
    case H_SUB_II: v = I::sub(A, B); break;
    case H_MUL_II: v = I::mul(A, B); break;
    case H_MIN_II: v = I::min_(A, B); break;
    case H_MAX_II: v = I::max_(A, B); break;
    case H_ADD_IF: v = I::add_f(A, lit); break;
    case H_SUB_IF: v = I::sub_f(A, lit); break;
    case H_MUL_IF: v = I::mul_f(A, lit); break;
    case H_MIN_IF: v = Iv{fm_min(A.lo, lit), fm_min(A.hi, lit)}; break;
    case H_MAX_IF: v = Iv{fm_max(A.lo, lit), fm_max(A.hi, lit)}; break;
    case H_SQR: v = I::sqr(A); break;
    case H_SQRT: v = I::sqrt_(A); break;
    case H_NEG: v = I::neg(A); break;
    case H_ABS: v = I::abs_(A); break;
    case H_SUB_FI: v = I::sub(iv(lit), A); break;
    default: return cold_forward<D>(h, A, B, lit);  // fixed inside
  }
  return I::fix(v);
}

template <bool D>
__device__ __noinline__ int cold_reverse_rule(uint32_t h, Iv A, Iv B, float lit, Iv &r0, Iv &r1) {
  return IA<D>::reverse_rule(h, A, B, lit, r0, r1);
}

template <bool D>
__device__ __forceinline__ void op_reverse_rule(uint32_t h, Iv A, Iv B, float lit, Iv &r0, Iv &r1) {
  using I = IA<D>;
  switch (h) {
    case H_COPY: r0 = iv(1.0f); break;
    case H_ADD_II: r0 = iv(1.0f); r1 = iv(1.0f); break;
    case H_SUB_II: r0 = iv(1.0f); r1 = iv(-1.0f); break;
    case H_MUL_II: r0 = B; r1 = A; break;
    case H_MIN_II: I::min_rr(A, B, r0, r1); break;
    case H_MAX_II: I::max_rr(A, B, r0, r1); break;
    case H_ADD_IF: r0 = iv(1.0f); break;
    case H_SUB_IF: r0 = iv(1.0f); break;
    case H_MUL_IF: r0 = iv(lit); break;
    case H_SQR: r0 = I::mul_f(A, 2.0f); break;
    case H_NEG: r0 = iv(-1.0f); break;
    case H_ABS: r0 = I::abs_rr(A); break;
    case H_SUB_FI: r0 = iv(-1.0f); break;
    case H_MIN_IF: { Iv t; I::min_rr(A, iv(lit), r0, t); break; }
    case H_MAX_IF: { Iv t; I::max_rr(A, iv(lit), r0, t); break; }
    default: cold_reverse_rule<D>(h, A, B, lit, r0, r1); break;
  }
}

// ---------------------------------------------------------------- passes
// Forward pass over `len` instructions (compute.wgsl:3633-3772).  Writes the
// operand log when `lg` is set and the min/max branch ballots when `dg` is
// set.  Returns the output register's value.
template <bool D>
__device__ __forceinline__ Iv forward_pass(const uint2 *__restrict__ code, uint32_t len, uint32_t out_reg, float2 *rf,
                                           uint32_t lane, Iv x, Iv y, Iv z, Iv t, float4 *lg, uint2 *dg) {
  st_reg(rf, 0, lane, x);
  st_reg(rf, 1, lane, y);
  st_reg(rf, 2, lane, z);
  st_reg(rf, 3, lane, t);
  uint32_t mm = 0;
  // the tape arrives 32 instructions per coalesced load, one chunk ahead
  uint2 cur = load_chunk(code, len, 0, lane), nxt = load_chunk(code, len, 1, lane);
  for (uint32_t c0 = 0; c0 < len; c0 += 32u) {
    const uint32_t n = min(32u, len - c0);
    for (uint32_t j = 0; j < n; ++j) {
      const uint2 w = chunk_word(cur, j);
      const uint32_t i = c0 + j;
      const uint32_t h = TSI_W0_H(w.x);
      const float lit = __uint_as_float(w.y);
      const Iv Av = ld_reg(rf, TSI_W0_A(w.x), lane);
      const Iv Bv = TSI_H_IS_II(h) ? ld_reg(rf, w.y & 255u, lane) : iv(lit);
      const Iv r = op_forward<D>(h, Av, Bv, lit);
      if (lg) lg[(size_t)i * 32u + lane] = make_float4(Av.lo, Av.hi, Bv.lo, Bv.hi);
      if (dg && TSI_H_IS_MINMAX(h)) {
        const bool amax = (h == H_MAX_II || h == H_MAX_IF);
        const bool a_below = Av.hi < Bv.lo, b_below = Bv.hi < Av.lo;
        const uint32_t ua = __ballot_sync(FULL_MASK, amax ? b_below : a_below);
        const uint32_t ub = __ballot_sync(FULL_MASK, amax ? a_below : b_below);
        if (lane == 0) dg[mm] = make_uint2(ua, ub);
        ++mm;
      }
      st_reg(rf, TSI_W0_DST(w.x), lane, r);
    }
    cur = nxt;
    nxt = load_chunk(code, len, (int)(c0 / 32u) + 2, lane);
  }
  return ld_reg(rf, out_reg, lane);
}

// Reverse pass (compute.wgsl:3785-3964): sensitivities reuse the register
// file; a register's accumulator is consumed and cleared at the definition
// it holds.  `bad` collects non-finite sensitivities.
template <bool D>
__device__ __forceinline__ void reverse_pass(const uint2 *__restrict__ code, uint32_t len, uint32_t nregs,
                                             uint32_t out_reg, float2 *rf, uint32_t lane, const float4 *lg,
                                             bool take, Iv sens[4], bool &bad) {
  using I = IA<D>;
  for (uint32_t r = 0; r < nregs; ++r) st_reg(rf, r, lane, iv(0.0f));
  st_reg(rf, out_reg, lane, iv(1.0f));
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  auto log_at = [&](int i) { return i >= 0 ? lg[(size_t)i * 32u + lane] : zero4; };
  // log entries three instructions ahead, the tape one 32-instruction chunk ahead
  float4 L0 = log_at((int)len - 1), L1 = log_at((int)len - 2), L2 = log_at((int)len - 3);
  const int nch = (int)((len + 31u) / 32u);
  uint2 cur = load_chunk(code, len, nch - 1, lane), nxt = load_chunk(code, len, nch - 2, lane);
  for (int k = nch - 1; k >= 0; --k) {
    const int c0 = 32 * k;
    for (int j = min(32, (int)len - c0) - 1; j >= 0; --j) {
      const int i = c0 + j;
      const uint2 w = chunk_word(cur, (uint32_t)j);
      const float4 L = L0;
      L0 = L1;
      L1 = L2;
      L2 = log_at(i - 3);
      const uint32_t h = TSI_W0_H(w.x);
      const uint32_t d = TSI_W0_DST(w.x), a = TSI_W0_A(w.x), b = w.y & 255u;
      const float lit = __uint_as_float(w.y);
      const Iv Av = Iv{L.x, L.y}, Bv = Iv{L.z, L.w};
      const Iv s = ld_reg(rf, d, lane);
      st_reg(rf, d, lane, iv(0.0f));
      if (take && h != H_CONST) {
        bad |= !finite2(s);
        const bool s0 = (s.lo == 0.0f && s.hi == 0.0f);
        if (TSI_H_IS_II(h)) {
          if (s0 && TSI_W0_FA(w.x) && TSI_W0_FB(w.x)) {
            st_reg(rf, a, lane, iv(0.0f));
            st_reg(rf, b, lane, iv(0.0f));
          } else {
            Iv r0, r1;
            op_reverse_rule<D>(h, Av, Bv, lit, r0, r1);
            r0 = I::mul(I::fix(r0), s);
            r1 = I::mul(I::fix(r1), s);
            const Iv n0 = I::add(r0, ld_reg(rf, a, lane));
            const Iv n1 = I::add(r1, ld_reg(rf, b, lane));
            st_reg(rf, a, lane, n0);
            st_reg(rf, b, lane, n1);
            bad |= !finite2(n0) || !finite2(n1);
          }
        } else if (s0 && TSI_W0_FA(w.x)) {
          st_reg(rf, a, lane, iv(0.0f));
        } else {
          Iv r0, r1;
          op_reverse_rule<D>(h, Av, Bv, lit, r0, r1);
          r0 = I::mul(I::fix(r0), s);
          const Iv n0 = I::add(r0, ld_reg(rf, a, lane));
          st_reg(rf, a, lane, n0);
          bad |= !finite2(n0);
        }
      } else if (take) {
        bad |= !finite2(s);
      }
    }
    cur = nxt;
    nxt = load_chunk(code, len, k - 2, lane);
  }
  for (int q = 0; q < 4; ++q) sens[q] = ld_reg(rf, q, lane);
}


}  // namespace tsi
