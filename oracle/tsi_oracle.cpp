/*
 * tsi_oracle.cpp — TEST INFRASTRUCTURE: CPU restatement of the reference's
 * hot path, used only by tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py.  The product never links or calls it.
 *
 * Parity status: UNPINNED against the reference's own outputs.  The
 * reference is WGSL run through wgpu/Vulkan (no cargo, no Vulkan driver on
 * this machine or the GPU machine) and ships no tests or golden vectors;
 * the only reference fixtures are the scene tapes scenes/{cables,cradle,piano,sponza}.ll, which fix
 * inputs, not outputs.  This file is therefore a line-by-line restatement
 * of the reference's algorithm, each function citing the lines it follows.
 * A second restatement written separately in numpy (tests/test_cpu_*_restatement.py:
 * interval ops and reverse rules, the whole-tape passes, the per-cell
 * temporal logic, point-sampled leaves, swept volume, the tracer and
 * cameras) agrees with it bit for bit; that checks the restatement, not the
 * reference's own outputs.  The parts restated:
 *
 *   interval ops           src/compute.wgsl:2474-2975, fix 3462-3472
 *   refinement `main`      src/compute.wgsl:3513-4056 (run level by level)
 *   root seeding           src/main.rs:749-766, compute.wgsl:4690-4708
 *   ray tracer             src/compute.wgsl:4059-4107, 4189-4403
 *   camera + shading       src/compute.wgsl:4590-4594, 4620-4688
 *   cinematic path tracing src/compute.wgsl:4429-4523 (bounces, shadow rays),
 *                          2451-2472 (frand), 497-677 (sky), 4600-4607 (sRGB)
 *
 * It consumes the tape in the reference's own 32-byte GPUInstruction layout
 * (src/ir.rs:88-97) and decodes it per instruction exactly as the shader
 * does (unpack2x16, op_top switch); it shares no code with the library.
 *
 * Deliberate, documented choices where the reference is not deterministic:
 *  - WGSL built-ins sin/exp/log/atan2/pow are replaced by oracle_fmath.h;
 *    min/max use IEEE minimumNumber/maximumNumber (NaN loses, -0 < +0).
 *  - mallocV (compute.wgsl:3437-3450) leaves dx/dy/dz of a recycled voxel
 *    stale (scheduling dependent); here a new voxel starts with zero normal.
 *  - the trace stack holds 32 entries instead of 16 (compute.wgsl:4075),
 *    so octrees deeper than 8 levels are traversed without overflow.
 * Built with -O2 -ffp-contract=off -fno-fast-math (no FMA contraction).
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

#include "oracle_fmath.h"

namespace {

struct I {
  float lo, hi;
};

/* ---------- compute.wgsl:2474-2975, RN f32 ---------- */
const float PI_F = 3.1415927410125732f;
const float TWOPI_F = 6.2831854820251465f;
const float HALFPI_F = 1.5707963705062866f;
const float BIG_F = 1000000.0f;

inline I IF(float a) { return I{a, a}; }
inline I I_FROM_UNORDERED(float a, float b) { return I{of_min(a, b), of_max(a, b)}; }
inline bool I_CONTAINS_ZERO(I a) { return a.lo <= 0.0f && 0.0f <= a.hi; }
inline bool I_CONTAINS_X(I a, float x) { return a.lo <= x && x <= a.hi; }
inline float DIAMETER(I a) { return a.hi - a.lo; }
inline float MID(I a) { return (a.lo + a.hi) / 2.0f; }
inline bool is_nan(float a) { return !(a < 0.0f || a > 0.0f || a == 0.0f); }
inline I ADD_II(I a, I b) { return I{a.lo + b.lo, a.hi + b.hi}; }
inline I ADD_IF(I a, float b) { return I{a.lo + b, a.hi + b}; }
inline I SUB_II(I a, I b) { return I{a.lo - b.hi, a.hi - b.lo}; }
inline I SUB_IF(I a, float b) { return I{a.lo - b, a.hi - b}; }
inline I MUL_II(I a, I b) {
  float x = a.lo * b.lo, y = a.lo * b.hi, z = a.hi * b.lo, w = a.hi * b.hi;
  return I{of_min(of_min(x, y), of_min(z, w)), of_max(of_max(x, y), of_max(z, w))};
}
inline I MUL_IF(I a, float b) {
  if (b >= 0.0f) return I{a.lo * b, a.hi * b};
  return I{a.hi * b, a.lo * b};
}
inline I SQRT_I(I a) { return I{sqrtf(of_max(a.lo, 0.0f)), sqrtf(of_max(a.hi, 0.0f))}; }
inline I EXP_I(I a) { return I{of_exp(a.lo), of_exp(a.hi)}; }
inline I LOG_I(I a) { return I{of_log(of_max(a.lo, 0.0f)), of_log(of_max(a.hi, 0.0f))}; }
inline I NEG_I(I a) { return I{-a.hi, -a.lo}; }
inline I DIV_II(I a, I b) {
  float x = a.lo / b.lo, y = a.lo / b.hi, z = a.hi / b.lo, w = a.hi / b.hi;
  return I{of_min(of_min(x, y), of_min(z, w)), of_max(of_max(x, y), of_max(z, w))};
}
inline I DIV_IF(I a, float b) { return DIV_II(a, IF(b)); }
inline I MIN_II(I a, I b) { return I{of_min(a.lo, b.lo), of_min(a.hi, b.hi)}; }
inline I MIN_IF(I a, float b) { return I{of_min(a.lo, b), of_min(a.hi, b)}; }
inline I MAX_IF(I a, float b) { return I{of_max(a.lo, b), of_max(a.hi, b)}; }
inline I MAX_II(I a, I b) { return I{of_max(a.lo, b.lo), of_max(a.hi, b.hi)}; }
inline I ABS_I(I a) {
  if (I_CONTAINS_ZERO(a)) return I{0.0f, of_max(-a.lo, a.hi)};
  if (a.hi < 0.0f) return I{-a.hi, -a.lo};
  return a;
}
inline I ABS_I_RR(I a) {
  if (I_CONTAINS_ZERO(a)) return I{-1.0f, 1.0f};
  if (a.hi < 0.0f) return IF(-1.0f);
  return IF(1.0f);
}
inline I I_EMPTY() { return I{OF_INF, -OF_INF}; }
inline I CAP_II(I a, I b) {
  if (a.hi < b.lo || b.hi < a.lo) return I_EMPTY();
  return I{of_max(a.lo, b.lo), of_min(a.hi, b.hi)};
}
inline I SQR_I(I a) {
  float x = a.lo * a.lo, y = a.hi * a.hi;
  if (I_CONTAINS_ZERO(a)) return I{0.0f, of_max(x, y)};
  return I{of_min(x, y), of_max(x, y)};
}
inline I FLOOR_I(I a) { return I{floorf(a.lo), floorf(a.hi)}; }
inline I FLOOR_I_RR(I a) {
  if (floorf(a.hi) != floorf(a.lo)) return I{-BIG_F, BIG_F};
  return IF(0.0f);
}
inline float wgsl_atan2(float y, float x) { return of_atan2(y, x); }
inline I ATAN2_II(I x, I y) { /* compute.wgsl:2724-2804 */
  I range_atan = I{-PI_F, PI_F};
  I half_range_atan = I{-HALFPI_F, HALFPI_F};
  if (y.lo == 0.0f) return I{0.0f, y.hi};
  if (y.hi == 0.0f) return I{y.lo, 0.0f};
  if (x.lo == 0.0f && x.hi == 0.0f) {
    if (y.lo == 0.0f && y.hi == 0.0f) return I_EMPTY();
    if (y.lo >= 0.0f) return IF(HALFPI_F);
    if (y.hi <= 0.0f) return IF(-HALFPI_F);
    return half_range_atan;
  } else if (x.lo > 0.0f) {
    if (y.lo == 0.0f && y.hi == 0.0f) return y;
    if (y.lo >= 0.0f) return I{wgsl_atan2(y.lo, x.hi), wgsl_atan2(y.hi, x.lo)};
    if (y.hi <= 0.0f) return I{wgsl_atan2(y.lo, x.lo), wgsl_atan2(y.hi, x.hi)};
    return I{wgsl_atan2(y.lo, x.lo), wgsl_atan2(y.hi, x.lo)};
  } else if (x.hi < 0.0f) {
    if (y.lo == 0.0f && y.hi == 0.0f) return IF(PI_F);
    if (y.lo >= 0.0f) return I{wgsl_atan2(y.hi, x.hi), wgsl_atan2(y.lo, x.lo)};
    if (y.hi < 0.0f) return I{wgsl_atan2(y.hi, x.lo), wgsl_atan2(y.lo, x.hi)};
    return range_atan;
  } else {
    if (x.lo == 0.0f) {
      if (y.lo == 0.0f && y.hi == 0.0f) return y;
      if (y.lo >= 0.0f) return I{wgsl_atan2(y.lo, x.hi), half_range_atan.hi};
      if (y.hi <= 0.0f) return I{half_range_atan.lo, wgsl_atan2(y.hi, x.hi)};
      return half_range_atan;
    } else if (x.hi == 0.0f) {
      if (y.lo == 0.0f && y.hi == 0.0f) return IF(PI_F);
      if (y.lo >= 0.0f) return I{HALFPI_F, wgsl_atan2(y.lo, x.lo)};
      if (y.hi < 0.0f) return I{wgsl_atan2(y.hi, x.lo), -HALFPI_F};
      return range_atan;
    } else {
      if (y.lo >= 0.0f) return I{wgsl_atan2(y.lo, x.hi), wgsl_atan2(y.lo, x.lo)};
      if (y.hi < 0.0f) return I{wgsl_atan2(y.hi, x.lo), wgsl_atan2(y.hi, x.hi)};
      return range_atan;
    }
  }
}
inline void ATAN2_II_RR(I larg, I rarg, I out[2]) {
  I den = ADD_II(SQR_I(rarg), SQR_I(larg));
  out[0] = DIV_II(NEG_I(larg), den);
  out[1] = DIV_II(rarg, den);
}
inline I SQR_I_RR(I a) { return MUL_IF(a, 2.0f); }
inline I MOD_II(I a, I b) { return SUB_II(a, MUL_II(b, FLOOR_I(DIV_II(a, b)))); }
inline void MOD_II_RR(I larg, I rarg, I out[2]) {
  I a = FLOOR_I(DIV_II(larg, rarg));
  out[0] = IF(1.0f);
  out[1] = NEG_I(ADD_II(a, MUL_II(rarg, FLOOR_I_RR(a))));
}
inline I POW_II(I a, I b) { /* compute.wgsl:2829-2860 */
  /* i32(round(x)) saturates; NaN converts to 0 */
  int power;
  float rb = rintf(b.lo);
  if (rb != rb) power = 0;
  else if (rb >= 2147483520.0f) power = 2147483647;
  else if (rb <= -2147483648.0f) power = -2147483647 - 1;
  else power = (int)rb;
  float lower, higher;
  if (a.lo <= 0.0f) {
    lower = (power % 2 == 0) ? of_powi(-a.lo, power) : -of_powi(-a.lo, power);
  } else {
    lower = of_powi(a.lo, power);
  }
  if (a.hi <= 0.0f) {
    higher = (power % 2 == 0) ? of_powi(-a.hi, power) : -of_powi(-a.hi, power);
  } else {
    higher = of_powi(a.hi, power);
  }
  if (I_CONTAINS_ZERO(a)) return I{0.0f, of_max(lower, higher)};
  return I{of_min(lower, higher), of_max(lower, higher)};
}
inline void POW_II_RR(I larg, I rarg, I out[2]) {
  out[0] = MUL_II(rarg, POW_II(larg, SUB_IF(rarg, 1.0f)));
  out[1] = MUL_II(POW_II(larg, rarg), LOG_I(larg));
}
inline I LOG_I_RR(I a) { return DIV_II(IF(1.0f), a); }
inline I EXP_I_RR(I a) { return EXP_I(a); }
inline I SQRT_I_RR(I a) {
  I res = DIV_II(IF(1.0f), MUL_IF(SQRT_I(a), 2.0f));
  res.hi = of_min(res.hi, BIG_F);
  return res;
}
inline void MIN_II_RR(I l, I r, I out[2]) {
  if (l.hi < r.lo) { out[0] = IF(1.0f); out[1] = IF(0.0f); }
  else if (r.hi < l.lo) { out[0] = IF(0.0f); out[1] = IF(1.0f); }
  else { out[0] = IF(1.0f); out[1] = IF(1.0f); }
}
inline void MAX_II_RR(I l, I r, I out[2]) {
  if (l.hi < r.lo) { out[0] = IF(0.0f); out[1] = IF(1.0f); }
  else if (r.hi < l.lo) { out[0] = IF(1.0f); out[1] = IF(0.0f); }
  else { out[0] = IF(1.0f); out[1] = IF(1.0f); }
}
inline void DIV_II_RR(I l, I r, I out[2]) {
  out[0] = DIV_II(IF(1.0f), r);
  out[1] = NEG_I(DIV_II(l, SQR_I(r)));
}
inline float mymod(float x, float y) { return x - y * floorf(x / y); }
inline I SIN_I(I a) { /* compute.wgsl:2926-2957 */
  I whole_range = I{-1.0f, 1.0f};
  if (DIAMETER(a) > TWOPI_F) return whole_range;
  float lo_q = floorf(a.lo / HALFPI_F);
  float hi_q = floorf(a.hi / HALFPI_F);
  if (hi_q - lo_q > 4.0f) return whole_range;
  lo_q = mymod(lo_q, 4.0f);
  hi_q = mymod(hi_q, 4.0f);
  if (lo_q == hi_q) {
    if (a.hi - a.lo > PI_F) return whole_range;
    return I_FROM_UNORDERED(of_sin(a.lo), of_sin(a.hi));
  } else if ((lo_q == 3.0f && hi_q == 0.0f) || (lo_q == 1.0f && hi_q == 2.0f)) {
    return I_FROM_UNORDERED(of_sin(a.lo), of_sin(a.hi));
  } else if ((lo_q == 0.0f || lo_q == 3.0f) && (hi_q == 1.0f || hi_q == 2.0f)) {
    return I{of_min(of_sin(a.lo), of_sin(a.hi)), 1.0f};
  } else if ((lo_q == 1.0f || lo_q == 2.0f) && (hi_q == 3.0f || hi_q == 0.0f)) {
    return I{-1.0f, of_max(of_sin(a.lo), of_sin(a.hi))};
  }
  return whole_range;
}
inline I COS_I(I a) { return SIN_I(ADD_II(a, IF(HALFPI_F))); }
inline I SIN_I_RR(I a) { return COS_I(a); }
inline I COS_I_RR(I a) { return NEG_I(SIN_I(a)); }
inline I fix(I x) { /* compute.wgsl:3462-3472 */
  float lo = x.lo, hi = x.hi;
  if (is_nan(x.hi)) hi = BIG_F;
  if (is_nan(x.lo)) lo = -BIG_F;
  return I{of_max(lo, -BIG_F), of_min(hi, BIG_F)};
}

/* ---------- tape, decoded as the shader does ---------- */
struct GInstr { /* ir.rs:90-97 */
  uint32_t index_, opcode_uses, larg_rarg;
  float literal, val[2], sens[2];
};

enum {
  OP_NOP = 0, OP_ADD = 5, OP_SUB = 6, OP_MUL = 7, OP_DIV = 8, OP_EXP = 9, OP_LOG = 10, OP_SQR = 11,
  OP_SQRT = 12, OP_POW = 13, OP_SIN = 14, OP_COS = 15, OP_NEG = 16, OP_MIN = 17, OP_MAX = 18,
  OP_ABS = 19, OP_FLOOR = 25, OP_RET = 28, OP_MOD = 29, OP_ATAN2 = 30
};

struct Scratch {
  std::vector<I> val, sens;
};

struct EvalOut {
  I field;
  I sens[4];
  uint64_t instr;
};

/* compute.wgsl:3632-3970 for one cell; args = slots 0..3. */
void eval_cell(const GInstr *tape, uint32_t count, const I args[4], bool take_derivative,
               Scratch &s, EvalOut &o) {
  if (s.val.size() < count) {
    s.val.resize(count);
    s.sens.resize(count);
  }
  I *val = s.val.data();
  I *sens = s.sens.data();
  for (int j = 0; j < 4; ++j) {
    val[j] = args[j];
    sens[j] = IF(0.0f);
  }
  for (uint32_t j = 4; j < count; ++j) {
    const uint32_t opu = tape[j].opcode_uses >> 16;
    const uint32_t op = opu & ~(3u << 14);
    const uint32_t op_top = opu >> 14;
    const uint32_t lx = tape[j].larg_rarg >> 16, ry = tape[j].larg_rarg & 65535u;
    const float lit = tape[j].literal;
    I v = IF(0.0f);
    switch (op_top) {
      case 1u: {
        I larg = val[lx];
        float rarg = lit;
        switch (op) {
          case OP_SQR: v = SQR_I(larg); break;
          case OP_SQRT: v = SQRT_I(larg); break;
          case OP_EXP: v = EXP_I(larg); break;
          case OP_LOG: v = LOG_I(larg); break;
          case OP_NEG: v = NEG_I(larg); break;
          case OP_ABS: v = ABS_I(larg); break;
          case OP_FLOOR: v = FLOOR_I(larg); break;
          case OP_SIN: v = SIN_I(larg); break;
          case OP_COS: v = COS_I(larg); break;
          case OP_ADD: v = ADD_IF(larg, rarg); break;
          case OP_SUB: v = SUB_IF(larg, rarg); break;
          case OP_DIV: v = DIV_IF(larg, rarg); break;
          case OP_MUL: v = MUL_IF(larg, rarg); break;
          case OP_MIN: v = MIN_IF(larg, rarg); break;
          case OP_MAX: v = MAX_IF(larg, rarg); break;
          case OP_POW: v = POW_II(larg, IF(rarg)); break;
          case OP_RET: v = larg; break;
          case OP_MOD: v = MOD_II(larg, IF(rarg)); break;
          case OP_ATAN2: v = ATAN2_II(larg, IF(rarg)); break;
          default: v = IF(-OF_INF); break;
        }
        break;
      }
      case 0u: {
        I larg = val[lx], rarg = val[ry];
        switch (op) {
          case OP_ADD: v = ADD_II(larg, rarg); break;
          case OP_SUB: v = SUB_II(larg, rarg); break;
          case OP_DIV: v = DIV_II(larg, rarg); break;
          case OP_MUL: v = MUL_II(larg, rarg); break;
          case OP_MIN: v = MIN_II(larg, rarg); break;
          case OP_MAX: v = MAX_II(larg, rarg); break;
          case OP_POW: v = POW_II(larg, rarg); break;
          case OP_MOD: v = MOD_II(larg, rarg); break;
          case OP_ATAN2: v = ATAN2_II(larg, rarg); break;
          case OP_NOP: v = IF(lit); break;
          default: v = IF(-OF_INF); break;
        }
        break;
      }
      case 2u: {
        float larg = lit;
        I rarg = val[ry];
        switch (op) {
          case OP_SUB: v = SUB_II(IF(larg), rarg); break;
          case OP_DIV: v = DIV_II(IF(larg), rarg); break;
          default: v = IF(-OF_INF); break;
        }
        break;
      }
      default: break;
    }
    val[j] = fix(v);
    sens[j] = IF(0.0f);
  }
  o.field = val[count - 1];
  sens[count - 1] = IF(1.0f);
  o.instr = count > 4 ? count - 4 : 0;
  if (take_derivative) {
    for (uint32_t j = count - 1; j >= 4 && j < count; --j) { /* compute.wgsl:3786-3964 */
      const uint32_t opu = tape[j].opcode_uses >> 16;
      const uint32_t op = opu & ~(3u << 14);
      const uint32_t op_top = opu >> 14;
      const uint32_t lx = tape[j].larg_rarg >> 16, ry = tape[j].larg_rarg & 65535u;
      const uint32_t larg_uses = tape[lx].opcode_uses & 65535u;
      const uint32_t rarg_uses = tape[ry].opcode_uses & 65535u;
      const float lit = tape[j].literal;
      const I sj = sens[j];
      switch (op_top) {
        case 1u: {
          I larg = val[lx];
          float rarg = lit;
          if (sj.lo == 0.0f && sj.hi == 0.0f && larg_uses == 1u) {
            sens[lx] = IF(0.0f);
          } else {
            I s, two[2];
            switch (op) {
              case OP_SQR: s = SQR_I_RR(larg); break;
              case OP_SQRT: s = SQRT_I_RR(larg); break;
              case OP_NEG: s = IF(-1.0f); break;
              case OP_SIN: s = SIN_I_RR(larg); break;
              case OP_COS: s = COS_I_RR(larg); break;
              case OP_ADD: s = IF(1.0f); break;
              case OP_SUB: s = IF(1.0f); break;
              case OP_MUL: s = IF(rarg); break;
              case OP_DIV: DIV_II_RR(larg, IF(rarg), two); s = two[0]; break;
              case OP_EXP: s = EXP_I_RR(larg); break;
              case OP_LOG: s = LOG_I_RR(larg); break;
              case OP_FLOOR: s = FLOOR_I_RR(larg); break;
              case OP_ABS: s = ABS_I_RR(larg); break;
              case OP_MIN: MIN_II_RR(larg, IF(rarg), two); s = two[0]; break;
              case OP_MAX: MAX_II_RR(larg, IF(rarg), two); s = two[0]; break;
              case OP_POW: POW_II_RR(larg, IF(rarg), two); s = two[0]; break;
              case OP_RET: s = IF(1.0f); break;
              case OP_MOD: s = IF(1.0f); break;
              case OP_ATAN2: ATAN2_II_RR(larg, IF(rarg), two); s = two[0]; break;
              default: s = IF(-OF_INF); break;
            }
            s = fix(s);
            s = MUL_II(s, sj);
            s = ADD_II(s, sens[lx]);
            sens[lx] = s;
          }
          break;
        }
        case 0u: {
          I larg = val[lx], rarg = val[ry];
          if (sj.lo == 0.0f && sj.hi == 0.0f && larg_uses == 1u && rarg_uses == 1u) {
            sens[lx] = IF(0.0f);
            sens[ry] = IF(0.0f);
          } else {
            I s[2];
            switch (op) {
              case OP_MIN: MIN_II_RR(larg, rarg, s); break;
              case OP_MUL: s[0] = rarg; s[1] = larg; break;
              case OP_DIV: DIV_II_RR(larg, rarg, s); break;
              case OP_ADD: s[0] = IF(1.0f); s[1] = IF(1.0f); break;
              case OP_SUB: s[0] = IF(1.0f); s[1] = IF(-1.0f); break;
              case OP_MAX: MAX_II_RR(larg, rarg, s); break;
              case OP_POW: POW_II_RR(larg, rarg, s); break;
              case OP_ATAN2: ATAN2_II_RR(larg, rarg, s); break;
              case OP_NOP: s[0] = IF(0.0f); s[1] = IF(0.0f); break;
              default: s[0] = IF(-OF_INF); s[1] = IF(-OF_INF); break;
            }
            s[0] = fix(s[0]);
            s[1] = fix(s[1]);
            s[0] = MUL_II(s[0], sj);
            s[1] = MUL_II(s[1], sj);
            s[0] = ADD_II(s[0], sens[lx]);
            s[1] = ADD_II(s[1], sens[ry]);
            sens[lx] = s[0];
            sens[ry] = s[1];
          }
          break;
        }
        case 2u: {
          float larg = lit;
          I rarg = val[ry];
          if (sj.lo == 0.0f && sj.hi == 0.0f && rarg_uses == 1u) {
            sens[ry] = IF(0.0f);
          } else {
            I s, two[2];
            switch (op) {
              case OP_SUB: s = IF(-1.0f); break;
              case OP_DIV: DIV_II_RR(IF(larg), rarg, two); s = two[1]; break;
              default: s = IF(-OF_INF); break;
            }
            s = fix(s);
            s = MUL_II(s, sj);
            s = ADD_II(s, sens[ry]);
            sens[ry] = s;
          }
          break;
        }
        default: break;
      }
    }
  }
  for (int k = 0; k < 4; ++k) o.sens[k] = sens[k];
}

/* ---------- octree (compute.wgsl:3003-3016) ---------- */
struct Voxel {
  I x, y, z;
  float t;
  uint32_t child_count;
  uint32_t children[8];
  float f, dx, dy, dz, time_err, fast;
};

struct Params { /* mirrors tsi_params (include/tsi.h) field by field */
  int32_t localsubdiv;
  float delta;
  int32_t pointsample, fastenabled, lipschitz_corrected, swept_volume, fast_normals, normal_viz,
      rounding_mode;
  float fast_multiplier;
  int32_t scene_id;
  float octree_darken_factor;
  float root_lo[3], root_hi[3];
  int32_t pruning;
  float swept_dt;
  int32_t cinematic, samples, see_background;
};

struct Stats { /* subset of tsi_stats, same field order for the counters */
  uint64_t parents_expanded, cells_evaluated, cells_reverse, cells_skipped, cells_ambiguous,
      cells_empty, cells_full, cells_enqueued, cells_reused, instr_forward, instr_reverse;
  uint32_t levels;
  uint32_t pad;
};

struct Scene {
  std::vector<GInstr> tape;
  Params p;
  std::vector<Voxel> vox;
  std::vector<uint32_t> free_list;
};

uint32_t malloc_voxel(Scene &S) { /* compute.wgsl:3437-3450, zero normal (see header) */
  uint32_t a;
  if (!S.free_list.empty()) {
    a = S.free_list.back();
    S.free_list.pop_back();
  } else {
    a = (uint32_t)S.vox.size();
    S.vox.push_back(Voxel{});
  }
  Voxel &v = S.vox[a];
  v.child_count = 0;
  v.f = 1.0f;
  v.t = 0.0f;
  v.time_err = 0.0f;
  v.fast = 0.0f;
  v.dx = v.dy = v.dz = 0.0f;
  return a;
}

void free_subtree(Scene &S, uint32_t a) { /* compute.wgsl:3533-3543, 3452-3460 */
  std::vector<uint32_t> st{a};
  while (!st.empty()) {
    uint32_t v = st.back();
    st.pop_back();
    Voxel &x = S.vox[v];
    if (x.child_count != 0) {
      x.child_count = 0;
      for (int j = 0; j < 8; ++j) st.push_back(x.children[j]);
    }
    x.f = 0.0f;
    x.t = 0.0f;
    x.time_err = 0.0f;
    x.fast = 0.0f;
    S.free_list.push_back(v);
  }
}

void reset_scene(Scene &S) { /* main.rs:730-766 */
  S.vox.clear();
  S.free_list.clear();
  Voxel root{};
  root.x = I{S.p.root_lo[0], S.p.root_hi[0]};
  root.y = I{S.p.root_lo[1], S.p.root_hi[1]};
  root.z = I{S.p.root_lo[2], S.p.root_hi[2]};
  root.t = 0.0f;
  root.child_count = 0;
  root.f = 0.0f;
  S.vox.push_back(root);
}

inline float epsilon_of(int L) { return 10.0f * ldexpf(1.0f, -L); } /* compute.wgsl:3521 */

struct ChildResult {
  bool enqueue;
  bool dealloc;
  uint32_t dealloc_voxel;
  int cls;  // 0 amb, 1 empty, 2 full, 3 skipped
  bool reverse;
  bool reused;
  uint64_t instr;
};

/* one thread of `main` (compute.wgsl:3558-4047) for child k of parent P */
void process_child(Scene &S, uint32_t P, int k, bool new_voxel, float time, float t0, Scratch &sc,
                   ChildResult &r) {
  const Params &p = S.p;
  const float eps = epsilon_of(p.localsubdiv);
  const int lx = k & 1, ly = (k >> 1) & 1, lz = k >> 2;
  Voxel &par = S.vox[P];
  uint32_t C = par.children[k];
  const I px = par.x, py = par.y, pz = par.z;
  const float pfast = par.fast;
  Voxel &c = S.vox[C];
  float dx = DIAMETER(px) / 2.0f, dy = DIAMETER(py) / 2.0f, dz = DIAMETER(pz) / 2.0f;
  float width = of_max(dx, of_max(dy, dz));
  I cx = I{px.lo + dx * (float)lx, px.lo + dx * (float)(1 + lx)};
  I cy = I{py.lo + dy * (float)ly, py.lo + dy * (float)(1 + ly)};
  I cz = I{pz.lo + dz * (float)lz, pz.lo + dz * (float)(1 + lz)};
  c.x = cx;
  c.y = cy;
  c.z = cz;
  I cur_t;
  if (new_voxel || pfast == 1.0f || width <= eps) {
    if (p.swept_volume) cur_t = I{t0, time};
    else cur_t = IF(time);
    c.fast = 0.0f;
  } else {
    cur_t = I{c.t, time};
  }
  c.t = time;
  if (p.pointsample && width <= eps) {
    cx = IF(MID(cx));
    cy = IF(MID(cy));
    cz = IF(MID(cz));
    width = 0.0f;
  }
  r = ChildResult{false, false, 0, 3, false, false, 0};
  if (!(new_voxel || c.f >= 0.0f || c.child_count == 0u)) return;
  I args[4] = {cx, cy, cz, I_FROM_UNORDERED(cur_t.lo, cur_t.hi)};
  bool take_derivative = (cur_t.lo != cur_t.hi) || (p.fast_normals == 0 && p.normal_viz != 0);
  EvalOut o;
  eval_cell(S.tape.data(), (uint32_t)S.tape.size(), args, take_derivative, sc, o);
  r.instr = o.instr;
  r.reverse = take_derivative;
  I field = o.field;
  I df = IF(0.0f), df_dt = IF(0.0f);
  const float delta = p.delta;
  if (take_derivative) { /* compute.wgsl:3966-3997 */
    c.dx = MID(o.sens[0]);
    c.dy = MID(o.sens[1]);
    c.dz = MID(o.sens[2]);
    df_dt = o.sens[3];
    float dt = DIAMETER(args[3]);
    df = MUL_IF(df_dt, dt);
    I W = MUL_IF(I{-1.0f, 1.0f}, DIAMETER(field));
    df = CAP_II(df, W);
    if (p.lipschitz_corrected && ABS_I(df).hi != 0.0f) {
      float lb = ABS_I(SQRT_I(ADD_II(SQR_I(o.sens[0]), ADD_II(SQR_I(o.sens[1]), SQR_I(o.sens[2]))))).lo;
      if (!is_nan(lb)) df = DIV_IF(df, lb);
    }
    if (df.lo == -OF_INF || df.hi == OF_INF || is_nan(df.lo) || is_nan(df.hi)) df = IF(delta);
    float a = ABS_I(df).hi;
    c.time_err = c.time_err + of_min(of_max(a, 0.0f), delta);
  }
  if (!p.swept_volume && p.fastenabled) { /* compute.wgsl:4003-4009 */
    c.fast = (ABS_I(df).hi >= delta * p.fast_multiplier) ? 1.0f : 0.0f;
  }
  const float thick = 0.0f;
  if (I_CONTAINS_X(field, delta * thick)) { /* compute.wgsl:4011-4045 */
    c.f = 0.0f;
    r.cls = 0;
    if (width > eps) {
      if (new_voxel || is_nan(df_dt.lo) || is_nan(df_dt.hi) || fabsf(df_dt.lo) == OF_INF ||
          fabsf(df_dt.hi) == OF_INF || pfast == 1.0f || cur_t.lo == cur_t.hi ||
          c.time_err >= delta || c.child_count == 0u) {
        c.time_err = 0.0f;
        r.enqueue = true;
      } else {
        r.reused = true;
      }
    }
  } else {
    if (field.hi <= delta * thick) {
      c.f = -1.0f;
      r.cls = 2;
    } else {
      r.cls = 1;
      if (!p.swept_volume) c.f = 1.0f;
    }
    if (!p.swept_volume && c.child_count != 0u) {
      c.child_count = 0;
      r.dealloc = true;
      r.dealloc_voxel = C;
    }
  }
}

/* one frame of `main`, level by level (compute.wgsl:3525-4056) */
void invert(Scene &S, float time, float t0_or_nan, Stats &st) {
  memset(&st, 0, sizeof(st));
  float t0 = (t0_or_nan != t0_or_nan) ? time - S.p.swept_dt : t0_or_nan;
  std::vector<uint32_t> cur{0}; /* buf_main: enqueue(0) */
  std::vector<uint32_t> dealloc_roots;
  while (!cur.empty()) {
    st.levels++;
    st.parents_expanded += cur.size();
    std::vector<uint8_t> is_new(cur.size());
    for (size_t i = 0; i < cur.size(); ++i) { /* mallocV x8 for new parents, 3564-3577 */
      uint32_t P = cur[i];
      is_new[i] = S.vox[P].child_count == 0u;
      if (is_new[i]) {
        uint32_t kids[8];
        for (int j = 0; j < 8; ++j) kids[j] = malloc_voxel(S);
        Voxel &par = S.vox[P];
        for (int j = 0; j < 8; ++j) par.children[j] = kids[j];
      }
      S.vox[P].child_count = 1u; /* 3579 */
    }
    const size_t n = cur.size();
    std::vector<ChildResult> res(n * 8);
#pragma omp parallel
    {
      Scratch sc;
#pragma omp for schedule(dynamic, 16)
      for (long long i = 0; i < (long long)n; ++i)
        for (int k = 0; k < 8; ++k) process_child(S, cur[i], k, is_new[i] != 0, time, t0, sc, res[i * 8 + k]);
    }
    std::vector<uint32_t> next;
    for (size_t i = 0; i < n; ++i) {
      for (int k = 0; k < 8; ++k) {
        const ChildResult &r = res[i * 8 + k];
        uint32_t C = S.vox[cur[i]].children[k];
        if (r.cls == 3) {
          st.cells_skipped++;
          continue;
        }
        st.cells_evaluated++;
        st.instr_forward += r.instr;
        if (r.reverse) {
          st.cells_reverse++;
          st.instr_reverse += r.instr;
        }
        if (r.cls == 0) st.cells_ambiguous++;
        else if (r.cls == 1) st.cells_empty++;
        else st.cells_full++;
        if (r.enqueue) {
          st.cells_enqueued++;
          next.push_back(C);
        }
        if (r.reused) st.cells_reused++;
        if (r.dealloc) {
          const Voxel &v = S.vox[C];
          for (int j = 0; j < 8; ++j) dealloc_roots.push_back(v.children[j]);
        }
      }
    }
    cur.swap(next);
  }
  for (uint32_t v : dealloc_roots) free_subtree(S, v);
}

/* ---------- trace (compute.wgsl:4059-4403) ---------- */
struct V3 {
  float x, y, z;
};
inline V3 v3(float a, float b, float c) { return V3{a, b, c}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 muls(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 divv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 rcp(V3 a) { return v3(1.0f / a.x, 1.0f / a.y, 1.0f / a.z); }
inline float len3(V3 a) { return sqrtf((a.x * a.x + a.y * a.y) + a.z * a.z); }
inline float sgn(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

inline V3 efficient_slabs(V3 p0, V3 p1, V3 ro, V3 inv) { /* 4059-4070 */
  V3 t0 = mul(sub(p0, ro), inv), t1 = mul(sub(p1, ro), inv);
  V3 tmin = v3(of_min(t0.x, t1.x), of_min(t0.y, t1.y), of_min(t0.z, t1.z));
  V3 tmax = v3(of_max(t0.x, t1.x), of_max(t0.y, t1.y), of_max(t0.z, t1.z));
  float d1 = of_max(tmin.x, of_max(tmin.y, tmin.z));
  float d2 = of_min(tmax.x, of_min(tmax.y, tmax.z));
  return v3((d1 <= d2 && d2 >= 0.0f) ? 1.0f : 0.0f, of_max(d1, 0.0f), of_max(d2, 0.0f));
}

struct TraceOut {
  V3 c;
  float d;
  V3 n;
  uint32_t visits;
};

const float TEPS = 0.0001f; /* compute.wgsl:4141 */

/* finite_diff_normal (compute.wgsl:4143-4184) for any tape: the tetrahedron
   of points p + k h, h = 0.01, k in {(1,-1,-1), (-1,-1,1), (-1,1,-1),
   (1,1,1)}, with f evaluated by the tape on point boxes, normalised as
   v / |v| (the reference pastes a per-scene function here). */
V3 tape_normal(const Scene &S, V3 p, float t) {
  static thread_local Scratch sc;
  const float h = 0.01f;
  const float kx[4] = {1.0f, -1.0f, -1.0f, 1.0f}, ky[4] = {-1.0f, -1.0f, 1.0f, 1.0f};
  const float kz[4] = {-1.0f, 1.0f, -1.0f, 1.0f};
  float f[4];
  for (int q = 0; q < 4; ++q) {
    const float ax = p.x + kx[q] * h, ay = p.y + ky[q] * h, az = p.z + kz[q] * h;
    const I args[4] = {{ax, ax}, {ay, ay}, {az, az}, {t, t}};
    EvalOut o;
    eval_cell(S.tape.data(), (uint32_t)S.tape.size(), args, false, sc, o);
    f[q] = o.field.lo;
  }
  V3 v = v3(kx[0] * f[0], ky[0] * f[0], kz[0] * f[0]);
  for (int q = 1; q < 4; ++q) v = add(v, v3(kx[q] * f[q], ky[q] * f[q], kz[q] * f[q]));
  const float l = len3(v);
  return v3(v.x / l, v.y / l, v.z / l);
}

void trace(const Scene &S, V3 ro, V3 rd, float time, TraceOut &out) { /* 4189-4403 */
  const Params &p = S.p;
  uint32_t stack[32];
  uint32_t sp = 0;
  V3 normal_at_hit = v3(0, 0, 0);
  V3 ro2 = ro;
  V3 c = v3(1, 1, 1);
  out.visits = 0;
  stack[sp++] = 0; /* push(0) */
  bool intersected = false;
  uint32_t region = stack[sp - 1];
  const Voxel *vx = S.vox.data();
  V3 p0 = v3(vx[region].x.lo, vx[region].y.lo, vx[region].z.lo);
  V3 p1 = v3(vx[region].x.hi, vx[region].y.hi, vx[region].z.hi);
  V3 hit = efficient_slabs(p0, p1, ro2, rcp(rd));
  if (hit.x == 0.0f) {
    out.c = c;
    out.d = -1.0f;
    out.n = normal_at_hit;
    return;
  }
  float spheremarchstep = 0.0f;
  for (uint32_t iter = 0; iter < 5000u; ++iter) {
    if (intersected) break;
    if (sp == 0) {
      out.c = c;
      out.d = -1.0f;
      out.n = normal_at_hit;
      return;
    }
    region = stack[--sp];
    if (hit.x == 0.0f) {
      if (sp == 0) continue; /* peak() of an empty stack: the next pass returns */
      uint32_t top = stack[sp - 1];
      p0 = v3(vx[top].x.lo, vx[top].y.lo, vx[top].z.lo);
      p1 = v3(vx[top].x.hi, vx[top].y.hi, vx[top].z.hi);
      hit = efficient_slabs(p0, p1, ro2, rcp(rd));
      continue;
    }
    V3 ro_l = divv(muls(sub(add(ro2, muls(rd, hit.y + TEPS)), p0), 2.0f), sub(p1, p0));
    V3 rd_l = mul(rd, divv(v3(2.0f, 2.0f, 2.0f), sub(p1, p0)));
    int mp[3] = {(int)floorf(ro_l.x), (int)floorf(ro_l.y), (int)floorf(ro_l.z)};
    V3 dd = rcp(v3(fabsf(rd_l.x), fabsf(rd_l.y), fabsf(rd_l.z)));
    float sg[3] = {sgn(rd_l.x), sgn(rd_l.y), sgn(rd_l.z)};
    int step[3] = {(int)sg[0], (int)sg[1], (int)sg[2]};
    float rol[3] = {ro_l.x, ro_l.y, ro_l.z};
    float ddv[3] = {dd.x, dd.y, dd.z};
    float sd[3];
    for (int a = 0; a < 3; ++a) sd[a] = ((sg[a] * ((float)mp[a] - rol[a]) + sg[a] * 0.5f) + 0.5f) * ddv[a];
    float mask[3] = {0, 0, 0};
    V3 old_ro2 = ro2;
    for (int i = 0; i < 32; ++i) {
      if (!p.normal_viz) {
        float ext = of_max(p1.x - p0.x, of_max(p1.y - p0.y, p1.z - p0.z));
        if (ext < 1.0f) c = muls(c, p.octree_darken_factor);
      }
      V3 mv = v3(mask[0] * (sd[0] - ddv[0]), mask[1] * (sd[1] - ddv[1]), mask[2] * (sd[2] - ddv[2]));
      float t = (len3(mv) + hit.y + TEPS) + spheremarchstep;
      ro2 = add(old_ro2, muls(rd, t));
      spheremarchstep = 0.0f;
      if (t >= hit.z - TEPS) { /* 4277-4292 */
        ro2 = add(old_ro2, muls(rd, hit.z));
        if (sp == 0) {
          hit = v3(0, 0, 0);
          break;
        }
        uint32_t top = stack[sp - 1];
        p0 = v3(vx[top].x.lo, vx[top].y.lo, vx[top].z.lo);
        p1 = v3(vx[top].x.hi, vx[top].y.hi, vx[top].z.hi);
        hit = efficient_slabs(p0, p1, ro2, rcp(rd));
        break;
      }
      int ci = mp[0] + 2 * mp[1] + 4 * mp[2];
      if (ci < 0 || ci >= 8) break;
      /* a node without children has no valid children[] (guarded; only a
         trace before the first inversion reaches it) */
      const bool has = vx[region].child_count != 0u;
      uint32_t child = has ? vx[region].children[ci] : region;
      if (has) out.visits++;
      const Voxel &cv = vx[child];
      if (has && cv.f <= 0.0f) {
        V3 tp0 = v3(cv.x.lo - TEPS, cv.y.lo - TEPS, cv.z.lo - TEPS);
        V3 tp1 = v3(cv.x.hi + TEPS, cv.y.hi + TEPS, cv.z.hi + TEPS);
        V3 th = efficient_slabs(tp0, tp1, ro2, rcp(rd));
        if (th.x == 1.0f) {
          if (cv.child_count != 0u) {
            if (sp < 32) stack[sp++] = region;
            if (sp < 32) stack[sp++] = child;
            p0 = tp0;
            p1 = tp1;
            hit = th;
            break;
          } else {
            intersected = true;
            normal_at_hit = v3(cv.dx, cv.dy, cv.dz);
            if (p.fast_normals) /* 4337-4342 */
              normal_at_hit = tape_normal(S, ro2, p.swept_volume ? vx[region].t : time);
            float timesince = time - cv.t;
            V3 movement = v3(1.0f, 0.0f, 0.0f);
            V3 base = v3(1.0f, 1.0f, 1.0f);
            if (p.normal_viz) {
              float nl = len3(normal_at_hit);
              V3 nv = v3(normal_at_hit.x / nl, normal_at_hit.y / nl, normal_at_hit.z / nl);
              c = add(muls(nv, 0.5f), v3(0.5f, 0.5f, 0.5f));
            } else {
              float tt = of_min(of_max(timesince * 60.0f, 0.0f), 1.0f);
              V3 a = sub(v3(1, 1, 1), movement), b = sub(v3(1, 1, 1), base);
              V3 lerp = v3(a.x * (1.0f - tt) + b.x * tt, a.y * (1.0f - tt) + b.y * tt, a.z * (1.0f - tt) + b.z * tt);
              c = sub(c, lerp);
            }
            break;
          }
        }
      }
      /* 4389-4391 */
      float m0 = (sd[0] <= of_min(sd[1], sd[2])) ? 1.0f : 0.0f;
      float m1 = (sd[1] <= of_min(sd[2], sd[0])) ? 1.0f : 0.0f;
      float m2 = (sd[2] <= of_min(sd[0], sd[1])) ? 1.0f : 0.0f;
      mask[0] = m0;
      mask[1] = m1;
      mask[2] = m2;
      for (int a = 0; a < 3; ++a) {
        sd[a] = sd[a] + mask[a] * ddv[a];
        mp[a] = mp[a] + (int)mask[a] * step[a];
      }
    }
  }
  c = v3(of_max(of_min(c.x, 1.0f), 0.0f), of_max(of_min(c.y, 1.0f), 0.0f), of_max(of_min(c.z, 1.0f), 0.0f));
  float dist = fabsf(len3(sub(ro2, ro)));
  if (!intersected) dist = -1.0f;
  out.c = c;
  out.d = dist;
  out.n = normal_at_hit;
}

struct Uniforms { /* uniforms.rs:8-17 */
  float view[16];
  uint32_t res[2];
  float time, lasttime, rendermode, pad[3];
};

struct Camera {
  V3 eye;
  float m[16]; /* view matrix after the scene rotation, column major */
  float zdist;
  float yshift;
};

void rotation_matrix(V3 axis, float angle, float out[16]) { /* compute.wgsl:4525-4588 */
  float l = len3(axis);
  axis = v3(axis.x / l, axis.y / l, axis.z / l);
  float s = sinf(angle), c = cosf(angle), oc = 1.0f - c;
  float m[16] = {oc * axis.x * axis.x + c, oc * axis.x * axis.y - axis.z * s, oc * axis.z * axis.x + axis.y * s, 0.0f,
                 oc * axis.x * axis.y + axis.z * s, oc * axis.y * axis.y + c, oc * axis.y * axis.z - axis.x * s, 0.0f,
                 oc * axis.z * axis.x - axis.y * s, oc * axis.y * axis.z + axis.x * s, oc * axis.z * axis.z + c, 0.0f,
                 0.0f, 0.0f, 0.0f, 1.0f};
  memcpy(out, m, sizeof(m));
}

void matmul4(const float a[16], const float b[16], float out[16]) { /* column major a*b */
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

void make_camera(const Params &p, const Uniforms &u, Camera &cam) { /* rt_main 4651-4685 */
  float view[16];
  memcpy(view, u.view, sizeof(view));
  V3 eye = v3(view[12], view[13], view[14]);
  const float PI = PI_F;
  if (p.scene_id == 3) {
    eye = add(eye, v3(7.7f, -2.21f, 7.7f));
    float r[16];
    rotation_matrix(v3(0.0f, 1.0f, 0.0f), (PI / 4.0f) * 3.0f, r);
    matmul4(r, view, view);
  } else if (p.scene_id == 4) {
    eye = add(eye, v3(0.0f, -0.78f, -7.0f));
  } else if (p.scene_id == 5) {
    eye = add(eye, v3(7.13f, 2.14f, -5.6f));
    float r[16];
    rotation_matrix(v3(0.0f, 1.0f, 0.0f), PI / 4.0f, r);
    matmul4(r, view, view);
    rotation_matrix(v3(-1.0f, 0.0f, -1.0f), (PI / 4.0f) * 0.45f, r);
    matmul4(r, view, view);
  }
  cam.eye = eye;
  memcpy(cam.m, view, sizeof(view));
  const float fov = 90.0f;
  float rad = fov * 0.017453292519943295474f; /* radians(), 2431-2433 */
  cam.zdist = (float)u.res[1] / tanf(rad / 2.0f);
  cam.yshift = (p.scene_id == 0) ? (float)u.res[1] * 0.32f : 0.0f;
}

V3 primary_ray(const Camera &cam, const Uniforms &u, uint32_t px, uint32_t py) { /* 4590-4631 */
  float pxf = (float)px, pyf = (float)py;
  pyf = pyf - cam.yshift;
  float xy0 = (pxf - (float)u.res[0] / 2.0f) + 0.5f;
  float xy1 = (pyf - (float)u.res[1] / 2.0f) + 0.5f;
  V3 d = v3(xy0, -xy1, -cam.zdist);
  float l = len3(d);
  d = v3(d.x / l, d.y / l, d.z / l);
  V3 g;
  /* view * vec4(d, 0.0), summed column by column */
  g.x = ((cam.m[0] * d.x + cam.m[4] * d.y) + cam.m[8] * d.z) + cam.m[12] * 0.0f;
  g.y = ((cam.m[1] * d.x + cam.m[5] * d.y) + cam.m[9] * d.z) + cam.m[13] * 0.0f;
  g.z = ((cam.m[2] * d.x + cam.m[6] * d.y) + cam.m[10] * d.z) + cam.m[14] * 0.0f;
  return g;
}

/* ---------------- cinematic path tracing ----------------
   rt_main with `cinematic` on (compute.wgsl:3499): per pixel, `samples`
   jittered rays (get_color_supersample 4620-4648), each a two-bounce path
   (get_color_single 4444-4523): at a hit the path continues in a
   cosine-power lobe around the normal (getSampleBiased 4429-4438), and a
   shadow ray towards a jittered sun direction adds sun light and a specular
   highlight when it escapes; a path that escapes sees the sky (sunsky
   520-677).  Random numbers: the PCG hash of frand / frand0to1
   (2451-2472) on the per-pixel seed of rt_main (4664). */
inline uint32_t pcg_word(uint32_t s) {
  uint32_t w = ((s >> ((s >> 28u) + 4u)) ^ s) * 277803737u;
  return (w >> 22u) ^ w;
}
inline float frand(uint32_t &seed) { /* -1 to 1 */
  seed = seed * 747796405u + 1u;
  return ((float)pcg_word(seed) / 4294967295.0f) * 2.0f - 1.0f;
}
inline float frand0to1(uint32_t &seed) {
  seed = seed * 747796405u + 1u;
  return (float)pcg_word(seed) / 4294967295.0f;
}
inline float dot3(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
inline V3 normalize3(V3 a) {
  const float l = len3(a);
  return v3(a.x / l, a.y / l, a.z / l);
}
inline V3 cross3(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline float clampf(float x, float lo, float hi) { return of_min(of_max(x, lo), hi); }
inline V3 exp3(V3 a) { return v3(of_exp(a.x), of_exp(a.y), of_exp(a.z)); }
inline V3 pow3(V3 a, V3 b) { return v3(of_powf(a.x, b.x), of_powf(a.y, b.y), of_powf(a.z, b.z)); }

V3 from_spherical(float px, float py) { /* 497-518 */
  return v3(of_cos(px) * of_sin(py), of_sin(px) * of_sin(py), of_cos(py));
}

V3 ortho(V3 v) { /* 4405-4427 */
  if (fabsf(v.x) > fabsf(v.z)) return v3(-v.y, v.x, 0.0f);
  return v3(0.0f, -v.z, v.y);
}

V3 sample_biased(V3 d, float power, uint32_t &seed) { /* getSampleBiased 4429-4438 */
  const V3 dir = normalize3(d);
  const V3 o1 = normalize3(ortho(dir));
  const V3 o2 = normalize3(cross3(dir, o1));
  float rx = frand0to1(seed);
  float ry = frand0to1(seed);
  rx = (rx * 2.0f) * PI_F;
  ry = of_powf(ry, 1.0f / (power + 1.0f));
  const float oneminus = sqrtf(1.0f - ry * ry);
  return add(add(muls(o1, of_cos(rx) * oneminus), muls(o2, of_sin(rx) * oneminus)), muls(dir, ry));
}

/* sunsky (520-677) with turbidity 1, sunSize 1, sky sun intensity 1000 (the
   private globals of 421-427); it returns 0.01 * sky (the sun disk term is
   computed there but not added).  pow with the constant exponent 2.0 is
   x * x, the rewrite shader compilers apply (Mesa's NIR among them); it is
   defined for the negative cosines between view and sun, where the
   exp(2 log x) form has no value. */
V3 sunsky(V3 view, float spx, float spy) {
  const float pi = 3.1415927410125732f;
  const float sun_cos = of_cos((1.0f * pi) / 180.0f);
  const V3 sun_dir = normalize3(from_spherical((spx - 0.0f) * 6.28000020980835f, (spy - 0.5f) * 3.140000104904175f));
  const float cos_view_sun = dot3(view, sun_dir);
  const float cos_sun_up = dot3(sun_dir, v3(0.0f, 0.0f, 1.0f));
  const float cos_up_view = dot3(v3(0.0f, 0.0f, 1.0f), view);
  if (sun_cos == 1.0f) return v3(1.0f, 0.0f, 0.0f);
  /* SunIntensity 482-495 */
  const float sunE = 1000.0f * of_max(0.0f, 1.0f - of_exp(-((1.6110731611233942f - of_acos(cos_sun_up)) / 1.5f)));
  const V3 rayleigh = v3(5.176821105123963e-6f, 1.2785348189936485e-5f, 2.8530756026157178e-5f);
  /* totalMie 438-456, T = 1 */
  const float c = (0.20000000298023224f * 1.0f) * 9.99999983775159e-18f;
  const V3 lambda = v3(6.800000278417428e-7f, 5.499999815583578e-7f, 4.4999998749517545e-7f);
  const V3 K = v3(0.6859999895095825f, 0.6779999732971191f, 0.6660000085830688f);
  const float two_pi = 2.0f * 3.1415927410125732f;
  const V3 q = divv(v3(two_pi, two_pi, two_pi), lambda); /* pow(q, vec3(4.0 - 2.0)) = q * q */
  const V3 tm = mul(muls(mul(q, q), (0.4339999854564667f * c) * 3.1415927410125732f), K);
  const V3 mie = muls(tm, 0.004999999888241291f);
  const float zenith = of_max(0.0f, cos_up_view);
  const float r_len = 8400.0f / zenith, m_len = 1250.0f / zenith;
  const V3 fex = exp3(v3(-(rayleigh.x * r_len + mie.x * m_len), -(rayleigh.y * r_len + mie.y * m_len),
                         -(rayleigh.z * r_len + mie.z * m_len)));
  /* RayleighPhase 429-436, hgPhase 458-480 */
  const float rphase = (3.0f / (16.0f * 3.1415927410125732f)) * (1.0f + (cos_view_sun * cos_view_sun));
  const float g = 0.800000011920929f;
  const float hg = (1.0f / (4.0f * 3.1415927410125732f)) *
                   ((1.0f - (g * g)) / of_powf((1.0f - (2.0f * g) * cos_view_sun) + (g * g), 1.5f));
  const V3 r_eye = muls(rayleigh, rphase), m_eye = muls(mie, hg);
  const V3 total = add(rayleigh, mie), light = add(r_eye, m_eye);
  const V3 se = muls(divv(light, total), sunE);
  V3 sky = mul(se, sub(v3(1.0f, 1.0f, 1.0f), fex));
  const float t = clampf(of_powf(1.0f - dot3(v3(0.0f, 0.0f, 1.0f), sun_dir), 5.0f), 0.0f, 1.0f);
  const V3 pw = pow3(mul(se, fex), v3(0.5f, 0.5f, 0.5f));
  /* mix(1, pw, t) = 1 (1 - t) + pw t */
  const V3 mx = v3(1.0f * (1.0f - t) + pw.x * t, 1.0f * (1.0f - t) + pw.y * t, 1.0f * (1.0f - t) + pw.z * t);
  sky = mul(sky, mx);
  return muls(sky, 0.009999999776482582f);
}

struct CineOut {
  float r, g, b, a;
};

/* get_color_single, cinematic (4444-4523) */
CineOut color_single(const Scene &S, V3 ro, V3 rd, float time, uint32_t &seed, float *d0, V3 *n0) {
  V3 frm = ro, dir = rd;
  V3 lum = v3(1.0f, 1.0f, 1.0f), direct = v3(0.0f, 0.0f, 0.0f);
  float spx = -0.1f, spy = 0.7f, sun_int = 3.0f, spec_int = 1.0f, albedo = 1.0f, sunsize = 0.01f, bg = 1.0f;
  if (S.p.scene_id == 3) {
    spx = 0.36f;
    spy = 0.72f;
    spec_int = 1.0f;
    sunsize = 0.1f;
    albedo = 1.5f;
    bg = 2.0f;
    sun_int = 2.0f;
  } else if (S.p.scene_id == 4) {
    spx = -0.1f;
    spy = 0.57f;
    sunsize = 0.01f;
  } else if (S.p.scene_id == 5) {
    spx = 0.63f;
    spy = 0.65f;
    sunsize = 0.02f;
  }
  for (int i = 0; i < 2; ++i) {
    TraceOut tr;
    trace(S, frm, dir, time, tr);
    if (i == 0) {
      *d0 = tr.d;
      *n0 = tr.n;
    }
    const V3 n = tr.n;
    const V3 hitpoint = add(frm, muls(dir, tr.d));
    if (tr.d >= 0.0f) {
      const V3 old = dir;
      dir = sample_biased(n, 3.0f, seed);
      lum = muls(mul(lum, tr.c), albedo);
      frm = add(hitpoint, muls(n, 0.05f));
      const V3 sd = normalize3(from_spherical((spx - 0.0f) * 6.28f, (spy - 0.5f) * 3.14f));
      const V3 sundir = v3(sd.x, sd.z, sd.y);
      const float jx = frand(seed), jy = frand(seed), jz = frand(seed);
      const V3 sample_dir = normalize3(add(sundir, muls(v3(jx, jy, jz), sunsize)));
      const float sunlight = dot3(n, sample_dir);
      TraceOut sh;
      trace(S, frm, sample_dir, time, sh);
      if (sunlight > 0.0f && sh.d < 0.0f) {
        direct = add(direct, muls(muls(lum, sunlight), sun_int));
        const V3 half = normalize3(add(v3(-old.x, -old.y, -old.z), sundir));
        const float spec = (100.0f * of_powf(of_max(dot3(n, half), 0.0f), 30.0f)) * spec_int;
        direct = add(direct, muls(lum, spec));
      }
    } else {
      if (i == 0 && !S.p.see_background) return CineOut{10.0f, 10.0f, 10.0f, 0.0f};
      const V3 sky = sunsky(v3(dir.x, dir.z, dir.y), spx, spy); /* getBackground 4440-4442 */
      const V3 c = add(direct, mul(lum, sky));
      return CineOut{c.x * bg, c.y * bg, c.z * bg, 1.0f * bg};
    }
  }
  return CineOut{direct.x, direct.y, direct.z, 1.0f};
}

/* primary ray through the (possibly jittered) pixel position (px, py),
   py already shifted for scene 0 (4590-4594, 4629-4631) */
V3 primary_ray_at(const Camera &cam, const Uniforms &u, float pxf, float pyf) {
  float xy0 = (pxf - (float)u.res[0] / 2.0f) + 0.5f;
  float xy1 = (pyf - (float)u.res[1] / 2.0f) + 0.5f;
  V3 d = v3(xy0, -xy1, -cam.zdist);
  float l = len3(d);
  d = v3(d.x / l, d.y / l, d.z / l);
  V3 g;
  g.x = ((cam.m[0] * d.x + cam.m[4] * d.y) + cam.m[8] * d.z) + cam.m[12] * 0.0f;
  g.y = ((cam.m[1] * d.x + cam.m[5] * d.y) + cam.m[9] * d.z) + cam.m[13] * 0.0f;
  g.z = ((cam.m[2] * d.x + cam.m[6] * d.y) + cam.m[10] * d.z) + cam.m[14] * 0.0f;
  return g;
}

/* LinearToSRGB (4600-4607) of one channel */
inline float linear_to_srgb(float x) {
  const float rgb = clampf(x, 0.0f, 1.0f);
  const float m = (rgb < 0.0031308f) ? 1.0f : 0.0f;
  const float a = of_powf(rgb, 1.0f / 2.4f) * 1.055f - 0.055f;
  const float b = rgb * 12.92f;
  return a * (1.0f - m) + b * m;
}

}  // namespace

/* ---------------- extern "C" API used by tests and bench ---------------- */
extern "C" {

struct OracleScene;

int oracle_eval_boxes(const void *instr, uint32_t count, uint32_t n, const float *boxes, int reverse,
                      float *out) {
  const GInstr *tape = (const GInstr *)instr;
  if (count < 4) return 1;
#pragma omp parallel
  {
    Scratch sc;
#pragma omp for schedule(static)
    for (long long i = 0; i < (long long)n; ++i) {
      const float *b = boxes + i * 8;
      I args[4] = {I{b[0], b[1]}, I{b[2], b[3]}, I{b[4], b[5]}, I{b[6], b[7]}};
      EvalOut o;
      eval_cell(tape, count, args, reverse != 0, sc, o);
      float *w = out + i * 10;
      w[0] = o.field.lo;
      w[1] = o.field.hi;
      for (int k = 0; k < 4; ++k) {
        w[2 + 2 * k] = reverse ? o.sens[k].lo : 0.0f;
        w[3 + 2 * k] = reverse ? o.sens[k].hi : 0.0f;
      }
    }
  }
  return 0;
}

void *oracle_scene_create(const void *instr, uint32_t count, const void *params) {
  Scene *S = new Scene();
  const GInstr *g = (const GInstr *)instr;
  S->tape.assign(g, g + count);
  memcpy(&S->p, params, sizeof(Params));
  reset_scene(*S);
  return S;
}

void oracle_scene_destroy(void *s) { delete (Scene *)s; }
void oracle_scene_reset(void *s) { reset_scene(*(Scene *)s); }

int oracle_scene_invert(void *s, float time, float t0_or_nan, void *stats) {
  Stats st;
  invert(*(Scene *)s, time, t0_or_nan, st);
  if (stats) memcpy(stats, &st, sizeof(st));
  return 0;
}

uint64_t oracle_scene_voxels_live(void *s) {
  Scene *S = (Scene *)s;
  return S->vox.size() - S->free_list.size();
}

/* cells in depth-first order keyed (level, ix, iy, iz); layout = tsi_cell */
struct OCell {
  uint32_t level, ix, iy, iz;
  float f, t, time_err, fast, dx, dy, dz;
  uint32_t has_children;
  float x[2], y[2], z[2];
};

uint64_t oracle_scene_cells(void *s, void *out, uint64_t cap) {
  Scene *S = (Scene *)s;
  OCell *o = (OCell *)out;
  uint64_t n = 0;
  struct E {
    uint32_t v, level, ix, iy, iz;
  };
  std::vector<E> st{{0, 0, 0, 0, 0}};
  while (!st.empty()) {
    E e = st.back();
    st.pop_back();
    const Voxel &v = S->vox[e.v];
    if (o && n < cap) {
      OCell c;
      c.level = e.level;
      c.ix = e.ix;
      c.iy = e.iy;
      c.iz = e.iz;
      c.f = v.f;
      c.t = v.t;
      c.time_err = v.time_err;
      c.fast = v.fast;
      c.dx = v.dx;
      c.dy = v.dy;
      c.dz = v.dz;
      c.has_children = v.child_count != 0;
      c.x[0] = v.x.lo; c.x[1] = v.x.hi;
      c.y[0] = v.y.lo; c.y[1] = v.y.hi;
      c.z[0] = v.z.lo; c.z[1] = v.z.hi;
      o[n] = c;
    }
    ++n;
    if (v.child_count != 0) {
      for (int k = 7; k >= 0; --k)
        st.push_back(E{v.children[k], e.level + 1, 2 * e.ix + (k & 1), 2 * e.iy + ((k >> 1) & 1), 2 * e.iz + (k >> 2)});
    }
  }
  return n;
}

/* rt_main over the whole image (compute.wgsl:4651-4688); rgba, depth,
 * normal may be NULL.  Rows [y0, y1) only, for bounded samples. */
int oracle_scene_trace(void *s, const void *uniforms, float *rgba, float *depth, float *normal, uint32_t y0,
                       uint32_t y1, uint64_t *visits) {
  Scene *S = (Scene *)s;
  const Uniforms &u = *(const Uniforms *)uniforms;
  Camera cam;
  make_camera(S->p, u, cam);
  const uint32_t W = u.res[0], H = u.res[1];
  if (y1 > H) y1 = H;
  uint64_t vis = 0;
  if (S->p.cinematic) { /* get_color_supersample 4620-4648 with cinematic on */
    const int samples = S->p.samples > 0 ? S->p.samples : 1;
    const uint32_t seed0 = (uint32_t)(12345.0f * (of_sin(u.time * 12345.0f) * 0.5f + 0.5f)); /* 4664 */
#pragma omp parallel for schedule(dynamic, 4)
    for (long long yy = y0; yy < (long long)y1; ++yy) {
      for (uint32_t x = 0; x < W; ++x) {
        const uint64_t i = (uint64_t)yy * W + x;
        uint32_t seed = (uint32_t)i + seed0;
        float cr = 0.0f, cg = 0.0f, cb = 0.0f, ca = 0.0f, d0 = -1.0f;
        V3 n0 = v3(0, 0, 0);
        for (int smp = 0; smp < samples; ++smp) {
          const float ox = frand(seed), oy = frand(seed);
          const float pxf = (float)x + (ox * 1.0f) * 0.5f;
          const float pyf = ((float)yy - cam.yshift) + (oy * 1.0f) * 0.5f;
          const V3 rd = primary_ray_at(cam, u, pxf, pyf);
          if (u.rendermode == 0.0f) {
            float dd = -1.0f;
            V3 nn = v3(0, 0, 0);
            const CineOut o = color_single(*S, cam.eye, rd, u.time, seed, &dd, &nn);
            cr = cr + o.r;
            cg = cg + o.g;
            cb = cb + o.b;
            ca = ca + o.a;
            if (smp == 0) {
              d0 = dd;
              n0 = nn;
            }
          }
        }
        const float fs = (float)samples;
        cr = cr / fs;
        cg = cg / fs;
        cb = cb / fs;
        ca = ca / fs;
        cr = linear_to_srgb(cr);
        cg = linear_to_srgb(cg);
        cb = linear_to_srgb(cb);
        if (rgba) {
          rgba[i * 4 + 0] = of_powf(cr, 0.45f);
          rgba[i * 4 + 1] = of_powf(cg, 0.45f);
          rgba[i * 4 + 2] = of_powf(cb, 0.45f);
          rgba[i * 4 + 3] = ca;
        }
        if (depth) depth[i] = d0;
        if (normal) {
          normal[i * 3 + 0] = n0.x;
          normal[i * 3 + 1] = n0.y;
          normal[i * 3 + 2] = n0.z;
        }
      }
    }
    if (visits) *visits = 0;
    return 0;
  }
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : vis)
  for (long long yy = y0; yy < (long long)y1; ++yy) {
    for (uint32_t x = 0; x < W; ++x) {
      uint64_t i = (uint64_t)yy * W + x;
      V3 rd = primary_ray(cam, u, x, (uint32_t)yy);
      TraceOut t;
      float cr = 0, cg = 0, cb = 0, ca = 0;
      if (u.rendermode == 0.0f) {
        trace(*S, cam.eye, rd, u.time, t);
        vis += t.visits;
        /* get_color_single, non-cinematic (4481-4516): colour with alpha 1 */
        cr = t.c.x;
        cg = t.c.y;
        cb = t.c.z;
        ca = 1.0f;
        if (S->p.normal_viz && t.d < 0.0f) {
          cr = cg = cb = 10.0f;
          ca = 0.0f;
        }
      } else {
        t.d = -1.0f;
        t.n = v3(0, 0, 0);
      }
      /* gamma, 4643-4645 */
      if (rgba) {
        rgba[i * 4 + 0] = of_powf(cr, 0.45f);
        rgba[i * 4 + 1] = of_powf(cg, 0.45f);
        rgba[i * 4 + 2] = of_powf(cb, 0.45f);
        rgba[i * 4 + 3] = ca;
      }
      if (depth) depth[i] = t.d;
      if (normal) {
        normal[i * 3 + 0] = t.n.x;
        normal[i * 3 + 1] = t.n.y;
        normal[i * 3 + 2] = t.n.z;
      }
    }
  }
  if (visits) *visits = vis;
  return 0;
}

/* cinematic pieces under test: the frand sequence, the sky, sRGB */
void oracle_frand_seq(uint32_t seed, uint32_t n, float *out) {
  for (uint32_t i = 0; i < n; ++i) out[i] = (i & 1u) ? frand0to1(seed) : frand(seed);
}
void oracle_sunsky(const float *view, float spx, float spy, float *out) {
  const V3 s = sunsky(v3(view[0], view[1], view[2]), spx, spy);
  out[0] = s.x;
  out[1] = s.y;
  out[2] = s.z;
}
float oracle_linear_to_srgb(float x) { return linear_to_srgb(x); }
float oracle_cos(float x) { return of_cos(x); }
float oracle_acos(float x) { return of_acos(x); }

/* f32 math under test */
float oracle_sin(float x) { return of_sin(x); }
float oracle_exp(float x) { return of_exp(x); }
float oracle_log(float x) { return of_log(x); }
float oracle_atan2(float y, float x) { return of_atan2(y, x); }
float oracle_powi(float x, int n) { return of_powi(x, n); }
float oracle_fmin(float a, float b) { return of_min(a, b); }
float oracle_fmax(float a, float b) { return of_max(a, b); }

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void oracle_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
