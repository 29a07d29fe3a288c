// fmath.cuh — f32 elementary functions for the interval kernels.
//
// compute.wgsl relies on WGSL built-ins (sin, exp, log, atan2, pow at
// compute.wgsl:2577-2581, 2753-2800, 2838-2853, 2947-2953) whose accuracy the
// WGSL spec only bounds.  The library fixes each one as a sequence of
// correctly rounded f32 operations (explicit __f*_rn intrinsics, so nothing
// contracts into FMA), which makes results reproducible bit for bit on any
// CPU that performs the same IEEE operations.  Methods:
//   sin  : Cody & Waite (1980) three-part reduction by pi/2, Taylor
//          polynomials (degree 11 / 12) on [-pi/4, pi/4]
//   exp  : x = k ln2 + r with a two-part ln2, Taylor polynomial of degree 8,
//          exact scaling by 2^k
//   log  : x = m 2^e, m in [sqrt(1/2), sqrt(2)], log m = 2 atanh((m-1)/(m+1))
//   atan2: octant reduction; atan(a) = pi/4 + atan((a-1)/(a+1)) above
//          tan(pi/8); Taylor series of atan to degree 17
//   powi : binary exponentiation (POW_II only uses integer exponents)
//   cos  : fm_sin's reduction and polynomials, quadrant shifted by one
//   acos : atan2(sqrt((1 - x)(1 + x)), x) (the cinematic sky model)
//   pow  : exp(y log x) for x > 0; 0 or 1 at x = 0; NaN for x < 0 (the
//          exp2(y log2 x) convention of GPU drivers for negative x)
// Error bounds used by the directed-rounding mode are in interval.cuh.
#pragma once
#include <stdint.h>

#define TSI_DEV __device__ __forceinline__

namespace tsi {

TSI_DEV float fm_mul(float a, float b) { return __fmul_rn(a, b); }
TSI_DEV float fm_add(float a, float b) { return __fadd_rn(a, b); }
TSI_DEV float fm_sub(float a, float b) { return __fsub_rn(a, b); }
TSI_DEV float fm_div(float a, float b) { return __fdiv_rn(a, b); }
TSI_DEV float fm_inf() { return __int_as_float(0x7f800000); }
TSI_DEV float fm_nan() { return __int_as_float(0x7fc00000); }

// IEEE 754-2019 minimumNumber / maximumNumber: a NaN operand loses and
// -0 < +0.  On sm_100 the hardware min/max (fminf/fmaxf) has exactly these
// semantics (both orders of -0/+0 and NaN are checked against the oracle's
// explicit rule by tests/test_gpu_ops.py::test_min_max_semantics), so one
// instruction implements it.
TSI_DEV float fm_min(float a, float b) { return fminf(a, b); }
TSI_DEV float fm_max(float a, float b) { return fmaxf(a, b); }

TSI_DEV float fm_sin(float x) {
  if (!(fabsf(x) <= 3.0e38f)) return fm_sub(x, x);
  const float two_over_pi = 0.6366197466850281f;
  const float p1 = 1.5703125f, p2 = 0.0004838705062866211f, p3 = -4.371138828673793e-08f;
  float k = rintf(fm_mul(x, two_over_pi));
  float r = fm_sub(x, fm_mul(k, p1));
  r = fm_sub(r, fm_mul(k, p2));
  r = fm_sub(r, fm_mul(k, p3));
  float qf = fm_sub(k, fm_mul(4.0f, floorf(fm_mul(k, 0.25f))));
  int q = (int)qf;
  float r2 = fm_mul(r, r);
  float ps = -2.5052107943679403e-08f;
  ps = fm_add(2.7557318844628753e-06f, fm_mul(r2, ps));
  ps = fm_add(-0.00019841270113829523f, fm_mul(r2, ps));
  ps = fm_add(0.008333333767950535f, fm_mul(r2, ps));
  ps = fm_add(-0.1666666716337204f, fm_mul(r2, ps));
  float s = fm_add(r, fm_mul(r, fm_mul(r2, ps)));
  float pc = 2.0876755879584152e-09f;
  pc = fm_add(-2.755731998149713e-07f, fm_mul(r2, pc));
  pc = fm_add(2.4801587642286904e-05f, fm_mul(r2, pc));
  pc = fm_add(-0.0013888889225199819f, fm_mul(r2, pc));
  pc = fm_add(0.0416666679084301f, fm_mul(r2, pc));
  pc = fm_add(-0.5f, fm_mul(r2, pc));
  float c = fm_add(1.0f, fm_mul(r2, pc));
  switch (q) {
    case 0: return s;
    case 1: return c;
    case 2: return -s;
    default: return -c;
  }
}

TSI_DEV float fm_cos(float x) {
  if (!(fabsf(x) <= 3.0e38f)) return fm_sub(x, x);
  const float two_over_pi = 0.6366197466850281f;
  const float p1 = 1.5703125f, p2 = 0.0004838705062866211f, p3 = -4.371138828673793e-08f;
  float k = rintf(fm_mul(x, two_over_pi));
  float r = fm_sub(x, fm_mul(k, p1));
  r = fm_sub(r, fm_mul(k, p2));
  r = fm_sub(r, fm_mul(k, p3));
  float qf = fm_sub(k, fm_mul(4.0f, floorf(fm_mul(k, 0.25f))));
  int q = (int)qf;
  float r2 = fm_mul(r, r);
  float ps = -2.5052107943679403e-08f;
  ps = fm_add(2.7557318844628753e-06f, fm_mul(r2, ps));
  ps = fm_add(-0.00019841270113829523f, fm_mul(r2, ps));
  ps = fm_add(0.008333333767950535f, fm_mul(r2, ps));
  ps = fm_add(-0.1666666716337204f, fm_mul(r2, ps));
  float s = fm_add(r, fm_mul(r, fm_mul(r2, ps)));
  float pc = 2.0876755879584152e-09f;
  pc = fm_add(-2.755731998149713e-07f, fm_mul(r2, pc));
  pc = fm_add(2.4801587642286904e-05f, fm_mul(r2, pc));
  pc = fm_add(-0.0013888889225199819f, fm_mul(r2, pc));
  pc = fm_add(0.0416666679084301f, fm_mul(r2, pc));
  pc = fm_add(-0.5f, fm_mul(r2, pc));
  float c = fm_add(1.0f, fm_mul(r2, pc));
  switch (q) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
  }
}

TSI_DEV float fm_pow2i(int e) { return __int_as_float((e + 127) << 23); }

TSI_DEV float fm_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283935546875f) return fm_inf();
  if (x < -103.97208404541016f) return 0.0f;
  const float log2e = 1.4426950216293335f;
  const float ln2_hi = 0.693145751953125f, ln2_lo = 1.428606765330187e-06f;
  float k = rintf(fm_mul(x, log2e));
  float r = fm_sub(x, fm_mul(k, ln2_hi));
  r = fm_sub(r, fm_mul(k, ln2_lo));
  float p = 2.4801587642286904e-05f;
  p = fm_add(0.00019841270113829523f, fm_mul(r, p));
  p = fm_add(0.0013888889225199819f, fm_mul(r, p));
  p = fm_add(0.008333333767950535f, fm_mul(r, p));
  p = fm_add(0.0416666679084301f, fm_mul(r, p));
  p = fm_add(0.1666666716337204f, fm_mul(r, p));
  p = fm_add(0.5f, fm_mul(r, p));
  p = fm_add(1.0f, fm_mul(r, p));
  p = fm_add(1.0f, fm_mul(r, p));
  int ki = (int)k;
  if (ki > 127) return fm_mul(fm_mul(p, fm_pow2i(127)), fm_pow2i(ki - 127));
  if (ki < -126) return fm_mul(fm_mul(p, fm_pow2i(-126)), fm_pow2i(ki + 126));
  return fm_mul(p, fm_pow2i(ki));
}

TSI_DEV float fm_log(float x) {
  if (x != x) return x;
  if (x < 0.0f) return fm_nan();
  if (x == 0.0f) return -fm_inf();
  if (x == fm_inf()) return x;
  int e = 0;
  if (x < 1.17549435e-38f) {
    x = fm_mul(x, 16777216.0f);
    e = -24;
  }
  uint32_t b = __float_as_uint(x);
  e += (int)(b >> 23) - 127;
  float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.4142135381698608f) {
    m = fm_mul(m, 0.5f);
    e += 1;
  }
  float s = fm_div(fm_sub(m, 1.0f), fm_add(m, 1.0f));
  float s2 = fm_mul(s, s);
  float p = 0.09090909361839294f;
  p = fm_add(0.1111111119389534f, fm_mul(s2, p));
  p = fm_add(0.1428571492433548f, fm_mul(s2, p));
  p = fm_add(0.20000000298023224f, fm_mul(s2, p));
  p = fm_add(0.3333333432674408f, fm_mul(s2, p));
  p = fm_add(1.0f, fm_mul(s2, p));
  float lm = fm_mul(fm_add(s, s), p);
  float fe = (float)e;
  const float ln2_hi = 0.693145751953125f, ln2_lo = 1.428606765330187e-06f;
  return fm_add(fm_mul(fe, ln2_hi), fm_add(lm, fm_mul(fe, ln2_lo)));
}

// C semantics atan2(y, x)
TSI_DEV float fm_atan2(float y, float x) {
  const float pi = 3.1415927410125732f, halfpi = 1.5707963705062866f, qpi = 0.7853981852531433f;
  if (x != x || y != y) return fm_add(x, y);
  float ax = fabsf(x), ay = fabsf(y);
  float r;
  const bool xneg = (__float_as_uint(x) >> 31) != 0;
  if (ay == 0.0f) {
    r = xneg ? pi : 0.0f;
    return copysignf(r, y);
  }
  if (ax == fm_inf()) {
    if (ay == fm_inf()) r = xneg ? fm_sub(pi, qpi) : qpi;
    else r = xneg ? pi : 0.0f;
    return copysignf(r, y);
  }
  if (ay == fm_inf() || ax == 0.0f) return copysignf(halfpi, y);
  bool swap = ay > ax;
  float num = swap ? ax : ay, den = swap ? ay : ax;
  float a = fm_div(num, den);
  float base = 0.0f, z = a;
  if (a > 0.4142135679721832f) {
    z = fm_div(fm_sub(a, 1.0f), fm_add(a, 1.0f));
    base = qpi;
  }
  float z2 = fm_mul(z, z);
  float p = 0.05882352963089943f;
  p = fm_add(-0.06666667014360428f, fm_mul(z2, p));
  p = fm_add(0.07692307978868484f, fm_mul(z2, p));
  p = fm_add(-0.09090909361839294f, fm_mul(z2, p));
  p = fm_add(0.1111111119389534f, fm_mul(z2, p));
  p = fm_add(-0.1428571492433548f, fm_mul(z2, p));
  p = fm_add(0.20000000298023224f, fm_mul(z2, p));
  p = fm_add(-0.3333333432674408f, fm_mul(z2, p));
  float at = fm_add(z, fm_mul(z, fm_mul(z2, p)));
  r = fm_add(base, at);
  if (swap) r = fm_sub(halfpi, r);
  if (xneg) r = fm_sub(pi, r);
  return copysignf(r, y);
}

TSI_DEV float fm_powi(float x, int n) {
  if (n == 0) return 1.0f;
  uint32_t m = (n < 0) ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  float r = 1.0f, b = x;
  while (m) {
    if (m & 1u) r = fm_mul(r, b);
    m >>= 1;
    if (m) b = fm_mul(b, b);
  }
  return (n < 0) ? fm_div(1.0f, r) : r;
}

TSI_DEV float fm_powf(float x, float y) {
  if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : fm_inf());
  if (x < 0.0f) return fm_nan();
  return fm_exp(fm_mul(y, fm_log(x)));
}

TSI_DEV float fm_acos(float x) { return fm_atan2(__fsqrt_rn(fm_mul(fm_sub(1.0f, x), fm_add(1.0f, x))), x); }

}  // namespace tsi
