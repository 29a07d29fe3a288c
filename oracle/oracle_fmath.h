/*
 * oracle_fmath.h — TEST INFRASTRUCTURE (CPU oracle).  Not part of the product.
 *
 * f32 elementary functions for the oracle.  compute.wgsl calls the WGSL
 * built-ins sin/exp/log/atan2/pow (compute.wgsl:2577-2581, 2753-2800,
 * 2838-2853, 2947-2953), which the Vulkan driver implements with bounded but
 * unspecified error.  The library pins them down instead: every function here
 * is a fixed sequence of correctly rounded f32 operations, restated
 * independently in the CUDA kernels, so the oracle and the GPU agree bit for
 * bit.  Methods (published, named):
 *   sin/cos : Cody & Waite (1980) three-part reduction by pi/2, Taylor
 *             polynomials on [-pi/4, pi/4] (Horner form)
 *   exp     : reduction x = k ln2 + r (Cody & Waite two-part ln2), Taylor
 *             polynomial of degree 8, exact scaling by 2^k
 *   log     : x = m 2^e, m in [sqrt(1/2), sqrt(2)], log m = 2 atanh(s),
 *             s = (m-1)/(m+1), odd series in s
 *   atan2   : octant reduction, atan(a) = pi/4 + atan((a-1)/(a+1)) above
 *             tan(pi/8), Taylor series of atan below
 *   powi    : binary exponentiation (integer exponents, POW_II's contract)
 *   acos    : atan2(sqrt((1 - x)(1 + x)), x) (cinematic sky model)
 *   pow     : exp(y log x) for x > 0, 0 or 1 at x = 0, NaN for x < 0 (the
 *             exp2(y log2 x) convention of GPU drivers for negative x)
 * The oracle is compiled with -ffp-contract=off so that no FMA contracts.
 */
#ifndef ORACLE_FMATH_H
#define ORACLE_FMATH_H
#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float of_bits(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t of_ubits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

#define OF_INF (of_bits(0x7f800000u))
#define OF_NAN (of_bits(0x7fc00000u))

/* sin via Cody-Waite */
static inline float of_sin(float x) {
  if (!(fabsf(x) <= 3.0e38f)) return x - x; /* inf, nan -> nan */
  const float two_over_pi = 0.6366197466850281f;
  const float p1 = 1.5703125f, p2 = 0.0004838705062866211f, p3 = -4.371138828673793e-08f;
  float k = rintf(x * two_over_pi);
  float r = x - k * p1;
  r = r - k * p2;
  r = r - k * p3;
  float qf = k - 4.0f * floorf(k * 0.25f);
  int q = (int)qf;
  float r2 = r * r;
  float ps = -2.5052107943679403e-08f;
  ps = 2.7557318844628753e-06f + r2 * ps;
  ps = -0.00019841270113829523f + r2 * ps;
  ps = 0.008333333767950535f + r2 * ps;
  ps = -0.1666666716337204f + r2 * ps;
  float s = r + r * (r2 * ps);
  float pc = 2.0876755879584152e-09f;
  pc = -2.755731998149713e-07f + r2 * pc;
  pc = 2.4801587642286904e-05f + r2 * pc;
  pc = -0.0013888889225199819f + r2 * pc;
  pc = 0.0416666679084301f + r2 * pc;
  pc = -0.5f + r2 * pc;
  float c = 1.0f + r2 * pc;
  switch (q) {
    case 0: return s;
    case 1: return c;
    case 2: return -s;
    default: return -c;
  }
}

/* cos: the same reduction and polynomials as of_sin, quadrant shifted by one */
static inline float of_cos(float x) {
  if (!(fabsf(x) <= 3.0e38f)) return x - x;
  const float two_over_pi = 0.6366197466850281f;
  const float p1 = 1.5703125f, p2 = 0.0004838705062866211f, p3 = -4.371138828673793e-08f;
  float k = rintf(x * two_over_pi);
  float r = x - k * p1;
  r = r - k * p2;
  r = r - k * p3;
  float qf = k - 4.0f * floorf(k * 0.25f);
  int q = (int)qf;
  float r2 = r * r;
  float ps = -2.5052107943679403e-08f;
  ps = 2.7557318844628753e-06f + r2 * ps;
  ps = -0.00019841270113829523f + r2 * ps;
  ps = 0.008333333767950535f + r2 * ps;
  ps = -0.1666666716337204f + r2 * ps;
  float s = r + r * (r2 * ps);
  float pc = 2.0876755879584152e-09f;
  pc = -2.755731998149713e-07f + r2 * pc;
  pc = 2.4801587642286904e-05f + r2 * pc;
  pc = -0.0013888889225199819f + r2 * pc;
  pc = 0.0416666679084301f + r2 * pc;
  pc = -0.5f + r2 * pc;
  float c = 1.0f + r2 * pc;
  switch (q) {
    case 0: return c;
    case 1: return -s;
    case 2: return -c;
    default: return s;
  }
}

static inline float of_pow2i(int e) { /* 2^e for e in [-126, 127] */
  return of_bits((uint32_t)(e + 127) << 23);
}

static inline float of_exp(float x) {
  if (x != x) return x;
  if (x > 88.72283935546875f) return OF_INF;
  if (x < -103.97208404541016f) return 0.0f;
  const float log2e = 1.4426950216293335f;
  const float ln2_hi = 0.693145751953125f, ln2_lo = 1.428606765330187e-06f;
  float k = rintf(x * log2e);
  float r = x - k * ln2_hi;
  r = r - k * ln2_lo;
  float p = 2.4801587642286904e-05f;
  p = 0.00019841270113829523f + r * p;
  p = 0.0013888889225199819f + r * p;
  p = 0.008333333767950535f + r * p;
  p = 0.0416666679084301f + r * p;
  p = 0.1666666716337204f + r * p;
  p = 0.5f + r * p;
  p = 1.0f + r * p;
  p = 1.0f + r * p;
  int ki = (int)k;
  if (ki > 127) return (p * of_pow2i(127)) * of_pow2i(ki - 127);
  if (ki < -126) return (p * of_pow2i(-126)) * of_pow2i(ki + 126);
  return p * of_pow2i(ki);
}

static inline float of_log(float x) {
  if (x != x) return x;
  if (x < 0.0f) return OF_NAN;
  if (x == 0.0f) return -OF_INF;
  if (x == OF_INF) return x;
  int e = 0;
  if (x < 1.17549435e-38f) {
    x = x * 16777216.0f;
    e = -24;
  }
  uint32_t b = of_ubits(x);
  e += (int)(b >> 23) - 127;
  float m = of_bits((b & 0x007fffffu) | 0x3f800000u);
  if (m > 1.4142135381698608f) {
    m = m * 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float s2 = s * s;
  float p = 0.09090909361839294f;
  p = 0.1111111119389534f + s2 * p;
  p = 0.1428571492433548f + s2 * p;
  p = 0.20000000298023224f + s2 * p;
  p = 0.3333333432674408f + s2 * p;
  p = 1.0f + s2 * p;
  float lm = (s + s) * p;
  float fe = (float)e;
  const float ln2_hi = 0.693145751953125f, ln2_lo = 1.428606765330187e-06f;
  return fe * ln2_hi + (lm + fe * ln2_lo);
}

/* C semantics: atan2(y, x) */
static inline float of_atan2(float y, float x) {
  const float pi = 3.1415927410125732f, halfpi = 1.5707963705062866f, qpi = 0.7853981852531433f;
  if (x != x || y != y) return x + y;
  float ax = fabsf(x), ay = fabsf(y);
  float r;
  if (ay == 0.0f) {
    r = signbit(x) ? pi : 0.0f;
    return copysignf(r, y);
  }
  if (ax == OF_INF) {
    if (ay == OF_INF) r = signbit(x) ? (pi - qpi) : qpi;
    else r = signbit(x) ? pi : 0.0f;
    return copysignf(r, y);
  }
  if (ay == OF_INF || ax == 0.0f) return copysignf(halfpi, y);
  int swap = ay > ax;
  float num = swap ? ax : ay, den = swap ? ay : ax;
  float a = num / den;
  float base = 0.0f, z = a;
  if (a > 0.4142135679721832f) {
    z = (a - 1.0f) / (a + 1.0f);
    base = qpi;
  }
  float z2 = z * z;
  float p = 0.05882352963089943f;
  p = -0.06666667014360428f + z2 * p;
  p = 0.07692307978868484f + z2 * p;
  p = -0.09090909361839294f + z2 * p;
  p = 0.1111111119389534f + z2 * p;
  p = -0.1428571492433548f + z2 * p;
  p = 0.20000000298023224f + z2 * p;
  p = -0.3333333432674408f + z2 * p;
  float at = z + z * (z2 * p);
  r = base + at;
  if (swap) r = halfpi - r;
  if (signbit(x)) r = pi - r;
  return copysignf(r, y);
}

static inline float of_powi(float x, int n) {
  if (n == 0) return 1.0f;
  uint32_t m = (n < 0) ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
  float r = 1.0f, b = x;
  while (m) {
    if (m & 1u) r = r * b;
    m >>= 1;
    if (m) b = b * b;
  }
  return (n < 0) ? 1.0f / r : r;
}

/* general pow for the gamma curve (x >= 0) */
static inline float of_powf(float x, float y) {
  if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : OF_INF);
  if (x < 0.0f) return OF_NAN;
  return of_exp(y * of_log(x));
}

static inline float of_acos(float x) { return of_atan2(sqrtf((1.0f - x) * (1.0f + x)), x); }

/* IEEE 754-2019 minimumNumber / maximumNumber: NaN loses, -0 < +0 */
static inline float of_min(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a < b) return a;
  if (b < a) return b;
  return signbit(a) ? a : b;
}
static inline float of_max(float a, float b) {
  if (a != a) return b;
  if (b != b) return a;
  if (a > b) return a;
  if (b > a) return b;
  return signbit(a) ? b : a;
}

#endif
