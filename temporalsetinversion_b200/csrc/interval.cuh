// interval.cuh — interval arithmetic for the tape interpreter.
//
// Template parameter D selects the rounding:
//   D = false : round to nearest, the plain f32 formulas of
//               compute.wgsl:2539-2975 (parity mode, bit-exact with the CPU
//               restatement of those formulas)
//   D = true  : outward rounding (lower bounds rounded down, upper bounds up
//               with __f*_rd / __f*_ru), division by an interval containing
//               0 gives the whole line, NaN means "anything", and the
//               library's elementary functions are widened by their error
//               bound; `fix` keeps infinities instead of clamping to 1e6, so
//               every result encloses the exact range.
#pragma once
#include "fmath.cuh"
#include "tape_format.h"

namespace tsi {

struct Iv {
  float lo, hi;
};

TSI_DEV Iv iv(float a) { return Iv{a, a}; }
TSI_DEV Iv iv(float a, float b) { return Iv{a, b}; }
TSI_DEV bool is_nan_f(float a) { return !(a < 0.0f || a > 0.0f || a == 0.0f); }

constexpr float kPI = 3.1415927410125732f;
constexpr float kTWOPI = 6.2831854820251465f;
constexpr float kHALFPI = 1.5707963705062866f;
constexpr float kBIG = 1000000.0f;
// Maximum error, in ulps, of fm_sin / fm_exp / fm_log / fm_atan2 over the
// argument ranges used below (measured against double precision by the
// GPU math tests, which assert it with a margin).
constexpr int kElemUlps = 4;
// fm_sin's argument reduction is exact below this magnitude (|k| < 2^12).
constexpr float kSinExactArg = 6000.0f;

template <bool D>
struct Rnd;
template <>
struct Rnd<false> {
  static TSI_DEV float add_dn(float a, float b) { return __fadd_rn(a, b); }
  static TSI_DEV float add_up(float a, float b) { return __fadd_rn(a, b); }
  static TSI_DEV float sub_dn(float a, float b) { return __fsub_rn(a, b); }
  static TSI_DEV float sub_up(float a, float b) { return __fsub_rn(a, b); }
  static TSI_DEV float mul_dn(float a, float b) { return __fmul_rn(a, b); }
  static TSI_DEV float mul_up(float a, float b) { return __fmul_rn(a, b); }
  static TSI_DEV float div_dn(float a, float b) { return __fdiv_rn(a, b); }
  static TSI_DEV float div_up(float a, float b) { return __fdiv_rn(a, b); }
  static TSI_DEV float sqrt_dn(float a) { return __fsqrt_rn(a); }
  static TSI_DEV float sqrt_up(float a) { return __fsqrt_rn(a); }
  static TSI_DEV float widen_dn(float a, int) { return a; }
  static TSI_DEV float widen_up(float a, int) { return a; }
};
template <>
struct Rnd<true> {
  static TSI_DEV float add_dn(float a, float b) { return __fadd_rd(a, b); }
  static TSI_DEV float add_up(float a, float b) { return __fadd_ru(a, b); }
  static TSI_DEV float sub_dn(float a, float b) { return __fsub_rd(a, b); }
  static TSI_DEV float sub_up(float a, float b) { return __fsub_ru(a, b); }
  static TSI_DEV float mul_dn(float a, float b) { return __fmul_rd(a, b); }
  static TSI_DEV float mul_up(float a, float b) { return __fmul_ru(a, b); }
  static TSI_DEV float div_dn(float a, float b) { return __fdiv_rd(a, b); }
  static TSI_DEV float div_up(float a, float b) { return __fdiv_ru(a, b); }
  static TSI_DEV float sqrt_dn(float a) { return __fsqrt_rd(a); }
  static TSI_DEV float sqrt_up(float a) { return __fsqrt_ru(a); }
  // step n ulps toward -inf / +inf (nextafter applied n times)
  static TSI_DEV float widen_dn(float a, int n) {
    if (a != a || a == -fm_inf()) return a;
    for (int i = 0; i < n; ++i) {
      if (a == 0.0f) a = -__int_as_float(1);
      else if (a > 0.0f) a = __int_as_float(__float_as_int(a) - 1);
      else a = __int_as_float(__float_as_int(a) + 1);
    }
    return a;
  }
  static TSI_DEV float widen_up(float a, int n) { return -widen_dn(-a, n); }
};

template <bool D>
struct IA {
  using R = Rnd<D>;
  static TSI_DEV Iv entire() { return Iv{-fm_inf(), fm_inf()}; }

  static TSI_DEV bool contains_zero(Iv a) { return a.lo <= 0.0f && 0.0f <= a.hi; }
  static TSI_DEV Iv unordered(float a, float b) { return Iv{fm_min(a, b), fm_max(a, b)}; }

  static TSI_DEV Iv add(Iv a, Iv b) { return Iv{R::add_dn(a.lo, b.lo), R::add_up(a.hi, b.hi)}; }
  static TSI_DEV Iv add_f(Iv a, float b) { return Iv{R::add_dn(a.lo, b), R::add_up(a.hi, b)}; }
  static TSI_DEV Iv sub(Iv a, Iv b) { return Iv{R::sub_dn(a.lo, b.hi), R::sub_up(a.hi, b.lo)}; }
  static TSI_DEV Iv sub_f(Iv a, float b) { return Iv{R::sub_dn(a.lo, b), R::sub_up(a.hi, b)}; }
  static TSI_DEV Iv mul(Iv a, Iv b) {
    if (!D) {
      float x = __fmul_rn(a.lo, b.lo), y = __fmul_rn(a.lo, b.hi);
      float z = __fmul_rn(a.hi, b.lo), w = __fmul_rn(a.hi, b.hi);
      return Iv{fm_min(fm_min(x, y), fm_min(z, w)), fm_max(fm_max(x, y), fm_max(z, w))};
    }
    float x = R::mul_dn(a.lo, b.lo), y = R::mul_dn(a.lo, b.hi);
    float z = R::mul_dn(a.hi, b.lo), w = R::mul_dn(a.hi, b.hi);
    float X = R::mul_up(a.lo, b.lo), Y = R::mul_up(a.lo, b.hi);
    float Z = R::mul_up(a.hi, b.lo), W = R::mul_up(a.hi, b.hi);
    if (x != x || y != y || z != z || w != w) return entire();
    return Iv{fminf(fminf(x, y), fminf(z, w)), fmaxf(fmaxf(X, Y), fmaxf(Z, W))};
  }
  static TSI_DEV Iv mul_f(Iv a, float b) {
    if (!D) {
      if (b >= 0.0f) return Iv{__fmul_rn(a.lo, b), __fmul_rn(a.hi, b)};
      return Iv{__fmul_rn(a.hi, b), __fmul_rn(a.lo, b)};
    }
    return mul(a, iv(b));
  }
  static TSI_DEV Iv div(Iv a, Iv b) {
    if (!D) {
      float x = __fdiv_rn(a.lo, b.lo), y = __fdiv_rn(a.lo, b.hi);
      float z = __fdiv_rn(a.hi, b.lo), w = __fdiv_rn(a.hi, b.hi);
      return Iv{fm_min(fm_min(x, y), fm_min(z, w)), fm_max(fm_max(x, y), fm_max(z, w))};
    }
    if (contains_zero(b) || b.lo != b.lo || b.hi != b.hi) return entire();
    float x = R::div_dn(a.lo, b.lo), y = R::div_dn(a.lo, b.hi);
    float z = R::div_dn(a.hi, b.lo), w = R::div_dn(a.hi, b.hi);
    float X = R::div_up(a.lo, b.lo), Y = R::div_up(a.lo, b.hi);
    float Z = R::div_up(a.hi, b.lo), W = R::div_up(a.hi, b.hi);
    if (x != x || y != y || z != z || w != w) return entire();
    return Iv{fminf(fminf(x, y), fminf(z, w)), fmaxf(fmaxf(X, Y), fmaxf(Z, W))};
  }
  static TSI_DEV Iv sqrt_(Iv a) { return Iv{R::sqrt_dn(fm_max(a.lo, 0.0f)), R::sqrt_up(fm_max(a.hi, 0.0f))}; }
  static TSI_DEV Iv exp_(Iv a) {
    if (!D) return Iv{fm_exp(a.lo), fm_exp(a.hi)};
    return Iv{fm_max(R::widen_dn(fm_exp(a.lo), kElemUlps), 0.0f), R::widen_up(fm_exp(a.hi), kElemUlps)};
  }
  static TSI_DEV Iv log_(Iv a) {
    return Iv{R::widen_dn(fm_log(fm_max(a.lo, 0.0f)), kElemUlps),
              R::widen_up(fm_log(fm_max(a.hi, 0.0f)), kElemUlps)};
  }
  static TSI_DEV Iv neg(Iv a) { return Iv{-a.hi, -a.lo}; }
  static TSI_DEV Iv min_(Iv a, Iv b) { return Iv{fm_min(a.lo, b.lo), fm_min(a.hi, b.hi)}; }
  static TSI_DEV Iv max_(Iv a, Iv b) { return Iv{fm_max(a.lo, b.lo), fm_max(a.hi, b.hi)}; }
  static TSI_DEV Iv abs_(Iv a) {
    if (contains_zero(a)) return Iv{0.0f, fm_max(-a.lo, a.hi)};
    if (a.hi < 0.0f) return Iv{-a.hi, -a.lo};
    return a;
  }
  static TSI_DEV Iv abs_rr(Iv a) {
    if (contains_zero(a)) return Iv{-1.0f, 1.0f};
    if (a.hi < 0.0f) return iv(-1.0f);
    return iv(1.0f);
  }
  static TSI_DEV Iv empty() { return Iv{fm_inf(), -fm_inf()}; }
  static TSI_DEV Iv cap(Iv a, Iv b) {
    if (a.hi < b.lo || b.hi < a.lo) return empty();
    return Iv{fm_max(a.lo, b.lo), fm_min(a.hi, b.hi)};
  }
  static TSI_DEV Iv sqr(Iv a) {
    float x = R::mul_dn(a.lo, a.lo), y = R::mul_dn(a.hi, a.hi);
    if (!D) {
      if (contains_zero(a)) return Iv{0.0f, fm_max(x, y)};
      return Iv{fm_min(x, y), fm_max(x, y)};
    }
    float X = R::mul_up(a.lo, a.lo), Y = R::mul_up(a.hi, a.hi);
    if (contains_zero(a)) return Iv{0.0f, fm_max(X, Y)};
    return Iv{fm_min(x, y), fm_max(X, Y)};
  }
  static TSI_DEV Iv floor_(Iv a) { return Iv{floorf(a.lo), floorf(a.hi)}; }
  static TSI_DEV Iv floor_rr(Iv a) {
    if (floorf(a.hi) != floorf(a.lo)) return Iv{-kBIG, kBIG};
    return iv(0.0f);
  }
  static TSI_DEV float at2_dn(float y, float x) { return R::widen_dn(fm_atan2(y, x), kElemUlps); }
  static TSI_DEV float at2_up(float y, float x) { return R::widen_up(fm_atan2(y, x), kElemUlps); }
  // ATAN2_II(x = larg, y = rarg), compute.wgsl:2724-2804
  static TSI_DEV Iv atan2_(Iv x, Iv y) {
    const Iv range_atan = Iv{D ? -kPI * 1.0000002f : -kPI, D ? kPI * 1.0000002f : kPI};
    const Iv half_range = Iv{-kHALFPI, kHALFPI};
    if (D) {
      // The reference's case analysis is not an enclosure (2729-2734 return
      // [0, y.hi] for y.lo == 0).  Directed mode encloses atan2(y, x) over
      // the box: monotone pieces away from the branch cut, else [-pi, pi].
      if (x.lo > 0.0f) {
        float lo = fminf(at2_dn(y.lo, x.lo), at2_dn(y.lo, x.hi));
        float hi = fmaxf(at2_up(y.hi, x.lo), at2_up(y.hi, x.hi));
        return Iv{lo, hi};
      }
      if (y.lo > 0.0f) {
        float lo = fminf(at2_dn(y.lo, x.hi), at2_dn(y.hi, x.hi));
        float hi = fmaxf(at2_up(y.lo, x.lo), at2_up(y.hi, x.lo));
        return Iv{lo, hi};
      }
      if (y.hi < 0.0f) {
        float lo = fminf(at2_dn(y.hi, x.lo), at2_dn(y.lo, x.lo));
        float hi = fmaxf(at2_up(y.hi, x.hi), at2_up(y.lo, x.hi));
        return Iv{lo, hi};
      }
      return range_atan;
    }
    if (y.lo == 0.0f) return Iv{0.0f, y.hi};
    if (y.hi == 0.0f) return Iv{y.lo, 0.0f};
    if (x.lo == 0.0f && x.hi == 0.0f) {
      if (y.lo == 0.0f && y.hi == 0.0f) return empty();
      if (y.lo >= 0.0f) return iv(kHALFPI);
      if (y.hi <= 0.0f) return iv(-kHALFPI);
      return half_range;
    } else if (x.lo > 0.0f) {
      if (y.lo == 0.0f && y.hi == 0.0f) return y;
      if (y.lo >= 0.0f) return Iv{fm_atan2(y.lo, x.hi), fm_atan2(y.hi, x.lo)};
      if (y.hi <= 0.0f) return Iv{fm_atan2(y.lo, x.lo), fm_atan2(y.hi, x.hi)};
      return Iv{fm_atan2(y.lo, x.lo), fm_atan2(y.hi, x.lo)};
    } else if (x.hi < 0.0f) {
      if (y.lo == 0.0f && y.hi == 0.0f) return iv(kPI);
      if (y.lo >= 0.0f) return Iv{fm_atan2(y.hi, x.hi), fm_atan2(y.lo, x.lo)};
      if (y.hi < 0.0f) return Iv{fm_atan2(y.hi, x.lo), fm_atan2(y.lo, x.hi)};
      return range_atan;
    } else {
      if (x.lo == 0.0f) {
        if (y.lo == 0.0f && y.hi == 0.0f) return y;
        if (y.lo >= 0.0f) return Iv{fm_atan2(y.lo, x.hi), half_range.hi};
        if (y.hi <= 0.0f) return Iv{half_range.lo, fm_atan2(y.hi, x.hi)};
        return half_range;
      } else if (x.hi == 0.0f) {
        if (y.lo == 0.0f && y.hi == 0.0f) return iv(kPI);
        if (y.lo >= 0.0f) return Iv{kHALFPI, fm_atan2(y.lo, x.lo)};
        if (y.hi < 0.0f) return Iv{fm_atan2(y.hi, x.lo), -kHALFPI};
        return range_atan;
      } else {
        if (y.lo >= 0.0f) return Iv{fm_atan2(y.lo, x.hi), fm_atan2(y.lo, x.lo)};
        if (y.hi < 0.0f) return Iv{fm_atan2(y.hi, x.lo), fm_atan2(y.hi, x.hi)};
        return range_atan;
      }
    }
  }
  static TSI_DEV void atan2_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    Iv den = add(sqr(r), sqr(l));
    o0 = div(neg(l), den);
    o1 = div(r, den);
  }
  static TSI_DEV Iv mod_(Iv a, Iv b) { return sub(a, mul(b, floor_(div(a, b)))); }
  static TSI_DEV void mod_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    Iv a = floor_(div(l, r));
    o0 = iv(1.0f);
    o1 = neg(add(a, mul(r, floor_rr(a))));
  }
  static TSI_DEV float powi_dn(float x, int n) {  // x >= 0
    if (!D) return fm_powi(x, n);
    if (n == 0) return 1.0f;
    uint32_t m = (n < 0) ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
    float r = 1.0f, b = x, R_ = 1.0f, B_ = x;
    while (m) {
      if (m & 1u) {
        r = __fmul_rd(r, b);
        R_ = __fmul_ru(R_, B_);
      }
      m >>= 1;
      if (m) {
        b = __fmul_rd(b, b);
        B_ = __fmul_ru(B_, B_);
      }
    }
    return (n < 0) ? __fdiv_rd(1.0f, R_) : r;
  }
  static TSI_DEV float powi_up(float x, int n) {
    if (!D) return fm_powi(x, n);
    if (n == 0) return 1.0f;
    uint32_t m = (n < 0) ? (uint32_t)(-(int64_t)n) : (uint32_t)n;
    float r = 1.0f, b = x, R_ = 1.0f, B_ = x;
    while (m) {
      if (m & 1u) {
        r = __fmul_rd(r, b);
        R_ = __fmul_ru(R_, B_);
      }
      m >>= 1;
      if (m) {
        b = __fmul_rd(b, b);
        B_ = __fmul_ru(B_, B_);
      }
    }
    return (n < 0) ? __fdiv_ru(1.0f, r) : R_;
  }
  static TSI_DEV int round_power(float b) {  // i32(round(b)), saturating, NaN -> 0
    float rb = rintf(b);
    if (rb != rb) return 0;
    if (rb >= 2147483520.0f) return 2147483647;
    if (rb <= -2147483648.0f) return -2147483647 - 1;
    return (int)rb;
  }
  // POW_II, compute.wgsl:2829-2860 (integer exponent round(b.lo))
  static TSI_DEV Iv pow_(Iv a, Iv b) {
    int p = round_power(b.lo);
    const bool even = (p % 2 == 0);
    if (!D) {
      float lower, higher;
      if (a.lo <= 0.0f) lower = even ? fm_powi(-a.lo, p) : -fm_powi(-a.lo, p);
      else lower = fm_powi(a.lo, p);
      if (a.hi <= 0.0f) higher = even ? fm_powi(-a.hi, p) : -fm_powi(-a.hi, p);
      else higher = fm_powi(a.hi, p);
      if (contains_zero(a)) return Iv{0.0f, fm_max(lower, higher)};
      return Iv{fm_min(lower, higher), fm_max(lower, higher)};
    }
    // enclosure of x^p over a for integer p
    if (p == 0) return iv(1.0f);
    if (p < 0 && contains_zero(a)) return entire();
    float l_lo, l_hi, h_lo, h_hi;  // bounds of f(a.lo) and f(a.hi)
    if (a.lo <= 0.0f) {
      float m = powi_dn(-a.lo, p), M = powi_up(-a.lo, p);
      if (even) { l_lo = m; l_hi = M; } else { l_lo = -M; l_hi = -m; }
    } else {
      l_lo = powi_dn(a.lo, p);
      l_hi = powi_up(a.lo, p);
    }
    if (a.hi <= 0.0f) {
      float m = powi_dn(-a.hi, p), M = powi_up(-a.hi, p);
      if (even) { h_lo = m; h_hi = M; } else { h_lo = -M; h_hi = -m; }
    } else {
      h_lo = powi_dn(a.hi, p);
      h_hi = powi_up(a.hi, p);
    }
    if (even && p > 0 && contains_zero(a)) return Iv{0.0f, fm_max(l_hi, h_hi)};
    return Iv{fm_min(l_lo, h_lo), fm_max(l_hi, h_hi)};
  }
  static TSI_DEV void pow_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    o0 = mul(r, pow_(l, sub_f(r, 1.0f)));
    o1 = mul(pow_(l, r), log_(l));
  }
  static TSI_DEV Iv log_rr(Iv a) { return div(iv(1.0f), a); }
  static TSI_DEV Iv sqrt_rr(Iv a) {
    Iv res = div(iv(1.0f), mul_f(sqrt_(a), 2.0f));
    if (!D) res.hi = fm_min(res.hi, kBIG);
    return res;
  }
  static TSI_DEV void min_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    if (l.hi < r.lo) { o0 = iv(1.0f); o1 = iv(0.0f); }
    else if (r.hi < l.lo) { o0 = iv(0.0f); o1 = iv(1.0f); }
    else if (D) { o0 = Iv{0.0f, 1.0f}; o1 = Iv{0.0f, 1.0f}; }
    else { o0 = iv(1.0f); o1 = iv(1.0f); }
  }
  static TSI_DEV void max_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    if (l.hi < r.lo) { o0 = iv(0.0f); o1 = iv(1.0f); }
    else if (r.hi < l.lo) { o0 = iv(1.0f); o1 = iv(0.0f); }
    else if (D) { o0 = Iv{0.0f, 1.0f}; o1 = Iv{0.0f, 1.0f}; }
    else { o0 = iv(1.0f); o1 = iv(1.0f); }
  }
  static TSI_DEV void div_rr(Iv l, Iv r, Iv &o0, Iv &o1) {
    o0 = div(iv(1.0f), r);
    o1 = neg(div(l, sqr(r)));
  }
  static TSI_DEV float mymod(float x, float y) { return __fsub_rn(x, __fmul_rn(y, floorf(__fdiv_rn(x, y)))); }
  // SIN_I, compute.wgsl:2926-2957 (quadrant method)
  static TSI_DEV Iv sin_(Iv a) {
    const Iv whole = Iv{-1.0f, 1.0f};
    if (!D) {
      if (__fsub_rn(a.hi, a.lo) > kTWOPI) return whole;
      float lo_q = floorf(__fdiv_rn(a.lo, kHALFPI));
      float hi_q = floorf(__fdiv_rn(a.hi, kHALFPI));
      if (__fsub_rn(hi_q, lo_q) > 4.0f) return whole;
      lo_q = mymod(lo_q, 4.0f);
      hi_q = mymod(hi_q, 4.0f);
      if (lo_q == hi_q) {
        if (__fsub_rn(a.hi, a.lo) > kPI) return whole;
        return unordered(fm_sin(a.lo), fm_sin(a.hi));
      } else if ((lo_q == 3.0f && hi_q == 0.0f) || (lo_q == 1.0f && hi_q == 2.0f)) {
        return unordered(fm_sin(a.lo), fm_sin(a.hi));
      } else if ((lo_q == 0.0f || lo_q == 3.0f) && (hi_q == 1.0f || hi_q == 2.0f)) {
        return Iv{fm_min(fm_sin(a.lo), fm_sin(a.hi)), 1.0f};
      } else if ((lo_q == 1.0f || lo_q == 2.0f) && (hi_q == 3.0f || hi_q == 0.0f)) {
        return Iv{-1.0f, fm_max(fm_sin(a.lo), fm_sin(a.hi))};
      }
      return whole;
    }
    // directed: quadrants of a slightly widened interval decide which
    // extrema (+-1 at pi/2 + k pi) the interval may contain
    if (!(a.hi - a.lo <= 3.0f) || !(fabsf(a.lo) < kSinExactArg) || !(fabsf(a.hi) < kSinExactArg)) return whole;
    // the f32 constant pi/2 differs from pi/2 by < 3e-8 relative: a relative
    // margin keeps every true extremum inside the widened quadrant range
    float qlo = floorf(__fdiv_rd(__fsub_rd(a.lo, __fmaf_ru(fabsf(a.lo), 1e-6f, 1e-6f)), kHALFPI));
    float qhi = floorf(__fdiv_ru(__fadd_ru(a.hi, __fmaf_ru(fabsf(a.hi), 1e-6f, 1e-6f)), kHALFPI));
    float slo = fm_sin(a.lo), shi = fm_sin(a.hi);
    // ulp error of the polynomial plus an absolute allowance for the
    // three-part reduction constant (|k| < 2^12 here)
    float lo = __fsub_rd(R::widen_dn(fminf(slo, shi), kElemUlps), 1e-7f);
    float hi = __fadd_ru(R::widen_up(fmaxf(slo, shi), kElemUlps), 1e-7f);
    // maxima at q = 4m+0 -> 4m+1 boundary (pi/2 + 2 m pi), minima at 4m+2 -> 4m+3
    for (float q = qlo; q < qhi; q += 1.0f) {
      float r = q - 4.0f * floorf(q * 0.25f);
      if (r == 0.0f) hi = 1.0f;
      if (r == 2.0f) lo = -1.0f;
    }
    return Iv{fm_max(lo, -1.0f), fm_min(hi, 1.0f)};
  }
  static TSI_DEV Iv cos_(Iv a) {
    if (!D) return sin_(add(a, iv(kHALFPI)));
    // shift by an enclosure of pi/2
    return sin_(Iv{__fadd_rd(a.lo, kHALFPI * 0.99999994f), __fadd_ru(a.hi, kHALFPI * 1.0000001f)});
  }
  // fix, compute.wgsl:3462-3472; directed mode keeps the enclosure
  static TSI_DEV Iv fix(Iv x) {
    // a NaN bound loses against +-BIG in minimumNumber/maximumNumber, which
    // is exactly the reference's NaN -> +-BIG replacement followed by the clamp
    if (!D) return Iv{fm_max(x.lo, -kBIG), fm_min(x.hi, kBIG)};
    return Iv{is_nan_f(x.lo) ? -fm_inf() : x.lo, is_nan_f(x.hi) ? fm_inf() : x.hi};
  }

  // ---- one tape instruction (compute.wgsl:3642-3768) ----
  static TSI_DEV Iv forward(uint32_t h, Iv A, Iv B, float lit) {
    Iv v;
    switch (h) {
      case H_CONST: v = iv(lit); break;
      case H_COPY: v = A; break;
      case H_ADD_II: v = add(A, B); break;
      case H_SUB_II: v = sub(A, B); break;
      case H_MUL_II: v = mul(A, B); break;
      case H_DIV_II: v = div(A, B); break;
      case H_MIN_II: v = min_(A, B); break;
      case H_MAX_II: v = max_(A, B); break;
      case H_POW_II: v = pow_(A, B); break;
      case H_MOD_II: v = mod_(A, B); break;
      case H_ATAN2_II: v = atan2_(A, B); break;
      case H_ADD_IF: v = add_f(A, lit); break;
      case H_SUB_IF: v = sub_f(A, lit); break;
      case H_MUL_IF: v = mul_f(A, lit); break;
      case H_DIV_IF: v = div(A, iv(lit)); break;
      case H_MIN_IF: v = Iv{fm_min(A.lo, lit), fm_min(A.hi, lit)}; break;
      case H_MAX_IF: v = Iv{fm_max(A.lo, lit), fm_max(A.hi, lit)}; break;
      case H_POW_IF: v = pow_(A, iv(lit)); break;
      case H_MOD_IF: v = mod_(A, iv(lit)); break;
      case H_ATAN2_IF: v = atan2_(A, iv(lit)); break;
      case H_SQR: v = sqr(A); break;
      case H_SQRT: v = sqrt_(A); break;
      case H_EXP: v = exp_(A); break;
      case H_LOG: v = log_(A); break;
      case H_NEG: v = neg(A); break;
      case H_ABS: v = abs_(A); break;
      case H_FLOOR: v = floor_(A); break;
      case H_SIN: v = sin_(A); break;
      case H_COS: v = cos_(A); break;
      case H_SUB_FI: v = sub(iv(lit), A); break;
      case H_DIV_FI: v = div(iv(lit), A); break;
      default: v = D ? entire() : iv(-fm_inf()); break;  // unsupported (op, op_top)
    }
    return fix(v);
  }

  // reverse rule of the register operand(s); compute.wgsl:3809-3869,
  // 3890-3920, 3944-3953.  Returns the number of rules written (0, 1, 2).
  static TSI_DEV int reverse_rule(uint32_t h, Iv A, Iv B, float lit, Iv &r0, Iv &r1) {
    switch (h) {
      case H_CONST: return 0;
      case H_COPY: r0 = iv(1.0f); return 1;
      case H_SQR: r0 = mul_f(A, 2.0f); return 1;
      case H_SQRT: r0 = sqrt_rr(A); return 1;
      case H_NEG: r0 = iv(-1.0f); return 1;
      case H_SIN: r0 = cos_(A); return 1;
      case H_COS: r0 = neg(sin_(A)); return 1;
      case H_ADD_IF: r0 = iv(1.0f); return 1;
      case H_SUB_IF: r0 = iv(1.0f); return 1;
      case H_MUL_IF: r0 = iv(lit); return 1;
      case H_DIV_IF: { Iv t; div_rr(A, iv(lit), r0, t); return 1; }
      case H_EXP: r0 = exp_(A); return 1;
      case H_LOG: r0 = log_rr(A); return 1;
      case H_FLOOR: r0 = floor_rr(A); return 1;
      case H_ABS: r0 = abs_rr(A); return 1;
      case H_MIN_IF: { Iv t; min_rr(A, iv(lit), r0, t); return 1; }
      case H_MAX_IF: { Iv t; max_rr(A, iv(lit), r0, t); return 1; }
      case H_POW_IF: { Iv t; pow_rr(A, iv(lit), r0, t); return 1; }
      case H_MOD_IF: r0 = iv(1.0f); return 1;
      case H_ATAN2_IF: { Iv t; atan2_rr(A, iv(lit), r0, t); return 1; }
      case H_BAD_I: r0 = D ? entire() : iv(-fm_inf()); return 1;
      case H_MIN_II: min_rr(A, B, r0, r1); return 2;
      case H_MUL_II: r0 = B; r1 = A; return 2;
      case H_DIV_II: div_rr(A, B, r0, r1); return 2;
      case H_ADD_II: r0 = iv(1.0f); r1 = iv(1.0f); return 2;
      case H_SUB_II: r0 = iv(1.0f); r1 = iv(-1.0f); return 2;
      case H_MAX_II: max_rr(A, B, r0, r1); return 2;
      case H_POW_II: pow_rr(A, B, r0, r1); return 2;
      case H_ATAN2_II: atan2_rr(A, B, r0, r1); return 2;
      case H_MOD_II:  // op_top 0 has no MOD case in the reverse switch (3890-3920)
      case H_BAD_II: r0 = D ? entire() : iv(-fm_inf()); r1 = r0; return 2;
      case H_SUB_FI: r0 = iv(-1.0f); return 1;
      case H_DIV_FI: { Iv t; div_rr(iv(lit), A, t, r0); return 1; }
      default: r0 = D ? entire() : iv(-fm_inf()); return 1;  // H_BAD_FI
    }
  }
};

}  // namespace tsi
