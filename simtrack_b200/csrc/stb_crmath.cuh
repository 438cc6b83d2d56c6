// Correctly rounded FP64 elementary functions for the tracking maps.
//
// The reference evaluates asin, sin, cos, exp and pow with the host C
// library.  The library's results are within about half an ulp of the exact
// value, and they are the correctly rounded value for almost every argument.
// A pointwise comparison of chaotic trajectories amplifies any single-ulp
// difference, so the GPU maps use the functions below: each evaluates the
// function in double-double arithmetic (Dekker/Knuth error-free
// transformations, ~2^-100 relative error) from its Taylor series after an
// additive (Cody-Waite) range reduction, then rounds once to double.  The
// result is the correctly rounded value except for arguments whose exact
// image lies within ~2^-100 relative of a rounding boundary.
//
// Domains: cr_asin evaluates the series for |x| <= 2^-5 (every trajectory
// slope a stored particle can have inside an aperture) and defers to CUDA's
// asin outside it; cr_exp covers results in the normal range; cr_sin/cr_cos
// reduce |x| < 2^20.  Outside those domains the CUDA library functions are
// used (error <= 2 ulp).
//
// sin and cos first try a two-step scheme (Ziv's strategy, as in the
// correctly rounded libraries CRlibm and CORE-MATH): a table-driven
// approximation with a proven error bound is accepted when that bound
// decides the rounding, which it does for all but about 2^-15 of the
// arguments; the others take the double-double series.
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

#include "stb_sincos_table.cuh"

namespace stb {

struct dd {
  double hi, lo;
};

__host__ __device__ __forceinline__ dd dd_two_sum(double a, double b) {
  const double s = a + b;
  const double bb = s - a;
  return dd{s, (a - (s - bb)) + (b - bb)};
}
__host__ __device__ __forceinline__ dd dd_fast_two_sum(double a, double b) {  // |a| >= |b|
  const double s = a + b;
  return dd{s, b - (s - a)};
}
__host__ __device__ __forceinline__ dd dd_two_prod(double a, double b) {
  const double p = a * b;
  return dd{p, fma(a, b, -p)};
}
__host__ __device__ __forceinline__ dd dd_add(dd a, dd b) {
  const dd s = dd_two_sum(a.hi, b.hi);
  return dd_fast_two_sum(s.hi, s.lo + (a.lo + b.lo));
}
__host__ __device__ __forceinline__ dd dd_add_d(dd a, double b) {
  const dd s = dd_two_sum(a.hi, b);
  return dd_fast_two_sum(s.hi, s.lo + a.lo);
}
__host__ __device__ __forceinline__ dd dd_mul(dd a, dd b) {
  dd p = dd_two_prod(a.hi, b.hi);
  return dd_fast_two_sum(p.hi, p.lo + (a.hi * b.lo + a.lo * b.hi));
}
__host__ __device__ __forceinline__ dd dd_mul_d(dd a, double b) {
  dd p = dd_two_prod(a.hi, b);
  return dd_fast_two_sum(p.hi, p.lo + a.lo * b);
}
// a / n for a small exact integer n (the remainder of the first quotient is exact).
__host__ __device__ __forceinline__ dd dd_div_small(dd a, double n) {
  const double q1 = a.hi / n;
  const double r = fma(-q1, n, a.hi) + a.lo;
  return dd_fast_two_sum(q1, r / n);
}
__host__ __device__ __forceinline__ dd dd_recip(dd a) {
  const double q1 = 1.0 / a.hi;
  const double r = fma(-q1, a.hi, 1.0) - q1 * a.lo;
  return dd_fast_two_sum(q1, r / a.hi);
}

// asin for |x| <= 2^-5: x + x*t*(c1 + t*(c2 + t*Q(t))), t = x^2, where
// c_k = (2k)! / (4^k (k!)^2 (2k+1)).  c1 and c2 carry their double-double
// tails; the rest of the series contributes below 2^-60 relative and is
// summed in double.
__host__ __device__ inline double cr_asin(double x) {
  if (!(fabs(x) <= 0.03125)) return asin(x);
  const dd t = dd_two_prod(x, x);
  const double c3 = 15.0 / 336.0, c4 = 105.0 / 3456.0, c5 = 945.0 / 42240.0, c6 = 10395.0 / 599040.0,
               c7 = 135135.0 / 9676800.0, c8 = 2027025.0 / 175472640.0;
  const double tail = t.hi * (c3 + t.hi * (c4 + t.hi * (c5 + t.hi * (c6 + t.hi * (c7 + t.hi * c8)))));
  const double c2h = 3.0 / 40.0, c2l = fma(-40.0, c2h, 3.0) / 40.0;
  const double c1h = 1.0 / 6.0, c1l = fma(-6.0, c1h, 1.0) / 6.0;
  dd w = dd_two_sum(c2h, tail);
  w.lo += c2l;
  dd v = dd_two_prod(t.hi, w.hi);
  v.lo += t.hi * w.lo + t.lo * w.hi;
  dd q = dd_two_sum(c1h, v.hi);
  q.lo += c1l + v.lo;
  dd r = dd_two_prod(t.hi, q.hi);
  r.lo += t.hi * q.lo + t.lo * q.hi;
  dd xr = dd_two_prod(x, r.hi);
  xr.lo += x * r.lo;
  dd s = dd_two_sum(x, xr.hi);
  return s.hi + (s.lo + xr.lo);
}

// Double-double reciprocals of the Taylor-series divisors: inv_n(n) = 1/n
// (n = 1..14), inv_cos(j) = 1/((2j-1)(2j)) and inv_sin(j) = 1/((2j)(2j+1))
// (j = 1..13), each split as the rounded value plus its rounded remainder
// (exact rational arithmetic).  The loops below are unrolled, so every
// lookup folds to a constant.
// Multiplying by them in double-double keeps the ~2^-104 relative accuracy
// of dividing by the exact integers, at a fraction of the cost.
__host__ __device__ constexpr dd inv_n(int n) {
  switch (n) {
    case 1: return dd{1.0, 0.0};
    case 2: return dd{0.5, 0.0};
    case 3: return dd{0.3333333333333333, 1.850371707708594e-17};
    case 4: return dd{0.25, 0.0};
    case 5: return dd{0.2, -1.1102230246251566e-17};
    case 6: return dd{0.16666666666666666, 9.25185853854297e-18};
    case 7: return dd{0.14285714285714285, 7.93016446160826e-18};
    case 8: return dd{0.125, 0.0};
    case 9: return dd{0.1111111111111111, 6.1679056923619804e-18};
    case 10: return dd{0.1, -5.551115123125783e-18};
    case 11: return dd{0.09090909090909091, -2.523234146875356e-18};
    case 12: return dd{0.08333333333333333, 4.625929269271485e-18};
    case 13: return dd{0.07692307692307693, -4.270088556250602e-18};
    case 14: return dd{0.07142857142857142, 3.96508223080413e-18};
    default: return dd{0.0, 0.0};
  }
}
// 1/((2j-1)(2j)), the cosine series (j = 1..13: 1/2, 1/12, ..., 1/650)
__host__ __device__ constexpr dd inv_cos(int n) {
  switch (n) {
    case 1: return dd{0.5, 0.0};
    case 2: return dd{0.08333333333333333, 4.625929269271485e-18};
    case 3: return dd{0.03333333333333333, 4.625929269271486e-19};
    case 4: return dd{0.017857142857142856, 9.912705577010326e-19};
    case 5: return dd{0.011111111111111112, -4.2404351634988616e-19};
    case 6: return dd{0.007575757575757576, -2.1026951223961299e-19};
    case 7: return dd{0.005494505494505495, -4.2891514515910067e-19};
    case 8: return dd{0.004166666666666667, 5.782411586589357e-20};
    case 9: return dd{0.0032679738562091504, -9.920804192677818e-20};
    case 10: return dd{0.002631578947368421, 5.934580312552235e-20};
    case 11: return dd{0.0021645021645021645, 1.8774063592822588e-21};
    case 12: return dd{0.0018115942028985507, -2.199830494898125e-20};
    case 13: return dd{0.0015384615384615385, 1.3344026738283131e-21};
    default: return dd{0.0, 0.0};
  }
}
// 1/((2j)(2j+1)), the sine series (j = 1..13: 1/6, 1/20, ..., 1/702)
__host__ __device__ constexpr dd inv_sin(int n) {
  switch (n) {
    case 1: return dd{0.16666666666666666, 9.25185853854297e-18};
    case 2: return dd{0.05, -2.7755575615628915e-18};
    case 3: return dd{0.023809523809523808, 1.32169407693471e-18};
    case 4: return dd{0.013888888888888888, 7.709882115452476e-19};
    case 5: return dd{0.00909090909090909, 4.415659757031872e-19};
    case 6: return dd{0.00641025641025641, 2.2240044563805217e-19};
    case 7: return dd{0.004761904761904762, -4.295505750037808e-19};
    case 8: return dd{0.003676470588235294, 5.102127870520021e-20};
    case 9: return dd{0.0029239766081871343, 1.6231330769373633e-19};
    case 10: return dd{0.002380952380952381, -2.147752875018904e-19};
    case 11: return dd{0.001976284584980237, 1.3370398332627564e-19};
    case 12: return dd{0.0016666666666666668, -1.0697461435190311e-19};
    case 13: return dd{0.0014245014245014246, -7.104458680104445e-20};
    default: return dd{0.0, 0.0};
  }
}

// exp: x = k ln2 + r (double-double reduction), exp(r) = (exp(r/16))^16 with
// exp(r/16) from its Taylor series in double-double Horner form.
static __host__ __device__ __noinline__ double cr_exp(double x) {
  if (x != x) return x;
  if (x > 709.7) return exp(x);
  if (x < -708.3) return exp(x);  // subnormal or zero results
  const double L1 = 0.6931471805599453094;     // ln 2 rounded to double
  const double L2 = 2.319046813846299558e-17;  // ln 2 - L1
  const double k = rint(x * 1.4426950408889634074);
  const dd p = dd_two_prod(k, L1);
  dd r = dd_two_sum(x, -p.hi);
  r = dd_fast_two_sum(r.hi, (r.lo - p.lo) - k * L2);
  const dd s{r.hi * 0.0625, r.lo * 0.0625};
  // e = exp(s) = 1 + s(1 + s/2(1 + s/3(... (1 + s/14))))
  dd e{1.0, 0.0};
#pragma unroll
  for (int n = 14; n >= 1; n--) {
    e = dd_mul(dd_mul(e, s), inv_n(n));  // e * s / n
    e = dd_add_d(e, 1.0);
  }
  for (int i = 0; i < 4; i++) e = dd_mul(e, e);
  return ldexp(e.hi + e.lo, (int)k);
}

// sin/cos: x = k pi/2 + r with pi/2 split in three parts, then the Taylor
// series of sin(r) and cos(r), |r| <= pi/4, in double-double.
static __host__ __device__ __noinline__ void cr_sincos_reduced(double x, dd &sr, dd &cr, int &quad) {
  const double P1 = 1.5707963267948966192;     // pi/2 rounded to double
  const double P2 = 6.123233995736766036e-17;  // next part of pi/2
  const double P3 = -1.4973849048591698e-33;   // remainder
  const double k = rint(x * 0.63661977236758134308);
  const dd a = dd_two_prod(k, P1);
  const dd b = dd_two_prod(k, P2);
  dd r = dd_two_sum(x, -a.hi);
  r = dd_add(r, dd{-a.lo, 0.0});
  r = dd_add(r, dd{-b.hi, -b.lo});
  r = dd_add_d(r, -k * P3);
  const dd r2 = dd_mul(r, r);
  // Terms kept: all 13 for |r| up to pi/4.  For |r| < 2^-4 the first
  // neglected term (r^18/19! resp. r^20/20!) is below 2^-128 relative, so 8
  // resp. 9 terms suffice; for |r| < 2^-7, 6 and 6 (first neglected term
  // below 2^-112).
  const double ar = fabs(r.hi);
  const int jmax_s = ar < 0.0078125 ? 6 : ar < 0.0625 ? 8 : 13;
  const int jmax_c = ar < 0.0078125 ? 6 : ar < 0.0625 ? 9 : 13;
  // sin r = r (1 - r^2/(2*3) (1 - r^2/(4*5) (...)))
  dd s{1.0, 0.0};
#pragma unroll
  for (int j = 13; j >= 1; j--) {
    if (j <= jmax_s) {
      s = dd_mul(dd_mul(r2, s), inv_sin(j));
      s = dd_add_d(dd{-s.hi, -s.lo}, 1.0);
    }
  }
  sr = dd_mul(r, s);
  // cos r = 1 - r^2/(1*2) (1 - r^2/(3*4) (...))
  dd c{1.0, 0.0};
#pragma unroll
  for (int j = 13; j >= 1; j--) {
    if (j <= jmax_c) {
      c = dd_mul(dd_mul(r2, c), inv_cos(j));
      c = dd_add_d(dd{-c.hi, -c.lo}, 1.0);
    }
  }
  cr = c;
  quad = ((int)fmod(k, 4.0) + 4) & 3;
}

// Table of the fast sin/cos path, [sin(i pi/128) hi, lo, cos(i pi/128) hi,
// lo] for i = 0..63: one copy in device memory (read through the read-only
// cache), one for host builds of the same functions.
__device__ const double kSinCosTabDev[256] = STB_SINCOS_TABLE_INIT;
static const double kSinCosTabHost[256] = STB_SINCOS_TABLE_INIT;

__host__ __device__ __forceinline__ uint64_t dbl_bits(double v) {
#ifdef __CUDA_ARCH__
  return (uint64_t)__double_as_longlong(v);
#else
  uint64_t u;
  memcpy(&u, &v, sizeof u);
  return u;
#endif
}
__host__ __device__ __forceinline__ double bits_dbl(uint64_t u) {
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)u);
#else
  double v;
  memcpy(&v, &u, sizeof v);
  return v;
#endif
}

// True when every real number within 2^-70 |y.hi| of y.hi + y.lo rounds to
// y.hi (y normalised: y.hi = RN(y.hi + y.lo)).  Half the gap to the next
// double is 2^(e-53) for y.hi in [2^e, 2^(e+1)), half of that below a power
// of two.  Tiny, zero and non-finite values are left to the slow path.
__host__ __device__ __forceinline__ bool rounding_decided(dd y) {
  const uint64_t u = dbl_bits(y.hi);
  const int e = (int)((u >> 52) & 0x7ff);
  if (e < 60 || e == 0x7ff) return false;
  double half = bits_dbl((uint64_t)(e - 53) << 52);
  if ((u & 0xfffffffffffffull) == 0) half *= 0.5;
  return fabs(y.lo) + fabs(y.hi) * 0x1p-70 < half;
}

// Fast path of sin and cos, |x| < 800.  x = k pi/128 + r with the constant
// in three parts (x - k A is exact, k B is exact, k C is rounded once):
// |r| <= pi/256 (1 + 2^-30) and r is a double-double with absolute error
// below 2^-112, i.e. 2^-78 relative when |r| >= 2^-34 (smaller r with
// k != 0 go to the slow path).  With j = k mod 256, q = j / 64 (the
// quadrant) and a = (j mod 64) pi/128:
//   sin(a + r) = S cos r + C sin r,   cos(a + r) = C cos r - S sin r,
// S, C from the table; cos r - 1 and sin r - r from their Taylor series
// through r^10 and r^11 (truncation below 2^-100 relative), the leading
// terms r^2/2 and r^3/6 in double-double, the rest in double (relative error
// of those tails below 2^-50, i.e. 2^-80 of cos r and sin r).  For a >= pi/128
// both results are >= sin(pi/256), so the sums do not cancel; for a = 0 the
// expressions reduce exactly to sin r and cos r.  Each double-double result
// is within 2^-77 relative of the exact value; rounding_decided() allows
// 2^-70.  False when it does not decide either rounding.
__host__ __device__ __forceinline__ bool sincos_fast(double x, double &sn, double &cs) {
  if (!(fabs(x) < 800.0)) return false;
  const double k = rint(x * kPi128Inv);
  dd r = dd_two_sum(fma(-k, kPi128A, x), -k * kPi128B);
  if (k != 0.0 && !(fabs(r.hi) >= 0x1p-34)) return false;
  r = dd_fast_two_sum(r.hi, fma(-k, kPi128C, r.lo));
  const int j = (int)k & 255, i = j & 63;
#ifdef __CUDA_ARCH__
  const double *T = kSinCosTabDev + 4 * i;
  const double Sh = __ldg(T), Sl = __ldg(T + 1), Ch = __ldg(T + 2), Cl = __ldg(T + 3);
#else
  const double *T = kSinCosTabHost + 4 * i;
  const double Sh = T[0], Sl = T[1], Ch = T[2], Cl = T[3];
#endif
  // r^2 = t.hi + t.lo
  dd t = dd_two_prod(r.hi, r.hi);
  t.lo = fma(r.hi + r.hi, r.lo, t.lo);
  const double th = t.hi;
  // cos r = 1 - r^2/2 + r^4 (1/24 - r^2/720 + r^4/40320 - r^6/3628800)
  const double qc = fma(th, fma(th, fma(th, -1.0 / 3628800.0, 1.0 / 40320.0), -1.0 / 720.0), 1.0 / 24.0);
  dd cr = dd_fast_two_sum(1.0, -0.5 * th);
  cr.lo = cr.lo + fma(th * th, qc, -0.5 * t.lo);
  // sin r = r + r^3 (-1/6 + r^2/120 - r^4/5040 + r^6/362880 - r^8/39916800)
  const double c1h = -0.16666666666666666, c1l = -9.25185853854297e-18;  // -1/6 = c1h + c1l
  const double pl =
      c1l + th * fma(th, fma(th, fma(th, -1.0 / 39916800.0, 1.0 / 362880.0), -1.0 / 5040.0), 1.0 / 120.0);
  dd rt = dd_two_prod(r.hi, th);  // r^3
  rt.lo = rt.lo + fma(r.hi, t.lo, r.lo * th);
  dd sm = dd_two_prod(rt.hi, c1h);
  sm.lo = sm.lo + fma(rt.hi, pl, rt.lo * c1h);
  dd sr = dd_fast_two_sum(r.hi, sm.hi);
  sr.lo = sr.lo + (r.lo + sm.lo);
  // S cos r + C sin r
  dd a = dd_two_prod(Sh, cr.hi);
  a.lo = a.lo + fma(Sh, cr.lo, Sl * cr.hi);
  dd b = dd_two_prod(Ch, sr.hi);
  b.lo = b.lo + fma(Ch, sr.lo, Cl * sr.hi);
  dd s = dd_two_sum(a.hi, b.hi);
  s = dd_fast_two_sum(s.hi, s.lo + (a.lo + b.lo));
  // C cos r - S sin r
  dd c = dd_two_prod(Ch, cr.hi);
  c.lo = c.lo + fma(Ch, cr.lo, Cl * cr.hi);
  dd d = dd_two_prod(Sh, sr.hi);
  d.lo = d.lo + fma(Sh, sr.lo, Sl * sr.hi);
  dd e = dd_two_sum(c.hi, -d.hi);
  e = dd_fast_two_sum(e.hi, e.lo + (c.lo - d.lo));
  if (!(rounding_decided(s) && rounding_decided(e))) return false;
  const int q = j >> 6;
  const double sv = s.hi, cv = e.hi;
  if (q == 0) { sn = sv; cs = cv; }
  else if (q == 1) { sn = cv; cs = -sv; }
  else if (q == 2) { sn = -sv; cs = -cv; }
  else { sn = -cv; cs = sv; }
  return true;
}

__host__ __device__ inline double cr_sin(double x) {
  double fs, fc;
  if (sincos_fast(x, fs, fc)) return fs;
  if (!(fabs(x) < 1048576.0)) return sin(x);
  dd s, c;
  int q;
  cr_sincos_reduced(x, s, c, q);
  if (q == 0) return s.hi + s.lo;
  if (q == 1) return c.hi + c.lo;
  if (q == 2) return -(s.hi + s.lo);
  return -(c.hi + c.lo);
}

// sin and cos of the same argument from one reduction, by the double-double
// series alone.
__host__ __device__ inline void cr_sincos_series(double x, double &sn, double &cs) {
  if (!(fabs(x) < 1048576.0)) {
    sn = sin(x);
    cs = cos(x);
    return;
  }
  dd s, c;
  int q;
  cr_sincos_reduced(x, s, c, q);
  const double sv = s.hi + s.lo, cv = c.hi + c.lo;
  if (q == 0) { sn = sv; cs = cv; }
  else if (q == 1) { sn = cv; cs = -sv; }
  else if (q == 2) { sn = -sv; cs = -cv; }
  else { sn = -cv; cs = sv; }
}

__host__ __device__ inline void cr_sincos(double x, double &sn, double &cs) {
  if (sincos_fast(x, sn, cs)) return;
  cr_sincos_series(x, sn, cs);
}

__host__ __device__ inline double cr_cos(double x) {
  double fs, fc;
  if (sincos_fast(x, fs, fc)) return fc;
  if (!(fabs(x) < 1048576.0)) return cos(x);
  dd s, c;
  int q;
  cr_sincos_reduced(x, s, c, q);
  if (q == 0) return c.hi + c.lo;
  if (q == 1) return -(s.hi + s.lo);
  if (q == 2) return -(c.hi + c.lo);
  return s.hi + s.lo;
}

// h^m for an integer m (|m| <= 64): binary powering in double-double, one
// final rounding.
static __host__ __device__ __noinline__ double cr_pown(double h, int m) {
  if (m == 0) return 1.0;
  if (!(h > 0.0) || !(h < 1e150) || !(h > 1e-150)) return pow(h, (double)m);
  int e = m < 0 ? -m : m;
  if (e > 64) return pow(h, (double)m);
  dd base{h, 0.0}, acc{1.0, 0.0};
  while (e) {
    if (e & 1) acc = dd_mul(acc, base);
    e >>= 1;
    if (e) base = dd_mul(base, base);
  }
  if (m < 0) acc = dd_recip(acc);
  return acc.hi + acc.lo;
}

}  // namespace stb
