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
#pragma once
#include <cmath>

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
  for (int n = 14; n >= 1; n--) {
    e = dd_div_small(dd_mul(e, s), (double)n);
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
  // sin r = r (1 - r^2/(2*3) (1 - r^2/(4*5) (...)))
  dd s{1.0, 0.0};
  for (int n = 26; n >= 2; n -= 2) {
    s = dd_div_small(dd_mul(r2, s), (double)(n * (n + 1)));
    s = dd_add_d(dd{-s.hi, -s.lo}, 1.0);
  }
  sr = dd_mul(r, s);
  // cos r = 1 - r^2/(1*2) (1 - r^2/(3*4) (...))
  dd c{1.0, 0.0};
  for (int n = 25; n >= 1; n -= 2) {
    c = dd_div_small(dd_mul(r2, c), (double)(n * (n + 1)));
    c = dd_add_d(dd{-c.hi, -c.lo}, 1.0);
  }
  cr = c;
  quad = ((int)fmod(k, 4.0) + 4) & 3;
}

__host__ __device__ inline double cr_sin(double x) {
  if (!(fabs(x) < 1048576.0)) return sin(x);
  dd s, c;
  int q;
  cr_sincos_reduced(x, s, c, q);
  if (q == 0) return s.hi + s.lo;
  if (q == 1) return c.hi + c.lo;
  if (q == 2) return -(s.hi + s.lo);
  return -(c.hi + c.lo);
}

__host__ __device__ inline double cr_cos(double x) {
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
