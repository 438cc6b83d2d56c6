// Correctly rounded asin / sin / cos / exp / pow for a variant of the
// reference oracle.  TEST INFRASTRUCTURE ONLY.
//
// The reference calls the host C library for its transcendentals.  That
// library returns the correctly rounded value for almost every argument but
// not for all of them (its asin differs from the correctly rounded value for
// about 1 argument in 1e5 between 1e-4 and 1e-3, the slopes of a sliced bend,
// and 1 in 300 between 3e-3 and 3e-2), and a single-ulp difference grows
// without bound in a chaotic trajectory.  Linked into
// oracle/_ref/libsimtrack_ref_cr.so (symbols bound inside the library), these
// definitions replace the C library's for the reference code only, so that
// long trajectories of the reference can be compared bit for bit with a
// tracker that uses correctly rounded functions.
//
// Method (independent of the tracker's own double-double code): evaluate in
// x87 extended precision (64-bit significand) with the C library's long
// double function, whose error is a few extended ulps; round that to double.
// The rounding is provably correct when the extended value lies more than
// kGuard extended ulps from the double rounding midpoint next to it.  Else
// evaluate again in binary128 (libquadmath, 113-bit significand) and apply
// the same test with kGuard binary128 ulps.  An argument that fails both
// tests (expected never: it needs the exact value within ~2^-105 relative of
// a midpoint) is counted in stb_crshim_unresolved() and gets the binary128
// rounding.
#include <quadmath.h>

#include <cmath>

namespace {

constexpr int kGuard = 8;  // error allowance in units of the wide format's ulp
long g_unresolved = 0;
long g_quad_calls = 0;

// RN(v) if it is certain that the exact value (|exact - v| <= kGuard ulps of
// v's format) rounds to it; `ok` false otherwise.
template <class W>
double round_checked(W v, int wide_digits, bool &ok) {
  const double d = (double)v;
  ok = true;
  if (!std::isfinite(d) || v == (W)d) return d;
  const double other = std::nextafter(d, v > (W)d ? INFINITY : -INFINITY);
  if (!std::isfinite(other)) return d;
  const W mid = ((W)d + (W)other) / 2;  // exact: the midpoint has one more bit than a double
  W ulp;
  if constexpr (sizeof(W) == sizeof(__float128)) {
    ulp = ldexpq(1, ilogbq(v) - (wide_digits - 1));
  } else {
    ulp = std::ldexp((W)1, std::ilogb(v) - (wide_digits - 1));
  }
  const W dist = v > mid ? v - mid : mid - v;
  ok = dist > (W)kGuard * ulp;
  return d;
}

template <class FL, class FQ>
double cr_eval(FL fl, FQ fq) {
  bool ok;
  const double d = round_checked<long double>(fl(), 64, ok);
  if (ok) return d;
  g_quad_calls++;
  const double q = round_checked<__float128>(fq(), 113, ok);
  if (!ok) g_unresolved++;
  return q;
}

}  // namespace

extern "C" {

double asin(double x) noexcept {
  return cr_eval([&] { return asinl((long double)x); }, [&] { return asinq((__float128)x); });
}

double exp(double x) noexcept {
  return cr_eval([&] { return expl((long double)x); }, [&] { return expq((__float128)x); });
}

double sin(double x) noexcept {
  return cr_eval([&] { return sinl((long double)x); }, [&] { return sinq((__float128)x); });
}

double cos(double x) noexcept {
  return cr_eval([&] { return cosl((long double)x); }, [&] { return cosq((__float128)x); });
}

double pow(double h, double e) noexcept {
  return cr_eval([&] { return powl((long double)h, (long double)e); },
                 [&] { return powq((__float128)h, (__float128)e); });
}

// Evaluation entry for tests: fn 0 asin, 1 exp, 2 sin, 3 cos, 4 pow(x, y).
double stb_crshim_eval(int fn, double x, double y) {
  switch (fn) {
    case 0: return asin(x);
    case 1: return exp(x);
    case 2: return sin(x);
    case 3: return cos(x);
    case 4: return pow(x, y);
    default: return NAN;
  }
}

// Arguments whose rounding neither the extended nor the binary128 evaluation
// could decide, and how many needed the binary128 evaluation.
long stb_crshim_unresolved(void) { return g_unresolved; }
long stb_crshim_quad_calls(void) { return g_quad_calls; }

}  // extern "C"
