// Correctly rounded asin / sin / cos / exp / integer pow for a variant of the
// reference oracle.  TEST INFRASTRUCTURE ONLY.
//
// The reference calls the host C library for its transcendentals.  That
// library returns the correctly rounded value for almost every argument but
// not for all of them (its asin differs from the correctly rounded value for
// about 1 argument in 1e5 between 1e-4 and 1e-3, the slopes of a sliced bend,
// and 1 in 300 between 3e-3 and 3e-2), and a single-ulp difference grows
// without bound in a chaotic trajectory.  Linked into oracle/_ref/libsimtrack_ref_cr.so (symbols
// bound inside the library), these definitions replace the C library's for
// the reference code only, so that long trajectories of the reference can be
// compared bit for bit with a tracker that uses correctly rounded functions.
// Inside each function's covered domain the value is the double-double
// evaluation of the product's device code (simtrack_b200/csrc/stb_crmath.cuh,
// compiled here for the host); outside it the C library's own function is
// called.
#include <dlfcn.h>

#include <cmath>

#ifndef __CUDACC__
#define __host__
#define __device__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))
#endif
#include "../simtrack_b200/csrc/stb_crmath.cuh"

namespace {

template <class F>
F libm(const char *name) {
  static void *h = dlopen("libm.so.6", RTLD_NOW | RTLD_LOCAL);
  return reinterpret_cast<F>(dlsym(h, name));
}

using fn1 = double (*)(double);
using fn2 = double (*)(double, double);

}  // namespace

extern "C" {

double asin(double x) noexcept {
  static fn1 f = libm<fn1>("asin");
  if (!(std::fabs(x) <= 0.03125)) return f(x);
  return stb::cr_asin(x);
}

double exp(double x) noexcept {
  static fn1 f = libm<fn1>("exp");
  if (x != x || x > 709.7 || x < -708.3) return f(x);
  return stb::cr_exp(x);
}

double sin(double x) noexcept {
  static fn1 f = libm<fn1>("sin");
  if (!(std::fabs(x) < 1048576.0)) return f(x);
  return stb::cr_sin(x);
}

double cos(double x) noexcept {
  static fn1 f = libm<fn1>("cos");
  if (!(std::fabs(x) < 1048576.0)) return f(x);
  return stb::cr_cos(x);
}

double pow(double h, double e) noexcept {
  static fn2 f = libm<fn2>("pow");
  const double m = std::trunc(e);
  if (m == e && std::fabs(m) <= 64 && h > 1e-150 && h < 1e150) return stb::cr_pown(h, (int)m);
  return f(h, e);
}

}  // extern "C"
