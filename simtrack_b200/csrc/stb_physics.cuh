// Per-element particle maps executed by the tracking kernel.
//
// Each map restates one reference pass function (simtrack.cpp line cited per
// function) with the particle held in registers.  Operand order matches the
// reference expression by expression and this translation unit is compiled
// with -fmad=false, so every +, -, *, / and sqrt rounds exactly as in the
// reference's x86-64 build.  The transcendentals (asin, sin, cos, exp, pow)
// are the correctly rounded versions of stb_crmath.cuh, which agree with the
// host C library's results except on rare arguments where the library itself
// is not correctly rounded.
//
// Quantities that depend only on pt (delta, gamma, beta of the particle) are
// held in a PtCache and recomputed only when an element changes pt (RF,
// crab cavities, beam-beam, Lorentz boosts).  The reference recomputes them
// inside every DRIFT_Pass; the values are identical because kicks and drifts
// never modify pt.
//
// Divisions.  A quotient a/b whose divisor b is reused (an element constant,
// a pt-only quantity, or a value shared by several quotients of one map) is
// formed from y = RN(1/b), computed once by an IEEE division, as
//   q0 = RN(a*y),  r = a - b*q0 (exact, one FMA),  q = RN(q0 + r*y),
// Markstein's correction step (P. Markstein, IBM J. Res. Dev. 34 (1990) 111).
// q is the correctly rounded a/b unless a/b lies within about 2^-52 ulp of a
// rounding midpoint (probability ~2^-50 per quotient), so it reproduces the
// reference's IEEE division while costing one multiply and two FMAs instead
// of a full division sequence.  Operands stay far from overflow/underflow.
#pragma once
#include <cstdint>

#include "stb_crmath.cuh"
#include "stb_rng.cuh"
#include "stb_table.hpp"

namespace stb {

struct Particle {
  double x, px, y, py, z, pt;
};

struct PtCache {
  double opd;     // 1.0 + delta1
  double opd2;    // (1.0 + delta1) * (1.0 + delta1)
  double beta1;   // particle velocity / c
  double iopd;    // RN(1 / opd)
  double ibeta1;  // RN(1 / beta1)
  double opd_ibeta1;  // RN(opd * ibeta1), for 1/betaz in the drift
};

// RN(a * b), a product that no contraction policy fuses into an FMA.
__host__ __device__ __forceinline__ double mul_rn(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);  // never contracted into an FMA, whatever the unit's flags
#else
  return a * b;
#endif
}

// a / b given y = RN(1/b) (see the division note above).
__device__ __forceinline__ double qdiv(double a, double b, double y) {
  const double q0 = __dmul_rn(a, y);
  const double r = fma(-q0, b, a);
  return fma(r, y, q0);
}

// delta1/gamma1/beta1 exactly as DRIFT_Pass computes them (simtrack.cpp:3755-3757).
__device__ __forceinline__ void pt_refresh(const RefConsts &R, double pt, PtCache &c) {
  const double delta1 = sqrt(1.0 + 2 * pt / R.beta + pt * pt) - 1.0;
  const double gamma1 = R.gamma + R.sqrt_g2m1 * pt;
  c.beta1 = sqrt(1.0 - 1.0 / gamma1 / gamma1);
  c.opd = 1.0 + delta1;
  c.opd2 = c.opd * c.opd;
  c.iopd = 1.0 / c.opd;
  c.ibeta1 = 1.0 / c.beta1;
  c.opd_ibeta1 = mul_rn(c.opd, c.ibeta1);
}

// Square root and reciprocal of a drift from the cached seed.  With
// v = (1+delta1)^2 - px^2 - py^2 and y0 = RN(1/(1+delta1)), y0 is within
// e0 = (px^2 + py^2) / (2 (1+delta1)^2) relative of 1/sqrt(v).  Newton steps
// for the reciprocal square root in FMA form, y <- y + (y/2)(1 - v y^2),
// square the error (times 3/2): one step suffices when |px| and |py| are below
// kSeedSlope1 (e0 <= 6.4e-7, then 2^-40), a second one up to kSeedSlope2
// (e0 <= 5e-5).  The square root s = RN(v y) is then corrected once with its
// exact remainder, s + (v - s^2) y/2 (Markstein's square-root step, IBM J.
// Res. Dev. 34 (1990) 111), and the reciprocal once with its remainder,
// y + y (1 - s y).  Both are the correctly rounded values unless the exact
// one lies within about 2^-50 ulp of a rounding midpoint (the same order as
// qdiv above); they are checked against IEEE sqrt and division on random
// drift arguments on the host and on the GPU.  Steeper slopes return false:
// the caller then takes IEEE sqrt and division.  10 or 14 FP64 operations and
// no MUFU, where sqrt and a reciprocal cost two MUFU seeds and two Newton
// sequences with range checks.  The step count is chosen per lane; the lanes
// of a warp usually agree, so the branch rarely diverges.
constexpr double kSeedSlope1 = 8e-4;
constexpr double kSeedSlope2 = 7e-3;

__host__ __device__ __forceinline__ bool seeded_sqrt_recip(double v, double y0, double px, double py, double &s,
                                                           double &is) {
  const double apx = fabs(px), apy = fabs(py);
  if (!(apx < kSeedSlope2 && apy < kSeedSlope2)) return false;
  double y = y0;
  {
    const double t = mul_rn(v, y);
    const double e = fma(-t, y, 1.0);
    y = fma(mul_rn(0.5, y), e, y);
  }
  if (!(apx < kSeedSlope1 && apy < kSeedSlope1)) {
    const double t = mul_rn(v, y);
    const double e = fma(-t, y, 1.0);
    y = fma(mul_rn(0.5, y), e, y);
  }
  const double s0 = mul_rn(v, y);
  const double d = fma(-s0, s0, v);
  s = fma(d, mul_rn(0.5, y), s0);
  is = fma(y, fma(-s, y, 1.0), y);
  return true;
}

// a / b with y within a few ulp of 1/b (here a product of correctly rounded
// reciprocals): q0 = RN(a y) and one correction with the exact remainder,
// correctly rounded unless a/b lies within about 2^-48 ulp of a rounding
// midpoint.
__host__ __device__ __forceinline__ double qdiv_near(double a, double b, double y) {
  const double q0 = mul_rn(a, y);
  const double r = fma(-q0, b, a);
  return fma(r, y, q0);
}

// The divisions and square root of DRIFT_Pass's exact branch: pz =
// sqrt((1+delta1)^2 - px^2 - py^2), 1/pz, betaz = pz*beta1/(1+delta1) and
// L/betaz.  The reciprocal of betaz is ((1+delta1)/beta1) * (1/pz) from the
// cached RN((1+delta1) * RN(1/beta1)), within ~2.5 ulp.
__host__ __device__ __forceinline__ void drift_quotients(double opd, double opd2, double beta1, double iopd,
                                                         double opd_ibeta1, double px, double py, double L,
                                                         double &pz, double &ipz, double &betaz, double &L_betaz) {
  const double v = opd2 - px * px - py * py;
  if (seeded_sqrt_recip(v, iopd, px, py, pz, ipz)) {
    const double t = mul_rn(pz, beta1);
    betaz = qdiv_near(t, opd, iopd);
    L_betaz = qdiv_near(L, betaz, mul_rn(opd_ibeta1, ipz));
  } else {
    pz = sqrt(v);
    ipz = 1.0 / pz;
    const double t = mul_rn(pz, beta1);
    betaz = qdiv_near(t, opd, iopd);
    L_betaz = L / betaz;
  }
}

// The increments of one drift: x += dx, y += dy, z -= dz.
struct DriftStep {
  double dx, dy, dz;
};

// A drift's increments depend on px, py, pt and L only, none of which the
// drift changes: a second drift of the same length with no kick between
// (the last drift of a Yoshida slice and the first of the next one) adds the
// very same three values, so it can reuse them (drift_again) and round
// exactly as the reference's recomputation does.
__device__ __forceinline__ DriftStep drift_step(const Particle &p, const PtCache &c, double L, double Lb) {
  double pz, ipz, betaz, L_betaz;
  drift_quotients(c.opd, c.opd2, c.beta1, c.iopd, c.opd_ibeta1, p.px, p.py, L, pz, ipz, betaz, L_betaz);
  return DriftStep{qdiv(p.px * L, pz, ipz), qdiv(p.py * L, pz, ipz), L_betaz - Lb};
}

__device__ __forceinline__ void drift_again(Particle &p, const DriftStep &d) {
  p.x = p.x + d.dx;
  p.y = p.y + d.dy;
  p.z = p.z - d.dz;
}

// DRIFT_Pass exact branch, simtrack.cpp:3759-3764.  L and Lb = L/GP.beta.
// The two quotients by pz share one reciprocal; (pz*beta1)/(1+delta1) uses
// the cached reciprocal of 1+delta1.
__device__ __forceinline__ DriftStep drift(Particle &p, const PtCache &c, double L, double Lb) {
  const DriftStep d = drift_step(p, c, L, Lb);
  drift_again(p, d);
  return d;
}

// sbend_exact_pass, simtrack.cpp:3833-3858.  B = [L, L/beta, href, 1/href, cosA, sinA].
// Every quotient by href uses the element's RN(1/href); the two arcsine
// arguments share RN(1/temp); temp/beta uses the cached RN(1/beta1).
__device__ __forceinline__ void bend_exact(Particle &p, const PtCache &c, const double *B) {
  const double L = B[0], Lb = B[1], href = B[2], invh = B[3], cosA = B[4], sinA = B[5];
  const double x0 = p.x, px0 = p.px, py0 = p.py;
  const double pz0 = sqrt(c.opd2 - px0 * px0 - py0 * py0);
  const double npx = px0 * cosA + (pz0 - 1. - href * x0) * sinA;
  const double pz1 = sqrt(c.opd2 - npx * npx - py0 * py0);
  const double der = (-px0) * sinA * href + (pz0 - 1. - x0 * href) * cosA * href;
  p.x = qdiv(pz1, href, invh) - qdiv(qdiv(der, href, invh), href, invh) - invh;
  double temp, itemp;
  if (!seeded_sqrt_recip(c.opd2 - py0 * py0, c.iopd, 0.0, py0, temp, itemp)) {
    temp = sqrt(c.opd2 - py0 * py0);
    itemp = 1.0 / temp;
  }
  const double as1 = cr_asin(qdiv(px0, temp, itemp));
  const double as2 = cr_asin(qdiv(npx, temp, itemp));
  const double das = as1 - as2;
  p.y = p.y + py0 * L + qdiv(py0 * das, href, invh);
  const double t2 = c.opd * L + qdiv(c.opd * das, href, invh);
  p.z = p.z - (qdiv(t2, c.beta1, c.ibeta1) - Lb);
  p.px = npx;
}

// general_sbend_exact_pass, simtrack.cpp:3974-4010.
// G = [L, L/beta, rhoc, b0, b0*rhoc, cosA, sinA, 1/rhoc, 1/b0]
static __device__ __forceinline__ void gbend_exact(Particle &p, const PtCache &c, const double *G) {
  const double L = G[0], Lb = G[1], rhoc = G[2], b0 = G[3], b0r = G[4], cosA = G[5], sinA = G[6];
  const double irhoc = G[7], ib0 = G[8];
  const double x0 = p.x, px0 = p.px, py0 = p.py;
  const double pz0 = sqrt(c.opd2 - px0 * px0 - py0 * py0);
  const double w = pz0 - b0r - b0 * x0;
  const double npx = px0 * cosA + w * sinA;
  const double pz1 = sqrt(c.opd2 - npx * npx - py0 * py0);
  const double der = qdiv((-px0) * sinA, rhoc, irhoc) + qdiv(w * cosA, rhoc, irhoc);
  p.x = qdiv(pz1, b0, ib0) - qdiv(der * rhoc, b0, ib0) - rhoc;
  const double temp = sqrt(c.opd2 - py0 * py0);
  const double itemp = 1.0 / temp;
  const double as1 = cr_asin(qdiv(px0, temp, itemp));
  const double as2 = cr_asin(qdiv(npx, temp, itemp));
  const double das = as1 - as2;
  p.y = p.y + qdiv(qdiv(py0 * L, b0, ib0), rhoc, irhoc) + qdiv(py0 * das, b0, ib0);
  const double t2 = qdiv(qdiv(c.opd * L, b0, ib0), rhoc, irhoc) + qdiv(c.opd * das, b0, ib0);
  p.z = p.z - (qdiv(t2, c.beta1, c.ibeta1) - Lb);
  p.px = npx;
}

// quad_kick_pass, simtrack.cpp:4046-4058
__device__ __forceinline__ void quad_kick(Particle &p, double kl, double ksl) {
  const double Bx = ksl * p.x + kl * p.y;
  const double By = kl * p.x - ksl * p.y;
  p.px = p.px - By;
  p.py = p.py + Bx;
}

// sext_kick_pass, simtrack.cpp:4060-4071
__device__ __forceinline__ void sext_kick(Particle &p, double kl, double ksl) {
  const double pr = p.x * p.x - p.y * p.y;
  const double pi = 2. * p.x * p.y;
  // x / 2. and x * 0.5 are the same exact scaling (also for subnormal results)
  const double Bx = (ksl * pr + kl * pi) * 0.5;
  const double By = (kl * pr - ksl * pi) * 0.5;
  p.px = p.px - By;
  p.py = p.py + Bx;
}

// oct_kick_pass, simtrack.cpp:4073-4084
__device__ __forceinline__ void oct_kick(Particle &p, double kl, double ksl) {
  const double pr = p.x * p.x * p.x - 3 * p.x * p.y * p.y;
  const double pi = 3 * p.x * p.x * p.y - p.y * p.y * p.y;
  const double Bx = qdiv(ksl * pr + kl * pi, 6., 1. / 6.);
  const double By = qdiv(kl * pr - ksl * pi, 6., 1. / 6.);
  p.px = p.px - By;
  p.py = p.py + Bx;
}

// mult_kick_pass, simtrack.cpp:4086-4111.  K = [KNL0, KNSL0, (KNLi, KNSLi, 1/i!) i=1..norder]
__device__ __forceinline__ void mult_kick(Particle &p, int norder, const double *K) {
  double Xn = 1., Yn = 0.;
  double By = K[0], Bx = K[1];
  double fac = 1.;
#pragma unroll 1
  for (int i = 1; i <= norder; i++) {
    const double Xn0 = Xn, Yn0 = Yn;
    Xn = Xn0 * p.x - Yn0 * p.y;
    Yn = Xn0 * p.y + Yn0 * p.x;
    fac = fac * (double)i;
    const double kn = K[3 * i - 1], ks = K[3 * i], ifac = K[3 * i + 1];
    if (kn != 0. || ks != 0.) {
      By = By + qdiv(kn * Xn - ks * Yn, fac, ifac);
      Bx = Bx + qdiv(kn * Yn + ks * Xn, fac, ifac);
    }
  }
  p.px = p.px - By;
  p.py = p.py + Bx;
}

// Field sum of cal_Bfield (simtrack.cpp:4169-4196) at (x, y) for the
// multipole block K = [KNL0, KNSL0, (KNLi, KNSLi, 1/i!) i = 1..norder] of the
// element's own strengths: By + i Bx, the divisions by i! exact IEEE ones as
// in the reference (an integer factorial converted to double).
__device__ __forceinline__ void bfield_sum(double x, double y, int norder, const double *K, double &By, double &Bx) {
  double Xn = 1., Yn = 0.;
  By = K[0];
  Bx = K[1];
  double fac = 1.;
#pragma unroll 1
  for (int i = 1; i <= norder; i++) {
    const double Xn0 = Xn, Yn0 = Yn;
    Xn = Xn0 * x - Yn0 * y;
    Yn = Xn0 * y + Yn0 * x;
    fac = fac * (double)i;
    const double kn = K[3 * i - 1], ks = K[3 * i];
    if (kn != 0. || ks != 0.) {
      By = By + (kn * Xn - ks * Yn) / fac;
      Bx = Bx + (kn * Yn + ks * Xn) / fac;
    }
  }
}

// Synchrotron radiation over one integration step: radiate()
// (simtrack.cpp:4198-4234) and, with `quantum`, radiate1() (4236-4288),
// whose fluctuation term takes the normal deviate `gauss`.  L: the step's
// length on the reference orbit; href: the reference orbit's curvature;
// (B0, B1, B2): the field integrated over the step over (B rho)_0; E3 =
// pow(GP.energy/1000, 3) and Cf (simtrack.cpp:26) from the host.  Every
// operation is the reference's, in its order, with IEEE division and square
// root; the pt cache is refreshed for the new pt.
constexpr double kCr = 8.84627632682e-5;          // simtrack.cpp:25
constexpr double kRadPI = 3.14159265358979323;    // PI, simtrack.cpp:23
constexpr double kSpeedLight = 299792458.;        // speed_light, simtrack.cpp:24
__device__ __forceinline__ void radiate_step(Particle &p, PtCache &c, const RefConsts &R, double L, double href,
                                             double B0, double B1, double B2, double E3, bool quantum, double Cf,
                                             double gauss) {
  const double px0 = p.px, py0 = p.py, pt0 = p.pt;
  const double pz = sqrt(c.opd2 - p.px * p.px - p.py * p.py);
  const double xp = (1 + p.x * href) * p.px / pz;
  const double yp = (1 + p.x * href) * p.py / pz;
  const double temp1 = sqrt((1 + p.x * href) * (1 + p.x * href) + xp * xp + yp * yp);
  const double u0 = xp / temp1, u1 = yp / temp1, u2 = (1 + p.x * href) / temp1;
  // vector_cross_product(BLbrho, u, BLper), simtrack.cpp:1639-1644
  const double b0 = B1 * u2 - B2 * u1;
  const double b1 = -1.0 * B0 * u2 + B2 * u0;
  const double b2 = B0 * u1 - B1 * u0;
  const double bper2 = b0 * b0 + b1 * b1 + b2 * b2;
  const double temp2 = kCr * c.opd * c.opd * E3 / 2 / kRadPI;
  if (quantum) {
    const double ptloss = temp2 * bper2 * temp1 / L;
    const double gamma1 = R.gamma + R.sqrt_g2m1 * pt0;
    const double dtdl = temp1 / c.beta1 / kSpeedLight;
    const double g1 = sqrt(bper2 / L / L) / c.opd;
    const double ptfluct = sqrt(Cf * gamma1 * gamma1 * gamma1 * gamma1 * gamma1 * g1 * g1 * g1 * dtdl * L) * gauss;
    p.pt = p.pt - ptloss + ptfluct;
  } else {
    p.pt = p.pt - temp2 * bper2 * temp1 / L;
  }
  const double delta2 = sqrt(1.0 + 2 * p.pt / R.beta + p.pt * p.pt) - 1.0;
  const double ratio = (1 + delta2) / c.opd;
  p.px = px0 * ratio;
  p.py = py0 * ratio;
  pt_refresh(R, p.pt, c);
}

// splint (simtrack.cpp:333-358): linear interpolation in a table by bisection.
__device__ __forceinline__ double splint_dev(const double *XA, const double *YA, int N, double X) {
  int klo = 0, khi = N - 1;
  while (khi - klo > 1) {
    const int k = (khi + klo) / 2;
    if (XA[k] > X) khi = k;
    else klo = k;
  }
  const double H = XA[khi] - XA[klo];
  const double A = (XA[khi] - X) / H;
  const double B = (X - XA[klo]) / H;
  return A * YA[klo] + B * YA[khi];
}

// radiate2 (simtrack.cpp:4290-4372): photon emission over one step by Monte
// Carlo, for the field (0, B1, 0): the critical energy Ec and mean photon
// count Nr of the step, Ng photons drawn with mean Nr, each photon's energy
// from the spectrum table (or (u/facg)^3 below u = 0.26).  `draws(j)` returns
// the step's j-th uniform (j = 0: the photon count).  As in the reference,
// the vertical slope uses x[1] (px) in place of x[3] (simtrack.cpp:4328).
template <class Draws>
__device__ __forceinline__ void radiate2_step(Particle &p, PtCache &c, const RefConsts &R, double L, double href,
                                              double B1, double facg, const double *XA, const double *YA, int N,
                                              Draws draws) {
  const double px0 = p.px, py0 = p.py;
  const double alpha = 1.0 / 137.0359997;
  const double gamma1 = R.gamma + R.sqrt_g2m1 * p.pt;
  const double pz = sqrt(c.opd2 - p.px * p.px - p.py * p.py);
  const double xp = (1 + p.x * href) * p.px / pz;
  const double yp = (1 + p.x * href) * p.px / pz;
  const double temp1 = sqrt((1 + p.x * href) * (1 + p.x * href) + xp * xp + yp * yp);
  const double u0 = xp / temp1, u1 = yp / temp1, u2 = (1 + p.x * href) / temp1;
  const double B0 = 0., B2 = 0.;
  const double b0 = B1 * u2 - B2 * u1;
  const double b1 = -1.0 * B0 * u2 + B2 * u0;
  const double b2 = B0 * u1 - B1 * u0;
  const double bper2 = b0 * b0 + b1 * b1 + b2 * b2;
  const double rho1 = (1 + p.pt) / sqrt(bper2) * L;
  const double Ec = 1.5 * 6.582119e-16 * 2.99792458e8 * gamma1 * gamma1 * gamma1 / rho1 / 1.0e6;
  const double Nr = 5. * alpha * gamma1 / 2. / sqrt(3.) / rho1 * L * temp1 / c.beta1;
  const int Ng = rad_poisson(draws(0u), Nr);
  double Etot = 0.;
  for (int i = 0; i < Ng; i++) {
    const double rtemp = draws((uint32_t)i + 1u);
    const double Etemp = rtemp < 0.26 ? cr_pown(rtemp / facg, 3) : splint_dev(XA, YA, N, rtemp);
    Etot = Etot + Etemp;
  }
  Etot = Etot * Ec;
  p.pt = p.pt - Etot / R.energy;
  const double delta2 = sqrt(1.0 + 2 * p.pt / R.beta + p.pt * p.pt) - 1.0;
  const double ratio = (1 + delta2) / c.opd;
  p.px = px0 * ratio;
  p.py = py0 * ratio;
  pt_refresh(R, p.pt, c);
}

// Hard-edge quadrupole fringe maps, simtrack.cpp:4906-4920 (entry) and 4948-4956 (exit).
static __device__ __forceinline__ void quad_fringe(Particle &p, double k, bool entry) {
  const double x0 = p.x, px0 = p.px, y0 = p.y, py0 = p.py, z0 = p.z, d0 = p.pt;
  const double a = k * (x0 * x0 * x0 + 3 * x0 * y0 * y0) / 12 / (1 + d0);
  const double b = k * ((x0 * x0 + y0 * y0) * px0 - 2 * x0 * y0 * py0) / 4 / (1 + d0);
  const double cc = k * (3 * x0 * x0 * y0 + y0 * y0 * y0) / 12 / (1 + d0);
  const double d = k * ((x0 * x0 + y0 * y0) * py0 - 2 * x0 * y0 * px0) / 4 / (1 + d0);
  const double e = k * (y0 * y0 * y0 * py0 - x0 * x0 * x0 * px0 + 3 * x0 * x0 * y0 * py0 - 3 * y0 * y0 * x0 * px0) /
                   12 / (1 + d0) / (1 + d0);
  if (entry) {
    p.x = x0 + a; p.px = px0 - b; p.y = y0 - cc; p.py = py0 + d; p.z = z0 + e;
  } else {
    p.x = x0 - a; p.px = px0 + b; p.y = y0 + cc; p.py = py0 - d; p.z = z0 - e;
  }
}

// GtoL1 / LtoG1, simtrack.cpp:3443-3481.  M = [dx, dy, cos(dpsi), sin(dpsi)]
__device__ __forceinline__ void gtol1(Particle &p, const double *M, int flags) {
  if (flags & EF_MISALIGN_OFFSET) {
    p.x = p.x - M[0];
    p.y = p.y - M[1];
  }
  if (flags & EF_MISALIGN_ROLL) {
    const double c = M[2], s = M[3];
    const double t0 = p.x, t1 = p.px, t2 = p.y, t3 = p.py;
    p.x = c * t0 + s * t2;
    p.px = c * t1 + s * t3;
    p.y = c * t2 - s * t0;
    p.py = c * t3 - s * t1;
  }
}
__device__ __forceinline__ void ltog1(Particle &p, const double *M, int flags) {
  if (flags & EF_MISALIGN_ROLL) {
    const double c = M[2], s = M[3];
    const double t0 = p.x, t1 = p.px, t2 = p.y, t3 = p.py;
    p.x = c * t0 - s * t2;
    p.px = c * t1 - s * t3;
    p.y = s * t0 + c * t2;
    p.py = s * t1 + c * t3;
  }
  if (flags & EF_MISALIGN_OFFSET) {
    p.x = p.x + M[0];
    p.y = p.y + M[1];
  }
}

// cerrf (Faddeeva w(z)), simtrack.cpp:6258-6323.  The reference fills
// rx[n], ry[n] for n = nu..1 and then consumes them for n = nc..1 with
// nc < nu; both loops run downwards, so the two are fused here and the
// arrays are not materialised.  Values are unchanged.
static __device__ __forceinline__ void cerrf_dev(double xx, double yy, double &wx, double &wy) {
  const double cc = 1.12837916709551, xlim = 5.33, ylim = 4.29, fac1 = 3.2, fac2 = 23, fac3 = 21;
  const double x = fabs(xx), y = fabs(yy);
  if (y < ylim && x < xlim) {
    const double q = (1. - y / ylim) * sqrt(1. - (x / xlim) * (x / xlim));
    const double h = 1. / (fac1 * q);
    const int nc = 7 + int(fac2 * q);
    double xl = cr_pown(h, 1 - nc);
    const double xh = y + .5 / h;
    const double yh = x;
    const int nu = 10 + int(fac3 * q);
    double rxn = 0., ryn = 0., sx = 0., sy = 0.;
    for (int n = nu; n >= 1; n--) {
      const double tx = xh + n * rxn;
      const double ty = yh - n * ryn;
      const double tn = tx * tx + ty * ty;
      rxn = .5 * tx / tn;
      ryn = .5 * ty / tn;
      if (n <= nc) {
        const double saux = sx + xl;
        sx = rxn * saux - ryn * sy;
        sy = rxn * sy + ryn * saux;
        xl = h * xl;
      }
    }
    wx = cc * sx;
    wy = cc * sy;
  } else {
    const double xh = y, yh = x;
    double rx = 0., ry = 0.;
    for (int n = 9; n >= 1; n--) {
      const double tx = xh + n * rx;
      const double ty = yh - n * ry;
      const double tn = tx * tx + ty * ty;
      rx = .5 * tx / tn;
      ry = .5 * ty / tn;
    }
    wx = cc * rx;
    wy = cc * ry;
  }
  if (yy < 0.) {
    wx = 2. * cr_exp(y * y - x * x) * cr_cos(2. * x * y) - wx;
    wy = -2. * cr_exp(y * y - x * x) * cr_sin(2. * x * y) - wy;
    if (xx > 0.) wy = -wy;
  } else {
    if (xx < 0.) wy = -wy;
  }
}

// BB4D (x, y, gamma, N, sigmax, sigmay) overload, simtrack.cpp:6325-6377.
// c4 = 2*N*rp/gamma (the constant prefix of temp1).
__device__ __forceinline__ void bb4d(double x, double y, double c4, double sigmax, double sigmay, double &Dpx,
                                     double &Dpy) {
  const double PI = 3.14159265358979323;
  const double signx = (x >= 0.0) ? 1. : -1.;
  const double signy = (y >= 0.0) ? 1. : -1.;
  if (x == 0. && y == 0.) {
    Dpx = 0.;
    Dpy = 0.;
  } else if (fabs(sigmax - sigmay) / sigmax < 1.0e-6) {
    const double r2 = x * x + y * y;
    const double temp1 = c4 / r2;
    const double temp2 = 1 - cr_exp(-r2 / 2 / sigmax / sigmax);
    Dpx = temp1 * x * temp2;
    Dpy = temp1 * y * temp2;
  } else if (sigmax > sigmay) {
    const double temp1 = c4 * sqrt(PI / 2. / (sigmax * sigmax - sigmay * sigmay));
    const double temp2 = cr_exp(-x * x * 0.5 / sigmax / sigmax - y * y * 0.5 / sigmay / sigmay);
    const double temp3 = sqrt(2. * (sigmax * sigmax - sigmay * sigmay));
    double w1r, w1i, w2r, w2i;
    const double x1 = fabs(x) / temp3, y1 = fabs(y) / temp3;
    const double x2 = fabs(x) * sigmay / sigmax / temp3, y2 = fabs(y) * sigmax / sigmay / temp3;
    cerrf_dev(x1, y1, w1r, w1i);
    cerrf_dev(x2, y2, w2r, w2i);
    Dpy = temp1 * (w1r - temp2 * w2r) * signy;
    Dpx = temp1 * (w1i - temp2 * w2i) * signx;
  } else if (sigmax < sigmay) {
    const double temp1 = c4 * sqrt(PI / 2 / (sigmay * sigmay - sigmax * sigmax));
    const double temp2 = cr_exp(-x * x / 2 / sigmax / sigmax - y * y / 2 / sigmay / sigmay);
    const double temp3 = sqrt(2 * (sigmay * sigmay - sigmax * sigmax));
    double w1r, w1i, w2r, w2i;
    const double x1 = fabs(x) / temp3, y1 = fabs(y) / temp3;
    const double x2 = fabs(x) * sigmay / sigmax / temp3, y2 = fabs(y) * sigmax / sigmay / temp3;
    cerrf_dev(y1, x1, w1r, w1i);
    cerrf_dev(y2, x2, w2r, w2i);
    Dpy = temp1 * (w1i - temp2 * w2i) * signy;
    Dpx = temp1 * (w1r - temp2 * w2r) * signx;
  } else {
    // sigmax or sigmay is NaN: the reference leaves Dpx/Dpy unset; NaN marks the particle lost.
    Dpx = __longlong_as_double(0x7ff8000000000000LL);
    Dpy = Dpx;
  }
}

// BB6D, simtrack.cpp:6622-6677 (slice loop).  P layout (built by the flattener):
// [bbscale, emitx, emity, betax*, alfx*, betay*, alfy*, gx*, gy*, 2*emitx, 2*emity,
//  temp3, c4, z_star[0..N-1]]
static __device__ __forceinline__ void bb6d(Particle &p, const double *P, int nslice) {
  const double bbscale = P[0], emitx = P[1], emity = P[2];
  const double betax_s = P[3], alfx_s = P[4], betay_s = P[5], alfy_s = P[6];
  const double gx = P[7], gy = P[8], e2x = P[9], e2y = P[10], t3 = P[11], c4 = P[12];
  const double *zs = P + 13;
  for (int i = 0; i < nslice; i++) {
    const Particle q = p;
    const double S = (q.z - zs[i]) * 0.5;
    const double betax = betax_s + 2 * S * alfx_s + S * S * gx;
    const double betay = betay_s + 2 * S * alfy_s + S * S * gy;
    const double sigmax = sqrt(emitx * betax);
    const double sigmay = sqrt(emity * betay);
    const double dsx = e2x * (alfx_s + S * gx);
    const double dsy = e2y * (alfy_s + S * gy);
    const double X = q.x + q.px * S;
    const double Y = q.y + q.py * S;
    double Dpx, Dpy;
    bb4d(X, Y, c4, sigmax, sigmay, Dpx, Dpy);
    const double temp1 = 1.0 / 2. / (sigmax * sigmax - sigmay * sigmay);
    const double temp2 = X * Dpx + Y * Dpy;
    const double temp4 = cr_exp(-X * X * 0.5 / sigmax / sigmax - Y * Y * 0.5 / sigmay / sigmay);
    p.x = q.x - S * Dpx * bbscale;
    p.px = q.px + Dpx * bbscale;
    p.y = q.y - S * Dpy * bbscale;
    p.py = q.py + Dpy * bbscale;
    const double kx = 0.5 * Dpx * bbscale * (q.px + 0.5 * Dpx * bbscale);
    const double ky = 0.5 * Dpy * bbscale * (q.py + 0.5 * Dpy * bbscale);
    if (fabs(sigmax - sigmay) / sigmax < 1.0e-6) {
      p.pt = q.pt + kx + ky + (1.0 / sigmax / sigmax) * dsx * (t3 * bbscale / 4.) * temp4;
    } else {
      const double dUx = temp1 * bbscale * (temp2 + t3 * (sigmay / sigmax * temp4 - 1.));
      const double dUy = -temp1 * bbscale * (temp2 + t3 * (sigmax / sigmay * temp4 - 1.));
      p.pt = q.pt + kx + ky - (0.5 * dsx * dUx + 0.5 * dsy * dUy);
    }
  }
}

// LBT_Pass, simtrack.cpp:6069-6093.  P = [sin, cos, tan]
static __device__ __forceinline__ void lbt(Particle &p, const double *P) {
  const double st = P[0], ct = P[1], tt = P[2];
  const double x0 = p.x, px0 = p.px, y0 = p.y, py0 = p.py, z0 = p.z, pz0 = p.pt;
  const double ps0 = sqrt((1 + pz0) * (1 + pz0) - px0 * px0 - py0 * py0);
  const double h0 = (1 + pz0) - ps0;
  const double pxs = (px0 - tt * h0) / ct;
  const double pys = py0 / ct;
  const double pzs = pz0 - tt * px0 + tt * tt * h0;
  const double pss = sqrt((1 + pzs) * (1 + pzs) - pxs * pxs - pys * pys);
  const double hs = (1 + pzs) - pss;
  p.x = tt * z0 + (1 + (pxs / pss) * st) * x0;
  p.y = y0 + st * (pys / pss) * x0;
  p.z = z0 / ct + (-hs / pss) * st * x0;
  p.px = pxs;
  p.py = pys;
  p.pt = pzs;
}

// ILBT_Pass, simtrack.cpp:6095-6123.  P = [sin, cos]
static __device__ __forceinline__ void ilbt(Particle &p, const double *P) {
  const double st = P[0], ct = P[1];
  const double xs = p.x, pxs = p.px, ys = p.y, pys = p.py, zs = p.z, pzs = p.pt;
  const double pss = sqrt((1 + pzs) * (1 + pzs) - pxs * pxs - pys * pys);
  const double hs = 1 + pzs - pss;
  const double hxs = pxs / pss, hys = pys / pss, hzs = -hs / pss;
  const double px0 = (pxs + hs * st) * ct;
  const double py0 = pys * ct;
  const double pz0 = pzs + pxs * st;
  const double x0 = (xs - zs * st) / (1 + hxs * st - hzs * st * st);
  const double z0 = (zs - hzs * st * x0) * ct;
  const double y0 = ys - st * hys * x0;
  p.x = x0; p.px = px0; p.y = y0; p.py = py0; p.z = z0; p.pt = pz0;
}

// CCMULT_Pass kick part, simtrack.cpp:6037-6064.
// P = [kf, PHASE0, scale, brho, B2, A2, B3, A3, B4, A4, B5, A5]
static __device__ __forceinline__ void ccmult_kick(Particle &p, const double *P) {
  const double kf = P[0], PHASE0 = P[1], scale = P[2], brho = P[3];
  const double B2 = P[4], A2 = P[5], B3 = P[6], A3 = P[7], B4 = P[8], A4 = P[9], B5 = P[10], A5 = P[11];
  const double arg = kf * p.z / 2.99792458e8 + PHASE0;
  const double sinangle = cr_sin(arg);
  const double cosangle = cr_cos(arg);
  const double X = p.x, Y = p.y;
  const double x2 = X * X, x3 = x2 * X, x4 = x3 * X, x5 = x4 * X;
  const double y2 = Y * Y, y3 = y2 * Y, y4 = y3 * Y, y5 = y4 * Y;
  const double xy = X * Y, x2y = x2 * Y, xy2 = X * y2, x2y2 = X * xy2;
  const double x3y = Y * x3, xy3 = X * y3;
  const double x2y3 = x2y2 * Y, x3y2 = x2y2 * X, x4y = x4 * Y, xy4 = y4 * X;
  double px = p.px, py = p.py, pt = p.pt;
  px = px + (B2 * X + A2 * Y) * cosangle / brho;
  py = py + (A2 * X - B2 * Y) * cosangle / brho;
  pt = pt + (B2 * (x2 - y2) * sinangle + A2 * xy * sinangle) * scale;
  px = px + (B3 * (x2 - y2) + 2 * A3 * xy) * cosangle / brho;
  py = py + (2 * B3 * xy + A3 * (x2 - y2)) * cosangle / brho;
  pt = pt + (B3 * (x3 - 3 * xy2) * sinangle + A3 * (3 * x2y - y3) * sinangle) * scale / 3.;
  px = px + (B4 * (x3 - 3 * xy2) - A4 * (y3 - 3 * x2y)) * cosangle / brho;
  py = py + (B4 * (y3 - 3 * x2y) + A4 * (x3 - 3 * xy2)) * cosangle / brho;
  pt = pt + (B4 * (x4 - 6 * x2 * y2 + y4) * sinangle + A4 * (4 * x3y - 4 * xy3) * sinangle) * scale / 4.;
  px = px + (B5 * (x4 - 6 * x2y2 + y4) + A5 * (4 * x3y - 4 * xy3)) * cosangle / brho;
  py = py + (B5 * (4 * xy3 - 4 * x3y) + A5 * (x4 - 6 * x2y2 + y4)) * cosangle / brho;
  pt = pt + (B5 * (x5 - 10 * x3y2 + 5 * xy4) * sinangle + A5 * (5 * x4y - 10 * x2y3 + y5) * sinangle) * scale / 5.;
  p.px = px;
  p.py = py;
  p.pt = pt;
}

// PATCH_Pass, simtrack.cpp:6248-6256: TRANS_Pass (6140-6151) then, when
// |THETA| >= 1e-9, YROTAT_Pass (6192-6217).  P = [DX, DY, DS, cos, sin, tan].
__device__ __forceinline__ void patch_map(Particle &p, const PtCache &c, const double *P, bool rotate) {
  p.x = p.x - P[0];
  p.y = p.y - P[1];
  p.z = p.z - P[2];
  if (!rotate) return;
  const double cosT = P[3], sinT = P[4], tanT = P[5];
  const double x0 = p.x, px0 = p.px, py0 = p.py;
  const double pz = sqrt(c.opd2 - px0 * px0 - py0 * py0);
  const double temp = 1 - px0 * tanT / pz;
  p.x = x0 / cosT / temp;
  p.px = px0 * cosT + pz * sinT;
  p.y = p.y + py0 * x0 * tanT / pz / temp;
  p.z = p.z - c.opd * x0 * tanT / pz / temp / c.beta1;
}

// Solenoid body shared by SOLEN_Pass (simtrack.cpp:5804-5857) and
// SOLEN_sPass (8118-8183), KS != 0: hard-edge entrance kick, Nint slices of
// the 4x4 rotation matrix in (x, x', y, y'), exit kick, path length.
// P = [q*Bz/2, L, Nint, L/Nint, L/beta/c, m0, p0 (, Bz*Lint/brho for spin)].
// `slice(xt, px, py)` is called before every slice with the slice's entry
// state and its momenta converted back to (px, py), as SOLEN_sPass feeds
// spin().
template <class SliceHook>
__device__ __forceinline__ void solen_map(Particle &p, const PtCache &c, const RefConsts &R, const double *P, int nint,
                                          SliceHook slice) {
  const double qb2 = P[0], L = P[1], fnint = P[2], Lint = P[3], Lbc = P[4], m0 = P[5], p0 = P[6];
  const double gamma1 = R.gamma + R.sqrt_g2m1 * p.pt;
  const double ps = sqrt(c.opd2 - p.px * p.px - p.py * p.py);
  double x0 = p.x, x1 = p.px / ps, x2 = p.y, x3 = p.py / ps;
  const double vz = 2.99792458e8 * c.beta1 / sqrt(1.0 + x1 * x1 + x3 * x3);
  const double K = qb2 / gamma1 / m0 / vz;
  x1 = x1 + x2 * K;
  x3 = x3 - x0 * K;
  const double theta = -2.0 * K * L / fnint;
  double st, ct;
  cr_sincos(theta, st, ct);
  const double m01 = Lint * st / theta, m03 = -(1 - ct) * Lint / theta;
  const double m21 = (1 - ct) * Lint / theta, m23 = Lint * st / theta;
  const double m11 = ct, m13 = -st, m31 = st, m33 = ct;
  for (int i = 0; i < nint; i++) {
    const double t0 = x0, t1 = x1, t2 = x2, t3 = x3;
    slice(t0, t1, t2, t3, gamma1, vz);
    // the reference's 4x4 product, zero and unit entries included
    x0 = 0. + 1.0 * t0 + m01 * t1 + 0. * t2 + m03 * t3;
    x1 = 0. + 0. * t0 + m11 * t1 + 0. * t2 + m13 * t3;
    x2 = 0. + 0. * t0 + m21 * t1 + 1. * t2 + m23 * t3;
    x3 = 0. + 0. * t0 + m31 * t1 + 0. * t2 + m33 * t3;
  }
  x1 = x1 - x2 * K;
  x3 = x3 + x0 * K;
  p.x = x0;
  p.y = x2;
  p.px = gamma1 * m0 * x1 * vz / p0;
  p.py = gamma1 * m0 * x3 * vz / p0;
  p.z = p.z - 2.99792458e8 * (L / vz - Lbc);
}

}  // namespace stb
