/*
 * C restatement of SimTrack's tracking path.  TEST INFRASTRUCTURE ONLY.
 *
 * Each function cites the reference routine (simtrack.cpp file:line) whose
 * arithmetic it restates.  Expressions keep the reference's operand order
 * because the parity bar is bit-level for +,-,*,/,sqrt: C evaluates
 * same-precedence operators left to right exactly like the C++ original,
 * and the Makefile compiles with -ffp-contract=off.  Only the exact
 * Hamiltonian, non-radiating branches are restated (GP.H_expand == false,
 * GP.radiate == false), which is what every dynamic-aperture configuration
 * uses.  Pitch/yaw misalignments (GtoL2/LtoG2) are not restated: elements
 * carrying DTHETA or DPHI make port_pass return -1.
 */
#include "simtrack_port.h"

#include <math.h>
#include <string.h>

static const double PORT_PI = 3.14159265358979323; /* simtrack.cpp:23 */

/* Yoshida 4th-order coefficients, simtrack.cpp:29-32 */
static double Fdrift1, Fdrift2, Fkick1, Fkick2;
static int coeffs_ready = 0;

static void init_coeffs(void)
{
  if (coeffs_ready) return;
  Fdrift1 = 1.e0 / (2.e0 * (2.e0 - pow(2.e0, 1.0 / 3.0)));
  Fdrift2 = 0.5e0 - Fdrift1;
  Fkick1 = 2.e0 * Fdrift1;
  Fkick2 = 1.e0 - 2e0 * Fkick1;
  coeffs_ready = 1;
}

/* GtoL1, simtrack.cpp:3443-3461 */
static void gtol1(double *x, double DX, double DY, double DT)
{
  double t[6];
  int i;
  if (fabs(DX) + fabs(DY) > 1.0e-10) {
    x[0] = x[0] - DX;
    x[2] = x[2] - DY;
  }
  if (fabs(DT) > 1.0e-10) {
    double c = cos(DT), s = sin(DT);
    for (i = 0; i < 6; i++) t[i] = x[i];
    x[0] = c * t[0] + s * t[2];
    x[1] = c * t[1] + s * t[3];
    x[2] = c * t[2] - s * t[0];
    x[3] = c * t[3] - s * t[1];
  }
}

/* LtoG1, simtrack.cpp:3463-3481 */
static void ltog1(double *x, double DX, double DY, double DT)
{
  double t[6];
  int i;
  if (fabs(DT) > 1.0e-10) {
    double c = cos(DT), s = sin(DT);
    for (i = 0; i < 6; i++) t[i] = x[i];
    x[0] = c * t[0] - s * t[2];
    x[1] = c * t[1] - s * t[3];
    x[2] = s * t[0] + c * t[2];
    x[3] = s * t[1] + c * t[3];
  }
  if (fabs(DX) + fabs(DY) > 1.0e-10) {
    x[0] = x[0] + DX;
    x[2] = x[2] + DY;
  }
}

/* GtoL/LtoG dispatch, simtrack.cpp:3701-3741.  Returns -1 for pitch/yaw. */
static int misaligned(const port_elem *e)
{
  double s = fabs(e->dx) + fabs(e->dy) + fabs(e->ds) + fabs(e->dtheta) + fabs(e->dphi) + fabs(e->dpsi);
  if (s < 1.0e-9) return 0;
  if (fabs(e->dtheta) + fabs(e->dphi) < 1.0e-9) return 1;
  return -1;
}

/* DRIFT_Pass exact branch, simtrack.cpp:3752-3765 */
static void drift(double *x, double L, const port_gp *gp)
{
  double delta1 = sqrt(1.0 + 2 * x[5] / gp->beta + x[5] * x[5]) - 1.0;
  double gamma1 = gp->gamma + sqrt(gp->gamma * gp->gamma - 1.) * x[5];
  double beta1 = sqrt(1.0 - 1.0 / gamma1 / gamma1);
  double pz = sqrt((1.0 + delta1) * (1.0 + delta1) - x[1] * x[1] - x[3] * x[3]);
  double betaz = pz * beta1 / (1.0 + delta1);
  x[0] = x[0] + x[1] * L / pz;
  x[2] = x[2] + x[3] * L / pz;
  x[4] = x[4] - (L / betaz - L / gp->beta);
}

/* sbend_exact_pass, simtrack.cpp:3833-3858 */
static void sbend_exact(double *x, double L, double Angle, double cosA, double sinA, const port_gp *gp)
{
  double href = Angle / L;
  double x0[6], pz0, pz1, delta, gamma, beta, der, temp, as1, as2;
  int i;
  for (i = 0; i < 6; i++) x0[i] = x[i];
  delta = sqrt(1.0 + 2 * x[5] / gp->beta + x[5] * x[5]) - 1.0;
  gamma = gp->gamma + sqrt(gp->gamma * gp->gamma - 1) * x[5];
  beta = sqrt(1.0 - 1.0 / gamma / gamma);
  pz0 = sqrt((1. + delta) * (1. + delta) - x0[1] * x0[1] - x0[3] * x0[3]);
  x[1] = x0[1] * cosA + (pz0 - 1. - href * x0[0]) * sinA;
  pz1 = sqrt((1. + delta) * (1. + delta) - x[1] * x[1] - x[3] * x[3]);
  der = -1.0 * x0[1] * sinA * href + (pz0 - 1. - x[0] * href) * cosA * href;
  x[0] = pz1 / href - der / href / href - 1.0 / href;
  temp = sqrt((1. + delta) * (1. + delta) - x0[3] * x0[3]);
  as1 = asin(x0[1] / temp);
  as2 = asin(x[1] / temp);
  x[2] = x0[2] + x0[3] * L + x0[3] * (as1 - as2) / href;
  temp = (1 + delta) * L + (1 + delta) * (as1 - as2) / href;
  x[4] = x[4] - (temp / beta - L / gp->beta);
}

/* general_sbend_exact_pass, simtrack.cpp:3974-4010 */
static void gsbend_exact(double *x, double L, double Angle, double K0L, double cosA, double sinA,
                         const port_gp *gp)
{
  double rhoc = L / Angle;
  double b0 = K0L / L;
  double x0[6], pz0, pz1, delta, gamma, beta, der, temp, as1, as2;
  int i;
  for (i = 0; i < 6; i++) x0[i] = x[i];
  delta = sqrt(1.0 + 2 * x[5] / gp->beta + x[5] * x[5]) - 1.0;
  gamma = gp->gamma + sqrt(gp->gamma * gp->gamma - 1) * x[5];
  beta = sqrt(1.0 - 1.0 / gamma / gamma);
  pz0 = sqrt((1. + delta) * (1. + delta) - x0[1] * x0[1] - x0[3] * x0[3]);
  x[1] = x0[1] * cosA + (pz0 - b0 * rhoc - b0 * x0[0]) * sinA;
  pz1 = sqrt((1. + delta) * (1. + delta) - x[1] * x[1] - x[3] * x[3]);
  der = -x0[1] * sinA / rhoc + (pz0 - b0 * rhoc - b0 * x0[0]) * cosA / rhoc;
  x[0] = pz1 / b0 - der * rhoc / b0 - rhoc;
  temp = sqrt((1. + delta) * (1. + delta) - x0[3] * x0[3]);
  as1 = asin(x0[1] / temp);
  as2 = asin(x[1] / temp);
  x[2] = x0[2] + x0[3] * L / b0 / rhoc + x0[3] * (as1 - as2) / b0;
  temp = (1 + delta) * L / b0 / rhoc + (1 + delta) * (as1 - as2) / b0;
  x[4] = x[4] - (temp / beta - L / gp->beta);
}

/* quad_kick_pass, simtrack.cpp:4046-4058 */
static void quad_kick(double *x, double k1l, double k1sl)
{
  double pr = x[0], pi = x[2];
  double Bx = k1sl * pr + k1l * pi;
  double By = k1l * pr - k1sl * pi;
  x[1] = x[1] - By;
  x[3] = x[3] + Bx;
}

/* sext_kick_pass, simtrack.cpp:4060-4071 */
static void sext_kick(double *x, double k2l, double k2sl)
{
  double pr = x[0] * x[0] - x[2] * x[2];
  double pi = 2. * x[0] * x[2];
  double Bx = (k2sl * pr + k2l * pi) / 2.;
  double By = (k2l * pr - k2sl * pi) / 2.;
  x[1] = x[1] - By;
  x[3] = x[3] + Bx;
}

/* oct_kick_pass, simtrack.cpp:4073-4084 */
static void oct_kick(double *x, double k3l, double k3sl)
{
  double pr = x[0] * x[0] * x[0] - 3 * x[0] * x[2] * x[2];
  double pi = 3 * x[0] * x[0] * x[2] - x[2] * x[2] * x[2];
  double Bx = (k3sl * pr + k3l * pi) / 6.;
  double By = (k3l * pr - k3sl * pi) / 6.;
  x[1] = x[1] - By;
  x[3] = x[3] + Bx;
}

/* mult_kick_pass, simtrack.cpp:4086-4111 */
static void mult_kick(double *x, int Norder, const double *KNL, const double *KNSL)
{
  int i, fac = 1;
  double Xn = 1., Yn = 0., Xn0, Yn0;
  double By = KNL[0], Bx = KNSL[0];
  for (i = 1; i < Norder + 1; i++) {
    Xn0 = Xn;
    Yn0 = Yn;
    Xn = Xn0 * x[0] - Yn0 * x[2];
    Yn = Xn0 * x[2] + Yn0 * x[0];
    fac = fac * i;
    if (KNL[i] != 0. || KNSL[i] != 0.) {
      By = By + (KNL[i] * Xn - KNSL[i] * Yn) / fac;
      Bx = Bx + (KNL[i] * Yn + KNSL[i] * Xn) / fac;
    }
  }
  x[1] = x[1] - By;
  x[3] = x[3] + Bx;
}

/* Hard-edge quadrupole fringe maps, simtrack.cpp:4895-4921 (entry, sgn=+1)
 * and 4938-4957 (exit, sgn=-1). */
static void quad_fringe(double *x, double k, int entry)
{
  double x0[6];
  int i;
  for (i = 0; i < 6; i++) x0[i] = x[i];
  if (entry) {
    x[0] = x0[0] + k * (x0[0] * x0[0] * x0[0] + 3 * x0[0] * x0[2] * x0[2]) / 12 / (1 + x0[5]);
    x[1] = x0[1] - k * ((x0[0] * x0[0] + x0[2] * x0[2]) * x0[1] - 2 * x0[0] * x0[2] * x0[3]) / 4 / (1 + x0[5]);
    x[2] = x0[2] - k * (3 * x0[0] * x0[0] * x0[2] + x0[2] * x0[2] * x0[2]) / 12 / (1 + x0[5]);
    x[3] = x0[3] + k * ((x0[0] * x0[0] + x0[2] * x0[2]) * x0[3] - 2 * x0[0] * x0[2] * x0[1]) / 4 / (1 + x0[5]);
    x[4] = x0[4] + k * (x0[2] * x0[2] * x0[2] * x0[3] - x0[0] * x0[0] * x0[0] * x0[1]
                        + 3 * x0[0] * x0[0] * x0[2] * x0[3] - 3 * x0[2] * x0[2] * x0[0] * x0[1]) / 12 / (1 + x0[5]) / (1 + x0[5]);
  } else {
    x[0] = x0[0] - k * (x0[0] * x0[0] * x0[0] + 3 * x0[0] * x0[2] * x0[2]) / 12 / (1 + x0[5]);
    x[1] = x0[1] + k * ((x0[0] * x0[0] + x0[2] * x0[2]) * x0[1] - 2 * x0[0] * x0[2] * x0[3]) / 4 / (1 + x0[5]);
    x[2] = x0[2] + k * (3 * x0[0] * x0[0] * x0[2] + x0[2] * x0[2] * x0[2]) / 12 / (1 + x0[5]);
    x[3] = x0[3] - k * ((x0[0] * x0[0] + x0[2] * x0[2]) * x0[3] - 2 * x0[0] * x0[2] * x0[1]) / 4 / (1 + x0[5]);
    x[4] = x0[4] - k * (x0[2] * x0[2] * x0[2] * x0[3] - x0[0] * x0[0] * x0[0] * x0[1]
                        + 3 * x0[0] * x0[0] * x0[2] * x0[3] - 3 * x0[2] * x0[2] * x0[0] * x0[1]) / 12 / (1 + x0[5]) / (1 + x0[5]);
  }
}

/* QUAD_Pass / SEXT_Pass / OCT_Pass, simtrack.cpp:4882-4959, 5004-5034, 5077-5105:
 * Yoshida D(F1)K(K1)D(F2)K(K2)D(F2)K(K1)D(F1) per slice. order = 1, 2, 3. */
static void thick_pass(double *x, double L, int Nint, double kl, double ksl, int order,
                       const port_gp *gp)
{
  int i;
  double Lint, a1, s1, a2, s2;
  if (kl == 0. && ksl == 0.) {
    drift(x, L, gp);
    return;
  }
  if (L == 0.) {
    if (order == 1) quad_kick(x, kl, ksl);
    else if (order == 2) sext_kick(x, kl, ksl);
    else oct_kick(x, kl, ksl);
    return;
  }
  if (order == 1 && gp->quad_fringe) quad_fringe(x, kl / L, 1);
  Lint = L / Nint;
  a1 = Fkick1 * kl / Nint;
  s1 = Fkick1 * ksl / Nint;
  a2 = Fkick2 * kl / Nint;
  s2 = Fkick2 * ksl / Nint;
  for (i = 0; i < Nint; i++) {
    drift(x, Fdrift1 * Lint, gp);
    if (order == 1) quad_kick(x, a1, s1); else if (order == 2) sext_kick(x, a1, s1); else oct_kick(x, a1, s1);
    drift(x, Fdrift2 * Lint, gp);
    if (order == 1) quad_kick(x, a2, s2); else if (order == 2) sext_kick(x, a2, s2); else oct_kick(x, a2, s2);
    drift(x, Fdrift2 * Lint, gp);
    if (order == 1) quad_kick(x, a1, s1); else if (order == 2) sext_kick(x, a1, s1); else oct_kick(x, a1, s1);
    drift(x, Fdrift1 * Lint, gp);
  }
  if (order == 1 && gp->quad_fringe) quad_fringe(x, kl / L, 0);
}

/* MULT_Pass, simtrack.cpp:5152-5182 */
static void mult_pass(double *x, double L, int Nint, int Norder, const double *KNL, const double *KNSL,
                      const port_gp *gp)
{
  double k1[11], s1[11], k2[11], s2[11], Lint;
  int i;
  if (L == 0.) {
    mult_kick(x, Norder, KNL, KNSL);
    return;
  }
  Lint = L / Nint;
  for (i = 0; i < 11; i++) {
    k1[i] = Fkick1 * KNL[i] / Nint;
    s1[i] = Fkick1 * KNSL[i] / Nint;
  }
  for (i = 0; i < 11; i++) {
    k2[i] = Fkick2 * KNL[i] / Nint;
    s2[i] = Fkick2 * KNSL[i] / Nint;
  }
  for (i = 0; i < Nint; i++) {
    drift(x, Fdrift1 * Lint, gp);
    mult_kick(x, Norder, k1, s1);
    drift(x, Fdrift2 * Lint, gp);
    mult_kick(x, Norder, k2, s2);
    drift(x, Fdrift2 * Lint, gp);
    mult_kick(x, Norder, k1, s1);
    drift(x, Fdrift1 * Lint, gp);
  }
}

/* GMULT_Pass / SBENDMULT_Pass exact, non-radiating branch,
 * simtrack.cpp:5223-5346 (lines 5288-5311) and 5348-5470 (5413-5436). */
static void bendmult_pass(double *x, double L, int Nint, int Norder, double Angle, double E1, double E2,
                          const double *KNL, const double *KNSL, const port_gp *gp)
{
  double k1[11], s1[11], k2[11], s2[11], href, Lint, edge, cA, sA, cA1, sA1;
  int i;
  if (L == 0.) {
    mult_kick(x, Norder, KNL, KNSL);
    return;
  }
  href = Angle / L;
  Lint = L / Nint;
  edge = tan(E1) * href;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
  for (i = 0; i < 11; i++) {
    k1[i] = Fkick1 * KNL[i] / Nint;
    s1[i] = Fkick1 * KNSL[i] / Nint;
  }
  for (i = 0; i < 11; i++) {
    k2[i] = Fkick2 * KNL[i] / Nint;
    s2[i] = Fkick2 * KNSL[i] / Nint;
  }
  cA1 = cos(Fdrift1 * Angle / Nint);
  sA1 = sin(Fdrift1 * Angle / Nint);
  cA = cos(Fdrift2 * Angle / Nint);
  sA = sin(Fdrift2 * Angle / Nint);
  for (i = 0; i < Nint; i++) {
    sbend_exact(x, Fdrift1 * Lint, Fdrift1 * Angle / Nint, cA1, sA1, gp);
    mult_kick(x, Norder, k1, s1);
    sbend_exact(x, Fdrift2 * Lint, Fdrift2 * Angle / Nint, cA, sA, gp);
    mult_kick(x, Norder, k2, s2);
    sbend_exact(x, Fdrift2 * Lint, Fdrift2 * Angle / Nint, cA, sA, gp);
    mult_kick(x, Norder, k1, s1);
    sbend_exact(x, Fdrift1 * Lint, Fdrift1 * Angle / Nint, cA1, sA1, gp);
  }
  edge = tan(E2) * href;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
}

/* SBEND_Pass exact branch, simtrack.cpp:4693-4752 (line 4737) */
static void sbend_pass(double *x, double L, double Angle, double E1, double E2, const port_gp *gp)
{
  double href = Angle / L, edge;
  if (Angle == 0.) {
    drift(x, L, gp);
    return;
  }
  edge = tan(E1) * href;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
  sbend_exact(x, L, Angle, cos(Angle), sin(Angle), gp);
  edge = tan(E2) * href;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
}

/* GSBEND_Pass exact branch, simtrack.cpp:4818-4880 (line 4861) */
static void gsbend_pass(double *x, double L, double Angle, double K0L, double E1, double E2,
                        const port_gp *gp)
{
  double hreal = K0L / L, edge;
  if (Angle == 0.) {
    drift(x, L, gp);
    return;
  }
  edge = tan(E1) * hreal;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
  gsbend_exact(x, L, Angle, K0L, cos(Angle), sin(Angle), gp);
  edge = tan(E2) * hreal;
  x[1] = x[1] + edge * x[0];
  x[3] = x[3] - edge * x[2];
}

/* KICK_Pass, simtrack.cpp:5887-5893 */
static void kick_pass(double *x, double L, double hk, double vk, const port_gp *gp)
{
  drift(x, L / 2.0, gp);
  x[1] = x[1] + hk;
  x[3] = x[3] + vk;
  drift(x, L / 2.0, gp);
}

/* SOLEN_Pass, simtrack.cpp:5804-5857, with the solenoid's single slice
 * (SOLEN's constructor fixes Nint = 1, simtrack.cpp:9645-9660). */
static void solen_pass(double *x, double L, double KS, const port_gp *gp)
{
  const int Nint = 1;
  double Bz, delta1, gamma1, beta1, ps, vz, K, Lint, theta, sn, cs;
  double m[4][4], t[4];
  int i, j, k;
  if (KS == 0) {
    drift(x, L, gp);
    return;
  }
  Bz = KS * gp->brho;
  Lint = L / Nint;
  delta1 = sqrt(1.0 + 2 * x[5] / gp->beta + x[5] * x[5]) - 1.0;
  gamma1 = gp->gamma + sqrt(gp->gamma * gp->gamma - 1.) * x[5];
  beta1 = sqrt(1.0 - 1.0 / gamma1 / gamma1);
  /* (px, py) -> (x', y') */
  ps = sqrt((1 + delta1) * (1 + delta1) - x[1] * x[1] - x[3] * x[3]);
  x[1] = x[1] / ps;
  x[3] = x[3] / ps;
  vz = 2.99792458e8 * beta1 / sqrt(1.0 + x[1] * x[1] + x[3] * x[3]);
  K = gp->q * Bz / 2.0 / gamma1 / gp->m0 / vz;
  /* entrance fringe */
  x[1] = x[1] + x[2] * K;
  x[3] = x[3] - x[0] * K;
  /* body: rotation in the transverse plane */
  theta = -2.0 * K * L / Nint;
  sn = sin(theta);
  cs = cos(theta);
  for (i = 0; i < 4; i++)
    for (j = 0; j < 4; j++) m[i][j] = 0.;
  m[0][0] = 1.0;
  m[0][1] = Lint * sn / theta;
  m[0][3] = -(1 - cs) * Lint / theta;
  m[1][1] = cs;
  m[1][3] = -sn;
  m[2][1] = (1 - cs) * Lint / theta;
  m[2][2] = 1.;
  m[2][3] = Lint * sn / theta;
  m[3][1] = sn;
  m[3][3] = cs;
  for (i = 0; i < Nint; i++) {
    for (k = 0; k < 4; k++) t[k] = x[k];
    for (k = 0; k < 4; k++) {
      x[k] = 0.;
      for (j = 0; j < 4; j++) x[k] = x[k] + m[k][j] * t[j];
    }
  }
  /* exit fringe, then back to (px, py) */
  x[1] = x[1] - x[2] * K;
  x[3] = x[3] + x[0] * K;
  x[1] = gamma1 * gp->m0 * x[1] * vz / gp->p;
  x[3] = gamma1 * gp->m0 * x[3] * vz / gp->p;
  x[4] = x[4] - 2.99792458e8 * (L / vz - L / gp->beta / 2.99792458e8);
}

/* PATCH_Pass, simtrack.cpp:6248-6256: TRANS_Pass (6140-6151), then
 * YROTAT_Pass (6192-6217), which does nothing for |THETA| < 1e-9. */
static void patch_pass(double *x, double DX, double DY, double DS, double THETA, const port_gp *gp)
{
  double x0, px0, py0, delta1, gamma1, beta1, cosT, sinT, tanT, pz, temp;
  x[0] = x[0] - DX;
  x[2] = x[2] - DY;
  x[4] = x[4] - DS;
  if (fabs(THETA) < 1.0e-9) return;
  delta1 = sqrt(1.0 + 2 * x[5] / gp->beta + x[5] * x[5]) - 1.0;
  gamma1 = gp->gamma + sqrt(gp->gamma * gp->gamma - 1.) * x[5];
  beta1 = sqrt(1.0 - 1.0 / gamma1 / gamma1);
  cosT = cos(THETA);
  sinT = sin(THETA);
  tanT = tan(THETA);
  x0 = x[0];
  px0 = x[1];
  py0 = x[3];
  pz = sqrt((1 + delta1) * (1 + delta1) - px0 * px0 - py0 * py0);
  temp = 1 - px0 * tanT / pz;
  x[0] = x0 / cosT / temp;
  x[1] = px0 * cosT + pz * sinT;
  x[2] = x[2] + py0 * x0 * tanT / pz / temp;
  x[4] = x[4] - (1 + delta1) * x0 * tanT / pz / temp / beta1;
}

/* RFCAV_Pass, simtrack.cpp:6002-6012 */
static void rfcav_pass(double *x, double L, double VRF, double FRF, double PHASE0, const port_gp *gp)
{
  if (VRF == 0.) {
    drift(x, L, gp);
    return;
  }
  drift(x, L / 2., gp);
  x[5] = x[5] + fabs(VRF * gp->Q) * sin(-2.0 * PORT_PI * FRF * x[4] / 2.99792458e8 + PORT_PI - PHASE0)
                    / gp->beta / gp->energy;
  drift(x, L / 2., gp);
}

/* CRABRF_Pass, simtrack.cpp:6014-6025 */
static void crabrf_pass(double *x, double L, double VRF, double FRF, double PHASE0, const port_gp *gp)
{
  if (VRF == 0.) {
    drift(x, L, gp);
    return;
  }
  drift(x, L / 2., gp);
  x[1] = x[1] - (VRF * gp->Q) * sin(2.0 * PORT_PI * FRF * x[4] / 2.99792458e8 + PHASE0) / gp->beta / gp->energy;
  x[5] = x[5] - (VRF * gp->Q) * cos(2.0 * PORT_PI * FRF * x[4] / 2.99792458e8 + PHASE0) * x[0]
                    * (2.0 * PORT_PI * FRF / 2.99792458e8) / gp->beta / gp->energy;
  drift(x, L / 2., gp);
}

/* CCMULT_Pass, simtrack.cpp:6027-6067 (arguments B2..A5 receive the element's B1..A4) */
static void ccmult_pass(double *x, double L, double VRF, double FRF, double PHASE0, double B2, double A2,
                        double B3, double A3, double B4, double A4, double B5, double A5, const port_gp *gp)
{
  double c, scale, sn, cs, x2, x3, x4, x5, y2, y3, y4, y5, xy, x2y, xy2, x2y2, x3y, xy3, x2y3, x3y2, x4y, xy4;
  if (VRF == 0.) {
    drift(x, L, gp);
    return;
  }
  drift(x, L / 2., gp);
  c = 2.99792458e8;
  scale = 2 * PORT_PI * FRF / c / gp->brho;
  sn = sin(2.0 * PORT_PI * FRF * x[4] / 2.99792458e8 + PHASE0);
  cs = cos(2.0 * PORT_PI * FRF * x[4] / 2.99792458e8 + PHASE0);
  x2 = x[0] * x[0]; x3 = x2 * x[0]; x4 = x3 * x[0]; x5 = x4 * x[0];
  y2 = x[2] * x[2]; y3 = y2 * x[2]; y4 = y3 * x[2]; y5 = y4 * x[2];
  xy = x[0] * x[2]; x2y = x2 * x[2]; xy2 = x[0] * y2; x2y2 = x[0] * xy2;
  x3y = x[2] * x3; xy3 = x[0] * y3;
  x2y3 = x2y2 * x[2]; x3y2 = x2y2 * x[0]; x4y = x4 * x[2]; xy4 = y4 * x[0];
  (void)x3y2;

  x[1] = x[1] + (B2 * x[0] + A2 * x[2]) * cs / gp->brho;
  x[3] = x[3] + (A2 * x[0] - B2 * x[2]) * cs / gp->brho;
  x[5] = x[5] + (B2 * (x2 - y2) * sn + A2 * xy * sn) * scale;

  x[1] = x[1] + (B3 * (x2 - y2) + 2 * A3 * xy) * cs / gp->brho;
  x[3] = x[3] + (2 * B3 * xy + A3 * (x2 - y2)) * cs / gp->brho;
  x[5] = x[5] + (B3 * (x3 - 3 * xy2) * sn + A3 * (3 * x2y - y3) * sn) * scale / 3.;

  x[1] = x[1] + (B4 * (x3 - 3 * xy2) - A4 * (y3 - 3 * x2y)) * cs / gp->brho;
  x[3] = x[3] + (B4 * (y3 - 3 * x2y) + A4 * (x3 - 3 * xy2)) * cs / gp->brho;
  x[5] = x[5] + (B4 * (x4 - 6 * x2 * y2 + y4) * sn + A4 * (4 * x3y - 4 * xy3) * sn) * scale / 4.;

  x[1] = x[1] + (B5 * (x4 - 6 * x2y2 + y4) + A5 * (4 * x3y - 4 * xy3)) * cs / gp->brho;
  x[3] = x[3] + (B5 * (4 * xy3 - 4 * x3y) + A5 * (x4 - 6 * x2y2 + y4)) * cs / gp->brho;
  x[5] = x[5] + (B5 * (x5 - 10 * x3y2 + 5 * xy4) * sn + A5 * (5 * x4y - 10 * x2y3 + y5) * sn) * scale / 5.;
  drift(x, L / 2., gp);
}

/* LBT_Pass, simtrack.cpp:6069-6093 */
static void lbt_pass(double *x, double theta)
{
  double st = sin(theta), ct = cos(theta), tt = st / ct;
  double x0 = x[0], px0 = x[1], y0 = x[2], py0 = x[3], z0 = x[4], pz0 = x[5];
  double ps0 = sqrt((1 + pz0) * (1 + pz0) - px0 * px0 - py0 * py0);
  double h0 = (1 + pz0) - ps0;
  double pxs = (px0 - tt * h0) / cos(theta);
  double pys = py0 / ct;
  double pzs = pz0 - tt * px0 + tt * tt * h0;
  double pss = sqrt((1 + pzs) * (1 + pzs) - pxs * pxs - pys * pys);
  double hs = (1 + pzs) - pss;
  double xs = tt * z0 + (1 + (pxs / pss) * st) * x0;
  double ys = y0 + st * (pys / pss) * x0;
  double zs = z0 / ct + (-hs / pss) * st * x0;
  x[0] = xs; x[1] = pxs; x[2] = ys; x[3] = pys; x[4] = zs; x[5] = pzs;
}

/* ILBT_Pass, simtrack.cpp:6095-6123 */
static void ilbt_pass(double *x, double theta)
{
  double st = sin(theta), ct = cos(theta);
  double xs = x[0], pxs = x[1], ys = x[2], pys = x[3], zs = x[4], pzs = x[5];
  double pss = sqrt((1 + pzs) * (1 + pzs) - pxs * pxs - pys * pys);
  double hs = 1 + pzs - pss;
  double hxs = pxs / pss, hys = pys / pss, hzs = -hs / pss;
  double px0 = (pxs + hs * st) * ct;
  double py0 = pys * ct;
  double pz0 = pzs + pxs * st;
  double x0 = (xs - zs * st) / (1 + hxs * st - hzs * st * st);
  double z0 = (zs - hzs * st * x0) * ct;
  double y0 = ys - st * hys * x0;
  x[0] = x0; x[1] = px0; x[2] = y0; x[3] = py0; x[4] = z0; x[5] = pz0;
}

/* cerrf, simtrack.cpp:6258-6323 */
void port_cerrf(double xx, double yy, double *wx, double *wy)
{
  int n, nc, nu;
  double x, y, q, h, xl, xh, yh, tx, ty, tn, sx, sy, saux;
  double rx[33], ry[33];
  const double cc = 1.12837916709551, zero = 0, one = 1, two = 2, half = .5, xlim = 5.33, ylim = 4.29,
               fac1 = 3.2, fac2 = 23, fac3 = 21;
  x = fabs(xx);
  y = fabs(yy);
  if (y < ylim && x < xlim) {
    q = (one - y / ylim) * sqrt(one - (x / xlim) * (x / xlim));
    h = one / (fac1 * q);
    nc = 7 + (int)(fac2 * q);
    xl = pow(h, (1 - nc));
    xh = y + half / h;
    yh = x;
    nu = 10 + (int)(fac3 * q);
    rx[nu + 1] = zero;
    ry[nu + 1] = zero;
    for (n = nu; n >= 1; n--) {
      tx = xh + n * rx[n + 1];
      ty = yh - n * ry[n + 1];
      tn = tx * tx + ty * ty;
      rx[n] = half * tx / tn;
      ry[n] = half * ty / tn;
    }
    sx = zero;
    sy = zero;
    for (n = nc; n >= 1; n--) {
      saux = sx + xl;
      sx = rx[n] * saux - ry[n] * sy;
      sy = rx[n] * sy + ry[n] * saux;
      xl = h * xl;
    }
    *wx = cc * sx;
    *wy = cc * sy;
  } else {
    xh = y;
    yh = x;
    rx[1] = zero;
    ry[1] = zero;
    for (n = 9; n >= 1; n--) {
      tx = xh + n * rx[1];
      ty = yh - n * ry[1];
      tn = tx * tx + ty * ty;
      rx[1] = half * tx / tn;
      ry[1] = half * ty / tn;
    }
    *wx = cc * rx[1];
    *wy = cc * ry[1];
  }
  if (yy < zero) {
    *wx = two * exp(y * y - x * x) * cos(two * x * y) - *wx;
    *wy = -two * exp(y * y - x * x) * sin(two * x * y) - *wy;
    if (xx > zero) *wy = -*wy;
  } else {
    if (xx < zero) *wy = -*wy;
  }
}

/* BB4D (x, y, gamma, N, sigmax, sigmay) overload, simtrack.cpp:6325-6377 */
static void bb4d(double x, double y, double gamma, double N, double sigmax, double sigmay, double *Dpx,
                 double *Dpy)
{
  const double rp = 1.53469826769e-18;
  double x1, y1, x2, y2, signx, signy;
  signx = ((x >= 0.0) ? (1) : (-1));
  signy = ((y >= 0.0) ? (1) : (-1));
  if (x == 0. && y == 0.) {
    *Dpx = 0.;
    *Dpy = 0.;
  } else if (fabs(sigmax - sigmay) / sigmax < 1.0e-6) {
    double r2 = x * x + y * y;
    double t1 = 2 * N * rp / gamma / r2;
    double t2 = 1 - exp(-r2 / 2 / sigmax / sigmax);
    *Dpx = t1 * x * t2;
    *Dpy = t1 * y * t2;
  } else if (sigmax > sigmay) {
    double t1 = (2. * N * rp / gamma) * sqrt(PORT_PI / 2. / (sigmax * sigmax - sigmay * sigmay));
    double t2 = exp(-x * x / 2. / sigmax / sigmax - y * y / 2. / sigmay / sigmay);
    double t3 = sqrt(2. * (sigmax * sigmax - sigmay * sigmay));
    double w1r, w1i, w2r, w2i;
    x1 = fabs(x) / t3;
    y1 = fabs(y) / t3;
    x2 = fabs(x) * sigmay / sigmax / t3;
    y2 = fabs(y) * sigmax / sigmay / t3;
    port_cerrf(x1, y1, &w1r, &w1i);
    port_cerrf(x2, y2, &w2r, &w2i);
    *Dpy = t1 * (w1r - t2 * w2r) * signy;
    *Dpx = t1 * (w1i - t2 * w2i) * signx;
  } else if (sigmax < sigmay) {
    double t1 = (2 * N * rp / gamma) * sqrt(PORT_PI / 2 / (sigmay * sigmay - sigmax * sigmax));
    double t2 = exp(-x * x / 2 / sigmax / sigmax - y * y / 2 / sigmay / sigmay);
    double t3 = sqrt(2 * (sigmay * sigmay - sigmax * sigmax));
    double w1r, w1i, w2r, w2i;
    x1 = fabs(x) / t3;
    y1 = fabs(y) / t3;
    x2 = fabs(x) * sigmay / sigmax / t3;
    y2 = fabs(y) * sigmax / sigmay / t3;
    port_cerrf(y1, x1, &w1r, &w1i);
    port_cerrf(y2, x2, &w2r, &w2i);
    *Dpy = t1 * (w1i - t2 * w2i) * signy;
    *Dpx = t1 * (w1r - t2 * w2r) * signx;
  }
}

/* Inverse normal CDF (AS241) used for the slice centroids; the reference
 * takes it from GSL (simtrack.cpp:6614). */
static double as241_pinv(double P)
{
  static const double a[8] = {3.387132872796366608, 133.14166789178437745, 1971.5909503065514427,
                              13731.693765509461125, 45921.953931549871457, 67265.770927008700853,
                              33430.575583588128105, 2509.0809287301226727};
  static const double b[8] = {1.0, 42.313330701600911252, 687.1870074920579083, 5394.1960214247511077,
                              21213.794301586595867, 39307.89580009271061, 28729.085735721942674,
                              5226.495278852545925};
  static const double c[8] = {1.42343711074968357734, 4.6303378461565452959, 5.7694972214606914055,
                              3.64784832476320460504, 1.27045825245236838258, 0.24178072517745061177,
                              0.0227238449892691845833, 7.7454501427834140764e-4};
  static const double d[8] = {1.0, 2.05319162663775882187, 1.6763848301838038494, 0.68976733498510000455,
                              0.14810397642748007459, 0.0151986665636164571966, 5.475938084995344946e-4,
                              1.05075007164441684324e-9};
  static const double e[8] = {6.6579046435011037772, 5.4637849111641143699, 1.7848265399172913358,
                              0.29656057182850489123, 0.026532189526576123093, 0.0012426609473880784386,
                              2.71155556874348757815e-5, 2.01033439929228813265e-7};
  static const double f[8] = {1.0, 0.59983220655588793769, 0.13692988092273580531,
                              0.0148753612908506148525, 7.868691311456132591e-4, 1.8463183175100546818e-5,
                              1.4215117583164458887e-7, 2.04426310338993978564e-15};
  const double *num, *den;
  double q = P - 0.5, r, u, v;
  int i;
  if (fabs(q) <= 0.425) {
    r = 0.180625 - q * q;
    num = a; den = b;
  } else {
    r = sqrt(-log((P < 0.5) ? P : 1.0 - P));
    if (r <= 5.0) { r = r - 1.6; num = c; den = d; }
    else { r = r - 5.0; num = e; den = f; }
  }
  u = num[7];
  v = den[7];
  for (i = 7; i > 0; i--) u = r * u + num[i - 1];
  for (i = 7; i > 0; i--) v = r * v + den[i - 1];
  if (fabs(q) <= 0.425) return q * (u / v);
  return (P < 0.5) ? -(u / v) : (u / v);
}

/* BB6D, simtrack.cpp:6579-6678 */
static void bb6d(double *x, double gamma, double Np, double bbscale, double sigma_l, int N_slice,
                 double emitx, double betax_s, double alfx_s, double emity, double betay_s, double alfy_s)
{
  const double rp = 1.534698e-18;
  double x0[6], Np_slice[64], z_star[64], yv[64];
  double S, gx, gy, betax, alfx, betay, alfy, sigmax, sigmay, dsx, dsy, dUx, dUy;
  double X, Y, Dpx, Dpy, t1, t2, t3, t4;
  int i, j;
  (void)alfx; (void)alfy;
  for (i = 0; i < N_slice; i++) Np_slice[i] = 1.0 * Np / N_slice;
  if (N_slice == 11) {
    static const double tab[11] = {1.7996765362153655, 1.1049618149811977, 0.75072324235797372,
                                   0.47407703558819131, 0.23041113693387344, 0., -0.23041113693387344,
                                   -0.47407703558819131, -0.75072324235797372, -1.1049618149811977,
                                   -1.7996765362153655};
    for (i = 0; i < 11; i++) z_star[i] = tab[i] * sigma_l;
  } else {
    for (i = 0; i < N_slice - 1; i++) yv[i] = as241_pinv((i + 1) * 1.0 / N_slice);
    z_star[0] = N_slice * (exp(-yv[0] * yv[0] / 2)) / sqrt(2.0 * 3.14159265);
    z_star[N_slice - 1] = N_slice * (0 - exp(-yv[0] * yv[0] / 2)) / sqrt(2.0 * 3.14159265);
    for (i = 1; i < N_slice - 1; i++)
      z_star[i] = N_slice * (exp(-yv[i] * yv[i] / 2) - exp(-yv[i - 1] * yv[i - 1] / 2)) / sqrt(2.0 * 3.14159265);
    for (i = 0; i < N_slice; i++) z_star[i] = z_star[i] * sigma_l;
  }
  for (i = 0; i < N_slice; i++) {
    for (j = 0; j < 6; j++) x0[j] = x[j];
    S = (x0[4] - z_star[i]) / 2.0;
    gx = (1.0 + alfx_s * alfx_s) / betax_s;
    gy = (1.0 + alfy_s * alfy_s) / betay_s;
    betax = betax_s + 2 * S * alfx_s + S * S * gx;
    alfx = (alfx_s + gx * S);
    betay = betay_s + 2 * S * alfy_s + S * S * gy;
    alfy = (alfy_s + gy * S);
    sigmax = sqrt(emitx * betax);
    sigmay = sqrt(emity * betay);
    dsx = 2.0 * emitx * (alfx_s + S * gx);
    dsy = 2.0 * emity * (alfy_s + S * gy);
    X = x0[0] + x0[1] * S;
    Y = x0[2] + x0[3] * S;
    bb4d(X, Y, gamma, Np_slice[i], sigmax, sigmay, &Dpx, &Dpy);
    t1 = 1.0 / 2. / (sigmax * sigmax - sigmay * sigmay);
    t2 = X * Dpx + Y * Dpy;
    t3 = 2. * Np_slice[i] * rp / gamma;
    t4 = exp(-X * X / 2. / sigmax / sigmax - Y * Y / 2. / sigmay / sigmay);
    x[0] = x0[0] - S * Dpx * bbscale;
    x[1] = x0[1] + Dpx * bbscale;
    x[2] = x0[2] - S * Dpy * bbscale;
    x[3] = x0[3] + Dpy * bbscale;
    x[4] = x0[4];
    if (fabs(sigmax - sigmay) / sigmax < 1.0e-6) {
      x[5] = x0[5] + 0.5 * Dpx * bbscale * (x0[1] + 0.5 * Dpx * bbscale)
             + 0.5 * Dpy * bbscale * (x0[3] + 0.5 * Dpy * bbscale)
             + (1.0 / sigmax / sigmax) * dsx * (t3 * bbscale / 4.) * t4;
    } else if (sigmax > sigmay) {
      dUx = t1 * bbscale * (t2 + t3 * (sigmay / sigmax * t4 - 1.));
      dUy = -t1 * bbscale * (t2 + t3 * (sigmax / sigmay * t4 - 1.));
      x[5] = x0[5] + 0.5 * Dpx * bbscale * (x0[1] + 0.5 * Dpx * bbscale)
             + 0.5 * Dpy * bbscale * (x0[3] + 0.5 * Dpy * bbscale)
             - (0.5 * dsx * dUx + 0.5 * dsy * dUy);
    } else {
      dUy = -t1 * bbscale * (t2 + t3 * (sigmax / sigmay * t4 - 1.));
      dUx = t1 * bbscale * (t2 + t3 * (sigmay / sigmax * t4 - 1.));
      x[5] = x0[5] + 0.5 * Dpx * bbscale * (x0[1] + 0.5 * Dpx * bbscale)
             + 0.5 * Dpy * bbscale * (x0[3] + 0.5 * Dpy * bbscale)
             - (0.5 * dsx * dUx + 0.5 * dsy * dUy);
    }
  }
}

/* BEAMBEAM::Pass -> BEAMBEAM_Pass, simtrack.cpp:11191-11195, 7343-7356 */
static void beambeam_pass(double *x, const port_elem *e, const port_gp *gp)
{
  double NP = e->p[0], BBSCALE = e->p[1], SIGMAL = e->p[2];
  double EMITX = e->p[3], BETAX = e->p[4], ALFAX = e->p[5];
  double EMITY = e->p[6], BETAY = e->p[7], ALFAY = e->p[8];
  if (NP == 0.) return;
  if (e->treatment == 6) {
    bb6d(x, gp->gamma, NP, BBSCALE, SIGMAL, e->nslice, EMITX, BETAX, ALFAX, EMITY, BETAY, ALFAY);
  } else {
    double Dpx, Dpy;
    bb4d(x[0], x[2], gp->gamma, NP, sqrt(EMITX * BETAX), sqrt(EMITY * BETAY), &Dpx, &Dpy);
    x[1] = x[1] + Dpx * BBSCALE;
    x[3] = x[3] + Dpy * BBSCALE;
  }
}

int port_pass(const port_elem *e, const port_gp *gp, double *x)
{
  int mis;
  init_coeffs();
  if (e->type == PORT_DRIFT || e->type == PORT_MARKER) { /* DRIFT::Pass 8426, MARKER::Pass 10617 */
    drift(x, e->L, gp);
    return 0;
  }
  if (e->type == PORT_PATCH) { /* PATCH::Pass 12323: no GtoL */
    patch_pass(x, e->p[0], e->p[1], e->p[2], e->p[3], gp);
    return 0;
  }
  mis = misaligned(e);
  if (mis < 0) return -1;
  if (mis) gtol1(x, e->dx, e->dy, e->dpsi);
  switch (e->type) {
  case PORT_SBEND: sbend_pass(x, e->L, e->p[0], e->p[1], e->p[2], gp); break;
  case PORT_GSBEND: gsbend_pass(x, e->L, e->p[0], e->p[1], e->p[2], e->p[3], gp); break;
  case PORT_QUAD: thick_pass(x, e->L, e->nint, e->p[0], e->p[1], 1, gp); break;
  case PORT_SKEWQ: thick_pass(x, e->L, e->nint, 0., e->p[0], 1, gp); break;
  case PORT_SEXT: thick_pass(x, e->L, e->nint, e->p[0], e->p[1], 2, gp); break;
  case PORT_OCT: thick_pass(x, e->L, e->nint, e->p[0], e->p[1], 3, gp); break;
  case PORT_MULT: mult_pass(x, e->L, e->nint, e->norder, e->knl, e->knsl, gp); break;
  case PORT_GMULT:
  case PORT_SBENDMULT:
    bendmult_pass(x, e->L, e->nint, e->norder, e->p[0], e->p[1], e->p[2], e->knl, e->knsl, gp);
    break;
  case PORT_KICKER: kick_pass(x, e->L, e->p[0], e->p[1], gp); break;
  case PORT_HKICKER: kick_pass(x, e->L, e->p[0], 0., gp); break;
  case PORT_VKICKER: kick_pass(x, e->L, 0., e->p[0], gp); break;
  case PORT_RFCAV: rfcav_pass(x, e->L, e->p[0], e->p[1], e->p[2], gp); break;
  case PORT_CRABRF: crabrf_pass(x, e->L, e->p[0], e->p[1], e->p[2], gp); break;
  case PORT_CCMULT:
    ccmult_pass(x, e->L, e->p[0], e->p[1], e->p[2], e->p[3], e->p[4], e->p[5], e->p[6], e->p[7], e->p[8],
                e->p[9], e->p[10], gp);
    break;
  case PORT_LBT: lbt_pass(x, e->p[0]); break;
  case PORT_ILBT: ilbt_pass(x, e->p[0]); break;
  case PORT_BEAMBEAM: beambeam_pass(x, e, gp); break;
  case PORT_SOLEN: solen_pass(x, e->L, e->p[0], gp); break;
  default: return -1;
  }
  if (mis) ltog1(x, e->dx, e->dy, e->dpsi);
  return 0;
}

static int lost_check(const port_elem *e, const double *x, double r2)
{
  if (fabs(x[0]) > e->apx || fabs(x[2]) > e->apy || isnan(x[0]) || isnan(x[2])) return 1;
  if (r2 > 0.0 && x[0] * x[0] + x[2] * x[2] > r2) return 1;
  return 0;
}

/* Track, simtrack.cpp:20791-20814 */
void port_track(const port_elem *e, long ne, const port_gp *gp, double *x, long n, int nturn, double radius,
                int *stable, int *lost_turn, int *lost_post)
{
  const double r2 = radius > 0.0 ? radius * radius : 0.0;
  long i, j;
  int t;
  for (i = 0; i < n; i++) {
    double *xi = x + 6 * i;
    int lost = 0;
    lost_turn[i] = 0;
    lost_post[i] = 0;
    if (fabs(xi[0]) > 0.1 || fabs(xi[2]) > 0.1 || stable[i] == 0) {
      stable[i] = 0;
      continue;
    }
    stable[i] = 1;
    for (t = 0; t < nturn && !lost; t++) {
      for (j = 0; j < ne; j++) {
        port_pass(e + j, gp, xi);
        if (lost_check(e + j, xi, r2)) {
          stable[i] = 0; lost_turn[i] = t; lost_post[i] = (int)j; lost = 1;
          break;
        }
      }
    }
  }
}

void port_track_dump(const port_elem *e, long ne, const port_gp *gp, double *x, int nturn, double radius,
                     double *dump, int *stable, int *lost_turn, int *lost_post)
{
  const double r2 = radius > 0.0 ? radius * radius : 0.0;
  long j;
  int t;
  *stable = 1; *lost_turn = 0; *lost_post = 0;
  if (fabs(x[0]) > 0.1 || fabs(x[2]) > 0.1) { *stable = 0; return; }
  for (t = 0; t < nturn; t++) {
    for (j = 0; j < ne; j++) {
      port_pass(e + j, gp, x);
      memcpy(dump + ((long)t * ne + j) * 6, x, 6 * sizeof(double));
      if (lost_check(e + j, x, r2)) {
        *stable = 0; *lost_turn = t; *lost_post = (int)j;
        return;
      }
    }
  }
}

/* DFT power of the samples at one tune; the phase argument and the sums are
 * formed in the reference's order (simtrack.cpp:2302-2306, 2335-2339). */
static double dft_power(int n, const double *x, const double *px, double tune)
{
  const double pi_ref = 3.14159265358979323; /* PI, simtrack.cpp:23 */
  double re = 0.0, im = 0.0;
  int i;
  for (i = 0; i < n; i++) {
    const double arg = -2 * pi_ref * i * tune;
    const double c = cos(arg), s = sin(arg);
    if (px) {
      re = re + x[i] * c - px[i] * s;
      im = im + x[i] * s + px[i] * c;
    } else {
      re = re + x[i] * c;
      im = im + x[i] * s;
    }
  }
  return re * re + im * im;
}

/* Coarse scan with step 1e-3 over [lower, upper), then repeated zooms to
 * [peak - step, peak + step) with a ten times finer step, until the step is
 * no longer above 1e-12; the first strict maximum of each scan wins. */
double port_fine_tune(int n, const double *x, const double *px, double tune_lower, double tune_upper)
{
  double step = 0.001, lo = tune_lower, hi = tune_upper, peak = tune_lower;
  for (;;) {
    double best = 0.0, t = lo;
    peak = lo;
    do {
      const double p = dft_power(n, x, px, t);
      if (p > best) { best = p; peak = t; }
      t = t + step;
    } while (t < hi);
    lo = peak - step;
    hi = peak + step;
    step = step / 10.;
    if (!(step > 1.0e-12)) break;
  }
  return peak;
}
