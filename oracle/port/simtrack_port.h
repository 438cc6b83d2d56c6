/*
 * C restatement of SimTrack's element-by-element tracking path.
 * TEST INFRASTRUCTURE ONLY: the CUDA product never links or calls this.
 *
 * The restatement follows the reference's arithmetic operation by operation
 * (simtrack.cpp, file:line cited per function in simtrack_port.c) so that,
 * compiled for x86-64 without FMA contraction, it rounds exactly as the
 * reference does.  Scope: the exact-Hamiltonian path (GP.H_expand == false,
 * GP.radiate == false) used by the dynamic-aperture configurations, offset
 * and roll misalignments (GtoL1/LtoG1), and the Track() loss convention.
 */
#ifndef SIMTRACK_PORT_H
#define SIMTRACK_PORT_H

#ifdef __cplusplus
extern "C" {
#endif

enum port_type {
  PORT_DRIFT = 0, PORT_MARKER, PORT_SBEND, PORT_GSBEND, PORT_QUAD, PORT_SKEWQ, PORT_SEXT,
  PORT_OCT, PORT_MULT, PORT_GMULT, PORT_SBENDMULT, PORT_KICKER, PORT_HKICKER, PORT_VKICKER,
  PORT_RFCAV, PORT_CRABRF, PORT_CCMULT, PORT_LBT, PORT_ILBT, PORT_BEAMBEAM, PORT_SOLEN, PORT_PATCH
};

/* One element in "as constructed" form: the reference constructor's
 * arguments plus the public Element fields the Pass functions read. */
typedef struct {
  int type;
  int nint;     /* Nint (thick elements) */
  int norder;   /* Norder (MULT family) */
  int nslice;   /* BEAMBEAM NSLICE */
  int treatment;/* BEAMBEAM TREATMENT */
  int pad;
  double L;
  double p[16]; /* type-specific constructor scalars, in constructor order after L */
  double knl[11], knsl[11];
  double dx, dy, ds, dtheta, dphi, dpsi;
  double apx, apy;
} port_elem;

typedef struct {
  double gamma, beta, energy, brho, G;
  double Q;
  int quad_fringe;
  int pad;
  double m0, q, p; /* GP.m0 [kg], GP.q [C], GP.p [kg m/s] (solenoid) */
} port_gp;

/* Track n particles (AoS x[n*6]) for nturn turns: Track() semantics
 * (simtrack.cpp:20791-20814) plus an optional circular aperture radius
 * (radius <= 0 disables it).  stable[i] is overwritten. */
void port_track(const port_elem *e, long ne, const port_gp *gp, double *x, long n, int nturn,
                double radius, int *stable, int *lost_turn, int *lost_post);

/* One particle; dump[(turn*ne + j)*6 + k] after element j. */
void port_track_dump(const port_elem *e, long ne, const port_gp *gp, double *x, int nturn,
                     double radius, double *dump, int *stable, int *lost_turn, int *lost_post);

/* Single element pass (Element::Pass). Returns 0, or -1 for an unsupported element. */
int port_pass(const port_elem *e, const port_gp *gp, double *x);

/* Faddeeva function w(z) (cerrf, simtrack.cpp:6258-6323). */
void port_cerrf(double xx, double yy, double *wx, double *wy);

/* Peak-DFT tune of n samples (FineTuneFinder, simtrack.cpp:2288-2319; with
 * px != NULL the x/px form of simtrack.cpp:2321-2352). */
double port_fine_tune(int n, const double *x, const double *px, double tune_lower, double tune_upper);

#ifdef __cplusplus
}
#endif

#endif
