/*
 * GSL shim for the SimTrack reference oracle.  TEST INFRASTRUCTURE ONLY.
 *
 * The reference (simtrack.cpp) links GSL, which is absent here.  Only one GSL
 * routine lies on the tracking path: gsl_cdf_ugaussian_Pinv, the inverse of
 * the standard normal CDF, which BB6D (simtrack.cpp:6612-6619) evaluates for
 * the strong-bunch slice boundaries whenever NSLICE != 11.  It is restated
 * here from Wichura's published algorithm AS241 (PPND16, Applied Statistics
 * 37 (1988) 477-484): a rational approximation in three regions, evaluated
 * with Horner's rule from the highest coefficient, the central region scaled
 * as q * (P(r)/Q(r)).  GSL's gaussinv.c implements the same published
 * algorithm; its exact rounding sequence cannot be checked here, so the shim
 * is pinned instead against the N=11 centroid table hard-coded in BB6D
 * (simtrack.cpp:6593-6604), reproduced through the general centroid formula.
 *
 * Every other GSL entry point the reference declares aborts: the oracle
 * harness never calls random-number, radiation or eigen-solver code.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include "gsl/gsl_shim_all.h"

static double horner_ratio(const double *a, const double *b, int n, double r)
{
  double u = a[n - 1];
  double v = b[n - 1];
  int i;
  for (i = n - 1; i > 0; i--) u = r * u + a[i - 1];
  for (i = n - 1; i > 0; i--) v = r * v + b[i - 1];
  return u / v;
}

/* AS241 PPND16 coefficient sets (published with the algorithm). */
static const double as241_a[8] = {
  3.387132872796366608, 133.14166789178437745, 1971.5909503065514427,
  13731.693765509461125, 45921.953931549871457, 67265.770927008700853,
  33430.575583588128105, 2509.0809287301226727};
static const double as241_b[8] = {
  1.0, 42.313330701600911252, 687.1870074920579083, 5394.1960214247511077,
  21213.794301586595867, 39307.89580009271061, 28729.085735721942674,
  5226.495278852545925};
static const double as241_c[8] = {
  1.42343711074968357734, 4.6303378461565452959, 5.7694972214606914055,
  3.64784832476320460504, 1.27045825245236838258, 0.24178072517745061177,
  0.0227238449892691845833, 7.7454501427834140764e-4};
static const double as241_d[8] = {
  1.0, 2.05319162663775882187, 1.6763848301838038494, 0.68976733498510000455,
  0.14810397642748007459, 0.0151986665636164571966, 5.475938084995344946e-4,
  1.05075007164441684324e-9};
static const double as241_e[8] = {
  6.6579046435011037772, 5.4637849111641143699, 1.7848265399172913358,
  0.29656057182850489123, 0.026532189526576123093, 0.0012426609473880784386,
  2.71155556874348757815e-5, 2.01033439929228813265e-7};
static const double as241_f[8] = {
  1.0, 0.59983220655588793769, 0.13692988092273580531,
  0.0148753612908506148525, 7.868691311456132591e-4, 1.8463183175100546818e-5,
  1.4215117583164458887e-7, 2.04426310338993978564e-15};

double gsl_cdf_ugaussian_Pinv(double P)
{
  double q, r, x, pp;
  if (P == 1.0) return INFINITY;
  if (P == 0.0) return -INFINITY;
  q = P - 0.5;
  if (fabs(q) <= 0.425) {
    r = 0.180625 - q * q;
    return q * horner_ratio(as241_a, as241_b, 8, r);
  }
  pp = (P < 0.5) ? P : 1.0 - P;
  r = sqrt(-log(pp));
  if (r <= 5.0)
    x = horner_ratio(as241_c, as241_d, 8, r - 1.6);
  else
    x = horner_ratio(as241_e, as241_f, 8, r - 5.0);
  return (P < 0.5) ? -x : x;
}

static void not_in_shim(const char *fn)
{
  fprintf(stderr, "oracle gsl shim: %s is not provided (off the tracking path)\n", fn);
  abort();
}

static const gsl_rng_type shim_rng_type = {"shim-unavailable"};
const gsl_rng_type *gsl_rng_default = &shim_rng_type;

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2)
{
  gsl_matrix_view v;
  v.matrix.size1 = n1; v.matrix.size2 = n2; v.matrix.tda = n2; v.matrix.data = base;
  return v;
}
gsl_vector_complex *gsl_vector_complex_alloc(size_t n) { (void)n; not_in_shim("gsl_vector_complex_alloc"); return NULL; }
void gsl_vector_complex_free(gsl_vector_complex *v) { (void)v; not_in_shim("gsl_vector_complex_free"); }
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i)
{
  gsl_complex z = {{0.0, 0.0}};
  (void)v; (void)i; not_in_shim("gsl_vector_complex_get");
  return z;
}
gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2) { (void)n1; (void)n2; not_in_shim("gsl_matrix_complex_alloc"); return NULL; }
void gsl_matrix_complex_free(gsl_matrix_complex *m) { (void)m; not_in_shim("gsl_matrix_complex_free"); }
gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m, size_t j)
{
  gsl_vector_complex_view v = {{0, 0, NULL}};
  (void)m; (void)j; not_in_shim("gsl_matrix_complex_column");
  return v;
}
gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n) { (void)n; not_in_shim("gsl_eigen_nonsymmv_alloc"); return NULL; }
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w) { (void)w; not_in_shim("gsl_eigen_nonsymmv_free"); }
int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval, gsl_matrix_complex *evec,
                       gsl_eigen_nonsymmv_workspace *w)
{
  (void)A; (void)eval; (void)evec; (void)w; not_in_shim("gsl_eigen_nonsymmv"); return -1;
}
int gsl_eigen_nonsymmv_sort(gsl_vector_complex *eval, gsl_matrix_complex *evec, gsl_eigen_sort_t t)
{
  (void)eval; (void)evec; (void)t; not_in_shim("gsl_eigen_nonsymmv_sort"); return -1;
}
void gsl_rng_env_setup(void) { not_in_shim("gsl_rng_env_setup"); }
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) { (void)T; not_in_shim("gsl_rng_alloc"); return NULL; }
void gsl_rng_set(const gsl_rng *r, unsigned long s) { (void)r; (void)s; not_in_shim("gsl_rng_set"); }
/* radiate2's photon draws (simtrack.cpp:4345, 4349): the harness's streams
   (ref_harness.cpp, ref_rng_poisson / ref_rng_uniform) in place of GSL's. */
double ref_rng_uniform(void);
unsigned int ref_rng_poisson(double mu);
double gsl_rng_uniform(const gsl_rng *r) { (void)r; return ref_rng_uniform(); }
/* radiate1's quantum-excitation deviate (simtrack.cpp:4275): GSL's own
   stream does not exist here, so the harness supplies the tracker's
   per-particle counter-based stream (ref_harness.cpp, ref_rng_gaussian). */
double ref_rng_gaussian(void);
double gsl_ran_gaussian(const gsl_rng *r, double sigma) { (void)r; return sigma * ref_rng_gaussian(); }
unsigned int gsl_ran_poisson(const gsl_rng *r, double mu) { (void)r; return ref_rng_poisson(mu); }
