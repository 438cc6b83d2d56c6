/*
 * Minimal GSL declarations for compiling the SimTrack reference source as a
 * test oracle.  TEST INFRASTRUCTURE ONLY: nothing in the product links this.
 *
 * GSL itself is not installed in this environment.  The reference uses it at
 * these call sites (simtrack.cpp):
 *   - gsl_cdf_ugaussian_Pinv : BB6D slice centroids (6614), BB6D_Lumi (6716),
 *     BB6D_Angle (6958), BB6D_Angle_Lumi (7123), Zboundary_slices_Gaussian (3165)
 *   - gsl_rng_* / gsl_ran_*   : Init_GSL_Seeds (316-329), radiation (4275-4349)
 *   - gsl_eigen_nonsymmv*     : EigenSolver / EigenSolver_6D (1663-1733)
 * Only the inverse normal CDF is on the tracking path; it is implemented in
 * gsl_shim.c from Wichura's published algorithm AS241 (PPND16).  Every other
 * entry point aborts with a message, because the oracle never reaches it.
 */
#ifndef ORACLE_GSL_SHIM_ALL_H
#define ORACLE_GSL_SHIM_ALL_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double dat[2]; } gsl_complex;
#define GSL_REAL(z) ((z).dat[0])
#define GSL_IMAG(z) ((z).dat[1])

typedef struct {
  size_t size1, size2, tda;
  double *data;
} gsl_matrix;
typedef struct { gsl_matrix matrix; } gsl_matrix_view;

typedef struct {
  size_t size, stride;
  double *data; /* interleaved re/im */
} gsl_vector_complex;
typedef struct { gsl_vector_complex vector; } gsl_vector_complex_view;

typedef struct {
  size_t size1, size2, tda;
  double *data; /* interleaved re/im */
} gsl_matrix_complex;

typedef struct { size_t n; } gsl_eigen_nonsymmv_workspace;
typedef enum { GSL_EIGEN_SORT_VAL_ASC, GSL_EIGEN_SORT_VAL_DESC,
               GSL_EIGEN_SORT_ABS_ASC, GSL_EIGEN_SORT_ABS_DESC } gsl_eigen_sort_t;

typedef struct { const char *name; } gsl_rng_type;
typedef struct { const gsl_rng_type *type; unsigned long state; } gsl_rng;
extern const gsl_rng_type *gsl_rng_default;

double gsl_cdf_ugaussian_Pinv(double P);

gsl_matrix_view gsl_matrix_view_array(double *base, size_t n1, size_t n2);
gsl_vector_complex *gsl_vector_complex_alloc(size_t n);
void gsl_vector_complex_free(gsl_vector_complex *v);
gsl_complex gsl_vector_complex_get(const gsl_vector_complex *v, size_t i);
gsl_matrix_complex *gsl_matrix_complex_alloc(size_t n1, size_t n2);
void gsl_matrix_complex_free(gsl_matrix_complex *m);
gsl_vector_complex_view gsl_matrix_complex_column(gsl_matrix_complex *m, size_t j);
gsl_eigen_nonsymmv_workspace *gsl_eigen_nonsymmv_alloc(size_t n);
void gsl_eigen_nonsymmv_free(gsl_eigen_nonsymmv_workspace *w);
int gsl_eigen_nonsymmv(gsl_matrix *A, gsl_vector_complex *eval,
                       gsl_matrix_complex *evec, gsl_eigen_nonsymmv_workspace *w);
int gsl_eigen_nonsymmv_sort(gsl_vector_complex *eval, gsl_matrix_complex *evec,
                            gsl_eigen_sort_t sort_type);

void gsl_rng_env_setup(void);
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long s);
double gsl_rng_uniform(const gsl_rng *r);
double gsl_ran_gaussian(const gsl_rng *r, double sigma);
unsigned int gsl_ran_poisson(const gsl_rng *r, double mu);

#ifdef __cplusplus
}
#endif

#endif
