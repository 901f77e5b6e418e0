/*
 * GSL-API shim for building the QuickCBC reference as an oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  GSL is not installed in this image, but the
 * reference C files include <gsl/...> headers and call a small set of GSL
 * routines.  This header declares exactly that set, with the types and
 * semantics documented in the GSL reference manual (the public API; no GSL
 * source is used).  The implementations live in gslshim.c.
 *
 * Hot-path relevant routines (must match GSL's documented maths):
 *   gsl_interp_cspline  natural cubic spline (second derivative zero at both
 *                       ends) -- used by fring/fdamp in
 *                       IMRPhenomD_internals.c:479-513;
 *   gsl_linalg_LU_decomp / gsl_linalg_LU_invert (partial pivoting) -- used by
 *                       Inverse() in Utilities.c:962-1001 (heterodyne setup);
 *   gsl_eigen_symmv (+_sort) -- FisherEvec(), QuickCBC.c:2449-2546.
 * Everything else exists so that the reference translation units link.
 */
#ifndef QCBC_GSL_SHIM_H
#define QCBC_GSL_SHIM_H

#include <stddef.h>
#include <math.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846264338328
#endif

#define GSL_SUCCESS 0
#define GSL_EDOM 1

/* ---------- vectors, matrices, permutations ---------- */
typedef struct { size_t size; size_t stride; double *data; void *block; int owner; } gsl_vector;
typedef struct { size_t size1; size_t size2; size_t tda; double *data; void *block; int owner; } gsl_matrix;
typedef struct { size_t size; size_t *data; } gsl_permutation;

gsl_vector *gsl_vector_alloc(size_t n);
void gsl_vector_free(gsl_vector *v);
double gsl_vector_get(const gsl_vector *v, size_t i);
void gsl_vector_set(gsl_vector *v, size_t i, double x);

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2);
void gsl_matrix_free(gsl_matrix *m);
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j);
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x);

gsl_permutation *gsl_permutation_alloc(size_t n);
void gsl_permutation_free(gsl_permutation *p);

int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum);
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inverse);

/* ---------- symmetric eigensolver ---------- */
typedef struct { size_t size; } gsl_eigen_symmv_workspace;
typedef enum {
  GSL_EIGEN_SORT_VAL_ASC, GSL_EIGEN_SORT_VAL_DESC,
  GSL_EIGEN_SORT_ABS_ASC, GSL_EIGEN_SORT_ABS_DESC
} gsl_eigen_sort_t;
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n);
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w);
int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t sort_type);

/* ---------- interpolation ---------- */
typedef struct { const char *name; int kind; } gsl_interp_type;
extern const gsl_interp_type *gsl_interp_cspline;
extern const gsl_interp_type *gsl_interp_steffen;
typedef struct { size_t cache; } gsl_interp_accel;
typedef struct {
  const gsl_interp_type *type;
  size_t size;
  double *x, *y;
  double *b, *c, *d;   /* per-interval cubic coefficients */
} gsl_spline;
gsl_interp_accel *gsl_interp_accel_alloc(void);
void gsl_interp_accel_free(gsl_interp_accel *a);
gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size);
int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[], size_t size);
double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a);
void gsl_spline_free(gsl_spline *s);

/* ---------- random numbers ---------- */
typedef struct { const char *name; } gsl_rng_type;
typedef struct { const gsl_rng_type *type; unsigned long mt[624]; int mti; double gauss_spare; int has_spare; } gsl_rng;
extern const gsl_rng_type *gsl_rng_default;
extern const gsl_rng_type *gsl_rng_mt19937;
const gsl_rng_type *gsl_rng_env_setup(void);
gsl_rng *gsl_rng_alloc(const gsl_rng_type *T);
void gsl_rng_set(const gsl_rng *r, unsigned long seed);
void gsl_rng_free(gsl_rng *r);
double gsl_rng_uniform(const gsl_rng *r);
double gsl_ran_gaussian(const gsl_rng *r, double sigma);

/* ---------- sorting / statistics / cdf ---------- */
void gsl_sort(double *data, size_t stride, size_t n);
int gsl_sort_vector2(gsl_vector *v1, gsl_vector *v2);
double gsl_stats_median_from_sorted_data(const double sorted_data[], size_t stride, size_t n);
double gsl_cdf_ugaussian_P(double x);

/* ---------- radix-2 real FFT, half-complex storage ---------- */
int gsl_fft_real_radix2_transform(double data[], size_t stride, size_t n);
int gsl_fft_halfcomplex_radix2_inverse(double data[], size_t stride, size_t n);
int gsl_fft_halfcomplex_radix2_backward(double data[], size_t stride, size_t n);

#endif
