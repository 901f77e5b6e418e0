/*
 * Implementation of the GSL-API shim declared in gsl_shim.h.
 *
 * TEST INFRASTRUCTURE ONLY: linked into the reference oracle build
 * (oracle/_ref).  Written from the mathematical definitions that the GSL
 * manual documents for each routine:
 *   - natural cubic spline: tridiagonal system for the second derivatives
 *     with M_0 = M_{n-1} = 0, piecewise cubic y_i + b dx + c dx^2 + d dx^3;
 *   - Steffen (1990) monotone cubic interpolation;
 *   - LU with partial pivoting (P A = L U), inverse by forward/back solves;
 *   - symmetric eigenproblem by cyclic Jacobi rotations;
 *   - MT19937 (Matsumoto & Nishimura 1998) with the 2002 seeding recurrence;
 *   - radix-2 FFT with GSL's documented half-complex packing
 *     (r_0, r_1, ..., r_{n/2}, i_{n/2-1}, ..., i_1) and 1/n on the inverse.
 */
#include "gsl_shim.h"
#include <stdlib.h>
#include <string.h>
#include <stdio.h>

/* ------------------------------------------------------------------ */
gsl_vector *gsl_vector_alloc(size_t n) {
  gsl_vector *v = (gsl_vector *)calloc(1, sizeof(gsl_vector));
  v->size = n; v->stride = 1; v->data = (double *)calloc(n ? n : 1, sizeof(double)); v->owner = 1;
  return v;
}
void gsl_vector_free(gsl_vector *v) { if (!v) return; free(v->data); free(v); }
double gsl_vector_get(const gsl_vector *v, size_t i) { return v->data[i * v->stride]; }
void gsl_vector_set(gsl_vector *v, size_t i, double x) { v->data[i * v->stride] = x; }

gsl_matrix *gsl_matrix_alloc(size_t n1, size_t n2) {
  gsl_matrix *m = (gsl_matrix *)calloc(1, sizeof(gsl_matrix));
  m->size1 = n1; m->size2 = n2; m->tda = n2;
  m->data = (double *)calloc((n1 * n2) ? n1 * n2 : 1, sizeof(double)); m->owner = 1;
  return m;
}
void gsl_matrix_free(gsl_matrix *m) { if (!m) return; free(m->data); free(m); }
double gsl_matrix_get(const gsl_matrix *m, size_t i, size_t j) { return m->data[i * m->tda + j]; }
void gsl_matrix_set(gsl_matrix *m, size_t i, size_t j, double x) { m->data[i * m->tda + j] = x; }

gsl_permutation *gsl_permutation_alloc(size_t n) {
  gsl_permutation *p = (gsl_permutation *)calloc(1, sizeof(gsl_permutation));
  p->size = n; p->data = (size_t *)calloc(n ? n : 1, sizeof(size_t));
  for (size_t i = 0; i < n; i++) p->data[i] = i;
  return p;
}
void gsl_permutation_free(gsl_permutation *p) { if (!p) return; free(p->data); free(p); }

/* P A = L U, L unit lower triangular stored below the diagonal. */
int gsl_linalg_LU_decomp(gsl_matrix *A, gsl_permutation *p, int *signum) {
  size_t n = A->size1;
  *signum = 1;
  for (size_t i = 0; i < n; i++) p->data[i] = i;
  for (size_t j = 0; j < n; j++) {
    /* pivot: largest |a_ij| for i >= j */
    double amax = fabs(gsl_matrix_get(A, j, j));
    size_t ip = j;
    for (size_t i = j + 1; i < n; i++) {
      double a = fabs(gsl_matrix_get(A, i, j));
      if (a > amax) { amax = a; ip = i; }
    }
    if (ip != j) {
      for (size_t k = 0; k < n; k++) {
        double t = gsl_matrix_get(A, j, k);
        gsl_matrix_set(A, j, k, gsl_matrix_get(A, ip, k));
        gsl_matrix_set(A, ip, k, t);
      }
      size_t t = p->data[j]; p->data[j] = p->data[ip]; p->data[ip] = t;
      *signum = -*signum;
    }
    double ajj = gsl_matrix_get(A, j, j);
    if (ajj != 0.0) {
      for (size_t i = j + 1; i < n; i++) {
        double l = gsl_matrix_get(A, i, j) / ajj;
        gsl_matrix_set(A, i, j, l);
        for (size_t k = j + 1; k < n; k++)
          gsl_matrix_set(A, i, k, gsl_matrix_get(A, i, k) - l * gsl_matrix_get(A, j, k));
      }
    }
  }
  return GSL_SUCCESS;
}

/* Solve L U x = P b for each unit vector b = e_c; column c of the inverse. */
int gsl_linalg_LU_invert(const gsl_matrix *LU, const gsl_permutation *p, gsl_matrix *inverse) {
  size_t n = LU->size1;
  double *x = (double *)malloc(n * sizeof(double));
  for (size_t c = 0; c < n; c++) {
    for (size_t i = 0; i < n; i++) x[i] = (p->data[i] == c) ? 1.0 : 0.0;
    for (size_t i = 0; i < n; i++) {           /* forward, unit L */
      double s = x[i];
      for (size_t k = 0; k < i; k++) s -= gsl_matrix_get(LU, i, k) * x[k];
      x[i] = s;
    }
    for (size_t ii = n; ii-- > 0;) {           /* backward, U */
      double s = x[ii];
      for (size_t k = ii + 1; k < n; k++) s -= gsl_matrix_get(LU, ii, k) * x[k];
      x[ii] = s / gsl_matrix_get(LU, ii, ii);
    }
    for (size_t i = 0; i < n; i++) gsl_matrix_set(inverse, i, c, x[i]);
  }
  free(x);
  return GSL_SUCCESS;
}

/* ------------------------------------------------------------------ */
gsl_eigen_symmv_workspace *gsl_eigen_symmv_alloc(size_t n) {
  gsl_eigen_symmv_workspace *w = (gsl_eigen_symmv_workspace *)malloc(sizeof(*w));
  w->size = n; return w;
}
void gsl_eigen_symmv_free(gsl_eigen_symmv_workspace *w) { free(w); }

/* Cyclic Jacobi: A is destroyed; eigenvectors are the columns of evec. */
int gsl_eigen_symmv(gsl_matrix *A, gsl_vector *eval, gsl_matrix *evec, gsl_eigen_symmv_workspace *w) {
  (void)w;
  size_t n = A->size1;
  for (size_t i = 0; i < n; i++)
    for (size_t j = 0; j < n; j++) gsl_matrix_set(evec, i, j, i == j ? 1.0 : 0.0);
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (size_t i = 0; i < n; i++)
      for (size_t j = 0; j < n; j++) {
        double a = gsl_matrix_get(A, i, j);
        tot += a * a;
        if (i != j) off += a * a;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (size_t p = 0; p + 1 < n; p++)
      for (size_t q = p + 1; q < n; q++) {
        double apq = gsl_matrix_get(A, p, q);
        if (apq == 0.0) continue;
        double app = gsl_matrix_get(A, p, p), aqq = gsl_matrix_get(A, q, q);
        double theta = (aqq - app) / (2.0 * apq);
        double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (size_t k = 0; k < n; k++) {       /* A <- A J */
          double akp = gsl_matrix_get(A, k, p), akq = gsl_matrix_get(A, k, q);
          gsl_matrix_set(A, k, p, c * akp - s * akq);
          gsl_matrix_set(A, k, q, s * akp + c * akq);
        }
        for (size_t k = 0; k < n; k++) {       /* A <- J^T A */
          double apk = gsl_matrix_get(A, p, k), aqk = gsl_matrix_get(A, q, k);
          gsl_matrix_set(A, p, k, c * apk - s * aqk);
          gsl_matrix_set(A, q, k, s * apk + c * aqk);
        }
        for (size_t k = 0; k < n; k++) {       /* V <- V J */
          double vkp = gsl_matrix_get(evec, k, p), vkq = gsl_matrix_get(evec, k, q);
          gsl_matrix_set(evec, k, p, c * vkp - s * vkq);
          gsl_matrix_set(evec, k, q, s * vkp + c * vkq);
        }
      }
  }
  for (size_t i = 0; i < n; i++) gsl_vector_set(eval, i, gsl_matrix_get(A, i, i));
  return GSL_SUCCESS;
}

int gsl_eigen_symmv_sort(gsl_vector *eval, gsl_matrix *evec, gsl_eigen_sort_t sort_type) {
  size_t n = eval->size;
  for (size_t i = 0; i + 1 < n; i++) {         /* selection sort, swapping columns */
    size_t best = i;
    for (size_t j = i + 1; j < n; j++) {
      double a = gsl_vector_get(eval, j), b = gsl_vector_get(eval, best);
      int better = 0;
      switch (sort_type) {
        case GSL_EIGEN_SORT_VAL_ASC: better = a < b; break;
        case GSL_EIGEN_SORT_VAL_DESC: better = a > b; break;
        case GSL_EIGEN_SORT_ABS_ASC: better = fabs(a) < fabs(b); break;
        case GSL_EIGEN_SORT_ABS_DESC: better = fabs(a) > fabs(b); break;
      }
      if (better) best = j;
    }
    if (best != i) {
      double t = gsl_vector_get(eval, i);
      gsl_vector_set(eval, i, gsl_vector_get(eval, best));
      gsl_vector_set(eval, best, t);
      for (size_t k = 0; k < n; k++) {
        double u = gsl_matrix_get(evec, k, i);
        gsl_matrix_set(evec, k, i, gsl_matrix_get(evec, k, best));
        gsl_matrix_set(evec, k, best, u);
      }
    }
  }
  return GSL_SUCCESS;
}

/* ------------------------------------------------------------------ */
static const gsl_interp_type cspline_type = {"cspline", 1};
static const gsl_interp_type steffen_type = {"steffen", 2};
const gsl_interp_type *gsl_interp_cspline = &cspline_type;
const gsl_interp_type *gsl_interp_steffen = &steffen_type;

gsl_interp_accel *gsl_interp_accel_alloc(void) { return (gsl_interp_accel *)calloc(1, sizeof(gsl_interp_accel)); }
void gsl_interp_accel_free(gsl_interp_accel *a) { free(a); }

gsl_spline *gsl_spline_alloc(const gsl_interp_type *T, size_t size) {
  gsl_spline *s = (gsl_spline *)calloc(1, sizeof(gsl_spline));
  s->type = T; s->size = size;
  s->x = (double *)calloc(size, sizeof(double));
  s->y = (double *)calloc(size, sizeof(double));
  s->b = (double *)calloc(size, sizeof(double));
  s->c = (double *)calloc(size, sizeof(double));
  s->d = (double *)calloc(size, sizeof(double));
  return s;
}
void gsl_spline_free(gsl_spline *s) {
  if (!s) return;
  free(s->x); free(s->y); free(s->b); free(s->c); free(s->d); free(s);
}

static void natural_cubic(gsl_spline *s) {
  size_t n = s->size;
  double *x = s->x, *y = s->y;
  /* unknowns M_1..M_{n-2}; M_0 = M_{n-1} = 0.  Thomas algorithm. */
  double *M = (double *)calloc(n, sizeof(double));
  size_t m = n - 2;
  if (n >= 3) {
    double *diag = (double *)malloc(m * sizeof(double));
    double *rhs = (double *)malloc(m * sizeof(double));
    double *off = (double *)malloc(m * sizeof(double));
    for (size_t k = 0; k < m; k++) {
      size_t i = k + 1;
      double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
      diag[k] = 2.0 * (h0 + h1);
      off[k] = h1;
      rhs[k] = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
    }
    for (size_t k = 1; k < m; k++) {
      double w = off[k - 1] / diag[k - 1];
      diag[k] -= w * off[k - 1];
      rhs[k] -= w * rhs[k - 1];
    }
    M[m] = rhs[m - 1] / diag[m - 1];
    for (size_t k = m - 1; k-- > 0;) M[k + 1] = (rhs[k] - off[k] * M[k + 2]) / diag[k];
    free(diag); free(rhs); free(off);
  }
  for (size_t i = 0; i + 1 < n; i++) {
    double h = x[i + 1] - x[i];
    s->c[i] = 0.5 * M[i];
    s->d[i] = (M[i + 1] - M[i]) / (6.0 * h);
    s->b[i] = (y[i + 1] - y[i]) / h - h * (2.0 * M[i] + M[i + 1]) / 6.0;
  }
  free(M);
}

static double sgn(double a) { return (a > 0) - (a < 0); }

static void steffen(gsl_spline *s) {
  size_t n = s->size;
  double *x = s->x, *y = s->y;
  double *yp = (double *)calloc(n, sizeof(double));
  for (size_t i = 1; i + 1 < n; i++) {
    double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    double s0 = (y[i] - y[i - 1]) / h0, s1 = (y[i + 1] - y[i]) / h1;
    double p = (s0 * h1 + s1 * h0) / (h0 + h1);
    yp[i] = (sgn(s0) + sgn(s1)) * fmin(fmin(fabs(s0), fabs(s1)), 0.5 * fabs(p));
  }
  if (n >= 2) {
    double h0 = x[1] - x[0], s0 = (y[1] - y[0]) / h0;
    yp[0] = s0;
    double hl = x[n - 1] - x[n - 2], sl = (y[n - 1] - y[n - 2]) / hl;
    yp[n - 1] = sl;
  }
  for (size_t i = 0; i + 1 < n; i++) {
    double h = x[i + 1] - x[i], si = (y[i + 1] - y[i]) / h;
    s->b[i] = yp[i];
    s->c[i] = (3.0 * si - 2.0 * yp[i] - yp[i + 1]) / h;
    s->d[i] = (yp[i] + yp[i + 1] - 2.0 * si) / (h * h);
  }
  free(yp);
}

int gsl_spline_init(gsl_spline *s, const double xa[], const double ya[], size_t size) {
  memcpy(s->x, xa, size * sizeof(double));
  memcpy(s->y, ya, size * sizeof(double));
  if (s->type->kind == 1) natural_cubic(s); else steffen(s);
  return GSL_SUCCESS;
}

double gsl_spline_eval(const gsl_spline *s, double x, gsl_interp_accel *a) {
  size_t n = s->size;
  if (x < s->x[0] || x > s->x[n - 1]) return NAN;
  /* largest i with x_i <= x, clamped to the last interval */
  size_t lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    size_t mid = (lo + hi) / 2;
    if (s->x[mid] > x) hi = mid; else lo = mid;
  }
  if (a) a->cache = lo;
  double dx = x - s->x[lo];
  return s->y[lo] + dx * (s->b[lo] + dx * (s->c[lo] + dx * s->d[lo]));
}

/* ------------------------------------------------------------------ */
static const gsl_rng_type mt_type = {"mt19937"};
const gsl_rng_type *gsl_rng_mt19937 = &mt_type;
const gsl_rng_type *gsl_rng_default = &mt_type;
const gsl_rng_type *gsl_rng_env_setup(void) { return gsl_rng_default; }

gsl_rng *gsl_rng_alloc(const gsl_rng_type *T) {
  gsl_rng *r = (gsl_rng *)calloc(1, sizeof(gsl_rng));
  r->type = T;
  gsl_rng_set(r, 0);
  return r;
}
void gsl_rng_free(gsl_rng *r) { free(r); }

void gsl_rng_set(const gsl_rng *rc, unsigned long seed) {
  gsl_rng *r = (gsl_rng *)rc;
  if (seed == 0) seed = 4357;
  r->mt[0] = seed & 0xffffffffUL;
  for (int i = 1; i < 624; i++)
    r->mt[i] = (1812433253UL * (r->mt[i - 1] ^ (r->mt[i - 1] >> 30)) + (unsigned long)i) & 0xffffffffUL;
  r->mti = 624;
  r->has_spare = 0;
}

static unsigned long mt_next(gsl_rng *r) {
  static const unsigned long mag01[2] = {0x0UL, 0x9908b0dfUL};
  unsigned long y;
  if (r->mti >= 624) {
    int k;
    for (k = 0; k < 624 - 397; k++) {
      y = (r->mt[k] & 0x80000000UL) | (r->mt[k + 1] & 0x7fffffffUL);
      r->mt[k] = r->mt[k + 397] ^ (y >> 1) ^ mag01[y & 1];
    }
    for (; k < 623; k++) {
      y = (r->mt[k] & 0x80000000UL) | (r->mt[k + 1] & 0x7fffffffUL);
      r->mt[k] = r->mt[k + 397 - 624] ^ (y >> 1) ^ mag01[y & 1];
    }
    y = (r->mt[623] & 0x80000000UL) | (r->mt[0] & 0x7fffffffUL);
    r->mt[623] = r->mt[396] ^ (y >> 1) ^ mag01[y & 1];
    r->mti = 0;
  }
  y = r->mt[r->mti++];
  y ^= (y >> 11);
  y ^= (y << 7) & 0x9d2c5680UL;
  y ^= (y << 15) & 0xefc60000UL;
  y ^= (y >> 18);
  return y & 0xffffffffUL;
}

double gsl_rng_uniform(const gsl_rng *rc) { return (double)mt_next((gsl_rng *)rc) / 4294967296.0; }

double gsl_ran_gaussian(const gsl_rng *rc, double sigma) {
  gsl_rng *r = (gsl_rng *)rc;
  double x, y, s;
  do {                                    /* Marsaglia polar method */
    x = -1.0 + 2.0 * gsl_rng_uniform(r);
    y = -1.0 + 2.0 * gsl_rng_uniform(r);
    s = x * x + y * y;
  } while (s > 1.0 || s == 0.0);
  return sigma * y * sqrt(-2.0 * log(s) / s);
}

/* ------------------------------------------------------------------ */
static int cmp_double(const void *a, const void *b) {
  double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}
void gsl_sort(double *data, size_t stride, size_t n) {
  if (stride == 1) { qsort(data, n, sizeof(double), cmp_double); return; }
  double *tmp = (double *)malloc(n * sizeof(double));
  for (size_t i = 0; i < n; i++) tmp[i] = data[i * stride];
  qsort(tmp, n, sizeof(double), cmp_double);
  for (size_t i = 0; i < n; i++) data[i * stride] = tmp[i];
  free(tmp);
}
typedef struct { double k, v; } pair2;
static int cmp_pair(const void *a, const void *b) { return cmp_double(&((const pair2 *)a)->k, &((const pair2 *)b)->k); }
int gsl_sort_vector2(gsl_vector *v1, gsl_vector *v2) {
  size_t n = v1->size;
  pair2 *p = (pair2 *)malloc(n * sizeof(pair2));
  for (size_t i = 0; i < n; i++) { p[i].k = gsl_vector_get(v1, i); p[i].v = gsl_vector_get(v2, i); }
  qsort(p, n, sizeof(pair2), cmp_pair);
  for (size_t i = 0; i < n; i++) { gsl_vector_set(v1, i, p[i].k); gsl_vector_set(v2, i, p[i].v); }
  free(p);
  return GSL_SUCCESS;
}
double gsl_stats_median_from_sorted_data(const double d[], size_t stride, size_t n) {
  if (n == 0) return 0.0;
  size_t lhs = (n - 1) / 2, rhs = n / 2;
  return lhs == rhs ? d[lhs * stride] : 0.5 * (d[lhs * stride] + d[rhs * stride]);
}
double gsl_cdf_ugaussian_P(double x) { return 0.5 * erfc(-x / sqrt(2.0)); }

/* ------------------------------------------------------------------ */
/* In-place complex radix-2 FFT, sign = -1 forward, +1 backward (unscaled). */
static void cfft(double *re, double *im, size_t n, int sign) {
  for (size_t i = 1, j = 0; i < n; i++) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) { double t = re[i]; re[i] = re[j]; re[j] = t; t = im[i]; im[i] = im[j]; im[j] = t; }
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    double ang = sign * 2.0 * M_PI / (double)len;
    for (size_t i = 0; i < n; i += len)
      for (size_t k = 0; k < len / 2; k++) {
        double wr = cos(ang * (double)k), wi = sin(ang * (double)k);
        size_t a = i + k, b = i + k + len / 2;
        double xr = re[b] * wr - im[b] * wi, xi = re[b] * wi + im[b] * wr;
        re[b] = re[a] - xr; im[b] = im[a] - xi;
        re[a] += xr; im[a] += xi;
      }
  }
}

int gsl_fft_real_radix2_transform(double data[], size_t stride, size_t n) {
  double *re = (double *)malloc(n * sizeof(double)), *im = (double *)calloc(n, sizeof(double));
  for (size_t i = 0; i < n; i++) re[i] = data[i * stride];
  cfft(re, im, n, -1);
  data[0] = re[0];
  for (size_t k = 1; k < n / 2; k++) { data[k * stride] = re[k]; data[(n - k) * stride] = im[k]; }
  if (n > 1) data[(n / 2) * stride] = re[n / 2];
  free(re); free(im);
  return GSL_SUCCESS;
}

int gsl_fft_halfcomplex_radix2_backward(double data[], size_t stride, size_t n) {
  double *re = (double *)malloc(n * sizeof(double)), *im = (double *)calloc(n, sizeof(double));
  re[0] = data[0]; im[0] = 0.0;
  for (size_t k = 1; k < n / 2; k++) {
    re[k] = data[k * stride]; im[k] = data[(n - k) * stride];
    re[n - k] = re[k]; im[n - k] = -im[k];
  }
  if (n > 1) { re[n / 2] = data[(n / 2) * stride]; im[n / 2] = 0.0; }
  cfft(re, im, n, +1);
  for (size_t i = 0; i < n; i++) data[i * stride] = re[i];
  free(re); free(im);
  return GSL_SUCCESS;
}

int gsl_fft_halfcomplex_radix2_inverse(double data[], size_t stride, size_t n) {
  gsl_fft_halfcomplex_radix2_backward(data, stride, n);
  for (size_t i = 0; i < n; i++) data[i * stride] /= (double)n;
  return GSL_SUCCESS;
}
