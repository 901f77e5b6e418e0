/*
 * Flat-array harness around the QuickCBC reference, compiled together with
 * the reference's own sources (by path, unmodified) into oracle/_ref.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this.  It turns
 * the reference's row-pointer (double**) interface into flat row-major
 * buffers that ctypes can pass, and adds an OpenMP batch loop over
 * parameter sets that mirrors the reference's own per-chain
 * `#pragma omp parallel for` (QuickCBC.c:2063-2067).
 *
 * Functions called (reference file:line):
 *   fulltemplates        QuickCBC.c:3683     fullphaseamp   QuickCBC.c:3780
 *   log_likelihood_full  QuickCBC.c:4236     heterodyne     QuickCBC.c:5112
 *   log_likelihood_het   QuickCBC.c:5303     het_space      QuickCBC.c:4570
 *   IMRPhenomDGenerateh22FDAmpPhase  IMRPhenomD.c:186
 *   F_ant / Times        Utilities.c:995 / 1078     fbegin Utilities.c:587
 *   fourier_nwip         Utilities.c:716
 *   templates            QuickCBC.c:3527     AmpPhase       QuickCBC.c:3395
 *   log_likelihood_intrinsic  QuickCBC.c:4093
 *   het_diff             QuickCBC.c:4966     Fisher_Het     QuickCBC.c:5446
 *   tukey                Utilities.c:635     makespec       Utilities.c:1908 (called directly)
 * and two restatements of input steps that live inside QuickCBC.c's main():
 *   ref_framed_count     the row count of QuickCBC.c:205-211 (same fscanf / feof loop)
 *   ref_condition        QuickCBC.c:244-258 + 309-313: tukey, gsl_fft_real_radix2_transform,
 *                        times sqrt(Tobs)/N
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>
#include "QuickCBC.h"
#include "Utilities.h"

/* The reference headers leave these undeclared in QuickCBC.h. */
void F_ant(double psi, double alpha, double sindelta, double GMST, double *Fplus, double *Fcross, int id);
void Times(double alpha, double sindelta, double GMST, double *dtimes);

static double **rows(double *flat, int nrow, int ncol) {
  double **r = (double **)malloc((size_t)(nrow + 1) * sizeof(double *));
  for (int i = 0; i < nrow; i++) r[i] = flat + (size_t)i * ncol;
  r[nrow] = NULL;
  return r;
}

struct Net *ref_net_new(int nifo, const int *labels, double Tobs, double GMST) {
  struct Net *net = (struct Net *)calloc(1, sizeof(struct Net));
  net->Nifo = nifo;
  net->Tobs = Tobs;
  net->GMST = GMST;
  net->labels = (int *)calloc((size_t)nifo + 1, sizeof(int));
  for (int i = 0; i < nifo; i++) net->labels[i] = labels[i];
  net->tds = (double *)calloc((size_t)nifo + 1, sizeof(double));
  net->tmin = Tobs - 3.5 < 1.5 ? 1.5 : Tobs - 3.5;   /* QuickCBC.c:178-183 */
  net->tmax = Tobs - 0.5;
  return net;
}

void ref_net_free(struct Net *net) {
  if (!net) return;
  free(net->labels); free(net->tds); free(net);
}

static RealVector *wrap_freq(const double *freq, int n) {
  RealVector *v = (RealVector *)malloc(sizeof(RealVector));
  v->data = (double *)freq;
  v->length = (size_t)n;
  return v;
}

int ref_amp_phase(const double *freq, int n, double phi0, double fRef, double m1_SI, double m2_SI,
                  double chi1, double chi2, double dist, double *amp, double *phase) {
  AmpPhaseFDWaveform *ap = NULL;
  RealVector *fv = wrap_freq(freq, n);
  int ret = IMRPhenomDGenerateh22FDAmpPhase(&ap, fv, phi0, fRef, m1_SI, m2_SI, chi1, chi2, dist);
  memcpy(amp, ap->amp, sizeof(double) * (size_t)n);
  memcpy(phase, ap->phase, sizeof(double) * (size_t)n);
  DestroyAmpPhaseFDWaveform(ap);
  free(fv);
  return ret;
}

double ref_fbegin(double *params) { return fbegin(params); }

void ref_F_ant(double psi, double alpha, double sindelta, double GMST, int id, double *out2) {
  F_ant(psi, alpha, sindelta, GMST, &out2[0], &out2[1], id);
}

void ref_Times(double alpha, double sindelta, double GMST, double *out3) {
  double t[5];
  Times(alpha, sindelta, GMST, t);
  out3[0] = t[0]; out3[1] = t[1]; out3[2] = t[2];
}

/* hflat: Nifo x N half-complex rows */
void ref_fulltemplates(struct Net *net, double *hflat, const double *freq, int nfreq, double *params, int N) {
  double **h = rows(hflat, net->Nifo, N);
  RealVector *fv = wrap_freq(freq, nfreq);
  fulltemplates(net, h, fv, params, N);
  free(fv); free(h);
}

/* amp/phase: Nifo x (N/2) rows; nfreq must be >= N/2 */
void ref_fullphaseamp(struct Net *net, double *aflat, double *pflat, const double *freq, int nfreq, double *params, int N) {
  double **a = rows(aflat, net->Nifo, N / 2);
  double **p = rows(pflat, net->Nifo, N / 2);
  RealVector *fv = wrap_freq(freq, nfreq);
  fullphaseamp(net, a, p, fv, params, N);
  free(fv); free(a); free(p);
}

double ref_fourier_nwip(double *a, double *b, double *Sn, int imin, int imax, int N) {
  return fourier_nwip(a, b, Sn, imin, imax, N);
}

/* D: Nifo x N, SN: Nifo x sn_stride (sn_stride >= N/2 + 1). */
double ref_lnl_full(struct Net *net, double *Dflat, double *params, const double *freq, double *SNflat,
                    int sn_stride, double *rho, int N, double Tobs) {
  double **D = rows(Dflat, net->Nifo, N);
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  double L = log_likelihood_full(net, D, params, fv, S, rho, N, Tobs);
  free(fv); free(D); free(S);
  return L;
}

/* OpenMP loop over B parameter sets (row-major B x 11); returns wall seconds. */
double ref_lnl_full_batch(struct Net *net, double *Dflat, const double *params, int B, const double *freq,
                          double *SNflat, int sn_stride, int N, double Tobs, double *lnl, int nthreads) {
  double **D = rows(Dflat, net->Nifo, N);
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 1)
  for (int b = 0; b < B; b++) {
    double p[11], rho[8];
    memcpy(p, params + (size_t)b * 11, sizeof(p));
    lnl[b] = log_likelihood_full(net, D, p, fv, S, rho, N, Tobs);
  }
  double t1 = omp_get_wtime();
  free(fv); free(D); free(S);
  return t1 - t0;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

/* intrinsic parametrisation: params of length NX + 3 (Nifo - 1) */
void ref_templates(struct Net *net, double *hflat, const double *freq, int nfreq, double *params, int N) {
  double **h = rows(hflat, net->Nifo, N);
  RealVector *fv = wrap_freq(freq, nfreq);
  templates(net, h, fv, params, N);
  free(fv); free(h);
}

double ref_lnl_intrinsic(struct Net *net, double *Dflat, double *params, const double *freq, double *SNflat,
                         int sn_stride, int N, double Tobs) {
  double **D = rows(Dflat, net->Nifo, N);
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  double L = log_likelihood_intrinsic(net, D, params, fv, S, N, Tobs);
  free(fv); free(D); free(S);
  return L;
}

/* Af, Pf: N/2 entries; entry 0 is left as passed in */
void ref_AmpPhase(double *Af, double *Pf, const double *freq, int nfreq, double *params, int N) {
  RealVector *fv = wrap_freq(freq, nfreq);
  AmpPhase(Af, Pf, fv, params, N);
  free(fv);
}

/* ---------------- heterodyne ---------------- */
struct Het *ref_het_new(void) { return (struct Het *)calloc(1, sizeof(struct Het)); }

/* het_space writes diagnostic files into the working directory. */
int ref_het_space(struct Net *net, struct Het *het, double *params, double *min, double *max,
                  const double *freq, double *SNflat, int sn_stride, int N, double Tobs) {
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  het_space(net, het, params, min, max, fv, S, N, Tobs);
  free(fv); free(S);
  return het->M;
}

/* Grid from the caller instead of het_space: fgrid[M] bin indices, MN, MM, J. */
void ref_het_set_grid(struct Het *het, const int *fgrid, int M, int MN, int MM, int J, double Tobs) {
  het->M = M; het->MN = MN; het->MM = MM; het->J = J;
  het->NR = (M - 1) / J;
  het->fgrid = int_vector(M);
  het->freq = CreateRealVector((size_t)M);
  for (int i = 0; i < M; i++) { het->fgrid[i] = fgrid[i]; het->freq->data[i] = (double)fgrid[i] / Tobs; }
}

void ref_heterodyne(struct Net *net, struct Het *het, double *Dflat, double *params, const double *freq,
                    double *SNflat, int sn_stride, int N, double Tobs) {
  double **D = rows(Dflat, net->Nifo, N);
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  heterodyne(net, het, D, params, fv, S, N, Tobs);
  free(fv); free(D); free(S);
}

/* sizes[0..5] = M, MN, MM, J, NR, Nifo */
void ref_het_sizes(struct Net *net, struct Het *het, int *sizes) {
  sizes[0] = het->M; sizes[1] = het->MN; sizes[2] = het->MM;
  sizes[3] = het->J; sizes[4] = het->NR; sizes[5] = net->Nifo;
}

/* Flatten the summary tables into caller buffers (row-major, same index order as struct Het). */
void ref_het_export(struct Net *net, struct Het *het, int *fgrid, double *freq, double *amp, double *phase,
                    double *IP, double *SL, double *lc, double *ls, double *aa, double *rc, double *rs,
                    double *logLb) {
  int M = het->M, J = het->J, NR = het->NR, nI = net->Nifo;
  for (int i = 0; i < M; i++) { fgrid[i] = het->fgrid[i]; freq[i] = het->freq->data[i]; }
  for (int id = 0; id < nI; id++)
    for (int j = 0; j < M; j++) {
      amp[id * M + j] = het->amp[id][j];
      phase[id * M + j] = het->phase[id][j];
    }
  for (int r = 0; r < NR; r++) {
    for (int a = 0; a <= J; a++)
      for (int b = 0; b <= J; b++) IP[(r * (J + 1) + a) * (J + 1) + b] = het->IP[r][a][b];
    for (int id = 0; id < nI; id++)
      for (int a = 0; a <= J; a++) {
        size_t o = ((size_t)r * nI + id) * (J + 1) + a;
        SL[o] = het->SL[r][id][a]; lc[o] = het->lc[r][id][a]; ls[o] = het->ls[r][id][a];
      }
  }
  for (int id = 0; id < nI; id++)
    for (int r = 0; r < NR; r++) {
      aa[id * NR + r] = het->aa[id][r]; rc[id * NR + r] = het->rc[id][r]; rs[id * NR + r] = het->rs[id][r];
    }
  *logLb = het->logLb;
}

double ref_lnl_het(struct Net *net, struct Het *het, double *params, double Tobs) {
  return log_likelihood_het(net, het, params, Tobs);
}

double ref_lnl_het_batch(struct Net *net, struct Het *het, const double *params, int B, double Tobs,
                         double *lnl, int nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 4)
  for (int b = 0; b < B; b++) {
    double p[11];
    memcpy(p, params + (size_t)b * 11, sizeof(p));
    lnl[b] = log_likelihood_het(net, het, p, Tobs);
  }
  return omp_get_wtime() - t0;
}

double ref_lnl_test(struct Net *net, struct Het *het, double *Dflat, double *params, const double *freq,
                    double *SNflat, int sn_stride, int N, double Tobs) {
  double **D = rows(Dflat, net->Nifo, N);
  double **S = rows(SNflat, net->Nifo, sn_stride);
  RealVector *fv = wrap_freq(freq, N / 2);
  double L = log_likelihood_test(net, het, D, params, fv, S, N, Tobs);
  free(fv); free(D); free(S);
  return L;
}

double ref_het_diff(struct Net *net, struct Het *het, double *params, double *dparams) {
  return het_diff(net, het, params, dparams);
}

/* fish: 11 x 11 (NP, ConstCBC.h:68) row-major */
void ref_Fisher_Het(struct Net *net, struct Het *het, double *fishflat, double *params, double Tobs) {
  double **F = rows(fishflat, 11, 11);
  Fisher_Het(net, het, F, params, Tobs);
  free(F);
}

void ref_het_free(struct Net *net, struct Het *het) {
  if (!het) return;
  if (het->IP) freehet(net, het);
  free(het);
}

/* Row count of a framed file by the loop of QuickCBC.c:205-211: one fscanf of two values per
 * pass until the end-of-file flag is set, starting from -1. */
int ref_framed_count(const char *path) {
  FILE *in = fopen(path, "r");
  if (!in) return -1;
  double x, y;
  int N = -1;
  while (!feof(in)) {
    if (fscanf(in, "%lf%lf", &x, &y) == 0) { N = -2; break; }   /* the reference would loop forever */
    N++;
  }
  fclose(in);
  return N;
}

/* D = FFT(tukey(x)) sqrt(Tobs)/N in GSL half-complex layout (QuickCBC.c:244-258, 309-313). */
void ref_condition(const double *x, int N, double Tobs, double *D) {
  memcpy(D, x, sizeof(double) * (size_t)N);
  double alpha = 2.0 * 0.4 / Tobs;
  tukey(D, alpha, N);
  gsl_fft_real_radix2_transform(D, 1, N);
  double fac = sqrt(Tobs) / (double)N;
  for (int i = 0; i < N; i++) D[i] *= fac;
}
