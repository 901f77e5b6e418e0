/*
 * The QuickCBC reference's own sampler code driven against the GPU drop-ins.
 *
 * TEST INFRASTRUCTURE ONLY.  `make -C oracle linked` compiles the reference's sources unmodified
 * (by path), weakens its definitions of the thirteen replaced functions with objcopy, and links
 * them with include/qcbc_forward.c (compiled with -DQCBC_FORWARD_COUNT), ref_harness.c, this
 * file and libqcbc_gpu.so into oracle/_ref/libquickcbc_linked.so.  Every call the reference's
 * code makes to a replaced name then goes through the forwarding stub to the GPU library;
 * tests/test_gpu_linked.py checks that with nm, the stub's call counters and the library's
 * launch counter, and checks the results against the library's own batched API.
 *
 * lk_mcmc runs the chain sequence of MCMC_all (QuickCBC.c:1781-2067) on NC = 12 chains:
 *   1. initial lnL of every chain by log_likelihood_full (QuickCBC.c:1898-1905);
 *   2. per chain Fisher_Het -> FisherEvec -> efix with het_diff (QuickCBC.c:1917-1923), inside
 *      `omp parallel for` as at QuickCBC.c:2019-2026;
 *   3. lnL reset by log_likelihood_het (QuickCBC.c:1944) and the history fill (1948-1955);
 *   4. `steps` sweeps of the reference's update() over all chains inside `omp parallel for`
 *      (QuickCBC.c:2050-2067), which proposes (Fisher, differential evolution, jiggle, sky ring),
 *      checks the prior and calls log_likelihood_het (QuickCBC.c:2372).
 * PT swaps (QuickCBC.c:2029-2049) are left out, so chain k touches only its own state and its own
 * random stream rvec[k]: the run with 12 threads must equal the run with 1 thread bit for bit.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <omp.h>
#include "QuickCBC.h"
#include "Utilities.h"
#include "ConstCBC.h"

/* The reference leaves these undeclared in its headers. */
void update(int k, struct Net *net, struct Het *het, double *lch, double *lht, double *logLx, double *logPx,
            double **rhox, double **paramx, double **paramy, double *min, double *max, int *who, double *heat,
            double ***history, double ***global, RealVector *freq, double **D, double **SN, double **SM,
            double **ejump, double ***evec, int N, double Tobs, int **cv, int **av, gsl_rng *r);
void FisherEvec(double **fish, double *ej, double **ev, int d);

/* libqcbc_gpu.so: kernel launches issued in the calling thread so far; data registration */
long long qcbc_launch_count(void);
int qcbc_bind_data(struct Net *net, double **D, double **SN, int N, double Tobs);
int qcbc_unbind_all(void);

static double **lk_rows(double *flat, int nrow, int ncol) {
  double **r = (double **)malloc((size_t)(nrow + 1) * sizeof(double *));
  for (int i = 0; i < nrow; i++) r[i] = flat + (size_t)i * ncol;
  r[nrow] = NULL;
  return r;
}

/* One analysis' data as the reference holds it for a whole run: row-pointer arrays made once
 * (QuickCBC.c:198-313 allocates D and SN with double_matrix before the samplers start) over the
 * caller's flat buffers, so every call passes the same D and SN pointers and writes into the
 * buffers (a PSD redraw) are seen by the next call. */
struct LkData {
  double **D, **SN;
  RealVector fv;
  int N;
  double Tobs;
};

struct LkData *lk_data_new(int nifo, double *Dflat, double *SNflat, int sn_stride, double *freq, int N, double Tobs) {
  struct LkData *d = (struct LkData *)calloc(1, sizeof(struct LkData));
  d->D = lk_rows(Dflat, nifo, N);
  d->SN = lk_rows(SNflat, nifo, sn_stride);
  d->fv.data = freq;
  d->fv.length = (size_t)(N / 2);
  d->N = N;
  d->Tobs = Tobs;
  return d;
}

void lk_data_free(struct LkData *d) {
  if (!d) return;
  free(d->D); free(d->SN); free(d);
}

/* log_likelihood_full at params on the data (QuickCBC.c:4236) */
double lk_lnl_full(struct Net *net, struct LkData *d, double *params, double *rho) {
  return log_likelihood_full(net, d->D, params, &d->fv, d->SN, rho, d->N, d->Tobs);
}

/* qcbc_bind_data on the data's row pointers (the optional fast path of INTEGRATION.md) */
int lk_bind(struct Net *net, struct LkData *d) { return qcbc_bind_data(net, d->D, d->SN, d->N, d->Tobs); }
int lk_unbind(void) { return qcbc_unbind_all(); }

/* p0, p_out: [NC][NP]; logL_out: [NC] (lnL after the steps); logL0_out: [NC] (log_likelihood_full
 * at p0); ejump_out: [NC][NP] (FisherEvec + efix jump sizes); accepted: [NC]; launches: GPU
 * kernels launched by all threads.  Returns wall seconds of the stepping phase. */
double lk_mcmc(struct Net *net, struct Het *het, struct LkData *data, const double *p0, double *min, double *max,
               int steps, int nthreads, unsigned long seed, double *p_out, double *logL_out, double *logL0_out,
               double *ejump_out, int *accepted, long long *launches) {
  const int nI = net->Nifo, N = data->N;
  const double Tobs = data->Tobs;
  double **D = data->D, **SN = data->SN;
  RealVector *freq = &data->fv;
  double **paramx = double_matrix(NC + 1, NP), **paramy = double_matrix(NC + 1, NP);
  double *logLx = double_vector(NC + 1), *logPx = double_vector(NC + 1);
  double *lch = double_vector(NC + 1), *lht = double_vector(NC + 1);
  double **rhox = double_matrix(NC + 1, nI);
  double *heat = double_vector(NC + 1);
  int *who = int_vector(NC + 1);
  double ***history = double_tensor(NC + 1, NH, NP);
  double **ejump = double_matrix(NC + 1, NP);
  double ***fish = double_tensor(NC + 1, NP, NP), ***evec = double_tensor(NC + 1, NP, NP);
  int **av = int_matrix(5, NC + 1), **cv = int_matrix(5, NC + 1);
  gsl_rng **rvec = (gsl_rng **)malloc(sizeof(gsl_rng *) * (NC + 1));
  for (int i = 0; i <= NC; i++) {                       /* QuickCBC.c:118-123 */
    rvec[i] = gsl_rng_alloc(gsl_rng_default);
    gsl_rng_set(rvec[i], seed + (unsigned long)i);
  }
  for (int k = 1; k <= NC; k++) {
    for (int i = 0; i < NP; i++) paramx[k][i] = p0[(size_t)(k - 1) * NP + i];
    who[k] = k;
  }
  for (int i = 1; i <= NCC; i++) heat[i] = 1.0;         /* QuickCBC.c:1025-1026 */
  for (int i = NCC + 1; i <= NC; i++) heat[i] = heat[i - 1] * ladder;
  for (int j = 0; j < 5; j++)
    for (int k = 0; k <= NC; k++) av[j][k] = cv[j][k] = 0;
  long long l0[NC + 1], l1[NC + 1];
  for (int k = 0; k <= NC; k++) l0[k] = l1[k] = 0;

  omp_set_num_threads(nthreads);
  /* 1. initial likelihoods (QuickCBC.c:1898-1905) */
#pragma omp parallel for schedule(static, 1)
  for (int k = 1; k <= NC; k++) {
    long long a = qcbc_launch_count();
    logLx[k] = log_likelihood_full(net, D, paramx[k], freq, SN, rhox[k], N, Tobs);
    l0[k] += qcbc_launch_count() - a;
  }
  for (int k = 1; k <= NC; k++) logL0_out[k - 1] = logLx[k];
  /* 2. Fisher matrices, eigen-directions and step sizes per chain (QuickCBC.c:2019-2026) */
#pragma omp parallel for schedule(static, 1)
  for (int k = 1; k <= NC; k++) {
    long long a = qcbc_launch_count();
    Fisher_Het(net, het, fish[k], paramx[k], Tobs);
    FisherEvec(fish[k], ejump[k], evec[k], NP);
    efix(net, het, paramx[k], min, max, freq, SN, N, Tobs, ejump[k], evec[k], 1.0, 1);
    l0[k] += qcbc_launch_count() - a;
  }
  /* 3. heterodyned lnL and the history (QuickCBC.c:1944-1955) */
  {
    long long a = qcbc_launch_count();
    for (int k = 1; k <= NC; k++) logLx[k] = log_likelihood_het(net, het, paramx[k], Tobs);
    l0[0] += qcbc_launch_count() - a;
  }
  for (int i = 0; i < NH; i++)
    for (int k = 1; k <= NC; k++) {
      int q = (int)(gsl_rng_uniform(rvec[0]) * (double)(NC)) + 1;
      for (int j = 0; j < NP; j++) history[k][i][j] = paramx[q][j];
    }
  /* 4. update sweeps (QuickCBC.c:2050-2067) */
  double t0 = omp_get_wtime();
  for (int mc = 0; mc < steps; mc++) {
    for (int j = 1; j <= NC; j++)
      for (int i = 0; i < NP; i++) paramy[j][i] = paramx[j][i];
#pragma omp parallel for schedule(static, 1)
    for (int k = 1; k <= NC; k++) {
      long long a = qcbc_launch_count();
      update(k, net, het, lch, lht, logLx, logPx, rhox, paramx, paramy, min, max, who, heat, history, NULL, freq,
             D, SN, SN, ejump, evec, N, Tobs, cv, av, rvec[k]);
      l1[k] += qcbc_launch_count() - a;
    }
  }
  double secs = omp_get_wtime() - t0;
  long long total = l0[0];
  for (int k = 1; k <= NC; k++) {
    for (int i = 0; i < NP; i++) {
      p_out[(size_t)(k - 1) * NP + i] = paramx[k][i];
      ejump_out[(size_t)(k - 1) * NP + i] = ejump[k][i];
    }
    logL_out[k - 1] = logLx[k];
    accepted[k - 1] = av[1][k] + av[2][k] + av[3][k] + av[4][k];
    total += l0[k] + l1[k];
  }
  *launches = total;
  for (int i = 0; i <= NC; i++) gsl_rng_free(rvec[i]);
  free(rvec);
  free_double_matrix(paramx, NC + 1); free_double_matrix(paramy, NC + 1);
  free_double_vector(logLx); free_double_vector(logPx); free_double_vector(lch); free_double_vector(lht);
  free_double_matrix(rhox, NC + 1); free_double_vector(heat); free_int_vector(who);
  free_double_tensor(history, NC + 1, NH); free_double_matrix(ejump, NC + 1);
  free_double_tensor(fish, NC + 1, NP); free_double_tensor(evec, NC + 1, NP);
  free_int_matrix(av, 5); free_int_matrix(cv, 5);
  return secs;
}

/* The reference's timing loop (QuickCBC.c:1931-1941) from `nthreads` threads at once: each thread
 * makes `calls` calls of log_likelihood_full (which == 0) or log_likelihood_het (which == 1) at
 * params.  Returns wall seconds; lnl_out[nthreads] gets each thread's last value. */
double lk_time_calls(struct Net *net, struct Het *het, struct LkData *d, double *params, int which, int calls,
                     int nthreads, double *lnl_out) {
  double t0 = omp_get_wtime();
#pragma omp parallel num_threads(nthreads)
  {
    double p[NP], rho[8], x = 0.0;
    memcpy(p, params, sizeof(p));
    for (int k = 0; k < calls; k++)
      x = which ? log_likelihood_het(net, het, p, d->Tobs) : log_likelihood_full(net, d->D, p, &d->fv, d->SN, rho,
                                                                                 d->N, d->Tobs);
    lnl_out[omp_get_thread_num()] = x;
  }
  return omp_get_wtime() - t0;
}
