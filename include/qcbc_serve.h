/*
 * qcbc_serve.h -- continuous-batching service for parallel-tempered MCMC
 * analyses on one GPU (no counterpart in the reference, whose samplers run one
 * analysis per process: QuickCBC.c:1781-2236 MCMC_all / 2238-2405 update).
 *
 * A run is one analysis: its data and PSD (copied at submission), a starting
 * point, a temperature ladder of n_temps temperatures for each of n_chains
 * independent ladders, and a number of steps.  Runs wait in a FIFO queue until
 * both an event slot and the device-memory budget allow admission; admitted
 * runs keep their data on the device and their chains on the host.  Every
 * qcbc_server_step() advances every live run by one step: one proposal per
 * chain (Gaussian, per-parameter scales adapted towards 25% acceptance during
 * burn-in, angles wrapped, sin/cos reflected; or the reference's mixture, see
 * qcbc_run_spec.proposal), all proposals of all live runs evaluated in ONE
 * multi-event launch (qcbc_lnl_multi), Metropolis acceptance at each chain's
 * temperature with the reference's prior density (flat in m1, m2, uniform in
 * volume: QuickCBC.c:2352-2381), one swap attempt between adjacent temperatures
 * per ladder, thinned samples of the T = 1 chains kept after burn-in.  Finished
 * runs release their slot and device memory.  A run's chains use their own
 * random stream and the lnL of a set does not depend on the other sets of the
 * launch, so a run evolves identically alone and in any mix.
 */
#ifndef QCBC_SERVE_H
#define QCBC_SERVE_H

#include "qcbc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct qcbc_server qcbc_server;

typedef struct {
  /* analysis data (copied at submission) */
  int nifo;
  const int* labels;        /* [nifo], 0 = H1, 1 = L1, 2 = V1 */
  double Tobs, GMST;
  int N;
  const double* D;          /* [nifo][N] half-complex */
  const double* SN;         /* [nifo][sn_stride] */
  int sn_stride;
  double fmin, fmax;
  /* sampler */
  const double* start;      /* [11] starting point of every chain */
  const double* scales;     /* [11] proposal scales at T = 1, or NULL for defaults */
  const double* prior_min;  /* [11] uniform prior box, or NULL for the reference's box */
  const double* prior_max;  /*      (MCMC_all, QuickCBC.c:1871-1896) */
  int n_temps, n_chains, n_steps, burn_in, thin;
  double ladder;            /* temperature ratio (1.15 in ConstCBC.h:44) */
  unsigned long long seed;
  int likelihood;           /* QCBC_LNL_FULL, or QCBC_LNL_HET: at admission the heterodyne grid search
                               and tables are built about `start` (het_space + heterodyne,
                               QuickCBC.c:4570, 5112) and every step uses the heterodyned lnL
                               (log_likelihood_het, QuickCBC.c:5303), as the reference's sampler does */
  int proposal;             /* QCBC_PROPOSE_GAUSS: Gaussian steps with scales adapted during burn-in;
                               QCBC_PROPOSE_REFERENCE (device-resident stepping only): the reference's
                               mixture (update, QuickCBC.c:2266-2333) of Fisher eigen-jumps, differential
                               evolution, jiggles and sky-ring moves; its Fisher matrix and jump sizes (Fisher_Het,
                               FisherEvec, efix) are computed at the starting point at admission, from
                               heterodyne tables built there for either likelihood */
} qcbc_run_spec;

#define QCBC_LNL_FULL 0
#define QCBC_LNL_HET 1
#define QCBC_PROPOSE_GAUSS 0
#define QCBC_PROPOSE_REFERENCE 1

#define QCBC_RUN_QUEUED 0
#define QCBC_RUN_LIVE 1
#define QCBC_RUN_DONE 2
#define QCBC_RUN_FAILED 3
#define QCBC_RUN_CANCELLED 4

typedef struct {
  int state;
  int steps_done;
  double t_arrival, t_admit, t_done;   /* server clock, seconds */
  double accept_cold;                  /* acceptance rate of the T = 1 chains */
  double swap_rate;
  long long device_bytes;
  long long lnl_evals;
  int n_samples;
} qcbc_run_info;

/* hbm_budget_bytes: admission limit on the device memory of live runs;
 * max_live: event slots; max_bins: largest N/2 accepted; precision QCBC_FP64/MIXED. */
qcbc_server* qcbc_server_create(long long hbm_budget_bytes, int max_live, int max_bins, int precision);
int qcbc_server_destroy(qcbc_server* s);
double qcbc_server_clock(const qcbc_server* s);
/* Returns the run id (>= 0) or a negative status (QCBC_EBUDGET when the run alone
 * needs more device memory than the budget; QCBC_EINVAL for a bad specification). */
long long qcbc_server_submit(qcbc_server* s, const qcbc_run_spec* spec);
int qcbc_server_cancel(qcbc_server* s, long long run);
/* One step of every live run (admits queued runs first). */
int qcbc_server_step(qcbc_server* s, int* n_live, int* n_queued, int* n_done);
int qcbc_server_run_info(qcbc_server* s, long long run, qcbc_run_info* out);
/* Rows of 12 doubles (11 parameters, lnL) of the run's T = 1 samples. */
int qcbc_server_run_samples(qcbc_server* s, long long run, double* out, int max_rows, int* n_rows);
int qcbc_server_stats(qcbc_server* s, long long* lnl_evals, long long* launches, long long* device_bytes_live);
/* Seconds spent so far in the three phases of the steps: building proposals, the
 * merged likelihood launch (including its copies), and the Metropolis/swap updates. */
int qcbc_server_timing(qcbc_server* s, double* propose_s, double* lnl_s, double* update_s);
/* Tiling of the merged launches (see qcbc_batch_set_tiling). */
int qcbc_server_set_tiling(qcbc_server* s, int tile_bins, int threads);
/* Device-resident stepping: with steps > 0 the chains of the live runs stay on the device and
 * every qcbc_server_step() queues up to `steps` whole steps on one stream (proposal, merged lnL
 * launches, acceptance, swaps, adaptation, thinning as kernels), stopping early when a run
 * finishes; 0 (the default) steps on the host.  Each chain draws from its own generator stream,
 * so a run evolves identically alone, in any mix and for any `steps`.  Set before submitting
 * runs; at most 64 temperatures per run in this mode. */
int qcbc_server_set_device_steps(qcbc_server* s, int steps);

#ifdef __cplusplus
}
#endif
#endif
