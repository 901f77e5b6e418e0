/*
 * qcbc_quickcbc.h -- drop-in replacements for the QuickCBC reference's
 * waveform and likelihood entry points, executed on the GPU.
 *
 * The functions keep the reference's names and signatures so the unchanged
 * host C (PT-MCMC, proposals, Fisher updates, heterodyne grid search) links
 * against them.  The struct layouts below are byte-compatible with the
 * reference's declarations; a program that already includes the reference's
 * QuickCBC.h / IMRPhenomD_internals.h uses its own definitions and only needs
 * the prototypes (define QCBC_HAVE_REFERENCE_TYPES before including this).
 *
 * Device residency: D, SN and freq are host arrays owned by the caller.
 * Arrays registered with qcbc_bind_data() are used from the device copies made
 * at registration (register again after changing their contents).  Otherwise a
 * call compares the caller's D and SN rows with a host copy of the rows its
 * cached device event was built from and uploads them only when a value
 * differs (the reference rewrites SN in place when it redraws the PSD,
 * QuickCBC.c:1994-2010), so results always follow the arrays' contents.  No
 * caller pointer is kept beyond a call except as a cache key.  freq must be the
 * reference's grid, freq[i] = i/Tobs (QuickCBC.c:419-420); another grid is
 * refused (-1e20, qcbc_last_error()).
 *
 * Threading: every function may be called from several host threads at once,
 * as the reference's OpenMP chains call the likelihoods (QuickCBC.c:2063-2067).
 * Each thread has its own CUDA stream and scratch; a cached event that is
 * replaced (new data, new heterodyne tables, a new binding) stays alive until
 * the calls still using it return.  Concurrent log_likelihood_het calls on the
 * same tables, and log_likelihood_full calls on the same data and geometry,
 * are merged: a caller that finds no launch running for that event takes the
 * sets of the callers waiting meanwhile into its own launch.  Each caller gets
 * the value it would get alone, bit for bit.
 *
 * Errors: the double-returning functions cannot report errors in-band; on a
 * failure they return -1e20 (the reference's rejected-sample value,
 * QuickCBC.c:2366) and qcbc_last_error() tells why.
 */
#ifndef QCBC_QUICKCBC_H
#define QCBC_QUICKCBC_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef QCBC_HAVE_REFERENCE_TYPES
/* QuickCBC.h:13-25 */
struct Net {
  int Nifo;
  double Tobs;
  double tmax;
  double tmin;
  double GMST;
  int* labels;
  double* tds;
  double** delays;
  int* lstart;
  int* lstop;
};

/* IMRPhenomD_internals.h:662-665 */
typedef struct tagRealVector {
  double* data;
  size_t length;
} RealVector;

/* IMRPhenomD_internals.h:649-654 */
typedef struct tagAmpPhaseFDWaveform {
  double* freq;
  double* amp;
  double* phase;
  size_t length;
} AmpPhaseFDWaveform;

/* QuickCBC.h:27-51 */
struct Het {
  int M;
  int MM;
  int MN;
  int ell;
  int J;
  int NR;
  double hh;
  double hr;
  double logLb;
  double*** IP;
  double*** SL;
  double** amp;
  double** phase;
  double** rc;
  double** rs;
  double** aa;
  double*** lc;
  double*** ls;
  double* pref;
  int* fgrid;
  RealVector* freq;
};
#endif

/* Band of the full likelihood: the reference's compile-time fmin/fmax
 * (ConstCBC.h:33-34, defaults 16 Hz and 1024 Hz). */
int qcbc_set_band(double fmin, double fmax);

/* Register caller arrays so later calls with the same pointers skip uploads. */
int qcbc_bind_data(struct Net* net, double** D, double** SN, int N, double Tobs);
int qcbc_unbind_all(void);

/* replaces QuickCBC.c:4236 */
double log_likelihood_full(struct Net* net, double** D, double* params, RealVector* freq, double** SN, double* rho,
                           int N, double Tobs);
/* replaces QuickCBC.c:5303; the struct Het tables are uploaded on first use and
 * re-uploaded when het->IP, het->M or het->logLb change (re-heterodyne).  Tables
 * of at most 32 structs stay on the device, least recently used evicted. */
double log_likelihood_het(struct Net* net, struct Het* het, double* params, double Tobs);
/* Drop the device copy of het's tables now (e.g. next to freehet, QuickCBC.c:5096);
 * optional. */
int qcbc_het_forget(const struct Het* het);
/* replaces QuickCBC.c:5112; needs het->M, MN, MM, J, NR, fgrid, freq from het_space.
 * Allocates the table arrays with the reference's row-pointer layout
 * (Utilities.c:2981-3015) so freehet() (QuickCBC.c:5096) releases them. */
void heterodyne(struct Net* net, struct Het* het, double** D, double* params, RealVector* freq, double** SN, int N,
                double Tobs);
/* replaces QuickCBC.c:3683 */
void fulltemplates(struct Net* net, double** hwave, RealVector* freq, double* params, int N);
/* replaces QuickCBC.c:3780 */
void fullphaseamp(struct Net* net, double** amp, double** phase, RealVector* freq, double* params, int N);
/* replaces IMRPhenomD.c:186; *h22 is malloc'd like CreateAmpPhaseFDWaveform
 * (IMRPhenomD_internals.c:130-146) so DestroyAmpPhaseFDWaveform frees it.
 * Returns 0 (PD_SUCCESS) or 33 (PD_EDOM) instead of exiting on bad input. */
int IMRPhenomDGenerateh22FDAmpPhase(AmpPhaseFDWaveform** h22, RealVector* freq, const double phi0,
                                    const double fRef_in, const double m1_SI, const double m2_SI, const double chi1,
                                    const double chi2, const double distance);
/* replaces Utilities.c:716 */
double fourier_nwip(double* a, double* b, double* Sn, int imin, int imax, int N);

/* Secondary consumers of the waveform (declared in QuickCBC.h:95-151). */
/* replaces QuickCBC.c:4093; params in the intrinsic layout (7 + 3 (Nifo - 1) entries) */
double log_likelihood_intrinsic(struct Net* net, double** D, double* params, RealVector* freq, double** SN, int N,
                                double Tobs);
/* replaces QuickCBC.c:3527; params in the intrinsic layout */
void templates(struct Net* net, double** hwave, RealVector* freq, double* params, int N);
/* replaces QuickCBC.c:3395; writes Af[i], Pf[i] for i in [1, N/2) */
void AmpPhase(double* Af, double* Pf, RealVector* freq, double* params, int N);
/* replaces QuickCBC.c:4966 (tables as for log_likelihood_het) */
double het_diff(struct Net* net, struct Het* het, double* params, double* dparams);
/* replaces QuickCBC.c:5446; fish is the reference's NP x NP row-pointer matrix */
void Fisher_Het(struct Net* net, struct Het* het, double** fish, double* params, double Tobs);
/* replaces QuickCBC.c:4570; sets het->MN, MM, J, NR, M, freq, fgrid (malloc'd as the reference
 * allocates them); writes no diagnostic files */
void het_space(struct Net* net, struct Het* het, double* params, double* min, double* max, RealVector* freq,
               double** SN, int N, double Tobs);

/* Times the reference-signature likelihood from `nthreads` native host threads
 * started together, as the reference's OpenMP chains call it: each thread makes
 * 4 untimed calls, then `calls` timed ones with parameter set (7 t + k) mod nsets
 * of params[nsets][11].  which = 0: log_likelihood_full(net, D, ., freq, SN, rho,
 * N, Tobs); which = 1: log_likelihood_het(net, het, ., Tobs).  *seconds is the
 * wall time of the timed calls of all threads; lnl_last[t] (optional) the last
 * lnL of thread t. */
int qcbc_time_dropin(int which, struct Net* net, struct Het* het, double** D, RealVector* freq, double** SN, int N,
                     double Tobs, const double* params, int nsets, int calls, int nthreads, double* seconds,
                     double* lnl_last);

/* The same functions under prefixed names, for a forwarding object that
 * gives an unchanged QuickCBC build strong definitions: a small C file that
 * defines each reference name as a call to its qcbc_gpu_ counterpart. */
double qcbc_gpu_log_likelihood_full(struct Net* net, double** D, double* params, RealVector* freq, double** SN,
                                    double* rho, int N, double Tobs);
double qcbc_gpu_log_likelihood_het(struct Net* net, struct Het* het, double* params, double Tobs);
void qcbc_gpu_heterodyne(struct Net* net, struct Het* het, double** D, double* params, RealVector* freq,
                         double** SN, int N, double Tobs);
void qcbc_gpu_fulltemplates(struct Net* net, double** hwave, RealVector* freq, double* params, int N);
void qcbc_gpu_fullphaseamp(struct Net* net, double** amp, double** phase, RealVector* freq, double* params, int N);
int qcbc_gpu_IMRPhenomDGenerateh22FDAmpPhase(AmpPhaseFDWaveform** h22, RealVector* freq, const double phi0,
                                             const double fRef_in, const double m1_SI, const double m2_SI,
                                             const double chi1, const double chi2, const double distance);
double qcbc_gpu_fourier_nwip(double* a, double* b, double* Sn, int imin, int imax, int N);
double qcbc_gpu_log_likelihood_intrinsic(struct Net* net, double** D, double* params, RealVector* freq, double** SN,
                                         int N, double Tobs);
void qcbc_gpu_templates(struct Net* net, double** hwave, RealVector* freq, double* params, int N);
void qcbc_gpu_AmpPhase(double* Af, double* Pf, RealVector* freq, double* params, int N);
double qcbc_gpu_het_diff(struct Net* net, struct Het* het, double* params, double* dparams);
void qcbc_gpu_Fisher_Het(struct Net* net, struct Het* het, double** fish, double* params, double Tobs);
void qcbc_gpu_het_space(struct Net* net, struct Het* het, double* params, double* min, double* max, RealVector* freq,
                        double** SN, int N, double Tobs);

#ifdef __cplusplus
}
#endif
#endif
