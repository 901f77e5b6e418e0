/*
 * qcbc_forward.c -- the reference-side binding: strong definitions of the thirteen QuickCBC
 * functions the GPU library replaces, each forwarding to the library's qcbc_gpu_ alias.
 *
 * A maintainer compiles this file next to the unchanged QuickCBC sources, weakens the
 * reference's own definitions of the same thirteen names with objcopy --weaken-symbol (or
 * guards them with #ifndef), and links libqcbc_gpu.so; the recipe is in INTEGRATION.md.  Every
 * call the reference makes to one of these names -- from update (QuickCBC.c:2372), MCMC_all
 * (1898-1941), het_space, efix, Fisher refreshes, log_likelihood_test -- then runs on the GPU.
 *
 * Compiled with -DQCBC_FORWARD_COUNT, each forward also counts its calls (atomically, any
 * thread) in qcbc_forward_calls[], indexed by the QCBC_FWD_* constants: a call counter showing
 * which replaced functions an unchanged program reached.
 *
 * The reference's own headers supply the types (QuickCBC.h:13-51, IMRPhenomD_internals.h:
 * 649-665); the qcbc_gpu_ prototypes come from qcbc_quickcbc.h.
 */
#include "QuickCBC.h"
#define QCBC_HAVE_REFERENCE_TYPES
#include "qcbc_quickcbc.h"

enum {
  QCBC_FWD_LOG_LIKELIHOOD_FULL, QCBC_FWD_LOG_LIKELIHOOD_HET, QCBC_FWD_HETERODYNE, QCBC_FWD_FULLTEMPLATES,
  QCBC_FWD_FULLPHASEAMP, QCBC_FWD_IMRPHENOMD, QCBC_FWD_FOURIER_NWIP, QCBC_FWD_LOG_LIKELIHOOD_INTRINSIC,
  QCBC_FWD_TEMPLATES, QCBC_FWD_AMPPHASE, QCBC_FWD_HET_DIFF, QCBC_FWD_FISHER_HET, QCBC_FWD_HET_SPACE,
  QCBC_FWD_N
};

#ifdef QCBC_FORWARD_COUNT
long long qcbc_forward_calls[QCBC_FWD_N];
#define COUNT(k) __atomic_fetch_add(&qcbc_forward_calls[k], 1, __ATOMIC_RELAXED)
#else
#define COUNT(k) ((void)0)
#endif

double log_likelihood_full(struct Net* net, double** D, double* params, RealVector* freq, double** SN, double* rho,
                           int N, double Tobs) {
  COUNT(QCBC_FWD_LOG_LIKELIHOOD_FULL);
  return qcbc_gpu_log_likelihood_full(net, D, params, freq, SN, rho, N, Tobs);
}

double log_likelihood_het(struct Net* net, struct Het* het, double* params, double Tobs) {
  COUNT(QCBC_FWD_LOG_LIKELIHOOD_HET);
  return qcbc_gpu_log_likelihood_het(net, het, params, Tobs);
}

void heterodyne(struct Net* net, struct Het* het, double** D, double* params, RealVector* freq, double** SN, int N,
                double Tobs) {
  COUNT(QCBC_FWD_HETERODYNE);
  qcbc_gpu_heterodyne(net, het, D, params, freq, SN, N, Tobs);
}

void fulltemplates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  COUNT(QCBC_FWD_FULLTEMPLATES);
  qcbc_gpu_fulltemplates(net, hwave, freq, params, N);
}

void fullphaseamp(struct Net* net, double** amp, double** phase, RealVector* freq, double* params, int N) {
  COUNT(QCBC_FWD_FULLPHASEAMP);
  qcbc_gpu_fullphaseamp(net, amp, phase, freq, params, N);
}

int IMRPhenomDGenerateh22FDAmpPhase(AmpPhaseFDWaveform** h22, RealVector* freq, const double phi0,
                                    const double fRef_in, const double m1_SI, const double m2_SI, const double chi1,
                                    const double chi2, const double distance) {
  COUNT(QCBC_FWD_IMRPHENOMD);
  return qcbc_gpu_IMRPhenomDGenerateh22FDAmpPhase(h22, freq, phi0, fRef_in, m1_SI, m2_SI, chi1, chi2, distance);
}

double fourier_nwip(double* a, double* b, double* Sn, int imin, int imax, int N) {
  COUNT(QCBC_FWD_FOURIER_NWIP);
  return qcbc_gpu_fourier_nwip(a, b, Sn, imin, imax, N);
}

double log_likelihood_intrinsic(struct Net* net, double** D, double* params, RealVector* freq, double** SN, int N,
                                double Tobs) {
  COUNT(QCBC_FWD_LOG_LIKELIHOOD_INTRINSIC);
  return qcbc_gpu_log_likelihood_intrinsic(net, D, params, freq, SN, N, Tobs);
}

void templates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  COUNT(QCBC_FWD_TEMPLATES);
  qcbc_gpu_templates(net, hwave, freq, params, N);
}

void AmpPhase(double* Af, double* Pf, RealVector* freq, double* params, int N) {
  COUNT(QCBC_FWD_AMPPHASE);
  qcbc_gpu_AmpPhase(Af, Pf, freq, params, N);
}

double het_diff(struct Net* net, struct Het* het, double* params, double* dparams) {
  COUNT(QCBC_FWD_HET_DIFF);
  return qcbc_gpu_het_diff(net, het, params, dparams);
}

void Fisher_Het(struct Net* net, struct Het* het, double** fish, double* params, double Tobs) {
  COUNT(QCBC_FWD_FISHER_HET);
  qcbc_gpu_Fisher_Het(net, het, fish, params, Tobs);
}

void het_space(struct Net* net, struct Het* het, double* params, double* min, double* max, RealVector* freq,
               double** SN, int N, double Tobs) {
  COUNT(QCBC_FWD_HET_SPACE);
  qcbc_gpu_het_space(net, het, params, min, max, freq, SN, N, Tobs);
}
