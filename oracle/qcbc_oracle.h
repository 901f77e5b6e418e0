/*
 * CPU restatement of the QuickCBC likelihood hot path (FP64).
 *
 * TEST INFRASTRUCTURE ONLY -- the checker for the CUDA kernels.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity is pinned against the reference itself (oracle/_ref, the reference
 * C compiled unmodified) by tests/test_oracle_vs_ref.py.
 *
 * Flat layouts (float64, row-major):
 *   D      [nifo][N]          half-complex (Re at i, Im at N-i)
 *   SN     [nifo][sn_stride]  PSD per bin, sn_stride >= N/2 + 1
 *   params [11]               ln Mc, ln Mt, chi1, chi2, phi0, tc, ln DL,
 *                             alpha, sin(delta), psi, cos(iota)
 */
#ifndef QCBC_ORACLE_H
#define QCBC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* QNM table (final spin, fring, fdamp) used by the natural spline of
 * fring/fdamp; must be set once before any waveform call. */
int ora_set_qnm(const double *a, const double *fring, const double *fdamp, int n);

int ora_amp_phase(const double *freq, int n, double phi0, double fRef, double m1_SI, double m2_SI,
                  double chi1, double chi2, double dist, double *amp, double *phase);
double ora_fbegin(const double *params);
void ora_antenna(double psi, double alpha, double sindelta, double GMST, int ifo, double *fpfc);
void ora_delays(double alpha, double sindelta, double GMST, double *dt3);

void ora_fulltemplates(const int *labels, int nifo, double GMST, const double *freq, const double *params,
                       int N, double *h);
void ora_fullphaseamp(const int *labels, int nifo, double GMST, double Tobs, const double *freq,
                      const double *params, int N, double *amp, double *phase);
double ora_fourier_nwip(const double *a, const double *b, const double *S, int imin, int imax, int N);
double ora_lnl_full(const int *labels, int nifo, double GMST, const double *D, const double *SN,
                    int sn_stride, const double *freq, const double *params, int N, double Tobs,
                    double fmin, double fmax, double *rho);
double ora_lnl_full_batch(const int *labels, int nifo, double GMST, const double *D, const double *SN,
                          int sn_stride, const double *freq, const double *params, int B, int N,
                          double Tobs, double fmin, double fmax, double *lnl, int nthreads);

/* Heterodyne summary tables for a given grid (fgrid[M] bin indices). */
int ora_heterodyne(const int *labels, int nifo, double GMST, const double *D, const double *SN,
                   int sn_stride, const double *freq, const double *params, int N, double Tobs,
                   const int *fgrid, int M, int MN, int MM, int J,
                   double *amp, double *phase, double *IP, double *SL, double *lc, double *ls,
                   double *aa, double *rc, double *rs, double *logLb);
double ora_lnl_het(const int *labels, int nifo, double GMST, double Tobs, const double *hfreq, int M, int J,
                   const double *amp, const double *phase, const double *IP, const double *SL,
                   const double *lc, const double *ls, const double *aa, const double *rc,
                   const double *rs, double logLb, const double *params);
double ora_lnl_het_batch(const int *labels, int nifo, double GMST, double Tobs, const double *hfreq, int M,
                         int J, const double *amp, const double *phase, const double *IP,
                         const double *SL, const double *lc, const double *ls, const double *aa,
                         const double *rc, const double *rs, double logLb, const double *params, int B,
                         double *lnl, int nthreads);

#ifdef __cplusplus
}
#endif
#endif
