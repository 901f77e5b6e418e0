/*
 * qcbc_ingest.h -- analysis inputs for the GPU likelihood path: QuickCBC's data
 * and PSD files, data conditioning, and the PSD redraw of noise marginalisation.
 *
 * Reference interfaces replaced (QuickCBC.c, Utilities.c):
 *   framed_<T>_<trig>_<ifo>.dat reader, N from its rows   QuickCBC.c:198-226
 *   spec_<T>_<trig>_<ifo>.dat reader (columns f, SN, SM, -) QuickCBC.c:233-242
 *   Tukey window + real FFT + sqrt(Tobs)/N scaling of D     QuickCBC.c:244-258, 309-313
 *                                                           (tukey, Utilities.c:635)
 *   summary_/sfile_/ffile_/lfile_ PSD-sample readers        QuickCBC.c:322-378
 *   makespec: natural-spline log PSD plus lines             Utilities.c:1908-1955
 *   noisemarg redraw: makespec per detector, heterodyne     QuickCBC.c:1994-2010
 *                     again about the reference point
 *
 * File readers are host code and need no GPU.  Conditioning and makespec run on
 * the GPU.  Status codes are those of qcbc_gpu.h.
 */
#ifndef QCBC_INGEST_H
#define QCBC_INGEST_H

#include "qcbc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- files (host) */

/* Number of samples N of a two-column framed file, counted as QuickCBC.c:205-211
 * counts them: every complete row, less one when the file ends directly after its
 * last number (no trailing newline). */
int qcbc_framed_length(const char* path, int* N);
/* The first N rows of a framed file: times t[N] (may be NULL) and strain x[N]. */
int qcbc_read_framed(const char* path, int N, double* t, double* x);
/* The first nh rows of a four-column spec file: SN (column 2) and SM (column 3);
 * SM may be NULL. */
int qcbc_read_spec(const char* path, int nh, double* SN, double* SM);
/* File names of one analysis, built as QuickCBC.c does: "<dir>/framed_%d_%d_%d.dat"
 * and "<dir>/spec_%d_%d_%d.dat" with (int)Tobs, (int)ttrig and the detector label. */
int qcbc_analysis_paths(const char* dir, double Tobs, double ttrig, int label, char* framed, char* spec,
                        int cap);

/* ---------------------------------------------------------------- conditioning (GPU) */

/* Time series x[nifo][x_stride] (N samples each, N a power of two >= 8) to the
 * likelihood's data D[nifo][d_stride]: Tukey window with a 0.4 s rise, real FFT in
 * GSL half-complex layout, times sqrt(Tobs)/N. */
int qcbc_condition_data(int nifo, int N, double Tobs, const double* x, int x_stride, double* D, int d_stride);

/* The whole input stage of one analysis: reads the framed and spec files of every
 * detector in `dir`, conditions the data.  N must be the value qcbc_framed_length
 * gives for the first detector's file.  SM may be NULL. */
int qcbc_load_analysis(const char* dir, double Tobs, double ttrig, int nifo, const int* labels, int N, double* D,
                       int d_stride, double* SN, double* SM, int sn_stride);

/* ---------------------------------------------------------------- PSD samples (GPU) */

typedef struct qcbc_psd_model qcbc_psd_model;

/* Reads summary_<ifo>.dat (Nspline Nlines Nsample), ffile_<ifo>.dat (Nspline knot
 * frequencies), sfile_<ifo>.dat (Nsample x Nspline log-PSD knot values) and
 * lfile_<ifo>.dat (Nsample x Nlines x {f, h, Q, w, deltafmax}) of each detector, as
 * QuickCBC.c:322-378 does (Nsample from the last detector's summary), and sets up
 * the natural splines of every sample on the device. */
qcbc_psd_model* qcbc_psd_model_open(const char* dir, int nifo, const int* labels);
/* The same from arrays: nspline[nifo], nlines[nifo]; ffit [nifo][nspline_max],
 * xspline [nifo][nsample][nspline_max], lines [nifo][nsample][nlines_max][5]. */
qcbc_psd_model* qcbc_psd_model_create(int nifo, const int* nspline, const int* nlines, int nsample,
                                      int nspline_max, int nlines_max, const double* ffit, const double* xspline,
                                      const double* lines);
int qcbc_psd_model_info(const qcbc_psd_model* m, int* nifo, int* nsample, int* nspline_max, int* nlines_max);
int qcbc_psd_model_close(qcbc_psd_model* m);
/* makespec (Utilities.c:1908) of sample k for every detector: SN[nifo][sn_stride],
 * N/2 bins at f = i/Tobs.  QCBC_EDOM when a bin lies outside a detector's knots. */
int qcbc_psd_draw(qcbc_psd_model* m, int k, double Tobs, int N, double* SN, int sn_stride);

/* noisemarg redraw on the device (QuickCBC.c:1994-2010): the event's PSD becomes
 * sample k of the model, its weighted data are rebuilt on the device, and when it
 * holds heterodyne tables they are rebuilt about the same reference point and grid. */
int qcbc_event_set_psd_sample(qcbc_event* ev, qcbc_psd_model* m, int k);
/* A new PSD from the host, SN[nifo][sn_stride], with the same rebuilds. */
int qcbc_event_set_psd(qcbc_event* ev, const double* SN, int sn_stride);

/* Reference signature (Utilities.c:1908): makespec on the GPU; also exported as
 * qcbc_gpu_makespec. */
void makespec(int Nspline, int Nlines, double* ffit, double* Sspline, double* linef, double* lineh, double* lineQ,
              double* linew, double* deltafmax, double* SN, double Tobs, int N);
void qcbc_gpu_makespec(int Nspline, int Nlines, double* ffit, double* Sspline, double* linef, double* lineh,
                       double* lineQ, double* linew, double* deltafmax, double* SN, double Tobs, int N);

#ifdef __cplusplus
}
#endif
#endif
