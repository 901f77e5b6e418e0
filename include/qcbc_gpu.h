/*
 * qcbc_gpu.h -- C ABI of the B200 likelihood engine for QuickCBC.
 *
 * Plain C types only (pointers, sizes, doubles); no CUDA or torch types.
 * Every function returns a status code (QCBC_OK on success) unless noted;
 * qcbc_last_error() gives the message of the calling thread's last failure.
 *
 * Data conventions are the QuickCBC reference's:
 *   D      [nifo][N]          half-complex FFT rows (Re at i, Im at N-i),
 *                             scaled by sqrt(Tobs)/N (QuickCBC.c:254-313)
 *   SN     [nifo][sn_stride]  one-sided PSD per bin, sn_stride >= N/2
 *   params [B][11]            ln(Mc kg), ln(Mt kg), chi1, chi2, phi0, tc,
 *                             ln(DL m), alpha, sin(delta), psi, cos(iota)
 *                             (QuickCBC.c:1867)
 *   lnL                       sum_ifo <d|h> - <h|h>/2 over
 *                             [Tobs*fmin, min(Tobs*fmax, N/2))  (QuickCBC.c:4236-4273)
 *
 * Reentrancy: calls on different events, or on the same event from different
 * host threads, may run concurrently (each thread has its own CUDA stream and
 * scratch).  Opening/closing an event or replacing its heterodyne tables must
 * not race with likelihood calls on that event.
 */
#ifndef QCBC_GPU_H
#define QCBC_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define QCBC_OK 0
#define QCBC_EINVAL (-1)   /* bad argument */
#define QCBC_ECUDA (-2)    /* CUDA runtime error */
#define QCBC_ENOMEM (-3)   /* device or host allocation failed */
#define QCBC_EBUDGET (-4)  /* admission refused by the device-memory budget */
#define QCBC_ETIMEOUT (-5) /* a bounded device wait ran out */
#define QCBC_EDOM 33       /* some parameter sets were outside the waveform's domain;
                              their lnL is -1e20 (IMRPhenomD.c:208-242 would exit) */

#define QCBC_FP64 0        /* plain form: every step in FP64 */
#define QCBC_MIXED 1       /* FP64 phase and 2 pi f tc shift, FP32 amplitude/sincos/accumulate */

typedef struct qcbc_event qcbc_event;

/* Heterodyne summary tables, flat row-major (the reference's struct Het,
 * QuickCBC.h:27-51, with its row-pointer arrays flattened):
 *   fgrid[M], freq[M], amp[nifo][M], phase[nifo][M], IP[NR][J+1][J+1],
 *   SL/lc/ls[NR][nifo][J+1], aa/rc/rs[nifo][NR], NR = (M-1)/J. */
typedef struct {
  int M, MN, MM, J, NR;
  double logLb;
  const int* fgrid;
  const double *freq, *amp, *phase, *IP, *SL, *lc, *ls, *aa, *rc, *rs;
} qcbc_het_tables;

const char* qcbc_last_error(void);
const char* qcbc_version(void);

/* Select the CUDA device for the calling thread and load the model tables
 * there (idempotent).  Every entry point calls it for device 0 if needed. */
int qcbc_init(int device);

/* QNM table override: final spin a[n] (strictly increasing), fring[n], fdamp[n].
 * The library ships the table of IMRPhenomD_internals.h:176-640. */
int qcbc_set_qnm_table(const double* a, const double* fring, const double* fdamp, int n);

/* ---- events: one analysis resident on the device ---- */
/* Copies D and SN to the device once (replaces QuickCBC.c:4254-4266's per-call
 * template and two inner-product passes).  d_stride / sn_stride are row strides. */
qcbc_event* qcbc_event_open(int nifo, const int* labels, double Tobs, double GMST, int N, const double* D,
                            int d_stride, const double* SN, int sn_stride, double fmin, double fmax);
int qcbc_event_close(qcbc_event* ev);
/* Device bytes held by an event (data, tables). */
long long qcbc_event_device_bytes(const qcbc_event* ev);

/* Full likelihood for B parameter sets (host arrays).  rho may be NULL
 * ([B][nifo] otherwise, rho = <d|h>/sqrt(<h|h>) per detector). */
int qcbc_lnl_full(qcbc_event* ev, const double* params, int B, double* lnl, double* rho, int precision);
/* Same with device pointers on a caller stream (cudaStream_t passed as void*, NULL = the thread's stream).
 * The work is queued on that stream with no synchronisation.  Calls from one host thread share
 * that thread's scratch, so calls on different streams from one thread must be ordered (each
 * after the previous one's work).  A call may be captured into a CUDA graph once the same call
 * (same B and precision) has run uncaptured on the thread, which sizes the scratch; replays
 * reuse the scratch of the thread that captured it. */
int qcbc_lnl_full_dev(qcbc_event* ev, const double* d_params, int B, double* d_lnl, double* d_rho, int precision,
                      void* stream);
/* Batched log_likelihood_intrinsic (QuickCBC.c:4093-4140): params [B][7 + 3 (nifo - 1)] in the
 * intrinsic layout of templates (QuickCBC.c:3527-3598: Mc, Mt, chi1, chi2, phic, tc, DL, then
 * phase offset, time offset and amplitude ratio of each detector after the first; phi0 =
 * params[4]).  lnL = sum over detectors of (HD - HH/2), set to 0 when nifo > 1 and fewer than
 * two detectors have SNR^2 = 2 (HD - HH/2) > 25.  snrsq [B][nifo] may be NULL. */
int qcbc_lnl_intrinsic(qcbc_event* ev, const double* params, int B, double* lnl, double* snrsq, int precision);

/* ---- many events in one launch ---- */
/* A batch groups open events (same device) so that parameter sets of different
 * analyses -- differing networks, durations, sample rates and bands -- are
 * evaluated together.  Each set's signal band is cut into tiles of tile_bins
 * bins; a persistent kernel takes (set, tile) work items from a device queue;
 * the sequence (copies, setup, work list, kernel, finalise) is one captured CUDA
 * graph per (batch-size bucket, precision), launched once per call.  A set's
 * lnL depends only on its own inputs and the tiling, not on the other sets in
 * the call.  Calls on one batch are serialised internally. */
typedef struct qcbc_batch qcbc_batch;
qcbc_batch* qcbc_batch_create(qcbc_event* const* events, int n_events);
/* A batch of `capacity` event slots, initially empty, for events of at most max_bins
 * frequency bins (N/2); slots are (re)filled with qcbc_batch_set_slot (NULL empties a
 * slot; sets naming an empty slot get lnL = -1e20).  The batch does not own events. */
qcbc_batch* qcbc_batch_create_slots(int capacity, int max_bins);
int qcbc_batch_set_slot(qcbc_batch* batch, int slot, qcbc_event* ev);
int qcbc_batch_destroy(qcbc_batch* batch);
/* tile_bins > 0 and threads in {64,128,256}; 0 keeps the current/automatic value */
int qcbc_batch_set_tiling(qcbc_batch* batch, int tile_bins, int threads);
int qcbc_batch_get_tiling(qcbc_batch* batch, int* tile_bins, int* threads);
/* Times each candidate tiling on the given call and keeps the fastest. */
int qcbc_batch_autotune(qcbc_batch* batch, const int* event_of, const double* params, int B, int precision);
/* event_of[B] indexes the batch's events; rho is [B][3] (unused detectors 0) or NULL. */
int qcbc_lnl_multi(qcbc_batch* batch, const int* event_of, const double* params, int B, double* lnl, double* rho,
                   int precision);
/* Heterodyned lnL (log_likelihood_het, QuickCBC.c:5303) of sets of many events: each set uses
 * the heterodyne tables its event had when its slot was set (qcbc_het_setup / qcbc_het_set
 * before qcbc_batch_set_slot; set the slot again after re-heterodyning).  Sets whose event has
 * no tables get lnL = -1e20 and the call returns QCBC_EDOM. */
int qcbc_lnl_multi_het(qcbc_batch* batch, const int* event_of, const double* params, int B, double* lnl,
                       int precision);
/* Device-buffer forms of qcbc_lnl_multi / qcbc_lnl_multi_het: event_of, params and lnl are device
 * pointers; the work is queued on `stream` (a cudaStream_t as void*, NULL = the batch's stream)
 * with no host copy and no synchronisation.  Sets outside the waveform domain or without an event
 * (or tables) get lnL = -1e20; no status is returned for them.  Calls on one batch share its
 * buffers: keep them on one stream. */
int qcbc_lnl_multi_dev(qcbc_batch* batch, const int* d_event_of, const double* d_params, int B, double* d_lnl,
                       int precision, void* stream);
int qcbc_lnl_multi_het_dev(qcbc_batch* batch, const int* d_event_of, const double* d_params, int B, double* d_lnl,
                           int precision, void* stream);
/* Sky-ring proposal map of the reference's sampler (update, QuickCBC.c:2299-2331) on the GPU: x's
 * sky position turned by `rot` radians about the line between detectors label1 and label2 (ring of
 * equal time delay, Ring_all), then the distance, polarisation, phase, inclination and geocentre
 * time that keep the signal in both detectors (skymap_all); *log_jacobian = log |det| of the map's
 * 4 x 4 Jacobian (skydensity_all).  x, y: [11] host arrays (y's angles not wrapped). */
int qcbc_sky_ring_map(const double* x, double* y, double GMST, int label1, int label2, double rot,
                      double* log_jacobian);
/* Device time of `iters` graph launches on inputs already uploaded by a previous
 * qcbc_lnl_multi call with the same B (no host copies inside the timed span). */
int qcbc_time_lnl_multi(qcbc_batch* batch, int B, int precision, int iters, int flush_l2, float* ms);

/* ---- heterodyned likelihood ---- */
/* Upload tables computed elsewhere (e.g. by the reference's heterodyne()). */
int qcbc_het_set(qcbc_event* ev, const qcbc_het_tables* t);
/* Compute the tables on the device in FP64 for reference parameters pref[11] and
 * grid fgrid[M] (bin indices, from het_space, QuickCBC.c:4570-4910); replaces
 * heterodyne(), QuickCBC.c:5112-5299. */
int qcbc_het_setup(qcbc_event* ev, const double* pref, const int* fgrid, int M, int MN, int MM, int J);
/* Copy the event's tables back: caller buffers sized from qcbc_het_sizes(). */
int qcbc_het_sizes(const qcbc_event* ev, int* M, int* J, int* NR, int* MN, int* MM);
int qcbc_het_export(const qcbc_event* ev, int* fgrid, double* freq, double* amp, double* phase, double* IP,
                    double* SL, double* lc, double* ls, double* aa, double* rc, double* rs, double* logLb);
int qcbc_lnl_het(qcbc_event* ev, const double* params, int B, double* lnl, int precision);
int qcbc_lnl_het_dev(qcbc_event* ev, const double* d_params, int B, double* d_lnl, int precision, void* stream);
/* Heterodyne grid search het_space (QuickCBC.c:4570-4910) on the event's PSD about params, within
 * the prior box [pmin, pmax] (11 each): limits (4275) -> Fisher_All (2695) -> eigen-directions
 * (FisherEvec, 2449) scaled by efix (4387) to a squared distance of ~30 -> adaptive grid with
 * J = 2 points per region.  The waveforms run on the device, the control logic on the host.
 * Returns the grid size M and the band [MN, MM]; qcbc_het_space_grid copies the M bins.
 * Feed them to qcbc_het_setup (J = 2). */
int qcbc_het_space(qcbc_event* ev, const double* params, const double* pmin, const double* pmax, int* M, int* MN,
                   int* MM);
int qcbc_het_space_grid(const qcbc_event* ev, int* fgrid);
/* Batched het_diff (QuickCBC.c:4966-5051): out[b] = heterodyned squared distance between the
 * templates of params_a[b] and params_b[b] ([B][11] each), FP64. */
int qcbc_het_diff(qcbc_event* ev, const double* params_a, const double* params_b, int B, double* out);
/* Batched Fisher_Het (QuickCBC.c:5446-5617): fish [B][11][11] for params [B][11], from central
 * differences with step 1e-5 of all 23 waveforms of each set computed in one launch.  A set with
 * |chi1| or |chi2| >= 0.9999 gets 1e4 on the diagonal and zeros elsewhere, as in the reference. */
int qcbc_het_fisher(qcbc_event* ev, const double* params, int B, double* fish);

/* ---- allocation-free form (no counterpart in the reference) ---- */
/* Some callers cannot allocate device memory at call time: code that runs inside
 * another framework's runtime, which owns all device memory and hands the
 * operation pre-allocated buffers, and long-running services that keep a fixed
 * device-memory budget (cudaMalloc can fail under fragmentation, and cudaFree
 * synchronises the whole device, stalling every other stream).  For them this
 * entry point runs the full likelihood on device pointers they own (d_params
 * [B][11], d_lnl [B], d_rho [B][nifo] or NULL) and allocates nothing: its
 * scratch (records, status, tile partials) is a fixed array of
 * QCBC_NOALLOC_SCRATCH_BYTES in device memory, part of the library, held by
 * every GPU that loads the library until the process exits.
 *  - B is limited to QCBC_NOALLOC_MAX_SETS; larger B returns QCBC_EINVAL.
 *  - The event must have been opened (that allocates, once) on the current device.
 *  - The first call on a device looks up the array's device address; make that
 *    first call before any stream capture.
 *  - All calls share the one array: calls whose GPU work overlaps (different
 *    streams, or host threads without ordering) race and corrupt each other's
 *    results.  Serialise them, e.g. on one stream.
 *  - stream is a cudaStream_t passed as void* (NULL = the default stream);
 *    results are ready when the work on that stream completes.  NULL here is
 *    the legacy default stream, unlike qcbc_lnl_full_dev, where NULL is the
 *    calling thread's own non-blocking stream: a caller moving between the
 *    two with NULL gets a different ordering against its other work. */
#define QCBC_NOALLOC_MAX_SETS 4096
#define QCBC_NOALLOC_MAX_TILE_SLOTS 16384
#define QCBC_NOALLOC_SCRATCH_BYTES 4734976
int qcbc_lnl_full_noalloc(qcbc_event* ev, const double* d_params, int B, double* d_lnl, double* d_rho,
                          int precision, void* stream);

/* ---- launch tuning ---- */
/* Blocks per parameter set and threads per block for the full likelihood
 * (0 = automatic: measured once per (bins, nifo, B, precision) and cached). */
int qcbc_set_full_launch(qcbc_event* ev, int tiles, int threads);
int qcbc_get_full_launch(qcbc_event* ev, int B, int precision, int* tiles, int* threads);

/* ---- device memory for callers that stage parameters themselves ---- */
void* qcbc_device_alloc(long long bytes);
int qcbc_device_free(void* p);
int qcbc_memcpy_h2d(void* dst, const void* src, long long bytes);
int qcbc_memcpy_d2h(void* dst, const void* src, long long bytes);
int qcbc_synchronize(void);

/* ---- measurement helpers (CUDA events on the launching stream) ---- */
/* Runs `iters` likelihood launches on device-resident params; between launches
 * writes a scratch buffer larger than L2 when flush_l2 != 0 (outside the timed
 * span).  ms[iters] receives each launch's device time; kernel_ms[iters] the
 * time of the fused inner-product kernel alone (may be NULL). */
int qcbc_time_lnl_full(qcbc_event* ev, const double* d_params, int B, int precision, int iters, int flush_l2,
                       float* ms, float* kernel_ms);
int qcbc_time_lnl_het(qcbc_event* ev, const double* d_params, int B, int precision, int iters, int flush_l2,
                      float* ms);
/* Kernel launches issued by this library in the calling thread so far. */
long long qcbc_launch_count(void);

#ifdef __cplusplus
}
#endif
#endif
