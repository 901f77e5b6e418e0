// Kernel launch interface shared by the C ABI (qcbc_capi.cu) and the kernels (qcbc_kernels.cu).
#pragma once
#include "qcbc_device.cuh"

namespace qcbc {

// Network geometry and band of one analysis (by value into every kernel).
struct NetGeom {
  int nifo;
  int labels[kMaxIfo];
  int N;                 // samples; bins are 0..N/2
  int imin, imax;        // analysis band [imin, imax) (QuickCBC.c:4250-4252)
  double GMST;
  double Tobs;           // used for ts = Tobs - tc and sqrt(Tobs)
  double df;             // 1/Tobs
  int div_exact;         // 1: f_i = i*df equals i/Tobs bit for bit (power-of-two Tobs)
  int pad;
};

// Device-resident data of one analysis, pre-weighted by the PSD and scaled by
// sigma[id] so that the FP32 copy stays in range:
//   wr = 4 sigma Re(D)/S,  wi = 4 sigma Im(D)/S,  ws = 4 sigma^2 / S  per bin.
struct EventData {
  const double* w64;     // [nifo][3][nh]: wr, wi, ws rows (FP64 kernels)
  // FP32 weighted data of the mixed kernel with the amplitude's bin factor folded in:
  // wr' = wr i^{-7/6}, wi' = wi i^{-7/6}, ws' = ws i^{-7/3}, 12 B per detector-bin in planes that
  // one thread reads with the fewest aligned loads (MixW):
  //   nifo 3: float4 (wr0', wi0', wr1', wi1') | float4 (wr2', wi2', ws0', ws1') | float ws2'
  //   nifo 2: float4 (wr0', wi0', wr1', wi1') | float2 (ws0', ws1')
  //   nifo 1: float2 (wr0', wi0') | float ws0'
  const float* wm;
  int nh;                // row length (N/2)
  double inv_sigma[kMaxIfo];
  // per-bin constants shared by all events on a device (index = bin number i >= 1):
  // tabA = (i^{1/3}, i^{-1/3}), tabB = (log i, i^{3/4}), tabC = (1/i, i^{3/4}) rounded to float
  const double2* tabA;
  const double2* tabB;
  const float2* tabC;
  int tab_n;
};
// Floats of the mixed kernel's planes for an event of nifo detectors: 3 per detector-bin over nh bins.
inline size_t mixed_plane_floats(int nifo, size_t nh) { return (size_t)3 * nifo * nh; }

// Heterodyne summary tables on the device (layouts as the reference's struct Het, flattened):
//   freq[M], amp/phase[nifo][M], IP[NR][J+1][J+1], SL/lc/ls[NR][nifo][J+1], aa/rc/rs[nifo][NR].
struct HetData {
  int M, J, NR, MN, MM;
  double logLb;
  const double *freq, *amp, *phase, *IP, *SL, *lc, *ls, *aa, *rc, *rs;
  // the device's per-bin tables (EventData::tabA/B/C): the mixed form evaluates the waveform at
  // the grid's bins with the folded polynomials of the mixed full-likelihood kernel
  const double2* tabA;
  const double2* tabB;
  const float2* tabC;
};

enum Precision { kFP64 = 0, kMixed = 1 };

// One entry of the device-resident event table of a multi-event launch.
struct EventDesc {
  NetGeom g;
  EventData ev;
};

// status bits written by the setup kernel per parameter set
enum RecStatus { kStOK = 0, kStBadMass = 1, kStBadSpin = 2, kStBadDist = 4, kStBadSpinFinal = 8, kStFcut = 16,
                 kStNoEvent = 32 };

struct FullLaunch {
  int tiles;             // blocks per parameter set
  int threads;           // threads per block
};

// Parameter models of a set.  Full: the 11 parameters of log_likelihood_full (sky position,
// polarisation, inclination -> antenna response; phi0 = params[4] / 2).  Intrinsic: the
// NX + 3 (Nifo - 1) parameters of log_likelihood_intrinsic / templates (QuickCBC.c:3527-3598):
// per-detector phase offset, time offset and amplitude ratio relative to detector 0 in place of
// the antenna response, phi0 = params[4].
enum ParamModel { kModelFull = 0, kModelIntrinsic = 1 };
constexpr int kNX = 7;
constexpr int kMaxParams = kNX + 3 * (kMaxIfo - 1);
__host__ __device__ constexpr int param_stride(int model, int nifo) {
  return model == kModelIntrinsic ? kNX + 3 * (nifo - 1) : 11;
}

// Tables of the launch that follows the setup, which the setup's threads pull into L2 while they
// start (one 128-byte line each): a contiguous range, and the per-bin table entries at `nbins`
// bins listed in `bins` (device memory).  Empty by default.
struct SetupPrefetch {
  const void* buf = nullptr;
  size_t bytes = 0;
  const int* bins = nullptr;
  int nbins = 0;
  const double2* tabA = nullptr;
  const double2* tabB = nullptr;
  const float2* tabC = nullptr;
  int tab_n = 0;                     // entries of each table; bins outside [0, tab_n) are skipped
};
void launch_setup(const double* d_params, int B, const NetGeom& g, const QnmTable& q, PhdRec* d_recs,
                  int* d_status, cudaStream_t s, int model = kModelFull, const SetupPrefetch& pf = SetupPrefetch{});
// Launch order of the sets: the setup files each set under its length class (its bin count in
// kOrderClasses classes of the band): cnt[c] counts class c, list[c * B + r] is its r-th set (r in
// no particular order).  Block k of the one-tile lnL launch then takes the k-th set with the
// classes longest first.  cnt must be zero before the setup (the caller clears it on the launch
// stream).
constexpr int kOrderClasses = 64;
struct SetOrder {
  int* cnt;        // [kOrderClasses]
  int* list;       // [kOrderClasses][B]
};
void launch_setup_ordered(const double* d_params, int B, const NetGeom& g, const QnmTable& q, PhdRec* d_recs,
                          int* d_status, const SetOrder& o, cudaStream_t s, int model = kModelFull);
void launch_lnl_full(const PhdRec* d_recs, int B, const NetGeom& g, const EventData& ev, Precision prec,
                     const FullLaunch& L, double* d_partials, cudaStream_t s);
// d_rho: full model rho[id] = HD / sqrt(HH); intrinsic model the per-detector SNR^2 = 2 (HD - HH/2)
// (and lnL = 0 unless at least two detectors exceed 25 when Nifo > 1, QuickCBC.c:4117-4128)
void launch_finalize_full(const double* d_partials, const PhdRec* d_recs, const int* d_status, int B, int tiles,
                          const NetGeom& g, const EventData& ev, Precision prec, double* d_lnl, double* d_rho,
                          cudaStream_t s, int model = kModelFull);
// lnL of B sets with the finaliser folded into the lnL kernel: when each set is one tile (L.tiles ==
// 1), longest first when order is given (filled by launch_setup_ordered); at several tiles per set
// when d_done (B ints, zero before the launch and left zero after it) is given, the set's last
// tile to finish finalises it.  Otherwise the lnL kernel and launch_finalize_full.  Returns true
// when one launch did both.
bool launch_lnl_full_final(const PhdRec* d_recs, const int* d_status, int B, const NetGeom& g, const EventData& ev,
                           Precision prec, const FullLaunch& L, double* d_partials, double* d_lnl, double* d_rho,
                           int model, const SetOrder* order, cudaStream_t s, int* d_done = nullptr);
// fill the per-bin tables for bins [0, n)
void launch_fill_bin_tables(double2* d_tabA, double2* d_tabB, float2* d_tabC, int n, cudaStream_t s);
void launch_lnl_het(const PhdRec* d_recs, const int* d_status, int B, const NetGeom& g, const HetData& h,
                    Precision prec, double* d_lnl, cudaStream_t s);
// shared memory of one set's warp in the heterodyned kernels (its record and [3][nifo][M] doubles)
size_t het_smem_bytes(const NetGeom& g, const HetData& h);
// heterodyned lnL of sets of many events (records from launch_setup_multi); d_het [n_events] (M = 0:
// no tables); smem = the largest het_smem_bytes over the events
void launch_lnl_het_multi(const PhdRec* d_recs, const int* d_status, int B, const EventDesc* d_events,
                          const HetData* d_het, size_t smem, Precision prec, double* d_lnl, cudaStream_t s);
// fullphaseamp on the heterodyne grid (QuickCBC.c:3850-3866) for B records:
// amp/phase [B][nifo][M]
void launch_het_waves(const PhdRec* d_recs, int B, const NetGeom& g, const HetData& h, double* d_amp,
                      double* d_phase, cudaStream_t s);
// fullphaseamp on any frequency list freq[0..M) for B records: amp/phase [B][nifo][M]
void launch_waves(const PhdRec* d_recs, int B, const NetGeom& g, const double* d_freq, int M, double* d_amp,
                  double* d_phase, cudaStream_t s);
// Fisher_All (QuickCBC.c:2695-2817) from the 23 wave sets per matrix (layout of launch_het_fisher) on n
// bins, PSD rows S [nifo][sn_stride], bins [imin, imax): upper triangle of d_fish[nmat][11][11]
void launch_fisher_full(const double* d_amp, const double* d_phase, int nmat, const NetGeom& g, int n,
                        const double* d_S, int sn_stride, int imin, int imax, double eps, double* d_fish,
                        cudaStream_t s);
// diff (QuickCBC.c:4913-4964) of B wave sets against one reference wave set, bins [imin, m) of n,
// as `chunks` partial sums per set: d_out[B][chunks] (sum them in order)
void launch_diff_full(const double* d_amp_ref, const double* d_ph_ref, const double* d_amp, const double* d_ph, int B,
                      const NetGeom& g, int n, int imin, int m, const double* d_S, int sn_stride, int chunks,
                      double* d_out, cudaStream_t s);
// het_space ratios Cs, Sn, DH (QuickCBC.c:4688-4702) of wave sets 1..nset-1 to set 0, bins [j0, j1),
// bin-major [j1-j0][nset-1][nifo]
void launch_hs_ratios(const double* d_amp, const double* d_ph, int nset, int nifo, int n, int j0, int j1,
                      double* d_Cs, double* d_Sn, double* d_DH, cudaStream_t s);
// het_space grid walk (QuickCBC.c:4720-4765) over the ratios (per = (nset-1) nifo values per bin) and
// the per-bin tolerance scale ratio[j]: d_grid[0..*d_count) (count -1 when it would exceed cap)
void launch_hs_walk(const double* d_Cs, const double* d_Sn, const double* d_DH, const double* d_ratio, int per, int MN,
                    int MM, int djmax, double tol, int cap, int* d_grid, int* d_count, cudaStream_t s);
// het_diff (QuickCBC.c:4966-5051) for npair pairs of wave sets (2p, 2p+1) -> d_out[npair]
void launch_het_diff(const double* d_amp, const double* d_phase, int npair, const NetGeom& g, const HetData& h,
                     double* d_out, cudaStream_t s);
// Fisher_Het (QuickCBC.c:5446-5617) for nmat matrices; matrix f uses the wave sets 23 f + k:
// k = 0 the point, k = 1 + 2 i / 2 + 2 i the point +/- eps along parameter i.  Writes the upper
// triangle (j >= i) of d_fish[nmat][11][11].
void launch_het_fisher(const double* d_amp, const double* d_phase, int nmat, const NetGeom& g, const HetData& h,
                       double eps, double* d_fish, cudaStream_t s);

// waveform outputs for the reference-signature entry points
void launch_amp_phase(const double* d_freq, int n, double phi0, double fRef, double m1_Msun, double m2_Msun,
                      double chi1, double chi2, double dist, const QnmTable& q, PhdRec* d_rec, double* d_amp,
                      double* d_phase, int* d_status, cudaStream_t s);
// 4 sum_{i in [imin,imax)} (a_i b_i + a_{N-i} b_{N-i}) / S_i  (Utilities.c:716-736) into d_out[0]
void launch_nwip(const double* d_a, const double* d_b, const double* d_S, int imin, int imax, int N, double* d_out,
                 cudaStream_t s);
void launch_fulltemplates(const double* d_params, const NetGeom& g, const QnmTable& q, const double* d_freq,
                          PhdRec* d_rec, int* d_status, double* d_h, cudaStream_t s, int model = kModelFull);
// AmpPhase outputs (QuickCBC.c:3435-3440): Pf[i] = 2 pi f_i ts - phase[i], Af[i] = h22fac amp[i], i in [1, n)
void launch_ampphase_out(const double* d_freq, const double* d_amp, const double* d_phase, int n, double ts,
                         double* d_Af, double* d_Pf, cudaStream_t s);
void launch_fullphaseamp(const double* d_params, const NetGeom& g, const QnmTable& q, const double* d_freq, int n,
                         PhdRec* d_rec, int* d_status, double* d_amp, double* d_phase, cudaStream_t s);

// heterodyne setup pieces (FP64)
void launch_het_bins(const double* d_h, const double* d_amp, const double* d_phase, const double* d_D,
                     const double* d_S, int sn_stride, int N, int nifo, double* d_RC, double* d_RS, double* d_AA,
                     cudaStream_t s);
void launch_het_region_sums(const double* d_RC, const double* d_RS, const double* d_AA, const int* d_fgrid, int M,
                            int J, int nifo, int nh, double* d_SL, double* d_lc, double* d_ls, cudaStream_t s);
void launch_nwip_pairs(const double* d_h, const double* d_D, const double* d_S, int sn_stride, int N, int nifo,
                       int imin, int imax, double* d_out /* nifo x 2: HH, HR */, cudaStream_t s);

// ---- multi-event launches: parameter set b belongs to event event_of[b]; its signal bins are cut
// into tiles of tile_bins bins; the (set, tile) work items are processed by a persistent kernel.
// A set's tiling depends only on its own bins, so its lnL is the same in any mix of events.
void launch_setup_multi(const double* d_params, const int* d_event_of, int B, const EventDesc* d_events, int n_events,
                        const QnmTable& q, int tile_bins, PhdRec* d_recs, int* d_status, int* d_ntile, cudaStream_t s);
// d_off[0] = 0, d_off[b+1] = d_off[b] + ntile[b]; then d_items[d_off[b] + t] = b
void launch_scan_expand(const int* d_ntile, int B, int* d_off, int* d_items, int items_cap, cudaStream_t s);
// persistent kernel: `blocks` blocks pull work items from *d_counter (zeroed by the caller)
void launch_lnl_multi(const PhdRec* d_recs, const EventDesc* d_events, const int* d_off, const int* d_items, int B,
                      int tile_bins, int items_cap, Precision prec, int threads, int blocks, int* d_counter,
                      double* d_partials, cudaStream_t s);
void launch_finalize_multi(const double* d_partials, const PhdRec* d_recs, const int* d_status, const int* d_off,
                           const EventDesc* d_events, int B, int items_cap, Precision prec, double* d_lnl,
                           double* d_rho, cudaStream_t s);
int multi_blocks_per_sm(Precision prec, int threads, int tile_bins);

void upload_tables();    // constant-memory tables; call once per device
void allow_dynamic_smem();
// One sky-ring proposal map (qcbc_sky_ring_map): x -> y on device buffers, log Jacobian in *d_lj.
void launch_sky_ring_map(const double* d_x, double* d_y, double GMST, int l1, int l2, double rot, double* d_lj,
                         cudaStream_t s);   // dynamic shared-memory limit of the mixed kernels; once per device

}  // namespace qcbc
