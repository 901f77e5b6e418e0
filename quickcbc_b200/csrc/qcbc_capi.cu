// C ABI of the QuickCBC likelihood engine: events resident on the device,
// batched likelihood calls, the reference-signature drop-ins and timing helpers.
#include <cuda_runtime.h>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>
#include <algorithm>
#include <atomic>
#include <chrono>
#include <thread>

#include "qcbc_kernels.cuh"
#include "qcbc_hetspace.h"
#include "qcbc_ingest_dev.h"
#include "../../include/qcbc_gpu.h"
#include "../../include/qcbc_quickcbc.h"
#include "_gen/qnm_table.h"

using namespace qcbc;

// ------------------------------------------------------------------ errors
static thread_local std::string tls_err;
static thread_local long long tls_launches = 0;

static int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  tls_err = buf;
  return code;
}
#define CU(call)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (call);                                                                   \
    if (e_ != cudaSuccess) return fail(QCBC_ECUDA, "%s: %s", #call, cudaGetErrorString(e_));   \
  } while (0)

extern "C" const char* qcbc_last_error(void) { return tls_err.c_str(); }
// error reporting for the library's other host files (the service)
extern "C" int qcbc_internal_fail(int code, const char* msg) {
  tls_err = msg;
  return code;
}
extern "C" const char* qcbc_version(void) { return "qcbc-b200 0.1 (sm_100a)"; }
extern "C" long long qcbc_launch_count(void) { return tls_launches; }

// ------------------------------------------------------------------ device state
struct DeviceState {
  bool ready = false;
  double* d_qnm = nullptr;   // x, yr, mr, yd, md (5 * n)
  int n = 0;
  QnmTable qnm{};
  // per-bin constants for the mixed kernel: (i^{1/3}, i^{-1/3}) and (log i, i^{3/4})
  double2* d_tabA = nullptr;
  double2* d_tabB = nullptr;
  float2* d_tabC = nullptr;
  int tab_n = 0;
  int* d_bucket = nullptr;   // QNM interval index per 0.001 of final spin
};
static std::mutex g_mu;
constexpr int kMaxDevices = 16;        // devices the library keeps state for (device ids 0..15)
static DeviceState g_dev[kMaxDevices];
static std::vector<double> g_qnm_host[3];   // a, fring, fdamp

static void natural_spline_m2(const std::vector<double>& x, const std::vector<double>& y, std::vector<double>& M) {
  int n = (int)x.size();
  M.assign(n, 0.0);
  if (n < 3) return;
  std::vector<double> diag(n), rhs(n);
  for (int i = 1; i < n - 1; i++) {
    double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    diag[i] = 2.0 * (h0 + h1);
    rhs[i] = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
  }
  for (int i = 2; i < n - 1; i++) {
    double h = x[i] - x[i - 1], w = h / diag[i - 1];
    diag[i] -= w * h;
    rhs[i] -= w * rhs[i - 1];
  }
  for (int i = n - 2; i >= 1; i--) M[i] = (rhs[i] - (x[i + 1] - x[i]) * M[i + 1]) / diag[i];
}

static int upload_qnm(DeviceState& ds) {
  if (g_qnm_host[0].empty()) {
    g_qnm_host[0].assign(QCBC_QNM_A, QCBC_QNM_A + QCBC_QNM_N);
    g_qnm_host[1].assign(QCBC_QNM_FRING, QCBC_QNM_FRING + QCBC_QNM_N);
    g_qnm_host[2].assign(QCBC_QNM_FDAMP, QCBC_QNM_FDAMP + QCBC_QNM_N);
  }
  int n = (int)g_qnm_host[0].size();
  std::vector<double> mr, md;
  natural_spline_m2(g_qnm_host[0], g_qnm_host[1], mr);
  natural_spline_m2(g_qnm_host[0], g_qnm_host[2], md);
  std::vector<double> all;
  all.reserve(5 * n);
  all.insert(all.end(), g_qnm_host[0].begin(), g_qnm_host[0].end());
  all.insert(all.end(), g_qnm_host[1].begin(), g_qnm_host[1].end());
  all.insert(all.end(), mr.begin(), mr.end());
  all.insert(all.end(), g_qnm_host[2].begin(), g_qnm_host[2].end());
  all.insert(all.end(), md.begin(), md.end());
  if (ds.d_qnm) cudaFree(ds.d_qnm);
  CU(cudaMalloc(&ds.d_qnm, all.size() * sizeof(double)));
  CU(cudaMemcpy(ds.d_qnm, all.data(), all.size() * sizeof(double), cudaMemcpyHostToDevice));
  // interval index for spins -1 + k/1000 (the table spacing is >= 0.001)
  const std::vector<double>& x = g_qnm_host[0];
  int nb = 2001;
  std::vector<int> bucket(nb);
  for (int k = 0, j = 0; k < nb; k++) {
    double sk = -1.0 + k / 1000.0;
    while (j < n - 2 && x[j + 1] <= sk) j++;
    bucket[k] = j;
  }
  if (ds.d_bucket) cudaFree(ds.d_bucket);
  CU(cudaMalloc(&ds.d_bucket, nb * sizeof(int)));
  CU(cudaMemcpy(ds.d_bucket, bucket.data(), nb * sizeof(int), cudaMemcpyHostToDevice));
  bool uniform_ok = x.front() >= -1.0 && x.back() <= 1.0;
  for (int i = 1; i < n && uniform_ok; i++) uniform_ok = (x[i] - x[i - 1]) >= 0.999e-3;
  ds.n = n;
  ds.qnm = QnmTable{ds.d_qnm, ds.d_qnm + n, ds.d_qnm + 2 * n, ds.d_qnm + 3 * n, ds.d_qnm + 4 * n,
                    uniform_ok ? ds.d_bucket : nullptr, n, nb};
  return QCBC_OK;
}

// Bin tables cover bins [0, n); grown (never shrunk) under g_mu when an event needs more.
static int ensure_bin_tables(DeviceState& ds, int n) {
  if (ds.tab_n >= n) return QCBC_OK;
  int want = std::max(n, 1 << 20);
  double2 *a = nullptr, *b = nullptr;
  float2* c = nullptr;
  CU(cudaMalloc(&a, (size_t)want * sizeof(double2)));
  CU(cudaMalloc(&b, (size_t)want * sizeof(double2)));
  CU(cudaMalloc(&c, (size_t)want * sizeof(float2)));
  launch_fill_bin_tables(a, b, c, want, 0);
  tls_launches += 1;
  CU(cudaDeviceSynchronize());
  // The smaller tables stay allocated: batches copy the table pointers into their device event
  // descriptors when a slot is set, and they must keep pointing at valid tables.
  ds.d_tabA = a;
  ds.d_tabB = b;
  ds.d_tabC = c;
  ds.tab_n = want;
  return QCBC_OK;
}

static int current_device() {
  int d = 0;
  cudaGetDevice(&d);
  return d;
}

extern "C" int qcbc_init(int device) {
  if (device < 0 || device >= kMaxDevices) return fail(QCBC_EINVAL, "device %d out of range 0..%d", device, kMaxDevices - 1);
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    return fail(QCBC_ECUDA, "no CUDA device available (%s)", cudaGetErrorString(e));
  if (device >= ndev) return fail(QCBC_EINVAL, "device %d >= device count %d", device, ndev);
  CU(cudaSetDevice(device));
  std::lock_guard<std::mutex> lk(g_mu);
  DeviceState& ds = g_dev[device];
  if (!ds.ready) {
    upload_tables();
    allow_dynamic_smem();
    int rc = upload_qnm(ds);
    if (rc) return rc;
    rc = ensure_bin_tables(ds, 1 << 20);
    if (rc) return rc;
    ds.ready = true;
  }
  return QCBC_OK;
}

// Every entry point calls this (directly or through workspace()) before it indexes per-device
// state with the current device, so the index is checked here.
static int ensure_init() {
  int d = current_device();
  if (d < 0 || d >= kMaxDevices) return fail(QCBC_EINVAL, "current device %d out of range 0..%d", d, kMaxDevices - 1);
  if (g_dev[d].ready) return QCBC_OK;
  return qcbc_init(d);
}

extern "C" int qcbc_internal_ensure_init(void) { return ensure_init(); }

extern "C" int qcbc_set_qnm_table(const double* a, const double* fring, const double* fdamp, int n) {
  if (!a || !fring || !fdamp || n < 4) return fail(QCBC_EINVAL, "bad QNM table");
  for (int i = 1; i < n; i++)
    if (!(a[i] > a[i - 1])) return fail(QCBC_EINVAL, "QNM spins must increase strictly");
  std::lock_guard<std::mutex> lk(g_mu);
  g_qnm_host[0].assign(a, a + n);
  g_qnm_host[1].assign(fring, fring + n);
  g_qnm_host[2].assign(fdamp, fdamp + n);
  for (auto& ds : g_dev)
    if (ds.ready) {
      int rc = upload_qnm(ds);
      if (rc) return rc;
    }
  return QCBC_OK;
}

// ------------------------------------------------------------------ per-thread workspace
template <typename T>
static int grow(T*& p, size_t& cap, size_t n) {
  if (n <= cap && p) return QCBC_OK;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  size_t want = std::max(n, (size_t)256);
  cudaError_t e = cudaMalloc(&p, want * sizeof(T));
  if (e != cudaSuccess) return fail(QCBC_ENOMEM, "cudaMalloc %zu B: %s", want * sizeof(T), cudaGetErrorString(e));
  cap = want;
  return QCBC_OK;
}
template <typename T>
static int grow_host(T*& p, size_t& cap, size_t n) {
  if (n <= cap && p) return QCBC_OK;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  size_t want = std::max(n, (size_t)256);
  cudaError_t e = cudaMallocHost(&p, want * sizeof(T));
  if (e != cudaSuccess) return fail(QCBC_ENOMEM, "cudaMallocHost %zu B: %s", want * sizeof(T), cudaGetErrorString(e));
  cap = want;
  return QCBC_OK;
}

struct Workspace {
  int device = -1;
  cudaStream_t stream = nullptr;
  double* d_params = nullptr; size_t c_params = 0;
  PhdRec* d_recs = nullptr; size_t c_recs = 0;
  int* d_status = nullptr; size_t c_status = 0;
  double* d_part = nullptr; size_t c_part = 0;
  double* d_lnl = nullptr; size_t c_lnl = 0;
  double* d_rho = nullptr; size_t c_rho = 0;
  // launch order of the sets (SetOrder): class counts, cleared on the call's stream before each
  // ordered setup, and the class lists
  int* d_ocnt = nullptr; size_t c_ocnt = 0;
  int* d_olist = nullptr; size_t c_olist = 0;
  // per-set tile counts of multi-tile launches that finalise in their last tile (FinalOut::done):
  // zeroed when allocated, left zero by every launch
  int* d_done = nullptr; size_t c_done = 0;
  double* h_params = nullptr; size_t ch_params = 0;
  double* h_lnl = nullptr; size_t ch_lnl = 0;
  double* h_rho = nullptr; size_t ch_rho = 0;
  // device addresses of the pinned buffers above (mapped_ptr), and the capacity of the buffer
  // each was taken from (a buffer is only reallocated to a larger capacity)
  double *m_params = nullptr, *m_lnl = nullptr, *m_rho = nullptr;
  size_t m_params_of = 0, m_lnl_of = 0, m_rho_of = 0;
  int* h_status = nullptr; size_t ch_status = 0;
  // generic scratch for the reference-signature entry points
  double* d_a = nullptr; size_t c_a = 0;
  double* d_b = nullptr; size_t c_b = 0;
  double* d_c = nullptr; size_t c_c = 0;
  double* h_a = nullptr; size_t ch_a = 0;
  double* h_b = nullptr; size_t ch_b = 0;
  unsigned char* d_flush = nullptr; size_t c_flush = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr, e2 = nullptr, e3 = nullptr;
};
static thread_local Workspace tls_ws;

static int workspace(Workspace*& w) {
  int rc = ensure_init();
  if (rc) return rc;
  w = &tls_ws;
  int d = current_device();
  if (w->device != d) {
    if (w->device >= 0) return fail(QCBC_EINVAL, "thread switched device (%d -> %d)", w->device, d);
    CU(cudaStreamCreateWithFlags(&w->stream, cudaStreamNonBlocking));
    CU(cudaEventCreate(&w->e0));
    CU(cudaEventCreate(&w->e1));
    CU(cudaEventCreate(&w->e2));
    CU(cudaEventCreate(&w->e3));
    w->device = d;
  }
  return QCBC_OK;
}

// ------------------------------------------------------------------ events
struct HetDev {
  int M = 0, J = 0, NR = 0, MN = 0, MM = 0;
  double logLb = 0.0;
  double* buf = nullptr;   // freq, amp, phase, IP, SL, lc, ls, aa, rc, rs
  int* d_fgrid = nullptr;
  size_t bytes = 0;
  std::vector<int> fgrid;
  double pref[11] = {0};       // reference point of tables built by qcbc_het_setup
  bool has_pref = false;
};

struct qcbc_event {
  int device = 0;
  // the last grid found by qcbc_het_space
  std::vector<int> space_grid;
  int space_MN = 0, space_MM = 0;
  NetGeom g{};
  double fmin = 16.0, fmax = 1024.0;
  int nh = 0;
  double* d_w64 = nullptr;
  float* d_wm = nullptr;     // FP32 planes of the mixed kernel (EventData::wm)
  double* d_D = nullptr;     // raw data [nifo][N] (heterodyne setup)
  double* d_S = nullptr;     // raw PSD [nifo][nh+1]
  double* d_freq = nullptr;  // canonical frequencies [nh]
  double inv_sigma[kMaxIfo] = {1, 1, 1};
  HetDev het;
  int fixed_tiles = 0, fixed_threads = 0;
  std::map<long long, FullLaunch> tuned;
  long long bytes = 0;
  bool has_data = false;
};

static EventData event_data(const qcbc_event* ev) {
  EventData d{};
  d.w64 = ev->d_w64;
  d.wm = ev->d_wm;
  d.nh = ev->nh;
  for (int k = 0; k < kMaxIfo; k++) d.inv_sigma[k] = ev->inv_sigma[k];
  const DeviceState& ds = g_dev[ev->device];
  d.tab_n = ds.tab_n;
  d.tabA = ds.d_tabA;
  d.tabB = ds.d_tabB;
  d.tabC = ds.d_tabC;
  return d;
}

static HetData het_data(const qcbc_event* ev) {
  const HetDev& h = ev->het;
  HetData d{};
  d.M = h.M; d.J = h.J; d.NR = h.NR; d.MN = h.MN; d.MM = h.MM; d.logLb = h.logLb;
  int nI = ev->g.nifo, J1 = h.J + 1;
  double* p = h.buf;
  d.freq = p; p += h.M;
  d.amp = p; p += (size_t)nI * h.M;
  d.phase = p; p += (size_t)nI * h.M;
  d.IP = p; p += (size_t)h.NR * J1 * J1;
  d.SL = p; p += (size_t)h.NR * nI * J1;
  d.lc = p; p += (size_t)h.NR * nI * J1;
  d.ls = p; p += (size_t)h.NR * nI * J1;
  d.aa = p; p += (size_t)nI * h.NR;
  d.rc = p; p += (size_t)nI * h.NR;
  d.rs = p;
  const DeviceState& ds = g_dev[ev->device];
  d.tabA = ds.d_tabA;
  d.tabB = ds.d_tabB;
  d.tabC = ds.d_tabC;
  return d;
}

static size_t het_doubles(int nifo, int M, int J) {
  int NR = (M - 1) / J, J1 = J + 1;
  return (size_t)M + 2 * (size_t)nifo * M + (size_t)NR * J1 * J1 + 3 * (size_t)NR * nifo * J1 + 3 * (size_t)nifo * NR;
}

static bool pow2_exact(double Tobs) {
  int e;
  double m = frexp(Tobs, &e);
  return m == 0.5;
}

static void fill_geom(NetGeom& g, int nifo, const int* labels, double Tobs, double GMST, int N, double fmin,
                      double fmax) {
  memset(&g, 0, sizeof(g));
  g.nifo = nifo;
  for (int i = 0; i < nifo && i < kMaxIfo; i++) g.labels[i] = labels[i];
  g.N = N;
  g.imin = (int)(Tobs * fmin);
  g.imax = (int)(Tobs * fmax);
  if (g.imax > N / 2) g.imax = N / 2;
  g.GMST = GMST;
  g.Tobs = Tobs;
  g.df = 1.0 / Tobs;
  g.div_exact = pow2_exact(Tobs) ? 1 : 0;
}

static int check_geom(int nifo, const int* labels, double Tobs, int N) {
  if (nifo < 1 || nifo > kMaxIfo) return fail(QCBC_EINVAL, "nifo=%d (1..3 supported)", nifo);
  if (!labels) return fail(QCBC_EINVAL, "labels is NULL");
  for (int i = 0; i < nifo; i++)
    if (labels[i] < 0 || labels[i] > 2) return fail(QCBC_EINVAL, "detector label %d (0=H,1=L,2=V)", labels[i]);
  if (!(Tobs > 0.0)) return fail(QCBC_EINVAL, "Tobs must be positive");
  if (N < 8 || (N & 1)) return fail(QCBC_EINVAL, "N=%d must be even and >= 8", N);
  return QCBC_OK;
}

// Data upload: raw D, S (rows gathered on the host), then the weighted FP64 data and the mixed
// kernel's FP32 planes built on the device by the kernel that rebuilds them after a PSD redraw
// (launch_event_weights), so both ways give the same bits.
static int event_upload(qcbc_event* ev, const double* const* Drows, const double* const* Srows) {
  const int nI = ev->g.nifo, N = ev->g.N, nh = N / 2;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    int rc = ensure_bin_tables(g_dev[ev->device], nh + 1);
    if (rc) return rc;
  }
  ev->nh = nh;
  std::vector<double> Dall((size_t)nI * N), Sall((size_t)nI * (nh + 1), 0.0);
  const int lo = std::max(ev->g.imin, 1), hi = std::min(ev->g.imax, nh);
  qcbc::Sigmas sg{{1.0, 1.0, 1.0}};
  for (int id = 0; id < nI; id++) {
    const double* D = Drows[id];
    const double* S = Srows[id];
    memcpy(&Dall[(size_t)id * N], D, sizeof(double) * N);
    for (int i = 0; i < nh; i++) Sall[(size_t)id * (nh + 1) + i] = S[i];
    // sigma^2 = smallest PSD in band keeps 4 sigma^2/S <= 4 and 4 sigma D/S = O(1)
    double smin = HUGE_VAL;
    for (int i = lo; i < hi; i++)
      if (S[i] > 0.0 && S[i] < smin) smin = S[i];
    if (!(smin < HUGE_VAL)) smin = 1.0;
    sg.v[id] = sqrt(smin);
    ev->inv_sigma[id] = 1.0 / sg.v[id];
  }
  std::vector<double> freq(nh);
  freq[0] = 1.0 / ev->g.Tobs;
  for (int i = 1; i < nh; i++) freq[i] = (double)i / ev->g.Tobs;
  const size_t b64 = (size_t)nI * 3 * nh * 8, bm = qcbc::mixed_plane_floats(nI, nh) * sizeof(float),
               bD = Dall.size() * 8, bS = Sall.size() * 8, bf = freq.size() * 8;
  if (!ev->d_w64) {
    CU(cudaMalloc(&ev->d_w64, b64));
    CU(cudaMalloc(&ev->d_wm, bm));
    CU(cudaMalloc(&ev->d_D, bD));
    CU(cudaMalloc(&ev->d_S, bS));
    CU(cudaMalloc(&ev->d_freq, bf));
  }
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  cudaStream_t s = w->stream;     // the calling thread's stream: other threads' work goes on
  CU(cudaMemsetAsync(ev->d_w64, 0, b64, s));
  CU(cudaMemsetAsync(ev->d_wm, 0, bm, s));
  CU(cudaMemcpyAsync(ev->d_D, Dall.data(), bD, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(ev->d_S, Sall.data(), bS, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(ev->d_freq, freq.data(), bf, cudaMemcpyHostToDevice, s));
  qcbc::launch_event_weights(ev->d_D, N, ev->d_S, nh + 1, nI, lo, hi, sg, ev->d_w64, ev->d_wm, s);
  tls_launches += 1;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(s));
  ev->bytes = (long long)(b64 + bm + bD + bS + bf);
  ev->has_data = true;
  return QCBC_OK;
}

static void event_free_device(qcbc_event* ev) {
  cudaFree(ev->d_w64); cudaFree(ev->d_wm); cudaFree(ev->d_D); cudaFree(ev->d_S); cudaFree(ev->d_freq);
  cudaFree(ev->het.buf); cudaFree(ev->het.d_fgrid);
  ev->d_w64 = nullptr; ev->d_wm = nullptr; ev->d_D = nullptr; ev->d_S = nullptr; ev->d_freq = nullptr;
  ev->het.buf = nullptr; ev->het.d_fgrid = nullptr;
}

extern "C" qcbc_event* qcbc_event_open(int nifo, const int* labels, double Tobs, double GMST, int N, const double* D,
                                       int d_stride, const double* SN, int sn_stride, double fmin, double fmax) {
  if (ensure_init()) return nullptr;
  if (check_geom(nifo, labels, Tobs, N)) return nullptr;
  if (!D || !SN) { fail(QCBC_EINVAL, "D and SN must not be NULL"); return nullptr; }
  if (d_stride < N || sn_stride < N / 2) { fail(QCBC_EINVAL, "row strides too small"); return nullptr; }
  if (!(fmin >= 0.0) || !(fmax > fmin)) { fail(QCBC_EINVAL, "bad band [%g, %g)", fmin, fmax); return nullptr; }
  qcbc_event* ev = new qcbc_event();
  ev->device = current_device();
  ev->fmin = fmin;
  ev->fmax = fmax;
  fill_geom(ev->g, nifo, labels, Tobs, GMST, N, fmin, fmax);
  std::vector<const double*> Dr(nifo), Sr(nifo);
  for (int i = 0; i < nifo; i++) { Dr[i] = D + (size_t)i * d_stride; Sr[i] = SN + (size_t)i * sn_stride; }
  if (event_upload(ev, Dr.data(), Sr.data())) { event_free_device(ev); delete ev; return nullptr; }
  return ev;
}

extern "C" int qcbc_event_close(qcbc_event* ev) {
  if (!ev) return QCBC_OK;
  event_free_device(ev);
  delete ev;
  return QCBC_OK;
}

extern "C" long long qcbc_event_device_bytes(const qcbc_event* ev) {
  if (!ev) return 0;
  return ev->bytes + (long long)ev->het.bytes;
}

// ------------------------------------------------------------------ launch choice
// Blocks per parameter set: enough blocks to fill 148 SMs several times over,
// but at least ~512 bins per block.  The measured variant (tune_full) overrides.
static FullLaunch heuristic_launch(const qcbc_event* ev, int B, int prec) {
  FullLaunch L;
  L.threads = 256;
  int bins = std::max(1, ev->g.imax - ev->g.imin);
  int want_blocks = 148 * 8;
  int tiles = (want_blocks + B - 1) / B;
  int max_tiles = std::max(1, bins / 512);
  L.tiles = std::max(1, std::min(tiles, max_tiles));
  (void)prec;
  return L;
}

static FullLaunch choose_launch(qcbc_event* ev, int B, int prec) {
  if (ev->fixed_tiles > 0) return FullLaunch{ev->fixed_tiles, ev->fixed_threads > 0 ? ev->fixed_threads : 256};
  long long key = ((long long)B << 2) | prec;
  auto it = ev->tuned.find(key);
  if (it != ev->tuned.end()) return it->second;
  return heuristic_launch(ev, B, prec);
}

extern "C" int qcbc_set_full_launch(qcbc_event* ev, int tiles, int threads) {
  if (!ev) return fail(QCBC_EINVAL, "event is NULL");
  if (tiles < 0 || (threads != 0 && (threads < 32 || threads > 256 || threads % 32)))
    return fail(QCBC_EINVAL, "tiles >= 0, threads in {32..256} multiple of 32");
  ev->fixed_tiles = tiles;
  ev->fixed_threads = threads;
  return QCBC_OK;
}

extern "C" int qcbc_get_full_launch(qcbc_event* ev, int B, int precision, int* tiles, int* threads) {
  if (!ev || !tiles || !threads) return fail(QCBC_EINVAL, "NULL argument");
  FullLaunch L = choose_launch(ev, B, precision);
  *tiles = L.tiles;
  *threads = L.threads;
  return QCBC_OK;
}

// ------------------------------------------------------------------ full likelihood
static int enqueue_full(Workspace* w, qcbc_event* ev, const double* d_params, int B, double* d_lnl, double* d_rho,
                        int prec, cudaStream_t s, const NetGeom& g, cudaEvent_t k0 = nullptr,
                        cudaEvent_t k1 = nullptr, int model = kModelFull, const FullLaunch* shape = nullptr) {
  FullLaunch L = shape ? *shape : choose_launch(ev, B, prec);
  int rc;
  if ((rc = grow(w->d_recs, w->c_recs, (size_t)B))) return rc;
  if ((rc = grow(w->d_status, w->c_status, (size_t)B))) return rc;
  if ((rc = grow(w->d_part, w->c_part, (size_t)B * L.tiles * 2 * kMaxIfo))) return rc;
  DeviceState& ds = g_dev[current_device()];
  EventData ed = event_data(ev);
  const Precision kp = prec == QCBC_MIXED ? kMixed : kFP64;
  if (L.tiles == 1) {
    // one tile per set: the sets run in order of length and the lnL kernel finalises each itself
    // The counts start at zero on this call's stream, whatever ran before: repeated calls, calls
    // on other streams and replays of a captured graph each clear their own.
    if ((rc = grow(w->d_ocnt, w->c_ocnt, (size_t)kOrderClasses))) return rc;
    if ((rc = grow(w->d_olist, w->c_olist, (size_t)kOrderClasses * B))) return rc;
    CU(cudaMemsetAsync(w->d_ocnt, 0, sizeof(int) * kOrderClasses, s));
    const SetOrder o{w->d_ocnt, w->d_olist};
    launch_setup_ordered(d_params, B, g, ds.qnm, w->d_recs, w->d_status, o, s, model);
    if (k0) cudaEventRecord(k0, s);
    launch_lnl_full_final(w->d_recs, w->d_status, B, g, ed, kp, L, w->d_part, d_lnl, d_rho, model, &o, s);
    if (k1) cudaEventRecord(k1, s);
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) return fail(QCBC_ECUDA, "lnL launch: %s", cudaGetErrorString(le));
    tls_launches += 2;
  } else {
    // several tiles per set: the last tile of each set to finish finalises it
    const size_t had = w->c_done;
    if ((rc = grow(w->d_done, w->c_done, (size_t)B))) return rc;
    if (w->c_done != had) CU(cudaMemsetAsync(w->d_done, 0, sizeof(int) * w->c_done, s));
    launch_setup(d_params, B, g, ds.qnm, w->d_recs, w->d_status, s, model);
    if (k0) cudaEventRecord(k0, s);
    launch_lnl_full_final(w->d_recs, w->d_status, B, g, ed, kp, L, w->d_part, d_lnl, d_rho, model, nullptr, s,
                          w->d_done);
    if (k1) cudaEventRecord(k1, s);
    tls_launches += 2;
  }
  CU(cudaGetLastError());
  return QCBC_OK;
}

// Device address of pinned buffer h of capacity cap, cached in m while the capacity is `of`.
static int mapped_ptr(double* h, size_t cap, double*& m, size_t& of) {
  if (of != cap || !m) {
    CU(cudaHostGetDevicePointer((void**)&m, h, 0));
    of = cap;
  }
  return QCBC_OK;
}

static int run_full(qcbc_event* ev, const double* params, int B, double* lnl, double* rho, int prec,
                    const NetGeom& g, int model = kModelFull, const FullLaunch* shape = nullptr) {
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  const size_t ps = (size_t)param_stride(model, g.nifo);
  if ((rc = grow_host(w->h_params, w->ch_params, (size_t)B * ps))) return rc;
  if ((rc = grow_host(w->h_lnl, w->ch_lnl, (size_t)B))) return rc;
  if ((rc = grow_host(w->h_rho, w->ch_rho, (size_t)B * kMaxIfo))) return rc;
  memcpy(w->h_params, params, sizeof(double) * ps * (size_t)B);
  cudaStream_t s = w->stream;
  // The setup reads the parameters from, and the lnL kernel writes lnL (and rho) into, the pinned
  // staging buffers directly (mapped host memory): the bytes cross the host link inside the
  // kernels, with no copy calls and their latency.
  if ((rc = mapped_ptr(w->h_params, w->ch_params, w->m_params, w->m_params_of))) return rc;
  if ((rc = mapped_ptr(w->h_lnl, w->ch_lnl, w->m_lnl, w->m_lnl_of))) return rc;
  if (rho && (rc = mapped_ptr(w->h_rho, w->ch_rho, w->m_rho, w->m_rho_of))) return rc;
  if ((rc = enqueue_full(w, ev, w->m_params, B, w->m_lnl, rho ? w->m_rho : nullptr, prec, s, g, nullptr, nullptr,
                         model, shape)))
    return rc;
  CU(cudaStreamSynchronize(s));
  memcpy(lnl, w->h_lnl, sizeof(double) * B);
  if (rho) memcpy(rho, w->h_rho, sizeof(double) * B * g.nifo);
  // a set fails the setup exactly when its lnL is the rejected-sample value
  int bad = 0;
  for (int b = 0; b < B; b++) bad += lnl[b] == -1.0e20;
  if (bad) return fail(QCBC_EDOM, "%d of %d parameter sets outside the waveform domain (lnL=-1e20)", bad, B);
  return QCBC_OK;
}

extern "C" int qcbc_lnl_full(qcbc_event* ev, const double* params, int B, double* lnl, double* rho, int precision) {
  if (!ev || !params || !lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (B < 0) return fail(QCBC_EINVAL, "B < 0");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B == 0) return QCBC_OK;
  return run_full(ev, params, B, lnl, rho, precision, ev->g);
}

extern "C" int qcbc_lnl_full_dev(qcbc_event* ev, const double* d_params, int B, double* d_lnl, double* d_rho,
                                 int precision, void* stream) {
  if (!ev || !d_params || !d_lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : w->stream;
  return enqueue_full(w, ev, d_params, B, d_lnl, d_rho, precision, s, ev->g);
}

extern "C" int qcbc_lnl_intrinsic(qcbc_event* ev, const double* params, int B, double* lnl, double* snrsq,
                                  int precision) {
  if (!ev || !params || !lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (B < 0) return fail(QCBC_EINVAL, "B < 0");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B == 0) return QCBC_OK;
  return run_full(ev, params, B, lnl, snrsq, precision, ev->g, kModelIntrinsic);
}

// ------------------------------------------------------------------ heterodyne
static int het_alloc(qcbc_event* ev, int M, int J, int MN, int MM) {
  HetDev& h = ev->het;
  if (M < J + 1 || J < 1 || J > 3) return fail(QCBC_EINVAL, "heterodyne grid M=%d J=%d", M, J);
  size_t need = het_doubles(ev->g.nifo, M, J);
  if (h.buf && h.M == M && h.J == J) {
    // same shape: reuse
  } else {
    cudaFree(h.buf);
    cudaFree(h.d_fgrid);
    h.buf = nullptr;
    h.d_fgrid = nullptr;
    CU(cudaMalloc(&h.buf, need * sizeof(double)));
    CU(cudaMalloc(&h.d_fgrid, (size_t)M * sizeof(int)));
  }
  h.M = M; h.J = J; h.NR = (M - 1) / J; h.MN = MN; h.MM = MM;
  h.bytes = need * sizeof(double) + (size_t)M * sizeof(int);
  size_t smem = het_smem_bytes(ev->g, het_data(ev));
  if (smem > 200 * 1024) return fail(QCBC_EINVAL, "heterodyne grid M=%d too large for one block (%zu B)", M, smem);
  return QCBC_OK;
}

extern "C" int qcbc_het_set(qcbc_event* ev, const qcbc_het_tables* t) {
  if (!ev || !t) return fail(QCBC_EINVAL, "NULL argument");
  int rc = ensure_init();
  if (rc) return rc;
  if ((rc = het_alloc(ev, t->M, t->J, t->MN, t->MM))) return rc;
  HetDev& h = ev->het;
  h.logLb = t->logLb;
  h.has_pref = false;
  h.fgrid.assign(t->fgrid, t->fgrid + t->M);
  HetData d = het_data(ev);
  int nI = ev->g.nifo, M = h.M, NR = h.NR, J1 = h.J + 1;
  struct { const double* src; const double* dst; size_t n; } parts[] = {
    {t->freq, d.freq, (size_t)M}, {t->amp, d.amp, (size_t)nI * M}, {t->phase, d.phase, (size_t)nI * M},
    {t->IP, d.IP, (size_t)NR * J1 * J1}, {t->SL, d.SL, (size_t)NR * nI * J1}, {t->lc, d.lc, (size_t)NR * nI * J1},
    {t->ls, d.ls, (size_t)NR * nI * J1}, {t->aa, d.aa, (size_t)nI * NR}, {t->rc, d.rc, (size_t)nI * NR},
    {t->rs, d.rs, (size_t)nI * NR}};
  for (auto& p : parts) {
    if (!p.src) return fail(QCBC_EINVAL, "heterodyne table pointer is NULL");
    CU(cudaMemcpy((void*)p.dst, p.src, p.n * sizeof(double), cudaMemcpyHostToDevice));
  }
  CU(cudaMemcpy(h.d_fgrid, t->fgrid, (size_t)M * sizeof(int), cudaMemcpyHostToDevice));
  return QCBC_OK;
}

extern "C" int qcbc_het_sizes(const qcbc_event* ev, int* M, int* J, int* NR, int* MN, int* MM) {
  if (!ev) return fail(QCBC_EINVAL, "NULL event");
  if (M) *M = ev->het.M;
  if (J) *J = ev->het.J;
  if (NR) *NR = ev->het.NR;
  if (MN) *MN = ev->het.MN;
  if (MM) *MM = ev->het.MM;
  return QCBC_OK;
}

extern "C" int qcbc_het_export(const qcbc_event* ev, int* fgrid, double* freq, double* amp, double* phase, double* IP,
                               double* SL, double* lc, double* ls, double* aa, double* rc, double* rs, double* logLb) {
  if (!ev || !ev->het.buf) return fail(QCBC_EINVAL, "event has no heterodyne tables");
  HetData d = het_data(ev);
  const HetDev& h = ev->het;
  int nI = ev->g.nifo, M = h.M, NR = h.NR, J1 = h.J + 1;
  struct { double* dst; const double* src; size_t n; } parts[] = {
    {freq, d.freq, (size_t)M}, {amp, d.amp, (size_t)nI * M}, {phase, d.phase, (size_t)nI * M},
    {IP, d.IP, (size_t)NR * J1 * J1}, {SL, d.SL, (size_t)NR * nI * J1}, {lc, d.lc, (size_t)NR * nI * J1},
    {ls, d.ls, (size_t)NR * nI * J1}, {aa, d.aa, (size_t)nI * NR}, {rc, d.rc, (size_t)nI * NR},
    {rs, d.rs, (size_t)nI * NR}};
  for (auto& p : parts)
    if (p.dst) CU(cudaMemcpy(p.dst, p.src, p.n * sizeof(double), cudaMemcpyDeviceToHost));
  if (fgrid) memcpy(fgrid, h.fgrid.data(), sizeof(int) * M);
  if (logLb) *logLb = h.logLb;
  return QCBC_OK;
}

// Transpose of the inverse of the sampled Legendre basis, per region (QuickCBC.c:5232-5253).
static void invert_small(const double* A, double* Ainv, int n) {
  double W[4][8];
  for (int i = 0; i < n; i++)
    for (int j = 0; j < 2 * n; j++) W[i][j] = j < n ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int col = 0; col < n; col++) {
    int piv = col;
    for (int i = col + 1; i < n; i++)
      if (fabs(W[i][col]) > fabs(W[piv][col])) piv = i;
    if (piv != col)
      for (int j = 0; j < 2 * n; j++) std::swap(W[col][j], W[piv][j]);
    double dd = W[col][col];
    for (int j = 0; j < 2 * n; j++) W[col][j] /= dd;
    for (int i = 0; i < n; i++) {
      if (i == col) continue;
      double f = W[i][col];
      for (int j = 0; j < 2 * n; j++) W[i][j] -= f * W[col][j];
    }
  }
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) Ainv[i * n + j] = W[i][n + j];
}

static void gram_values(int J, int U, int n, double* P) {
  double c0 = 0.0, c1 = (double)(U - 2 * n), c2 = (double)U;
  double d0 = c2, d1 = c1 + c1, d2 = d0;
  P[0] = 1.0;
  if (J >= 1) P[1] = c1 / (double)U;
  for (int i = 1; i < J; i++) {
    d0 += 2.0; d2 -= 2.0; c0 += d0; c1 += d1; c2 += d2;
    P[i + 1] = (c1 * P[i] - c0 * P[i - 1]) / c2;
  }
}

extern "C" int qcbc_het_setup(qcbc_event* ev, const double* pref, const int* fgrid, int M, int MN, int MM, int J) {
  if (!ev || !pref || !fgrid) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->has_data) return fail(QCBC_EINVAL, "event has no data");
  const int nI = ev->g.nifo, N = ev->g.N, nh = N / 2;
  for (int i = 0; i < M; i++)
    if (fgrid[i] < 1 || fgrid[i] >= nh || (i && fgrid[i] <= fgrid[i - 1]))
      return fail(QCBC_EINVAL, "fgrid must increase strictly inside [1, N/2)");
  if (MN < 1 || MM > nh || MN > MM) return fail(QCBC_EINVAL, "bad [MN, MM) = [%d, %d)", MN, MM);
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = het_alloc(ev, M, J, MN, MM))) return rc;
  cudaStream_t s = w->stream;
  DeviceState& ds = g_dev[current_device()];
  // scratch: h [nifo][N], amp/phase [nifo][nh], RC/RS/AA [nifo][nh]
  size_t nA = (size_t)nI * N + 5 * (size_t)nI * nh;
  if ((rc = grow(w->d_a, w->c_a, nA))) return rc;
  if ((rc = grow(w->d_params, w->c_params, 11))) return rc;
  if ((rc = grow(w->d_recs, w->c_recs, 1))) return rc;
  if ((rc = grow(w->d_status, w->c_status, 1))) return rc;
  if ((rc = grow(w->d_b, w->c_b, (size_t)2 * kMaxIfo))) return rc;
  double* d_h = w->d_a;
  double* d_amp = d_h + (size_t)nI * N;
  double* d_ph = d_amp + (size_t)nI * nh;
  double* d_RC = d_ph + (size_t)nI * nh;
  double* d_RS = d_RC + (size_t)nI * nh;
  double* d_AA = d_RS + (size_t)nI * nh;
  CU(cudaMemcpyAsync(w->d_params, pref, 11 * sizeof(double), cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(ev->het.d_fgrid, fgrid, (size_t)M * sizeof(int), cudaMemcpyHostToDevice, s));
  // fulltemplates uses Tobs = 1/freq[1]; the canonical grid has freq[1] = 1/Tobs
  NetGeom gt = ev->g;
  gt.Tobs = 1.0 / (1.0 / ev->g.Tobs);
  launch_fulltemplates(w->d_params, gt, ds.qnm, ev->d_freq, w->d_recs, w->d_status, d_h, s);
  launch_fullphaseamp(w->d_params, ev->g, ds.qnm, ev->d_freq, nh, w->d_recs, w->d_status, d_amp, d_ph, s);
  launch_het_bins(d_h, d_amp, d_ph, ev->d_D, ev->d_S, nh + 1, N, nI, d_RC, d_RS, d_AA, s);
  HetData hd = het_data(ev);
  launch_het_region_sums(d_RC, d_RS, d_AA, ev->het.d_fgrid, M, J, nI, nh, (double*)hd.SL, (double*)hd.lc,
                         (double*)hd.ls, s);
  launch_nwip_pairs(d_h, ev->d_D, ev->d_S, nh + 1, N, nI, MN, MM, w->d_b, s);
  tls_launches += 8;
  CU(cudaGetLastError());
  // grid gathers and per-region small tables on the host (FP64)
  std::vector<double> ampb((size_t)nI * nh), phb((size_t)nI * nh), RC((size_t)nI * nh), RS((size_t)nI * nh),
      AA((size_t)nI * nh);
  double pairs[2 * kMaxIfo];
  CU(cudaMemcpyAsync(ampb.data(), d_amp, ampb.size() * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(phb.data(), d_ph, phb.size() * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(RC.data(), d_RC, RC.size() * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(RS.data(), d_RS, RS.size() * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(AA.data(), d_AA, AA.size() * 8, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(pairs, w->d_b, sizeof(double) * 2 * nI, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  HetDev& h = ev->het;
  int NR = h.NR, J1 = J + 1;
  std::vector<double> freq(M), amp((size_t)nI * M), ph((size_t)nI * M), IP((size_t)NR * J1 * J1), aa((size_t)nI * NR),
      rcv((size_t)nI * NR), rsv((size_t)nI * NR);
  for (int j = 0; j < M; j++) freq[j] = (double)fgrid[j] / ev->g.Tobs;
  for (int id = 0; id < nI; id++)
    for (int j = 0; j < M; j++) {
      amp[(size_t)id * M + j] = ampb[(size_t)id * nh + fgrid[j]];
      ph[(size_t)id * M + j] = phb[(size_t)id * nh + fgrid[j]];
    }
  for (int id = 0; id < nI; id++)
    for (int r = 0; r < NR; r++) {
      int k = fgrid[r * J];
      rcv[(size_t)id * NR + r] = RC[(size_t)id * nh + k];
      rsv[(size_t)id * NR + r] = RS[(size_t)id * nh + k];
      aa[(size_t)id * NR + r] = AA[(size_t)id * nh + k];
    }
  for (int r = 0; r < NR; r++) {
    int U = fgrid[(r + 1) * J] - fgrid[r * J];
    double PP[16], inv[16], P[4];
    for (int k = 0; k <= J; k++) {
      gram_values(J, U, fgrid[r * J + k] - fgrid[r * J], P);
      for (int a = 0; a <= J; a++) PP[a * J1 + k] = P[a];
    }
    invert_small(PP, inv, J1);
    for (int a = 0; a <= J; a++)
      for (int b = 0; b <= J; b++) IP[((size_t)r * J1 + a) * J1 + b] = inv[b * J1 + a];
  }
  double L = 0.0;
  for (int id = 0; id < nI; id++) L += pairs[2 * id + 1] + 0.5 * pairs[2 * id];
  h.logLb = L;
  h.fgrid.assign(fgrid, fgrid + M);
  memcpy(h.pref, pref, sizeof(h.pref));
  h.has_pref = true;
  CU(cudaMemcpy((void*)hd.freq, freq.data(), M * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.amp, amp.data(), amp.size() * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.phase, ph.data(), ph.size() * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.IP, IP.data(), IP.size() * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.aa, aa.data(), aa.size() * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.rc, rcv.data(), rcv.size() * 8, cudaMemcpyHostToDevice));
  CU(cudaMemcpy((void*)hd.rs, rsv.data(), rsv.size() * 8, cudaMemcpyHostToDevice));
  return QCBC_OK;
}

static int enqueue_het(Workspace* w, qcbc_event* ev, const double* d_params, int B, double* d_lnl, int prec,
                       cudaStream_t s, const NetGeom& g) {
  int rc;
  if ((rc = grow(w->d_recs, w->c_recs, (size_t)B))) return rc;
  if ((rc = grow(w->d_status, w->c_status, (size_t)B))) return rc;
  DeviceState& ds = g_dev[current_device()];
  const HetData hd = het_data(ev);
  // the setup's threads pull the heterodyne tables (and, for the mixed form, the bin tables at the
  // grid's bins) into L2 for the heterodyned launch
  SetupPrefetch pf;
  pf.buf = ev->het.buf;
  pf.bytes = het_doubles(ev->g.nifo, ev->het.M, ev->het.J) * sizeof(double);
  if (prec == QCBC_MIXED) {
    pf.bins = ev->het.d_fgrid;
    pf.nbins = ev->het.M;
    pf.tabA = hd.tabA;
    pf.tabB = hd.tabB;
    pf.tabC = hd.tabC;
    pf.tab_n = g_dev[ev->device].tab_n;
  }
  launch_setup(d_params, B, g, ds.qnm, w->d_recs, w->d_status, s, kModelFull, pf);
  launch_lnl_het(w->d_recs, w->d_status, B, g, hd, prec == QCBC_MIXED ? kMixed : kFP64, d_lnl, s);
  tls_launches += 2;
  CU(cudaGetLastError());
  return QCBC_OK;
}

extern "C" int qcbc_lnl_het(qcbc_event* ev, const double* params, int B, double* lnl, int precision) {
  if (!ev || !params || !lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->het.buf) return fail(QCBC_EINVAL, "event has no heterodyne tables");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = grow_host(w->h_params, w->ch_params, (size_t)B * 11))) return rc;
  if ((rc = grow_host(w->h_lnl, w->ch_lnl, (size_t)B))) return rc;
  memcpy(w->h_params, params, sizeof(double) * 11 * (size_t)B);
  cudaStream_t s = w->stream;
  // as for the full likelihood: the setup reads the parameters from, and the heterodyned kernel
  // writes lnL into, the pinned staging buffers through their mapped addresses (no copy calls)
  if ((rc = mapped_ptr(w->h_params, w->ch_params, w->m_params, w->m_params_of))) return rc;
  if ((rc = mapped_ptr(w->h_lnl, w->ch_lnl, w->m_lnl, w->m_lnl_of))) return rc;
  if ((rc = enqueue_het(w, ev, w->m_params, B, w->m_lnl, precision, s, ev->g))) return rc;
  CU(cudaStreamSynchronize(s));
  memcpy(lnl, w->h_lnl, sizeof(double) * B);
  // a set fails the setup exactly when its lnL is the rejected-sample value
  int bad = 0;
  for (int b = 0; b < B; b++) bad += lnl[b] == -1.0e20;
  if (bad) return fail(QCBC_EDOM, "%d of %d parameter sets outside the waveform domain (lnL=-1e20)", bad, B);
  return QCBC_OK;
}

extern "C" int qcbc_lnl_het_dev(qcbc_event* ev, const double* d_params, int B, double* d_lnl, int precision,
                                void* stream) {
  if (!ev || !d_params || !d_lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->het.buf) return fail(QCBC_EINVAL, "event has no heterodyne tables");
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : w->stream;
  return enqueue_het(w, ev, d_params, B, d_lnl, precision, s, ev->g);
}

// Waves of the sets in d_params (FP64 fullphaseamp on the heterodyne grid) into w->d_a:
// amplitude [nset][nifo][M] followed by phase [nset][nifo][M].
static int het_waves(Workspace* w, qcbc_event* ev, const double* d_params, int nset, cudaStream_t s, double** amp,
                     double** ph) {
  const size_t per = (size_t)nset * ev->g.nifo * ev->het.M;
  int rc;
  if ((rc = grow(w->d_recs, w->c_recs, (size_t)nset))) return rc;
  if ((rc = grow(w->d_status, w->c_status, (size_t)nset))) return rc;
  if ((rc = grow(w->d_a, w->c_a, 2 * per))) return rc;
  DeviceState& ds = g_dev[current_device()];
  launch_setup(d_params, nset, ev->g, ds.qnm, w->d_recs, w->d_status, s);
  launch_het_waves(w->d_recs, nset, ev->g, het_data(ev), w->d_a, w->d_a + per, s);
  tls_launches += 2;
  *amp = w->d_a;
  *ph = w->d_a + per;
  return QCBC_OK;
}

extern "C" int qcbc_het_diff(qcbc_event* ev, const double* params_a, const double* params_b, int B, double* out) {
  if (!ev || !params_a || !params_b || !out) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->het.buf) return fail(QCBC_EINVAL, "event has no heterodyne tables");
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = grow(w->d_params, w->c_params, (size_t)2 * B * 11))) return rc;
  if ((rc = grow_host(w->h_params, w->ch_params, (size_t)2 * B * 11))) return rc;
  if ((rc = grow(w->d_lnl, w->c_lnl, (size_t)B))) return rc;
  if ((rc = grow_host(w->h_lnl, w->ch_lnl, (size_t)B))) return rc;
  for (int p = 0; p < B; p++) {
    memcpy(w->h_params + (size_t)(2 * p) * 11, params_a + (size_t)p * 11, 11 * sizeof(double));
    memcpy(w->h_params + (size_t)(2 * p + 1) * 11, params_b + (size_t)p * 11, 11 * sizeof(double));
  }
  cudaStream_t s = w->stream;
  CU(cudaMemcpyAsync(w->d_params, w->h_params, sizeof(double) * 22 * (size_t)B, cudaMemcpyHostToDevice, s));
  double *amp, *ph;
  if ((rc = het_waves(w, ev, w->d_params, 2 * B, s, &amp, &ph))) return rc;
  launch_het_diff(amp, ph, B, ev->g, het_data(ev), w->d_lnl, s);
  tls_launches += 1;
  CU(cudaMemcpyAsync(w->h_lnl, w->d_lnl, sizeof(double) * B, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  memcpy(out, w->h_lnl, sizeof(double) * B);
  return QCBC_OK;
}

extern "C" int qcbc_het_fisher(qcbc_event* ev, const double* params, int B, double* fish) {
  constexpr int NP = 11, NSET = 2 * NP + 1;
  constexpr double eps = 1.0e-5;                 // QuickCBC.c:5489
  if (!ev || !params || !fish) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->het.buf) return fail(QCBC_EINVAL, "event has no heterodyne tables");
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  const size_t nset = (size_t)B * NSET;
  if ((rc = grow(w->d_params, w->c_params, nset * NP))) return rc;
  if ((rc = grow_host(w->h_params, w->ch_params, nset * NP))) return rc;
  if ((rc = grow(w->d_b, w->c_b, (size_t)B * NP * NP))) return rc;
  if ((rc = grow_host(w->h_b, w->ch_b, (size_t)B * NP * NP))) return rc;
  for (int b = 0; b < B; b++) {
    double* q = w->h_params + (size_t)b * NSET * NP;
    for (int k = 0; k < NSET; k++) memcpy(q + (size_t)k * NP, params + (size_t)b * NP, NP * sizeof(double));
    for (int i = 0; i < NP; i++) {
      q[(size_t)(1 + 2 * i) * NP + i] += eps;
      q[(size_t)(2 + 2 * i) * NP + i] -= eps;
    }
  }
  cudaStream_t s = w->stream;
  CU(cudaMemcpyAsync(w->d_params, w->h_params, sizeof(double) * nset * NP, cudaMemcpyHostToDevice, s));
  double *amp, *ph;
  if ((rc = het_waves(w, ev, w->d_params, (int)nset, s, &amp, &ph))) return rc;
  launch_het_fisher(amp, ph, B, ev->g, het_data(ev), eps, w->d_b, s);
  tls_launches += 1;
  CU(cudaMemcpyAsync(w->h_b, w->d_b, sizeof(double) * B * NP * NP, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  for (int b = 0; b < B; b++) {
    double* F = fish + (size_t)b * NP * NP;
    const double* G = w->h_b + (size_t)b * NP * NP;
    const double* p = params + (size_t)b * NP;
    if (fabs(p[2]) < 0.9999 && fabs(p[3]) < 0.9999) {
      for (int i = 0; i < NP; i++)
        for (int j = i; j < NP; j++) F[i * NP + j] = F[j * NP + i] = G[i * NP + j];
    } else {                                     // QuickCBC.c:5459-5469
      for (int i = 0; i < NP * NP; i++) F[i] = 0.0;
      for (int i = 0; i < NP; i++) F[i * NP + i] = 1.0e4;
    }
  }
  return QCBC_OK;
}

// ------------------------------------------------------------------ heterodyne grid search
static int run_het_space(const NetGeom& g, const double* h_S, int sn_stride, const double* h_freq, int N, double Tobs,
                         double fmin, double fmax, const double* params, const double* pmin, const double* pmax,
                         HetSpaceOut& out) {
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  HetSpaceIn in{g, g_dev[current_device()].qnm, h_S, sn_stride, h_freq, N, Tobs, fmin, fmax, w->stream};
  std::string err;
  rc = het_space_run(in, params, pmin, pmax, out, err);
  tls_launches += out.launches;
  if (rc == -3) return fail(QCBC_ECUDA, "%s", err.c_str());
  if (rc) return fail(QCBC_EINVAL, "%s", err.c_str());
  return QCBC_OK;
}

extern "C" int qcbc_het_space(qcbc_event* ev, const double* params, const double* pmin, const double* pmax, int* M,
                              int* MN, int* MM) {
  if (!ev || !params || !pmin || !pmax) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->has_data) return fail(QCBC_EINVAL, "event has no data");
  const int nI = ev->g.nifo, nh = ev->nh;
  std::vector<double> S((size_t)nI * (nh + 1)), freq((size_t)nh);
  CU(cudaMemcpy(S.data(), ev->d_S, S.size() * sizeof(double), cudaMemcpyDeviceToHost));
  CU(cudaMemcpy(freq.data(), ev->d_freq, freq.size() * sizeof(double), cudaMemcpyDeviceToHost));
  HetSpaceOut out;
  int rc = run_het_space(ev->g, S.data(), nh + 1, freq.data(), ev->g.N, ev->g.Tobs, ev->fmin, ev->fmax, params, pmin,
                         pmax, out);
  if (rc) return rc;
  ev->space_grid = out.fgrid;
  ev->space_MN = out.MN;
  ev->space_MM = out.MM;
  if (M) *M = out.M;
  if (MN) *MN = out.MN;
  if (MM) *MM = out.MM;
  return QCBC_OK;
}

extern "C" int qcbc_het_space_grid(const qcbc_event* ev, int* fgrid) {
  if (!ev || !fgrid) return fail(QCBC_EINVAL, "NULL argument");
  if (ev->space_grid.empty()) return fail(QCBC_EINVAL, "no grid: call qcbc_het_space first");
  memcpy(fgrid, ev->space_grid.data(), ev->space_grid.size() * sizeof(int));
  return QCBC_OK;
}

// ------------------------------------------------------------------ device memory helpers
extern "C" void* qcbc_device_alloc(long long bytes) {
  if (ensure_init()) return nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, (size_t)bytes) != cudaSuccess) { fail(QCBC_ENOMEM, "cudaMalloc %lld", bytes); return nullptr; }
  return p;
}
extern "C" int qcbc_device_free(void* p) { CU(cudaFree(p)); return QCBC_OK; }
extern "C" int qcbc_memcpy_h2d(void* dst, const void* src, long long bytes) {
  CU(cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyHostToDevice));
  return QCBC_OK;
}
extern "C" int qcbc_memcpy_d2h(void* dst, const void* src, long long bytes) {
  CU(cudaMemcpy(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost));
  return QCBC_OK;
}
extern "C" int qcbc_synchronize(void) { CU(cudaDeviceSynchronize()); return QCBC_OK; }

// ------------------------------------------------------------------ timing helpers
static int flush_l2(Workspace* w, cudaStream_t s) {
  const size_t bytes = (size_t)512 << 20;   // 512 MiB > 126 MB L2
  int rc = grow(w->d_flush, w->c_flush, bytes);
  if (rc) return rc;
  CU(cudaMemsetAsync(w->d_flush, 0x5a, bytes, s));
  return QCBC_OK;
}

extern "C" int qcbc_time_lnl_full(qcbc_event* ev, const double* d_params, int B, int precision, int iters,
                                  int flush, float* ms, float* kernel_ms) {
  if (!ev || !d_params || !ms || iters <= 0) return fail(QCBC_EINVAL, "bad argument");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = grow(w->d_lnl, w->c_lnl, (size_t)B))) return rc;
  cudaStream_t s = w->stream;
  for (int it = 0; it < iters; it++) {
    if (flush && (rc = flush_l2(w, s))) return rc;
    CU(cudaEventRecord(w->e0, s));
    // the kernel's own events only when its time is asked for: an event recorded between the setup
    // and the lnL kernel also ends the programmatic overlap of the two launches
    if ((rc = enqueue_full(w, ev, d_params, B, w->d_lnl, nullptr, precision, s, ev->g, kernel_ms ? w->e2 : nullptr,
                           kernel_ms ? w->e3 : nullptr)))
      return rc;
    CU(cudaEventRecord(w->e1, s));
    CU(cudaEventSynchronize(w->e1));
    CU(cudaEventElapsedTime(&ms[it], w->e0, w->e1));
    if (kernel_ms) CU(cudaEventElapsedTime(&kernel_ms[it], w->e2, w->e3));
  }
  return QCBC_OK;
}

extern "C" int qcbc_time_lnl_het(qcbc_event* ev, const double* d_params, int B, int precision, int iters, int flush,
                                 float* ms) {
  if (!ev || !d_params || !ms || iters <= 0) return fail(QCBC_EINVAL, "bad argument");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = grow(w->d_lnl, w->c_lnl, (size_t)B))) return rc;
  cudaStream_t s = w->stream;
  for (int it = 0; it < iters; it++) {
    if (flush && (rc = flush_l2(w, s))) return rc;
    CU(cudaEventRecord(w->e0, s));
    if ((rc = enqueue_het(w, ev, d_params, B, w->d_lnl, precision, s, ev->g))) return rc;
    CU(cudaEventRecord(w->e1, s));
    CU(cudaEventSynchronize(w->e1));
    CU(cudaEventElapsedTime(&ms[it], w->e0, w->e1));
  }
  return QCBC_OK;
}

// ================================================================== multi-event batches
struct MultiGraph {
  int Bcap = 0, items_cap = 0, tile_bins = 0, threads = 0, blocks = 0;
  int prec = 0;
  double* d_params = nullptr; int* d_eof = nullptr; PhdRec* d_recs = nullptr; int* d_status = nullptr;
  int* d_ntile = nullptr; int* d_off = nullptr; int* d_items = nullptr; int* d_counter = nullptr;
  double* d_part = nullptr; double* d_lnl = nullptr; double* d_rho = nullptr;
  double* h_params = nullptr; int* h_eof = nullptr; double* h_lnl = nullptr; double* h_rho = nullptr;
  int* h_status = nullptr;
  cudaGraphExec_t exec_full = nullptr, exec_dev = nullptr;
};

// Scratch of the heterodyned multi-event path (grown on demand).
struct HetMultiScratch {
  int cap = 0;
  double* d_params = nullptr; int* d_eof = nullptr; PhdRec* d_recs = nullptr; int* d_status = nullptr;
  int* d_ntile = nullptr; double* d_lnl = nullptr;
  double* h_params = nullptr; int* h_eof = nullptr; double* h_lnl = nullptr; int* h_status = nullptr;
};

static void free_het_scratch(HetMultiScratch& h) {
  cudaFree(h.d_params); cudaFree(h.d_eof); cudaFree(h.d_recs); cudaFree(h.d_status); cudaFree(h.d_ntile);
  cudaFree(h.d_lnl);
  cudaFreeHost(h.h_params); cudaFreeHost(h.h_eof); cudaFreeHost(h.h_lnl); cudaFreeHost(h.h_status);
  h = HetMultiScratch();
}

struct qcbc_batch {
  int device = 0;
  std::vector<qcbc_event*> events;
  EventDesc* d_events = nullptr;
  HetData* d_het = nullptr;            // per slot: the event's heterodyne tables (M = 0: none)
  std::vector<size_t> het_smem;        // per slot: shared memory of its heterodyned lnL
  HetMultiScratch hs;
  int nh_max = 0;
  int tile_bins = 2048, threads = 256;
  cudaStream_t stream = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  unsigned char* d_flush = nullptr;
  std::mutex mu;
  std::map<long long, MultiGraph*> graphs;
};

extern "C" int qcbc_batch_destroy(qcbc_batch* bt);

static void free_graph(MultiGraph* m) {
  if (!m) return;
  if (m->exec_full) cudaGraphExecDestroy(m->exec_full);
  if (m->exec_dev) cudaGraphExecDestroy(m->exec_dev);
  cudaFree(m->d_params); cudaFree(m->d_eof); cudaFree(m->d_recs); cudaFree(m->d_status); cudaFree(m->d_ntile);
  cudaFree(m->d_off); cudaFree(m->d_items); cudaFree(m->d_counter); cudaFree(m->d_part); cudaFree(m->d_lnl);
  cudaFree(m->d_rho);
  cudaFreeHost(m->h_params); cudaFreeHost(m->h_eof); cudaFreeHost(m->h_lnl); cudaFreeHost(m->h_rho);
  cudaFreeHost(m->h_status);
  delete m;
}

extern "C" qcbc_batch* qcbc_batch_create_slots(int capacity, int max_bins) {
  if (capacity <= 0 || max_bins <= 0) { fail(QCBC_EINVAL, "capacity and max_bins must be positive"); return nullptr; }
  if (ensure_init()) return nullptr;
  qcbc_batch* bt = new qcbc_batch();
  bt->device = current_device();
  bt->nh_max = max_bins;
  bt->events.assign(capacity, nullptr);
  bt->het_smem.assign(capacity, 0);
  std::vector<EventDesc> h(capacity);
  memset(h.data(), 0, sizeof(EventDesc) * capacity);   // nifo = 0 marks an empty slot
  std::vector<HetData> hh(capacity);
  memset(hh.data(), 0, sizeof(HetData) * capacity);
  if (cudaMalloc(&bt->d_events, sizeof(EventDesc) * capacity) != cudaSuccess ||
      cudaMemcpy(bt->d_events, h.data(), sizeof(EventDesc) * capacity, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMalloc(&bt->d_het, sizeof(HetData) * capacity) != cudaSuccess ||
      cudaMemcpy(bt->d_het, hh.data(), sizeof(HetData) * capacity, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaStreamCreateWithFlags(&bt->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&bt->e0) != cudaSuccess || cudaEventCreate(&bt->e1) != cudaSuccess) {
    fail(QCBC_ECUDA, "batch allocation failed");
    cudaFree(bt->d_events);
    cudaFree(bt->d_het);
    delete bt;
    return nullptr;
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    if (ensure_bin_tables(g_dev[bt->device], max_bins + 1)) { qcbc_batch_destroy(bt); return nullptr; }
  }
  return bt;
}

extern "C" int qcbc_batch_set_slot(qcbc_batch* bt, int slot, qcbc_event* ev) {
  if (!bt || slot < 0 || slot >= (int)bt->events.size()) return fail(QCBC_EINVAL, "bad batch or slot");
  EventDesc d;
  memset(&d, 0, sizeof(d));
  HetData hd;
  memset(&hd, 0, sizeof(hd));
  size_t smem = 0;
  if (ev) {
    if (!ev->has_data || ev->device != bt->device) return fail(QCBC_EINVAL, "event has no data or another device");
    if (ev->nh > bt->nh_max) return fail(QCBC_EINVAL, "event has %d bins, batch holds at most %d", ev->nh, bt->nh_max);
    d.g = ev->g;
    d.ev = event_data(ev);
    if (ev->het.buf) {               // tables as of now; set the slot again after a re-heterodyne
      hd = het_data(ev);
      smem = het_smem_bytes(ev->g, hd);
    }
  }
  std::lock_guard<std::mutex> lk(bt->mu);
  CU(cudaMemcpyAsync(bt->d_events + slot, &d, sizeof(d), cudaMemcpyHostToDevice, bt->stream));
  CU(cudaMemcpyAsync(bt->d_het + slot, &hd, sizeof(hd), cudaMemcpyHostToDevice, bt->stream));
  CU(cudaStreamSynchronize(bt->stream));
  bt->events[slot] = ev;
  bt->het_smem[slot] = smem;
  return QCBC_OK;
}

extern "C" qcbc_batch* qcbc_batch_create(qcbc_event* const* events, int n_events) {
  if (!events || n_events <= 0) { fail(QCBC_EINVAL, "no events"); return nullptr; }
  if (ensure_init()) return nullptr;
  int dev = current_device(), nh = 1;
  for (int i = 0; i < n_events; i++) {
    qcbc_event* ev = events[i];
    if (!ev || !ev->has_data || ev->device != dev) {
      fail(QCBC_EINVAL, "event %d is NULL, has no data or lives on another device", i);
      return nullptr;
    }
    nh = std::max(nh, ev->nh);
  }
  qcbc_batch* bt = qcbc_batch_create_slots(n_events, nh);
  if (!bt) return nullptr;
  for (int i = 0; i < n_events; i++)
    if (qcbc_batch_set_slot(bt, i, events[i])) { qcbc_batch_destroy(bt); return nullptr; }
  return bt;
}

extern "C" int qcbc_batch_destroy(qcbc_batch* bt) {
  if (!bt) return QCBC_OK;
  {
    std::lock_guard<std::mutex> lk(bt->mu);
    cudaStreamSynchronize(bt->stream);
    for (auto& kv : bt->graphs) free_graph(kv.second);
    bt->graphs.clear();
  }
  cudaFree(bt->d_events);
  cudaFree(bt->d_het);
  free_het_scratch(bt->hs);
  cudaFree(bt->d_flush);
  cudaEventDestroy(bt->e0);
  cudaEventDestroy(bt->e1);
  cudaStreamDestroy(bt->stream);
  delete bt;
  return QCBC_OK;
}

extern "C" int qcbc_batch_set_tiling(qcbc_batch* bt, int tile_bins, int threads) {
  if (!bt) return fail(QCBC_EINVAL, "NULL batch");
  if (tile_bins < 0 || (threads != 0 && threads != 64 && threads != 128 && threads != 256))
    return fail(QCBC_EINVAL, "tile_bins >= 0, threads in {64, 128, 256}");
  std::lock_guard<std::mutex> lk(bt->mu);
  if (tile_bins > 0) bt->tile_bins = tile_bins;
  if (threads > 0) bt->threads = threads;
  return QCBC_OK;
}

extern "C" int qcbc_batch_get_tiling(qcbc_batch* bt, int* tile_bins, int* threads) {
  if (!bt || !tile_bins || !threads) return fail(QCBC_EINVAL, "NULL argument");
  *tile_bins = bt->tile_bins;
  *threads = bt->threads;
  return QCBC_OK;
}

// Buffers + captured graphs for (Bcap, precision, tiling); caller holds bt->mu.
static int multi_graph(qcbc_batch* bt, int Bcap, int prec, MultiGraph** out) {
  long long key = ((long long)Bcap << 24) ^ ((long long)bt->tile_bins << 4) ^ ((long long)bt->threads << 1) ^ prec;
  auto it = bt->graphs.find(key);
  if (it != bt->graphs.end()) { *out = it->second; return QCBC_OK; }
  MultiGraph* m = new MultiGraph();
  m->Bcap = Bcap;
  m->prec = prec;
  m->tile_bins = bt->tile_bins;
  m->threads = bt->threads;
  long long tiles_per_set = (bt->nh_max + m->tile_bins - 1) / m->tile_bins;
  long long cap = (long long)Bcap * tiles_per_set;
  if (cap > (1LL << 30)) { delete m; return fail(QCBC_EINVAL, "work list too large"); }
  m->items_cap = (int)cap;
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, bt->device));
  Precision P = prec == QCBC_MIXED ? kMixed : kFP64;
  m->blocks = prop.multiProcessorCount * multi_blocks_per_sm(P, m->threads, m->tile_bins);
  bool ok = cudaMalloc(&m->d_params, sizeof(double) * 11 * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_eof, sizeof(int) * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_recs, sizeof(PhdRec) * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_status, sizeof(int) * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_ntile, sizeof(int) * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_off, sizeof(int) * (Bcap + 1)) == cudaSuccess &&
            cudaMalloc(&m->d_items, sizeof(int) * cap) == cudaSuccess &&
            cudaMalloc(&m->d_counter, sizeof(int)) == cudaSuccess &&
            cudaMalloc(&m->d_part, sizeof(double) * 2 * kMaxIfo * cap) == cudaSuccess &&
            cudaMalloc(&m->d_lnl, sizeof(double) * Bcap) == cudaSuccess &&
            cudaMalloc(&m->d_rho, sizeof(double) * kMaxIfo * Bcap) == cudaSuccess &&
            cudaMallocHost(&m->h_params, sizeof(double) * 11 * Bcap) == cudaSuccess &&
            cudaMallocHost(&m->h_eof, sizeof(int) * Bcap) == cudaSuccess &&
            cudaMallocHost(&m->h_lnl, sizeof(double) * Bcap) == cudaSuccess &&
            cudaMallocHost(&m->h_rho, sizeof(double) * kMaxIfo * Bcap) == cudaSuccess &&
            cudaMallocHost(&m->h_status, sizeof(int) * Bcap) == cudaSuccess;
  if (!ok) { free_graph(m); return fail(QCBC_ENOMEM, "multi-event buffers for B=%d", Bcap); }
  DeviceState& ds = g_dev[bt->device];
  cudaStream_t s = bt->stream;
  for (int with_copies = 1; with_copies >= 0; with_copies--) {
    cudaGraph_t graph = nullptr;
    CU(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    if (with_copies) {
      cudaMemcpyAsync(m->d_params, m->h_params, sizeof(double) * 11 * Bcap, cudaMemcpyHostToDevice, s);
      cudaMemcpyAsync(m->d_eof, m->h_eof, sizeof(int) * Bcap, cudaMemcpyHostToDevice, s);
    }
    cudaMemsetAsync(m->d_counter, 0, sizeof(int), s);
    launch_setup_multi(m->d_params, m->d_eof, Bcap, bt->d_events, (int)bt->events.size(), ds.qnm, m->tile_bins,
                       m->d_recs, m->d_status, m->d_ntile, s);
    launch_scan_expand(m->d_ntile, Bcap, m->d_off, m->d_items, m->items_cap, s);
    launch_lnl_multi(m->d_recs, bt->d_events, m->d_off, m->d_items, Bcap, m->tile_bins, m->items_cap, P, m->threads,
                     m->blocks, m->d_counter, m->d_part, s);
    launch_finalize_multi(m->d_part, m->d_recs, m->d_status, m->d_off, bt->d_events, Bcap, m->items_cap, P, m->d_lnl,
                          m->d_rho, s);
    if (with_copies) {
      cudaMemcpyAsync(m->h_lnl, m->d_lnl, sizeof(double) * Bcap, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(m->h_rho, m->d_rho, sizeof(double) * kMaxIfo * Bcap, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(m->h_status, m->d_status, sizeof(int) * Bcap, cudaMemcpyDeviceToHost, s);
    }
    cudaError_t e = cudaStreamEndCapture(s, &graph);
    if (e != cudaSuccess) { free_graph(m); return fail(QCBC_ECUDA, "graph capture: %s", cudaGetErrorString(e)); }
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) { free_graph(m); return fail(QCBC_ECUDA, "graph instantiate: %s", cudaGetErrorString(e)); }
    if (with_copies) m->exec_full = exec; else m->exec_dev = exec;
  }
  bt->graphs[key] = m;
  *out = m;
  return QCBC_OK;
}

static int bucket_of(int B) { return std::max(256, (B + 255) / 256 * 256); }

static int run_multi(qcbc_batch* bt, const int* event_of, const double* params, int B, double* lnl, double* rho,
                     int precision) {
  MultiGraph* m = nullptr;
  int rc = multi_graph(bt, bucket_of(B), precision, &m);
  if (rc) return rc;
  memcpy(m->h_params, params, sizeof(double) * 11 * (size_t)B);
  memcpy(m->h_eof, event_of, sizeof(int) * (size_t)B);
  for (int b = B; b < m->Bcap; b++) m->h_eof[b] = -1;      // padding sets: no event, no work
  CU(cudaGraphLaunch(m->exec_full, bt->stream));
  tls_launches += 4;
  CU(cudaStreamSynchronize(bt->stream));
  memcpy(lnl, m->h_lnl, sizeof(double) * (size_t)B);
  if (rho) memcpy(rho, m->h_rho, sizeof(double) * kMaxIfo * (size_t)B);
  int bad = 0;
  for (int b = 0; b < B; b++) bad += m->h_status[b] != 0;
  if (bad) return fail(QCBC_EDOM, "%d of %d parameter sets invalid (bad input or event index; lnL=-1e20)", bad, B);
  return QCBC_OK;
}

extern "C" int qcbc_lnl_multi(qcbc_batch* bt, const int* event_of, const double* params, int B, double* lnl,
                              double* rho, int precision) {
  if (!bt || !event_of || !params || !lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  int dev = current_device();
  if (dev != bt->device) return fail(QCBC_EINVAL, "batch lives on device %d, %d is current", bt->device, dev);
  std::lock_guard<std::mutex> lk(bt->mu);
  return run_multi(bt, event_of, params, B, lnl, rho, precision);
}

// Device-buffer forms for callers that keep parameter sets and results on the device (the
// service's device-resident sampler): no host copies, no synchronisation; work is ordered on
// `stream`.  Calls on one batch must not overlap (they share the batch's graph buffers).
extern "C" int qcbc_lnl_multi_dev(qcbc_batch* bt, const int* d_event_of, const double* d_params, int B, double* d_lnl,
                                  int precision, void* stream) {
  if (!bt || !d_event_of || !d_params || !d_lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  std::lock_guard<std::mutex> lk(bt->mu);
  MultiGraph* m = nullptr;
  int rc = multi_graph(bt, bucket_of(B), precision, &m);
  if (rc) return rc;
  cudaStream_t s = stream ? (cudaStream_t)stream : bt->stream;
  CU(cudaMemcpyAsync(m->d_params, d_params, sizeof(double) * 11 * (size_t)B, cudaMemcpyDeviceToDevice, s));
  CU(cudaMemcpyAsync(m->d_eof, d_event_of, sizeof(int) * (size_t)B, cudaMemcpyDeviceToDevice, s));
  if (m->Bcap > B) CU(cudaMemsetAsync(m->d_eof + B, 0xFF, sizeof(int) * (size_t)(m->Bcap - B), s));   // -1: no work
  CU(cudaGraphLaunch(m->exec_dev, s));
  CU(cudaMemcpyAsync(d_lnl, m->d_lnl, sizeof(double) * (size_t)B, cudaMemcpyDeviceToDevice, s));
  tls_launches += 4;
  return QCBC_OK;
}

extern "C" int qcbc_lnl_multi_het_dev(qcbc_batch* bt, const int* d_event_of, const double* d_params, int B,
                                      double* d_lnl, int precision, void* stream) {
  if (!bt || !d_event_of || !d_params || !d_lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  std::lock_guard<std::mutex> lk(bt->mu);
  HetMultiScratch& h = bt->hs;
  cudaStream_t s = stream ? (cudaStream_t)stream : bt->stream;
  if (B > h.cap) {                 // grown once; device memory only
    CU(cudaStreamSynchronize(s));
    free_het_scratch(h);
    const size_t n = (size_t)B;
    CU(cudaMalloc(&h.d_params, n * 11 * sizeof(double)));
    CU(cudaMalloc(&h.d_eof, n * sizeof(int)));
    CU(cudaMalloc(&h.d_recs, n * sizeof(PhdRec)));
    CU(cudaMalloc(&h.d_status, n * sizeof(int)));
    CU(cudaMalloc(&h.d_ntile, n * sizeof(int)));
    CU(cudaMalloc(&h.d_lnl, n * sizeof(double)));
    CU(cudaMallocHost(&h.h_params, n * 11 * sizeof(double)));
    CU(cudaMallocHost(&h.h_eof, n * sizeof(int)));
    CU(cudaMallocHost(&h.h_lnl, n * sizeof(double)));
    CU(cudaMallocHost(&h.h_status, n * sizeof(int)));
    h.cap = B;
  }
  size_t smem = 0;
  for (size_t k = 0; k < bt->het_smem.size(); k++) smem = std::max(smem, bt->het_smem[k]);
  DeviceState& ds = g_dev[current_device()];
  launch_setup_multi(d_params, d_event_of, B, bt->d_events, (int)bt->events.size(), ds.qnm, bt->tile_bins, h.d_recs,
                     h.d_status, h.d_ntile, s);
  launch_lnl_het_multi(h.d_recs, h.d_status, B, bt->d_events, bt->d_het, smem,
                       precision == QCBC_MIXED ? kMixed : kFP64, d_lnl, s);
  tls_launches += 2;
  CU(cudaGetLastError());
  return QCBC_OK;
}

extern "C" int qcbc_lnl_multi_het(qcbc_batch* bt, const int* event_of, const double* params, int B, double* lnl,
                                  int precision) {
  if (!bt || !event_of || !params || !lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B <= 0) return B == 0 ? QCBC_OK : fail(QCBC_EINVAL, "B < 0");
  std::lock_guard<std::mutex> lk(bt->mu);
  HetMultiScratch& h = bt->hs;
  if (B > h.cap) {
    free_het_scratch(h);
    const size_t n = (size_t)B;
    CU(cudaMalloc(&h.d_params, n * 11 * sizeof(double)));
    CU(cudaMalloc(&h.d_eof, n * sizeof(int)));
    CU(cudaMalloc(&h.d_recs, n * sizeof(PhdRec)));
    CU(cudaMalloc(&h.d_status, n * sizeof(int)));
    CU(cudaMalloc(&h.d_ntile, n * sizeof(int)));
    CU(cudaMalloc(&h.d_lnl, n * sizeof(double)));
    CU(cudaMallocHost(&h.h_params, n * 11 * sizeof(double)));
    CU(cudaMallocHost(&h.h_eof, n * sizeof(int)));
    CU(cudaMallocHost(&h.h_lnl, n * sizeof(double)));
    CU(cudaMallocHost(&h.h_status, n * sizeof(int)));
    h.cap = B;
  }
  size_t smem = 0;
  for (size_t k = 0; k < bt->het_smem.size(); k++) smem = std::max(smem, bt->het_smem[k]);
  memcpy(h.h_params, params, sizeof(double) * 11 * (size_t)B);
  memcpy(h.h_eof, event_of, sizeof(int) * (size_t)B);
  cudaStream_t s = bt->stream;
  CU(cudaMemcpyAsync(h.d_params, h.h_params, sizeof(double) * 11 * (size_t)B, cudaMemcpyHostToDevice, s));
  CU(cudaMemcpyAsync(h.d_eof, h.h_eof, sizeof(int) * (size_t)B, cudaMemcpyHostToDevice, s));
  DeviceState& ds = g_dev[current_device()];
  launch_setup_multi(h.d_params, h.d_eof, B, bt->d_events, (int)bt->events.size(), ds.qnm, bt->tile_bins, h.d_recs,
                     h.d_status, h.d_ntile, s);
  launch_lnl_het_multi(h.d_recs, h.d_status, B, bt->d_events, bt->d_het, smem,
                       precision == QCBC_MIXED ? kMixed : kFP64, h.d_lnl, s);
  tls_launches += 2;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(h.h_lnl, h.d_lnl, sizeof(double) * (size_t)B, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(h.h_status, h.d_status, sizeof(int) * (size_t)B, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  memcpy(lnl, h.h_lnl, sizeof(double) * (size_t)B);
  int bad = 0;
  for (int b = 0; b < B; b++) bad += h.h_status[b] != 0 || h.h_lnl[b] <= -1.0e19;
  if (bad) return fail(QCBC_EDOM, "%d of %d sets without a valid event, heterodyne tables or waveform (lnL=-1e20)",
                       bad, B);
  return QCBC_OK;
}

extern "C" int qcbc_time_lnl_multi(qcbc_batch* bt, int B, int precision, int iters, int flush, float* ms) {
  if (!bt || !ms || iters <= 0 || B <= 0) return fail(QCBC_EINVAL, "bad argument");
  std::lock_guard<std::mutex> lk(bt->mu);
  MultiGraph* m = nullptr;
  int rc = multi_graph(bt, bucket_of(B), precision, &m);
  if (rc) return rc;
  size_t fb = (size_t)512 << 20;
  if (flush && !bt->d_flush) CU(cudaMalloc(&bt->d_flush, fb));
  for (int it = 0; it < iters; it++) {
    if (flush) CU(cudaMemsetAsync(bt->d_flush, 0x5a, fb, bt->stream));
    CU(cudaEventRecord(bt->e0, bt->stream));
    CU(cudaGraphLaunch(m->exec_dev, bt->stream));
    tls_launches += 4;
    CU(cudaEventRecord(bt->e1, bt->stream));
    CU(cudaEventSynchronize(bt->e1));
    CU(cudaEventElapsedTime(&ms[it], bt->e0, bt->e1));
  }
  return QCBC_OK;
}

extern "C" int qcbc_batch_autotune(qcbc_batch* bt, const int* event_of, const double* params, int B, int precision) {
  if (!bt || !event_of || !params || B <= 0) return fail(QCBC_EINVAL, "bad argument");
  static const int cand[][2] = {{1024, 128}, {2048, 256}, {4096, 256}, {8192, 256}, {2048, 128}, {1024, 256}};
  std::vector<double> lnl(B);
  float best = 1e30f;
  int bt_tiles = bt->tile_bins, bt_threads = bt->threads;
  for (auto& c : cand) {
    {
      std::lock_guard<std::mutex> lk(bt->mu);
      bt->tile_bins = c[0];
      bt->threads = c[1];
      int rc = run_multi(bt, event_of, params, B, lnl.data(), nullptr, precision);
      if (rc && rc != QCBC_EDOM) return rc;
    }
    float ms[5];
    int rc = qcbc_time_lnl_multi(bt, B, precision, 5, 0, ms);
    if (rc) return rc;
    std::sort(ms, ms + 5);
    if (ms[2] < best) { best = ms[2]; bt_tiles = c[0]; bt_threads = c[1]; }
  }
  std::lock_guard<std::mutex> lk(bt->mu);
  bt->tile_bins = bt_tiles;
  bt->threads = bt_threads;
  return QCBC_OK;
}

// ================================================================== reference-signature drop-ins
static double g_band_fmin = 16.0, g_band_fmax = 1024.0;   // ConstCBC.h:33-34

extern "C" int qcbc_set_band(double fmin, double fmax) {
  if (!(fmin >= 0.0) || !(fmax > fmin)) return fail(QCBC_EINVAL, "bad band");
  g_band_fmin = fmin;
  g_band_fmax = fmax;
  return QCBC_OK;
}

struct BindKey {
  const void *net, *D, *SN;
  int N;
  bool operator<(const BindKey& o) const {
    if (net != o.net) return net < o.net;
    if (D != o.D) return D < o.D;
    if (SN != o.SN) return SN < o.SN;
    return N < o.N;
  }
};

// The events the reference-signature entry points build from the caller's rows are held through
// shared pointers.  A call copies the pointer under the cache's lock and keeps the event alive
// while its kernels run, so replacing a cache entry (new data, new heterodyne tables, a new
// binding) never frees or rewrites memory that a concurrent call reads: the old event is closed
// when its last user returns.  Host threads may therefore call these entry points concurrently,
// as the reference's OpenMP chains do (QuickCBC.c:2063-2067).
static inline void cpu_relax() {
#if defined(__x86_64__) || defined(__i386__)
  __builtin_ia32_pause();
#endif
}

// A spin lock for sections of a few instructions that many threads enter at once: a thread that
// finds std::mutex taken may sleep in the kernel and wake tens of microseconds later.
struct SpinLock {
  std::atomic<bool> taken{false};
  void lock() {
    while (taken.exchange(true, std::memory_order_acquire))
      while (taken.load(std::memory_order_relaxed)) cpu_relax();
  }
  void unlock() { taken.store(false, std::memory_order_release); }
};

struct MergeReq;
struct EventRef {
  qcbc_event* ev;
  // calls waiting to be merged into one launch on this event (merge_call)
  SpinLock mu;                       // guards queue
  std::vector<MergeReq*> queue;
  std::atomic<int> queued{0};        // queue.size(), readable without the lock
  std::atomic<bool> busy{false};     // a caller is leading a batch
  std::atomic<int> last_batch{1};    // size of the previous batch: how many callers to wait for
  explicit EventRef(qcbc_event* e) : ev(e) {}
  EventRef(const EventRef&) = delete;
  EventRef& operator=(const EventRef&) = delete;
  ~EventRef() { qcbc_event_close(ev); }
};
using EventPtr = std::shared_ptr<EventRef>;

// ------------------------------------------------------------------ merging of concurrent calls
// The reference's sampler calls log_likelihood_het (QuickCBC.c:2372) and, while it sets up,
// log_likelihood_full (QuickCBC.c:948-1016) one parameter set at a time from each of its OpenMP
// threads.  Calls that arrive for the same event while a launch for it is running are merged:
// the first caller that finds no launch running takes every waiting set of its kind into one
// batch, runs it and hands each caller its lnL; the others wait, and when their set was not in
// that batch one of them leads the next.  A lone caller runs its set alone with no wait.  A set's
// lnL does not depend on the batch it runs in (the heterodyned kernel gives each set its own
// warp; a merged full-likelihood batch keeps the tiling of a one-set call), so a merged call
// returns the bits of a lone one.
struct MergeReq {
  int kind = 0;                  // kMergeHet or kMergeFull
  int device = 0;                // the calling thread's device (its batch runs there)
  const double* params = nullptr;
  const NetGeom* g = nullptr;    // full likelihood: the call's geometry (sets merge only when equal)
  double lnl = -1.0e20;
  double rho[kMaxIfo] = {0.0, 0.0, 0.0};
  int rc = QCBC_OK;
  std::string err;
  std::atomic<int> done{0};      // set by the batch's leader once lnl, rho, rc and err are written
};
constexpr int kMergeHet = 0, kMergeFull = 1;
constexpr int kMergeMax = 256;

// One launch for the sets of `batch` (same kind, device and geometry), each caller's result and
// error written into its request.
static void merge_launch(qcbc_event* ev, const std::vector<MergeReq*>& batch) {
  const int B = (int)batch.size();
  const MergeReq& lead = *batch[0];
  static thread_local std::vector<double> P, L, R;
  P.resize((size_t)B * 11);
  L.assign((size_t)B, -1.0e20);
  R.assign((size_t)B * kMaxIfo, 0.0);
  for (int b = 0; b < B; b++) memcpy(&P[(size_t)b * 11], batch[b]->params, 11 * sizeof(double));
  int rc;
  if (lead.kind == kMergeHet) {
    rc = qcbc_lnl_het(ev, P.data(), B, L.data(), QCBC_FP64);
  } else {
    const FullLaunch one = choose_launch(ev, 1, QCBC_FP64);
    rc = run_full(ev, P.data(), B, L.data(), R.data(), QCBC_FP64, *lead.g, kModelFull, &one);
  }
  const std::string err = rc ? tls_err : std::string();
  const int nifo = lead.g ? lead.g->nifo : 0;
  for (int b = 0; b < B; b++) {
    MergeReq& r = *batch[b];
    r.lnl = L[b];
    for (int i = 0; i < nifo; i++) r.rho[i] = R[(size_t)b * nifo + i];
    if (rc == QCBC_EDOM) {
      // only the sets outside the waveform domain fail, as each would alone
      r.rc = L[b] == -1.0e20 ? QCBC_EDOM : QCBC_OK;
      if (r.rc) r.err = "1 of 1 parameter sets outside the waveform domain (lnL=-1e20)";
    } else {
      r.rc = rc;
      r.err = err;
    }
  }
}

// How long a new leader waits for as many callers as the previous batch had (the reference's
// chains call again a few microseconds after their previous results come back).
constexpr double kMergeGatherSeconds = 20e-6;

// Lead one batch: wait briefly for the callers of the previous batch, take this request and the
// waiting ones of the same kind, device and geometry, run them, publish each result.
static void merge_lead(EventRef& er, MergeReq& me) {
  const int target = std::min(er.last_batch.load(std::memory_order_relaxed), kMergeMax);
  if (target > 1 && er.queued.load(std::memory_order_acquire) < target) {
    const auto t_end = std::chrono::steady_clock::now() + std::chrono::duration<double>(kMergeGatherSeconds);
    while (er.queued.load(std::memory_order_acquire) < target && std::chrono::steady_clock::now() < t_end)
      cpu_relax();
  }
  static thread_local std::vector<MergeReq*> batch;
  batch.clear();
  batch.reserve(kMergeMax);
  batch.push_back(&me);
  {
    std::lock_guard<SpinLock> lk(er.mu);
    size_t keep = 0;                 // the requests left for a later batch stay in place
    for (size_t i = 0; i < er.queue.size(); i++) {
      MergeReq* r = er.queue[i];
      if (r == &me) continue;
      const bool same = r->kind == me.kind && r->device == me.device &&
                        (me.kind == kMergeHet || memcmp(r->g, me.g, sizeof(NetGeom)) == 0);
      if (same && (int)batch.size() < kMergeMax) batch.push_back(r);
      else er.queue[keep++] = r;
    }
    er.queue.resize(keep);
    er.queued.store((int)keep, std::memory_order_release);
  }
  try {
    merge_launch(er.ev, batch);
  } catch (...) {                    // an allocation failed: every caller of the batch gets the error
    for (MergeReq* r : batch) {
      r->lnl = -1.0e20;
      r->rc = QCBC_ENOMEM;
      r->err = "host allocation failed in a merged likelihood call";
    }
  }
  er.last_batch.store((int)batch.size(), std::memory_order_relaxed);
  // a follower may return (and its request go out of scope) as soon as its flag is set
  for (MergeReq* r : batch) r->done.store(1, std::memory_order_release);
  er.busy.store(false, std::memory_order_release);
}

// Run request `me` on event `er`, merged with the requests of other threads that arrive meanwhile.
// Waiting callers spin (a launch takes tens of microseconds, shorter than a sleep and wake-up),
// yielding the core after the first few thousand rounds.  Returns the request's status, with its
// error message in this thread's error slot.
static int merge_call(EventRef& er, MergeReq& me) {
  {
    std::lock_guard<SpinLock> lk(er.mu);
    er.queue.push_back(&me);
    er.queued.store((int)er.queue.size(), std::memory_order_release);
  }
  for (unsigned spin = 0;; spin++) {
    if (me.done.load(std::memory_order_acquire)) break;
    bool idle = false;
    if (!er.busy.load(std::memory_order_relaxed) &&
        er.busy.compare_exchange_strong(idle, true, std::memory_order_acq_rel)) {
      // the previous leader may have taken and finished this request before releasing the flag
      if (me.done.load(std::memory_order_acquire)) {
        er.busy.store(false, std::memory_order_release);
        break;
      }
      merge_lead(er, me);
      break;
    }
    if (spin < 4096) cpu_relax();
    else std::this_thread::yield();
  }
  if (me.rc) tls_err = me.err;
  return me.rc;
}

// The caches below live until the process exits and are never destroyed: destroying them would
// close events after the CUDA runtime has shut down.
static std::map<BindKey, EventPtr>& g_bound = *new std::map<BindKey, EventPtr>();   // qcbc_bind_data
static std::mutex g_bind_mu;

static qcbc_event* open_from_rows(struct Net* net, double** D, double** SN, int N, double Tobs) {
  if (check_geom(net->Nifo, net->labels, Tobs, N)) return nullptr;
  qcbc_event* ev = new qcbc_event();
  ev->device = current_device();
  ev->fmin = g_band_fmin;
  ev->fmax = g_band_fmax;
  fill_geom(ev->g, net->Nifo, net->labels, Tobs, net->GMST, N, g_band_fmin, g_band_fmax);
  std::vector<const double*> Dr(net->Nifo), Sr(net->Nifo);
  for (int i = 0; i < net->Nifo; i++) { Dr[i] = D[i]; Sr[i] = SN[i]; }
  if (event_upload(ev, Dr.data(), Sr.data())) { event_free_device(ev); delete ev; return nullptr; }
  return ev;
}

// Unbound calls: events cached by the rows' addresses together with a host copy of the rows they
// were built from.  A call compares the caller's rows with that copy (the reference rewrites SN in
// place when it redraws the PSD, QuickCBC.c:1994-2010) and reuses the event only when every value
// is the same, so results never depend on stale data; anything else builds a new event.  At most
// kRowsCacheMax entries, least recently used evicted.
struct RowsSnap {
  int nifo = 0, N = 0;
  double Tobs = 0.0, GMST = 0.0, fmin = 0.0, fmax = 0.0;
  std::vector<int> labels;
  std::vector<double> D, S;     // [nifo][N], [nifo][N/2]
  EventPtr ev;
};
struct RowsEntry {
  std::shared_ptr<const RowsSnap> snap;
  unsigned long long used = 0;
};
static std::map<BindKey, RowsEntry>& g_rows = *new std::map<BindKey, RowsEntry>();
static unsigned long long g_rows_tick = 0;
constexpr size_t kRowsCacheMax = 16;

static bool rows_match(const RowsSnap& r, struct Net* net, double** D, double** SN, int N, double Tobs) {
  if (r.nifo != net->Nifo || r.N != N || r.Tobs != Tobs || r.GMST != net->GMST || r.fmin != g_band_fmin ||
      r.fmax != g_band_fmax)
    return false;
  const size_t nh = (size_t)N / 2;
  for (int i = 0; i < r.nifo; i++) {
    if (r.labels[i] != net->labels[i]) return false;
    if (memcmp(&r.D[(size_t)i * N], D[i], sizeof(double) * (size_t)N) != 0) return false;
    if (memcmp(&r.S[(size_t)i * nh], SN[i], sizeof(double) * nh) != 0) return false;
  }
  return true;
}

// The event holding (D, SN) for a reference-signature call: the bound one, else a cached one whose
// rows equal the caller's, else a new one (which enters the cache).
// The bound event this thread last used, valid while no binding was made or dropped since
// (g_bind_gen): a chain calling with the same registered arrays skips the cache's lock.
struct TlsBound {
  BindKey key{nullptr, nullptr, nullptr, 0};
  unsigned long long gen = 0;
  std::weak_ptr<EventRef> ev;
};
static thread_local TlsBound tls_bound;
static std::atomic<unsigned long long> g_bind_gen{1};

static EventPtr data_event(struct Net* net, double** D, double** SN, int N, double Tobs) {
  const BindKey key{net, D, SN, N};
  TlsBound& t = tls_bound;
  const unsigned long long gen = g_bind_gen.load(std::memory_order_acquire);
  if (t.gen == gen && !(t.key < key) && !(key < t.key))
    if (EventPtr ev = t.ev.lock()) return ev;
  {
    std::lock_guard<std::mutex> lk(g_bind_mu);
    auto it = g_bound.find(key);
    if (it != g_bound.end()) {
      t.key = key;
      t.gen = gen;
      t.ev = it->second;
      return it->second;
    }
  }
  std::shared_ptr<const RowsSnap> snap;
  {
    std::lock_guard<std::mutex> lk(g_bind_mu);
    auto it = g_rows.find(key);
    if (it != g_rows.end()) {
      it->second.used = ++g_rows_tick;
      snap = it->second.snap;
    }
  }
  if (snap && rows_match(*snap, net, D, SN, N, Tobs)) return snap->ev;   // compared outside the lock
  qcbc_event* ev = open_from_rows(net, D, SN, N, Tobs);
  if (!ev) return nullptr;
  auto fresh = std::make_shared<RowsSnap>();
  fresh->ev = std::make_shared<EventRef>(ev);
  fresh->nifo = net->Nifo;
  fresh->N = N;
  fresh->Tobs = Tobs;
  fresh->GMST = net->GMST;
  fresh->fmin = g_band_fmin;
  fresh->fmax = g_band_fmax;
  fresh->labels.assign(net->labels, net->labels + net->Nifo);
  const size_t nh = (size_t)N / 2;
  fresh->D.resize((size_t)net->Nifo * N);
  fresh->S.resize((size_t)net->Nifo * nh);
  for (int i = 0; i < net->Nifo; i++) {
    memcpy(&fresh->D[(size_t)i * N], D[i], sizeof(double) * (size_t)N);
    memcpy(&fresh->S[(size_t)i * nh], SN[i], sizeof(double) * nh);
  }
  EventPtr out = fresh->ev;
  std::lock_guard<std::mutex> lk(g_bind_mu);
  g_rows[key] = RowsEntry{std::move(fresh), ++g_rows_tick};
  while (g_rows.size() > kRowsCacheMax) {
    auto lru = g_rows.begin();
    for (auto it = g_rows.begin(); it != g_rows.end(); ++it)
      if (it->second.used < lru->second.used) lru = it;
    g_rows.erase(lru);
  }
  return out;
}

// The reference builds freq[i] = i/Tobs with freq[0] = 1/Tobs (QuickCBC.c:419-420) and the kernels
// use that grid; another grid is refused rather than silently replaced.
static bool reference_grid(const RealVector* freq, int N, double Tobs, int imin, int imax) {
  const size_t nh = (size_t)N / 2;
  if (!freq || !freq->data || freq->length < nh) return false;
  const size_t probe[] = {1, (size_t)std::max(imin, 1), (size_t)std::max(imax - 1, 1), nh - 1};
  for (size_t i : probe) {
    if (i >= nh) continue;
    const double want = (double)i / Tobs;
    if (!(fabs(freq->data[i] - want) <= 1e-12 * want)) return false;
  }
  return true;
}

extern "C" int qcbc_bind_data(struct Net* net, double** D, double** SN, int N, double Tobs) {
  if (!net || !D || !SN) return fail(QCBC_EINVAL, "NULL argument");
  int rc = ensure_init();
  if (rc) return rc;
  qcbc_event* ev = open_from_rows(net, D, SN, N, Tobs);
  if (!ev) return QCBC_ENOMEM;
  EventPtr p = std::make_shared<EventRef>(ev);
  std::lock_guard<std::mutex> lk(g_bind_mu);
  g_bound[BindKey{net, D, SN, N}] = std::move(p);    // a replaced binding closes after its last user
  g_bind_gen.fetch_add(1, std::memory_order_acq_rel);
  return QCBC_OK;
}

extern "C" int qcbc_unbind_all(void) {
  std::lock_guard<std::mutex> lk(g_bind_mu);
  g_bound.clear();
  g_rows.clear();
  g_bind_gen.fetch_add(1, std::memory_order_acq_rel);
  return QCBC_OK;
}

// Upload a caller frequency vector into thread scratch (legacy paths read freq[i] like the reference).
static int stage_freq(Workspace* w, const RealVector* freq, size_t n, double** d_out) {
  if (!freq || !freq->data || freq->length < n) return fail(QCBC_EINVAL, "freq shorter than needed (%zu)", n);
  int rc = grow(w->d_c, w->c_c, n);
  if (rc) return rc;
  CU(cudaMemcpyAsync(w->d_c, freq->data, n * sizeof(double), cudaMemcpyHostToDevice, w->stream));
  *d_out = w->d_c;
  return QCBC_OK;
}

extern "C" double log_likelihood_full(struct Net* net, double** D, double* params, RealVector* freq, double** SN,
                                      double* rho, int N, double Tobs) {
  if (!net || !D || !SN || !params) { fail(QCBC_EINVAL, "NULL argument"); return -1.0e20; }
  if (ensure_init()) return -1.0e20;
  EventPtr ep = data_event(net, D, SN, N, Tobs);
  if (!ep) return -1.0e20;
  qcbc_event* ev = ep->ev;
  NetGeom g = ev->g;
  fill_geom(g, net->Nifo, net->labels, Tobs, net->GMST, N, ev->fmin, ev->fmax);
  if (!reference_grid(freq, N, Tobs, g.imin, g.imax)) {
    fail(QCBC_EINVAL, "freq is not the reference grid i/Tobs (QuickCBC.c:419-420)");
    return -1.0e20;
  }
  MergeReq me;
  me.kind = kMergeFull;
  me.device = current_device();
  me.params = params;
  me.g = &g;
  const int rc = merge_call(*ep, me);
  if (rho && rc == QCBC_OK)
    for (int i = 0; i < net->Nifo; i++) rho[i] = me.rho[i];
  return rc == QCBC_OK ? me.lnl : -1.0e20;
}

// Heterodyne tables of the reference's struct Het, uploaded on first use and again when the
// struct's tables change (another IP array, M or logLb: heterodyne() rebuilt them).  Entries are
// keyed by the struct's address and evicted least recently used beyond kHetCacheMax, so the tables
// of structs the caller has freed do not stay on the device for the life of the process.
struct HetCacheEntry {
  EventPtr ev;
  const void* ip = nullptr;
  int M = 0;
  double logLb = 0.0;
  unsigned long long used = 0;
};
static std::map<const void*, HetCacheEntry>& g_het_cache = *new std::map<const void*, HetCacheEntry>();
static std::mutex g_het_mu;
static unsigned long long g_het_tick = 0;
constexpr size_t kHetCacheMax = 32;

// The last struct Het this thread used and a weak reference to its event: a chain that calls with
// the same tables again skips the cache's lock (twelve chains calling at once contend for it).
// Valid while the struct's IP, M and logLb are unchanged and the cache still holds the event.
struct TlsHet {
  const void* het = nullptr;
  const void* ip = nullptr;
  int M = 0;
  double logLb = 0.0;
  unsigned long long gen = 0;
  std::weak_ptr<EventRef> ev;
};
static thread_local TlsHet tls_het;
// bumped whenever the cache drops or replaces an entry: thread-local references older than that
// go back through the cache
static std::atomic<unsigned long long> g_het_gen{1};

static EventPtr het_event_locked(struct Net* net, struct Het* het);

static EventPtr het_event_for(struct Net* net, struct Het* het) {
  TlsHet& t = tls_het;
  const unsigned long long gen = g_het_gen.load(std::memory_order_acquire);
  if (t.gen == gen && t.het == het && t.ip == (const void*)het->IP && t.M == het->M && t.logLb == het->logLb)
    if (EventPtr ev = t.ev.lock()) return ev;
  EventPtr ev = het_event_locked(net, het);
  if (ev) {
    t.gen = gen;
    t.het = het;
    t.ip = het->IP;
    t.M = het->M;
    t.logLb = het->logLb;
    t.ev = ev;
  }
  return ev;
}

static EventPtr het_event_locked(struct Net* net, struct Het* het) {
  std::lock_guard<std::mutex> lk(g_het_mu);
  HetCacheEntry& e = g_het_cache[het];
  e.used = ++g_het_tick;
  if (e.ev && e.ip == (const void*)het->IP && e.M == het->M && e.logLb == het->logLb) return e.ev;
  int nI = net->Nifo, M = het->M, J = het->J, NR = het->NR, J1 = J + 1;
  if (J < 1 || NR != (M - 1) / J) { fail(QCBC_EINVAL, "het NR inconsistent with M, J"); return nullptr; }
  // a new event every time the tables change: calls still running on the old one keep it
  qcbc_event* raw = new qcbc_event();
  raw->device = current_device();
  EventPtr ev = std::make_shared<EventRef>(raw);
  fill_geom(raw->g, nI, net->labels, net->Tobs, net->GMST, 2 * het->M, 0.0, 1.0);
  std::vector<double> amp((size_t)nI * M), ph((size_t)nI * M), IP((size_t)NR * J1 * J1), SL((size_t)NR * nI * J1),
      lc(SL.size()), ls(SL.size()), aa((size_t)nI * NR), rcv(aa.size()), rsv(aa.size());
  for (int id = 0; id < nI; id++)
    for (int j = 0; j < M; j++) { amp[(size_t)id * M + j] = het->amp[id][j]; ph[(size_t)id * M + j] = het->phase[id][j]; }
  for (int r = 0; r < NR; r++) {
    for (int a = 0; a < J1; a++)
      for (int b = 0; b < J1; b++) IP[((size_t)r * J1 + a) * J1 + b] = het->IP[r][a][b];
    for (int id = 0; id < nI; id++)
      for (int a = 0; a < J1; a++) {
        size_t o = ((size_t)r * nI + id) * J1 + a;
        SL[o] = het->SL[r][id][a]; lc[o] = het->lc[r][id][a]; ls[o] = het->ls[r][id][a];
      }
  }
  for (int id = 0; id < nI; id++)
    for (int r = 0; r < NR; r++) {
      aa[(size_t)id * NR + r] = het->aa[id][r]; rcv[(size_t)id * NR + r] = het->rc[id][r];
      rsv[(size_t)id * NR + r] = het->rs[id][r];
    }
  qcbc_het_tables t{M, het->MN, het->MM, J, NR, het->logLb, het->fgrid, het->freq->data, amp.data(), ph.data(),
                    IP.data(), SL.data(), lc.data(), ls.data(), aa.data(), rcv.data(), rsv.data()};
  if (qcbc_het_set(raw, &t) != QCBC_OK) return nullptr;
  if (e.ev) g_het_gen.fetch_add(1, std::memory_order_acq_rel);   // replaces an entry's tables
  e.ev = ev;
  e.ip = het->IP;
  e.M = het->M;
  e.logLb = het->logLb;
  while (g_het_cache.size() > kHetCacheMax) {
    auto lru = g_het_cache.begin();
    for (auto it = g_het_cache.begin(); it != g_het_cache.end(); ++it)
      if (it->second.used < lru->second.used) lru = it;
    g_het_cache.erase(lru);
    g_het_gen.fetch_add(1, std::memory_order_acq_rel);
  }
  return ev;
}

// Forget the device copy of a struct Het's tables (e.g. before freehet); optional, since entries
// are also evicted when the cache is full.
extern "C" int qcbc_het_forget(const struct Het* het) {
  std::lock_guard<std::mutex> lk(g_het_mu);
  g_het_cache.erase(het);
  g_het_gen.fetch_add(1, std::memory_order_acq_rel);
  return QCBC_OK;
}

extern "C" double log_likelihood_het(struct Net* net, struct Het* het, double* params, double Tobs) {
  (void)Tobs;   // fullphaseamp inside the reference's het lnL uses net->Tobs (QuickCBC.c:3797)
  if (!net || !het || !params) { fail(QCBC_EINVAL, "NULL argument"); return -1.0e20; }
  if (ensure_init()) return -1.0e20;
  EventPtr ev = het_event_for(net, het);
  if (!ev) return -1.0e20;
  MergeReq me;
  me.kind = kMergeHet;
  me.device = current_device();
  me.params = params;
  const int rc = merge_call(*ev, me);
  return rc == QCBC_OK ? me.lnl : -1.0e20;
}

extern "C" int qcbc_time_dropin(int which, struct Net* net, struct Het* het, double** D, RealVector* freq,
                                double** SN, int N, double Tobs, const double* params, int nsets, int calls,
                                int nthreads, double* seconds, double* lnl_last) {
  if (!net || !params || !seconds || (which == 1 && !het) || (which == 0 && (!D || !SN || !freq)))
    return fail(QCBC_EINVAL, "NULL argument");
  if (which != 0 && which != 1) return fail(QCBC_EINVAL, "which=%d (0 full, 1 heterodyned)", which);
  if (nsets < 1 || calls < 1 || nthreads < 1 || nthreads > 256) return fail(QCBC_EINVAL, "nsets, calls, nthreads");
  int rc = ensure_init();
  if (rc) return rc;
  const int dev = current_device();
  std::atomic<int> ready{0}, bad{0};
  std::atomic<bool> go{false};
  std::vector<double> last((size_t)nthreads, -1.0e20);
  auto work = [&](int t) {
    cudaSetDevice(dev);
    double p[11], rho[kMaxIfo + 1];
    auto call = [&](int k) {
      memcpy(p, params + (size_t)((7 * t + k) % nsets) * 11, sizeof(p));
      return which ? log_likelihood_het(net, het, p, Tobs) : log_likelihood_full(net, D, p, freq, SN, rho, N, Tobs);
    };
    for (int k = 0; k < 4; k++) call(k);
    ready.fetch_add(1);
    while (!go.load(std::memory_order_acquire)) std::this_thread::yield();
    double x = -1.0e20;
    for (int k = 0; k < calls; k++) x = call(k);
    last[(size_t)t] = x;
    if (x == -1.0e20) bad.fetch_add(1);
  };
  std::vector<std::thread> ts;
  for (int t = 0; t < nthreads; t++) ts.emplace_back(work, t);
  while (ready.load() < nthreads) std::this_thread::yield();
  const auto t0 = std::chrono::steady_clock::now();
  go.store(true, std::memory_order_release);
  for (auto& th : ts) th.join();
  *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (lnl_last)
    for (int t = 0; t < nthreads; t++) lnl_last[t] = last[(size_t)t];
  return bad.load() ? fail(QCBC_EDOM, "%d threads ended on lnL=-1e20", bad.load()) : QCBC_OK;
}

// Allocation helpers with the reference's layout (Utilities.c:2941-3015): N+1 rows of M+1 entries.
static double** alloc_matrix(int N, int M) {
  double** m = (double**)malloc((size_t)(N + 1) * sizeof(double*));
  for (int i = 0; i < N + 1; i++) m[i] = (double*)malloc((size_t)(M + 1) * sizeof(double));
  return m;
}
static double*** alloc_tensor(int N, int M, int L) {
  double*** t = (double***)malloc((size_t)(N + 1) * sizeof(double**));
  for (int i = 0; i < N + 1; i++) t[i] = alloc_matrix(M, L);
  return t;
}

extern "C" void heterodyne(struct Net* net, struct Het* het, double** D, double* params, RealVector* freq,
                           double** SN, int N, double Tobs) {
  (void)freq;
  if (!net || !het || !D || !SN || !params || !het->fgrid) { fail(QCBC_EINVAL, "NULL argument"); return; }
  if (ensure_init()) return;
  qcbc_event* ev = open_from_rows(net, D, SN, N, Tobs);
  if (!ev) return;
  int M = het->M, J = het->J, NR = het->NR, nI = net->Nifo, J1 = J + 1;
  if (qcbc_het_setup(ev, params, het->fgrid, M, het->MN, het->MM, J) != QCBC_OK) { qcbc_event_close(ev); return; }
  std::vector<double> fr(M), amp((size_t)nI * M), ph((size_t)nI * M), IP((size_t)NR * J1 * J1),
      SL((size_t)NR * nI * J1), lc(SL.size()), ls(SL.size()), aa((size_t)nI * NR), rcv(aa.size()), rsv(aa.size());
  double logLb = 0.0;
  qcbc_het_export(ev, nullptr, fr.data(), amp.data(), ph.data(), IP.data(), SL.data(), lc.data(), ls.data(), aa.data(),
                  rcv.data(), rsv.data(), &logLb);
  qcbc_event_close(ev);
  het->IP = alloc_tensor(NR, J + 1, J + 1);
  het->SL = alloc_tensor(NR, nI, J + 1);
  het->amp = alloc_matrix(nI, M);
  het->phase = alloc_matrix(nI, M);
  het->rc = alloc_matrix(nI, NR);
  het->rs = alloc_matrix(nI, NR);
  het->aa = alloc_matrix(nI, NR);
  het->lc = alloc_tensor(NR, nI, J + 1);
  het->ls = alloc_tensor(NR, nI, J + 1);
  het->pref = (double*)malloc(12 * sizeof(double));
  for (int k = 0; k < 11; k++) het->pref[k] = params[k];
  for (int id = 0; id < nI; id++)
    for (int j = 0; j < M; j++) { het->amp[id][j] = amp[(size_t)id * M + j]; het->phase[id][j] = ph[(size_t)id * M + j]; }
  for (int r = 0; r < NR; r++) {
    for (int a = 0; a < J1; a++)
      for (int b = 0; b < J1; b++) het->IP[r][a][b] = IP[((size_t)r * J1 + a) * J1 + b];
    for (int id = 0; id < nI; id++)
      for (int a = 0; a < J1; a++) {
        size_t o = ((size_t)r * nI + id) * J1 + a;
        het->SL[r][id][a] = SL[o]; het->lc[r][id][a] = lc[o]; het->ls[r][id][a] = ls[o];
      }
  }
  for (int id = 0; id < nI; id++)
    for (int r = 0; r < NR; r++) {
      het->aa[id][r] = aa[(size_t)id * NR + r]; het->rc[id][r] = rcv[(size_t)id * NR + r];
      het->rs[id][r] = rsv[(size_t)id * NR + r];
    }
  het->logLb = logLb;
}

extern "C" void fulltemplates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  if (!net || !hwave || !freq || !params) { fail(QCBC_EINVAL, "NULL argument"); return; }
  Workspace* w;
  if (workspace(w)) return;
  if (check_geom(net->Nifo, net->labels, 1.0, N)) return;
  cudaStream_t s = w->stream;
  double* d_freq;
  if (stage_freq(w, freq, (size_t)N / 2, &d_freq)) return;
  double Tobs = 1.0 / freq->data[1];   // QuickCBC.c:3703
  NetGeom g;
  fill_geom(g, net->Nifo, net->labels, Tobs, net->GMST, N, 0.0, 1.0);
  int nI = net->Nifo;
  if (grow(w->d_a, w->c_a, (size_t)nI * N) || grow(w->d_params, w->c_params, 11) || grow(w->d_recs, w->c_recs, 1) ||
      grow(w->d_status, w->c_status, 1) || grow_host(w->h_a, w->ch_a, (size_t)nI * N))
    return;
  if (cudaMemcpyAsync(w->d_params, params, 11 * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess) return;
  DeviceState& ds = g_dev[current_device()];
  launch_fulltemplates(w->d_params, g, ds.qnm, d_freq, w->d_recs, w->d_status, w->d_a, s);
  tls_launches += 2;
  cudaMemcpyAsync(w->h_a, w->d_a, sizeof(double) * nI * N, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "fulltemplates failed"); return; }
  for (int id = 0; id < nI; id++) memcpy(hwave[id], w->h_a + (size_t)id * N, sizeof(double) * N);
}

extern "C" void fullphaseamp(struct Net* net, double** amp, double** phase, RealVector* freq, double* params, int N) {
  if (!net || !amp || !phase || !freq || !params) { fail(QCBC_EINVAL, "NULL argument"); return; }
  Workspace* w;
  if (workspace(w)) return;
  if (check_geom(net->Nifo, net->labels, net->Tobs, N)) return;
  cudaStream_t s = w->stream;
  int n = N / 2, nI = net->Nifo;
  double* d_freq;
  if (stage_freq(w, freq, (size_t)n, &d_freq)) return;
  NetGeom g;
  fill_geom(g, nI, net->labels, net->Tobs, net->GMST, N, 0.0, 1.0);
  if (grow(w->d_a, w->c_a, (size_t)2 * nI * n) || grow(w->d_params, w->c_params, 11) || grow(w->d_recs, w->c_recs, 1) ||
      grow(w->d_status, w->c_status, 1) || grow_host(w->h_a, w->ch_a, (size_t)2 * nI * n))
    return;
  cudaMemcpyAsync(w->d_params, params, 11 * sizeof(double), cudaMemcpyHostToDevice, s);
  DeviceState& ds = g_dev[current_device()];
  launch_fullphaseamp(w->d_params, g, ds.qnm, d_freq, n, w->d_recs, w->d_status, w->d_a, w->d_a + (size_t)nI * n, s);
  tls_launches += 2;
  cudaMemcpyAsync(w->h_a, w->d_a, sizeof(double) * 2 * nI * n, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "fullphaseamp failed"); return; }
  for (int id = 0; id < nI; id++) {
    memcpy(amp[id], w->h_a + (size_t)id * n, sizeof(double) * n);
    memcpy(phase[id], w->h_a + (size_t)(nI + id) * n, sizeof(double) * n);
  }
}

extern "C" int IMRPhenomDGenerateh22FDAmpPhase(AmpPhaseFDWaveform** h22, RealVector* freq, const double phi0,
                                               const double fRef_in, const double m1_SI, const double m2_SI,
                                               const double chi1, const double chi2, const double distance) {
  const int PD_EFAULT = 14, PD_EDOM = 33;
  if (!h22 || *h22 || !freq || !freq->data || freq->length == 0) { fail(QCBC_EINVAL, "bad pointers"); return PD_EFAULT; }
  double m1 = m1_SI / kMsun, m2 = m2_SI / kMsun;
  size_t n = freq->length;
  double fmin_ = freq->data[0];
  if (fRef_in < 0 || m1 <= 0 || m2 <= 0 || fmin_ <= 0 || distance <= 0 || chi1 > 1.0 || chi1 < -1.0 || chi2 > 1.0 ||
      chi2 < -1.0) {
    fail(QCBC_EDOM, "IMRPhenomD input outside its domain");
    return PD_EDOM;
  }
  double fCut = kFcut / ((m1 + m2) * kMtsun);
  if (fCut <= fmin_) { fail(QCBC_EDOM, "fCut %g <= f_min %g", fCut, fmin_); return PD_EDOM; }
  double fRef = (fRef_in == 0.0) ? fmin_ : fRef_in;
  Workspace* w;
  if (workspace(w)) return PD_EFAULT;
  cudaStream_t s = w->stream;
  double* d_freq;
  if (stage_freq(w, freq, n, &d_freq)) return PD_EFAULT;
  if (grow(w->d_a, w->c_a, 2 * n) || grow(w->d_recs, w->c_recs, 1) || grow(w->d_status, w->c_status, 1) ||
      grow_host(w->h_a, w->ch_a, 2 * n) || grow_host(w->h_status, w->ch_status, 1))
    return PD_EFAULT;
  DeviceState& ds = g_dev[current_device()];
  launch_amp_phase(d_freq, (int)n, phi0, fRef, m1, m2, chi1, chi2, distance, ds.qnm, w->d_recs, w->d_a, w->d_a + n,
                   w->d_status, s);
  tls_launches += 2;
  cudaMemcpyAsync(w->h_a, w->d_a, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(w->h_status, w->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "amp/phase failed"); return PD_EFAULT; }
  if (w->h_status[0] != 0) { fail(QCBC_EDOM, "IMRPhenomD input outside its domain"); return PD_EDOM; }
  AmpPhaseFDWaveform* wf = (AmpPhaseFDWaveform*)malloc(sizeof(AmpPhaseFDWaveform));
  wf->length = n;
  wf->freq = (double*)malloc(sizeof(double) * n);
  wf->amp = (double*)malloc(sizeof(double) * n);
  wf->phase = (double*)malloc(sizeof(double) * n);
  memcpy(wf->freq, freq->data, sizeof(double) * n);
  memcpy(wf->amp, w->h_a, sizeof(double) * n);
  memcpy(wf->phase, w->h_a + n, sizeof(double) * n);
  *h22 = wf;
  return 0;
}

extern "C" double fourier_nwip(double* a, double* b, double* Sn, int imin, int imax, int N) {
  if (!a || !b || !Sn) { fail(QCBC_EINVAL, "NULL argument"); return 0.0; }
  if (imin >= imax) return 0.0;
  if (imin < 1 || imax > N / 2 + 1 || N - imax + 1 < 0) { fail(QCBC_EINVAL, "bad band"); return 0.0; }
  Workspace* w;
  if (workspace(w)) return 0.0;
  cudaStream_t s = w->stream;
  if (grow(w->d_a, w->c_a, (size_t)2 * N + imax + 1) || grow(w->d_b, w->c_b, 2 * kMaxIfo)) return 0.0;
  double* d_x = w->d_a;
  double* d_y = d_x + N;
  double* d_s = d_y + N;
  cudaMemcpyAsync(d_x, a, sizeof(double) * N, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_y, b, sizeof(double) * N, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_s, Sn, sizeof(double) * imax, cudaMemcpyHostToDevice, s);
  launch_nwip(d_x, d_y, d_s, imin, imax, N, w->d_b, s);
  tls_launches += 1;
  double out = 0.0;
  cudaMemcpyAsync(&out, w->d_b, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "fourier_nwip failed"); return 0.0; }
  return out;
}

extern "C" double log_likelihood_intrinsic(struct Net* net, double** D, double* params, RealVector* freq,
                                           double** SN, int N, double Tobs) {
  if (!net || !D || !SN || !params) { fail(QCBC_EINVAL, "NULL argument"); return -1.0e20; }
  if (ensure_init()) return -1.0e20;
  EventPtr ep = data_event(net, D, SN, N, Tobs);
  if (!ep) return -1.0e20;
  qcbc_event* ev = ep->ev;
  NetGeom g = ev->g;
  fill_geom(g, net->Nifo, net->labels, Tobs, net->GMST, N, ev->fmin, ev->fmax);
  if (!reference_grid(freq, N, Tobs, g.imin, g.imax)) {
    fail(QCBC_EINVAL, "freq is not the reference grid i/Tobs (QuickCBC.c:419-420)");
    return -1.0e20;
  }
  double lnl = -1.0e20;
  int rc = run_full(ev, params, 1, &lnl, nullptr, QCBC_FP64, g, kModelIntrinsic);
  return rc == QCBC_OK ? lnl : -1.0e20;
}

extern "C" void templates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  if (!net || !hwave || !freq || !params) { fail(QCBC_EINVAL, "NULL argument"); return; }
  Workspace* w;
  if (workspace(w)) return;
  if (check_geom(net->Nifo, net->labels, 1.0, N)) return;
  cudaStream_t s = w->stream;
  double* d_freq;
  if (stage_freq(w, freq, (size_t)N / 2, &d_freq)) return;
  double Tobs = 1.0 / freq->data[1];   // QuickCBC.c:3539
  NetGeom g;
  fill_geom(g, net->Nifo, net->labels, Tobs, net->GMST, N, 0.0, 1.0);
  const int nI = net->Nifo, ps = param_stride(kModelIntrinsic, nI);
  if (grow(w->d_a, w->c_a, (size_t)nI * N) || grow(w->d_params, w->c_params, (size_t)ps) ||
      grow(w->d_recs, w->c_recs, 1) || grow(w->d_status, w->c_status, 1) || grow_host(w->h_a, w->ch_a, (size_t)nI * N))
    return;
  if (cudaMemcpyAsync(w->d_params, params, ps * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess) return;
  DeviceState& ds = g_dev[current_device()];
  launch_fulltemplates(w->d_params, g, ds.qnm, d_freq, w->d_recs, w->d_status, w->d_a, s, kModelIntrinsic);
  tls_launches += 2;
  cudaMemcpyAsync(w->h_a, w->d_a, sizeof(double) * nI * N, cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "templates failed"); return; }
  for (int id = 0; id < nI; id++) memcpy(hwave[id], w->h_a + (size_t)id * N, sizeof(double) * N);
}

extern "C" void AmpPhase(double* Af, double* Pf, RealVector* freq, double* params, int N) {
  if (!Af || !Pf || !freq || !freq->data || !params) { fail(QCBC_EINVAL, "NULL argument"); return; }
  const int n = N / 2;
  if (n < 2 || freq->length < (size_t)n) { fail(QCBC_EINVAL, "freq shorter than N/2"); return; }
  Workspace* w;
  if (workspace(w)) return;
  // physical parameters exactly as QuickCBC.c:3406-3431 forms them
  const double Tobs = 1.0 / freq->data[1];
  const double mc = exp(params[0]), mt = exp(params[1]);
  const double eta = pow((mc / mt), (5.0 / 3.0));
  const double dm = eta > 0.25 ? 0.0 : sqrt(1.0 - 4.0 * eta);
  const double m1_SI = mt * (1.0 + dm) / 2.0, m2_SI = mt * (1.0 - dm) / 2.0;
  const double ts = Tobs - params[5], distance = exp(params[6]);
  cudaStream_t s = w->stream;
  double* d_freq;
  if (stage_freq(w, freq, (size_t)n, &d_freq)) return;
  if (grow(w->d_a, w->c_a, (size_t)4 * n) || grow(w->d_recs, w->c_recs, 1) || grow(w->d_status, w->c_status, 1) ||
      grow_host(w->h_a, w->ch_a, (size_t)2 * n) || grow_host(w->h_status, w->ch_status, 1))
    return;
  DeviceState& ds = g_dev[current_device()];
  double *d_amp = w->d_a, *d_ph = w->d_a + n, *d_Af = w->d_a + 2 * n, *d_Pf = w->d_a + 3 * n;
  launch_amp_phase(d_freq, n, params[4], kFref, m1_SI / kMsun, m2_SI / kMsun, params[2], params[3], distance, ds.qnm,
                   w->d_recs, d_amp, d_ph, w->d_status, s);
  launch_ampphase_out(d_freq, d_amp, d_ph, n, ts, d_Af, d_Pf, s);
  tls_launches += 3;
  cudaMemcpyAsync(w->h_a, d_Af, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(w->h_status, w->d_status, sizeof(int), cudaMemcpyDeviceToHost, s);
  if (cudaStreamSynchronize(s) != cudaSuccess) { fail(QCBC_ECUDA, "AmpPhase failed"); return; }
  if (w->h_status[0] != 0) fail(QCBC_EDOM, "IMRPhenomD input outside its domain");
  memcpy(Af + 1, w->h_a + 1, sizeof(double) * (n - 1));
  memcpy(Pf + 1, w->h_a + n + 1, sizeof(double) * (n - 1));
}

extern "C" double het_diff(struct Net* net, struct Het* het, double* params, double* dparams) {
  if (!net || !het || !params || !dparams) { fail(QCBC_EINVAL, "NULL argument"); return 0.0; }
  if (ensure_init()) return 0.0;
  EventPtr ev = het_event_for(net, het);
  if (!ev) return 0.0;
  double out = 0.0;
  return qcbc_het_diff(ev->ev, params, dparams, 1, &out) == QCBC_OK ? out : 0.0;
}

extern "C" void Fisher_Het(struct Net* net, struct Het* het, double** fish, double* params, double Tobs) {
  (void)Tobs;   // fullphaseamp on the heterodyne grid uses net->Tobs (QuickCBC.c:3797)
  if (!net || !het || !fish || !params) { fail(QCBC_EINVAL, "NULL argument"); return; }
  if (ensure_init()) return;
  EventPtr ev = het_event_for(net, het);
  if (!ev) return;
  double F[11 * 11];
  if (qcbc_het_fisher(ev->ev, params, 1, F) != QCBC_OK) return;
  for (int i = 0; i < 11; i++)
    for (int j = 0; j < 11; j++) fish[i][j] = F[i * 11 + j];
}

extern "C" void het_space(struct Net* net, struct Het* het, double* params, double* min, double* max,
                          RealVector* freq, double** SN, int N, double Tobs) {
  if (!net || !het || !params || !min || !max || !freq || !freq->data || !SN) { fail(QCBC_EINVAL, "NULL argument"); return; }
  if (ensure_init()) return;
  if (check_geom(net->Nifo, net->labels, net->Tobs, N)) return;
  const int nI = net->Nifo, nh = N / 2;
  if (freq->length < (size_t)nh) { fail(QCBC_EINVAL, "freq shorter than N/2"); return; }
  std::vector<double> S((size_t)nI * nh);
  for (int id = 0; id < nI; id++) memcpy(&S[(size_t)id * nh], SN[id], sizeof(double) * nh);
  NetGeom g;
  fill_geom(g, nI, net->labels, net->Tobs, net->GMST, N, g_band_fmin, g_band_fmax);
  HetSpaceOut out;
  if (run_het_space(g, S.data(), nh, freq->data, N, Tobs, g_band_fmin, g_band_fmax, params, min, max, out)) return;
  // the struct Het fields het_space sets, allocated as CreateRealVector / int_vector do
  // (IMRPhenomD_internals.c:148-156, Utilities.c:2941-2944) so freehet releases them
  het->MN = out.MN;
  het->MM = out.MM;
  het->J = out.J;
  het->NR = out.NR;
  het->M = out.M;
  RealVector* fv = (RealVector*)malloc(sizeof(RealVector));
  fv->length = (size_t)out.M;
  fv->data = (double*)malloc(sizeof(double) * (size_t)out.M);
  het->fgrid = (int*)malloc(sizeof(int) * (size_t)(out.M + 1));
  for (int i = 0; i < out.M; i++) {
    het->fgrid[i] = out.fgrid[i];
    fv->data[i] = ((double)out.fgrid[i]) / Tobs;
  }
  het->freq = fv;
}

// ------------------------------------------------------------------ prefixed aliases
extern "C" double qcbc_gpu_log_likelihood_full(struct Net* net, double** D, double* params, RealVector* freq,
                                               double** SN, double* rho, int N, double Tobs) {
  return log_likelihood_full(net, D, params, freq, SN, rho, N, Tobs);
}
extern "C" double qcbc_gpu_log_likelihood_het(struct Net* net, struct Het* het, double* params, double Tobs) {
  return log_likelihood_het(net, het, params, Tobs);
}
extern "C" void qcbc_gpu_heterodyne(struct Net* net, struct Het* het, double** D, double* params, RealVector* freq,
                                    double** SN, int N, double Tobs) {
  heterodyne(net, het, D, params, freq, SN, N, Tobs);
}
extern "C" void qcbc_gpu_fulltemplates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  fulltemplates(net, hwave, freq, params, N);
}
extern "C" void qcbc_gpu_fullphaseamp(struct Net* net, double** amp, double** phase, RealVector* freq, double* params,
                                      int N) {
  fullphaseamp(net, amp, phase, freq, params, N);
}
extern "C" int qcbc_gpu_IMRPhenomDGenerateh22FDAmpPhase(AmpPhaseFDWaveform** h22, RealVector* freq, const double phi0,
                                                        const double fRef_in, const double m1_SI, const double m2_SI,
                                                        const double chi1, const double chi2, const double distance) {
  return IMRPhenomDGenerateh22FDAmpPhase(h22, freq, phi0, fRef_in, m1_SI, m2_SI, chi1, chi2, distance);
}
extern "C" double qcbc_gpu_fourier_nwip(double* a, double* b, double* Sn, int imin, int imax, int N) {
  return fourier_nwip(a, b, Sn, imin, imax, N);
}
extern "C" double qcbc_gpu_log_likelihood_intrinsic(struct Net* net, double** D, double* params, RealVector* freq,
                                                    double** SN, int N, double Tobs) {
  return log_likelihood_intrinsic(net, D, params, freq, SN, N, Tobs);
}
extern "C" void qcbc_gpu_templates(struct Net* net, double** hwave, RealVector* freq, double* params, int N) {
  templates(net, hwave, freq, params, N);
}
extern "C" void qcbc_gpu_AmpPhase(double* Af, double* Pf, RealVector* freq, double* params, int N) {
  AmpPhase(Af, Pf, freq, params, N);
}
extern "C" double qcbc_gpu_het_diff(struct Net* net, struct Het* het, double* params, double* dparams) {
  return het_diff(net, het, params, dparams);
}
extern "C" void qcbc_gpu_het_space(struct Net* net, struct Het* het, double* params, double* min, double* max,
                                   RealVector* freq, double** SN, int N, double Tobs) {
  het_space(net, het, params, min, max, freq, SN, N, Tobs);
}
extern "C" void qcbc_gpu_Fisher_Het(struct Net* net, struct Het* het, double** fish, double* params, double Tobs) {
  Fisher_Het(net, het, fish, params, Tobs);
}

// ------------------------------------------------------------------ allocation-free entry point
// Scratch of qcbc_lnl_full_noalloc in a file-scope device array: per-set records,
// per-set status and per-(set, tile) partial sums for up to QCBC_NOALLOC_MAX_SETS
// sets and QCBC_NOALLOC_MAX_TILE_SLOTS (set, tile) pairs.  Every GPU that loads
// this library holds it until the process exits.  Nothing in it needs to start at
// zero: each launch writes every record, status and partial it later reads.
constexpr size_t kNaRecBytes = (size_t)QCBC_NOALLOC_MAX_SETS * sizeof(PhdRec);
constexpr size_t kNaStatusOff = (kNaRecBytes + 255) / 256 * 256;
constexpr size_t kNaPartOff = (kNaStatusOff + (size_t)QCBC_NOALLOC_MAX_SETS * sizeof(int) + 255) / 256 * 256;
constexpr size_t kNaBytes = kNaPartOff + (size_t)QCBC_NOALLOC_MAX_TILE_SLOTS * 2 * kMaxIfo * sizeof(double);
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];
static_assert(kNaBytes == QCBC_NOALLOC_SCRATCH_BYTES, "header size constant out of date");

// Device address of g_noalloc_scratch per device.  In host code the array's name
// only stands in for the symbol; the address comes from cudaGetSymbolAddress,
// taken once per device with that device current.
static void* g_noalloc_addr[kMaxDevices] = {nullptr};
static std::mutex g_noalloc_mu;

extern "C" int qcbc_lnl_full_noalloc(qcbc_event* ev, const double* d_params, int B, double* d_lnl, double* d_rho,
                                     int precision, void* stream) {
  if (!ev || !d_params || !d_lnl) return fail(QCBC_EINVAL, "NULL argument");
  if (precision != QCBC_FP64 && precision != QCBC_MIXED) return fail(QCBC_EINVAL, "precision %d", precision);
  if (B < 0) return fail(QCBC_EINVAL, "B < 0");
  if (B == 0) return QCBC_OK;
  if (B > QCBC_NOALLOC_MAX_SETS)
    return fail(QCBC_EINVAL, "qcbc_lnl_full_noalloc: B=%d exceeds QCBC_NOALLOC_MAX_SETS=%d", B,
                QCBC_NOALLOC_MAX_SETS);
  int dev = 0;
  CU(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(QCBC_EINVAL, "current device %d out of range", dev);
  if (dev != ev->device)
    return fail(QCBC_EINVAL, "event lives on device %d but device %d is current", ev->device, dev);
  if (!g_dev[dev].ready) return fail(QCBC_EINVAL, "device %d not initialised (open an event first)", dev);
  void* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess)
        return fail(QCBC_ECUDA, "cudaGetSymbolAddress(g_noalloc_scratch): %s", cudaGetErrorString(e));
      g_noalloc_addr[dev] = p;
    }
    base = g_noalloc_addr[dev];
  }
  FullLaunch L = choose_launch(ev, B, precision);
  int max_tiles = QCBC_NOALLOC_MAX_TILE_SLOTS / B;
  if (L.tiles > max_tiles) L.tiles = max_tiles;
  if (L.tiles < 1) L.tiles = 1;
  unsigned char* b = static_cast<unsigned char*>(base);
  PhdRec* recs = reinterpret_cast<PhdRec*>(b);
  int* status = reinterpret_cast<int*>(b + kNaStatusOff);
  double* part = reinterpret_cast<double*>(b + kNaPartOff);
  cudaStream_t s = (cudaStream_t)stream;
  DeviceState& ds = g_dev[dev];
  EventData ed = event_data(ev);
  launch_setup(d_params, B, ev->g, ds.qnm, recs, status, s);
  launch_lnl_full(recs, B, ev->g, ed, precision == QCBC_MIXED ? kMixed : kFP64, L, part, s);
  launch_finalize_full(part, recs, status, B, L.tiles, ev->g, ed, precision == QCBC_MIXED ? kMixed : kFP64, d_lnl,
                       d_rho, s);
  tls_launches += 3;
  CU(cudaGetLastError());
  return QCBC_OK;
}

// ================================================================== PSD changes (noise marginalisation)
// After the event's device PSD rows changed: the in-band minimum of each detector (device reduction),
// sigma = sqrt(min) as at upload, the weighted data rebuilt on the device with the same arithmetic
// as event_upload, and heterodyne tables built by qcbc_het_setup rebuilt about the same reference
// point and grid (QuickCBC.c:1994-2010).  Tables given by qcbc_het_set are dropped.
static int event_psd_changed(qcbc_event* ev, Workspace* w) {
  const int nI = ev->g.nifo, nh = ev->nh;
  const int lo = std::max(ev->g.imin, 1), hi = std::min(ev->g.imax, nh);
  int rc;
  if ((rc = grow(w->d_b, w->c_b, (size_t)2 * kMaxIfo))) return rc;
  cudaStream_t s = w->stream;
  qcbc::launch_band_min(ev->d_S, nh + 1, nI, lo, hi, w->d_b, s);
  double smin[kMaxIfo];
  CU(cudaMemcpyAsync(smin, w->d_b, sizeof(double) * nI, cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  qcbc::Sigmas sg{{1.0, 1.0, 1.0}};
  for (int id = 0; id < nI; id++) {
    double m = smin[id];
    if (!(m < HUGE_VAL)) m = 1.0;
    sg.v[id] = sqrt(m);
    ev->inv_sigma[id] = 1.0 / sg.v[id];
  }
  qcbc::launch_event_weights(ev->d_D, ev->g.N, ev->d_S, nh + 1, nI, lo, hi, sg, ev->d_w64, ev->d_wm, s);
  tls_launches += 2;
  CU(cudaGetLastError());
  CU(cudaStreamSynchronize(s));
  HetDev& h = ev->het;
  if (h.buf && h.has_pref) {
    double pref[11];
    memcpy(pref, h.pref, sizeof(pref));
    std::vector<int> grid = h.fgrid;
    return qcbc_het_setup(ev, pref, grid.data(), h.M, h.MN, h.MM, h.J);
  }
  if (h.buf) {
    cudaFree(h.buf);
    cudaFree(h.d_fgrid);
    h = HetDev();
  }
  return QCBC_OK;
}

extern "C" int qcbc_event_set_psd_sample(qcbc_event* ev, qcbc_psd_model* m, int k) {
  if (!ev || !m) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->has_data) return fail(QCBC_EINVAL, "event has no data");
  if (qcbc::psd_model_nifo(m) != ev->g.nifo)
    return fail(QCBC_EINVAL, "model has %d detectors, event %d", qcbc::psd_model_nifo(m), ev->g.nifo);
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = qcbc::psd_model_draw_dev(m, k, ev->g.Tobs, ev->g.N, ev->d_S, ev->nh + 1, w->stream))) return rc;
  return event_psd_changed(ev, w);
}

extern "C" int qcbc_event_set_psd(qcbc_event* ev, const double* SN, int sn_stride) {
  if (!ev || !SN) return fail(QCBC_EINVAL, "NULL argument");
  if (!ev->has_data) return fail(QCBC_EINVAL, "event has no data");
  if (sn_stride < ev->nh) return fail(QCBC_EINVAL, "sn_stride < N/2");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  for (int id = 0; id < ev->g.nifo; id++)
    CU(cudaMemcpyAsync(ev->d_S + (size_t)id * (ev->nh + 1), SN + (size_t)id * sn_stride, sizeof(double) * ev->nh,
                       cudaMemcpyHostToDevice, w->stream));
  return event_psd_changed(ev, w);
}

// ================================================================== sky-ring map (one point)
extern "C" int qcbc_sky_ring_map(const double* x, double* y, double GMST, int label1, int label2, double rot,
                                 double* log_jacobian) {
  if (!x || !y || !log_jacobian) return fail(QCBC_EINVAL, "NULL argument");
  if (label1 < 0 || label1 > 2 || label2 < 0 || label2 > 2 || label1 == label2)
    return fail(QCBC_EINVAL, "two different detector labels in 0..2");
  Workspace* w;
  int rc = workspace(w);
  if (rc) return rc;
  if ((rc = grow(w->d_b, w->c_b, (size_t)2 * kMaxIfo))) return rc;
  if ((rc = grow(w->d_params, w->c_params, 24))) return rc;
  cudaStream_t s = w->stream;
  CU(cudaMemcpyAsync(w->d_params, x, sizeof(double) * 11, cudaMemcpyHostToDevice, s));
  launch_sky_ring_map(w->d_params, w->d_params + 12, GMST, label1, label2, rot, w->d_b, s);
  tls_launches += 1;
  CU(cudaGetLastError());
  CU(cudaMemcpyAsync(y, w->d_params + 12, sizeof(double) * 11, cudaMemcpyDeviceToHost, s));
  CU(cudaMemcpyAsync(log_jacobian, w->d_b, sizeof(double), cudaMemcpyDeviceToHost, s));
  CU(cudaStreamSynchronize(s));
  return QCBC_OK;
}
