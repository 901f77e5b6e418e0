// Continuous-batching PT-MCMC service over the multi-event likelihood
// (declared in include/qcbc_serve.h).  Host code only: every likelihood goes
// through the public C ABI (qcbc_event_open, qcbc_batch_*, qcbc_lnl_multi,
// qcbc_lnl_multi_het, qcbc_het_space, qcbc_het_setup).
//
// The sampler follows the reference's parallel-tempered scheme in outline
// (QuickCBC.c:1781-2236 MCMC_all, 2238-2405 update): Metropolis updates at
// temperatures T_t = ladder^t, swaps between adjacent temperatures, prior box
// of MCMC_all (QuickCBC.c:1871-1896, ConstCBC.h:48-57), angle wrapping as in
// het_space (QuickCBC.c:4650-4665).  Its proposal is a plain Gaussian with
// adapted scales; the reference's Fisher, differential-evolution and sky-ring
// moves are host logic outside the likelihood path.
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/qcbc_gpu.h"
#include "../../include/qcbc_serve.h"
#include "qcbc_hetspace.h"
#include "qcbc_ptstep.h"

extern "C" int qcbc_internal_fail(int code, const char* msg);

namespace {

int sfail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return qcbc_internal_fail(code, buf);
}

// xoshiro256** seeded by splitmix64: one independent stream per run
struct Rng {
  uint64_t s[4];
  static uint64_t splitmix(uint64_t& x) {
    uint64_t z = (x += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
  }
  void seed(uint64_t v) {
    for (auto& w : s) w = splitmix(v);
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  // Symmetric, zero-mean, unit-variance step: (u1 + u2 + u3 + u4 - 2) sqrt(3) from four 32-bit
  // uniforms (two generator calls).  Metropolis-Hastings needs only a symmetric proposal, not
  // an exact Gaussian, and this one costs a few ns instead of a log, a sqrt and a cos.
  double step() {
    uint64_t a = next(), b = next();
    constexpr double k = 1.0 / 4294967296.0;
    double s4 = ((double)(uint32_t)a + (double)(a >> 32) + (double)(uint32_t)b + (double)(b >> 32)) * k;
    return (s4 - 2.0) * 1.7320508075688772;
  }
};

constexpr double kMsun = 1.988546954961461467461011951140572744e30;
constexpr double kPc = 3.085677581491367278913937957796471611e16;
constexpr double kTwoPi = 6.2831853071795862319959269370884;
constexpr double kPi = 3.1415926535897931159979634685442;

struct Run {
  long long id = 0;
  int state = QCBC_RUN_QUEUED;
  // copied submission
  int nifo = 0, N = 0, sn_stride = 0;
  int labels[3] = {0, 0, 0};
  double Tobs = 0, GMST = 0, fmin = 0, fmax = 0;
  std::vector<double> D, SN;
  double start[11], sigma[11], pmin[11], pmax[11];
  int n_temps = 1, n_chains = 1, n_steps = 0, burn_in = 0, thin = 1;
  double ladder = 1.15;
  int likelihood = QCBC_LNL_FULL;
  int proposal = QCBC_PROPOSE_GAUSS;
  unsigned long long seed = 0;
  double ejump[11], evec[11][11];            // reference proposal: Fisher jumps at the start point
  // live state
  qcbc_event* ev = nullptr;
  int slot = -1;
  long long bytes = 0;
  bool initialised = false;
  int steps_done = 0;
  std::vector<double> x, lnl, temp, scale;   // per chain; scale per temperature
  std::vector<int> acc, prop;                // per temperature, reset each adaptation window
  long long cold_acc = 0, cold_prop = 0, swaps = 0, swap_tries = 0, evals = 0;
  std::vector<double> samples;               // rows of 12
  double t_arrival = 0, t_admit = -1, t_done = -1;
  Rng rng;
  // device-resident stepping: per-chain generator states and the kernels' view of the run
  std::vector<uint64_t> rng_chains;          // [nc][4]
  qcbc::PtRun pt{};
};

long long estimate_bytes(const Run& r) {
  long long nh = r.N / 2;
  return (long long)r.nifo * (3 * nh * 8 + nh * 16 + (long long)r.N * 8 + (nh + 1) * 8) + nh * 8;
}

}  // namespace

struct qcbc_server {
  long long budget = 0, bytes_live = 0, evals = 0, launches = 0;
  double t_propose = 0.0, t_lnl = 0.0, t_update = 0.0;   // seconds spent in each phase of a step
  int max_live = 0, max_bins = 0, precision = QCBC_MIXED;
  qcbc_batch* batch = nullptr;
  std::vector<long long> slot_run;             // run id per slot or -1
  std::map<long long, Run*> runs;
  std::deque<long long> queue;
  std::vector<long long> live;
  long long next_id = 0;
  std::chrono::steady_clock::time_point t0;
  std::mutex mu;
  // launch staging: full and heterodyned sets
  std::vector<int> eo, eo_h;
  std::vector<double> params, out, params_h, out_h;
  // device-resident stepping (dev_steps > 0): the live runs packed into flat device arrays,
  // full-likelihood runs first; repacked when the live set changes
  int dev_steps = 0;
  cudaStream_t dstream = nullptr;
  qcbc::PtChains dc{};
  qcbc::PtRun* d_runs = nullptr;
  int capB = 0, capR = 0, Bpk = 0, Bfpk = 0;
  std::vector<long long> packed;
  bool dirty = true;
  bool any_ref = false;                        // a packed run uses the reference proposal
};

static void free_dev(qcbc_server* s);
static int dev_init_run(Run* r, unsigned long long seed);
static int dev_pull(qcbc_server* s);
static int dev_samples(Run* r);

static double now_s(const qcbc_server* s) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - s->t0).count();
}

extern "C" qcbc_server* qcbc_server_create(long long budget, int max_live, int max_bins, int precision) {
  if (budget <= 0 || max_live <= 0 || max_bins <= 0 || (precision != QCBC_FP64 && precision != QCBC_MIXED)) {
    sfail(QCBC_EINVAL, "bad server settings");
    return nullptr;
  }
  qcbc_batch* b = qcbc_batch_create_slots(max_live, max_bins);
  if (!b) return nullptr;
  qcbc_server* s = new qcbc_server();
  s->budget = budget;
  s->max_live = max_live;
  s->max_bins = max_bins;
  s->precision = precision;
  s->batch = b;
  s->slot_run.assign(max_live, -1);
  s->t0 = std::chrono::steady_clock::now();
  return s;
}

static void retire(qcbc_server* s, Run* r, int state) {
  if (r->pt.samples) {
    cudaFree(r->pt.samples);
    r->pt.samples = nullptr;
  }
  if (r->pt.hist) {
    cudaFree(r->pt.hist);
    r->pt.hist = nullptr;
  }
  s->dirty = true;
  if (r->slot >= 0) {
    qcbc_batch_set_slot(s->batch, r->slot, nullptr);
    s->slot_run[r->slot] = -1;
    r->slot = -1;
  }
  if (r->ev) {
    qcbc_event_close(r->ev);
    r->ev = nullptr;
    s->bytes_live -= r->bytes;
  }
  r->state = state;
  r->t_done = now_s(s);
  r->D.clear();
  r->D.shrink_to_fit();
  r->SN.clear();
  r->SN.shrink_to_fit();
}

extern "C" int qcbc_server_destroy(qcbc_server* s) {
  if (!s) return QCBC_OK;
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->dstream) cudaStreamSynchronize(s->dstream);
  for (auto& kv : s->runs) {
    if (kv.second->state == QCBC_RUN_LIVE) retire(s, kv.second, QCBC_RUN_CANCELLED);
    delete kv.second;
  }
  free_dev(s);
  if (s->dstream) cudaStreamDestroy(s->dstream);
  qcbc_batch_destroy(s->batch);
  delete s;
  return QCBC_OK;
}

extern "C" double qcbc_server_clock(const qcbc_server* s) { return s ? now_s(s) : 0.0; }

extern "C" int qcbc_server_set_tiling(qcbc_server* s, int tile_bins, int threads) {
  if (!s) return sfail(QCBC_EINVAL, "NULL server");
  return qcbc_batch_set_tiling(s->batch, tile_bins, threads);
}

extern "C" long long qcbc_server_submit(qcbc_server* s, const qcbc_run_spec* sp) {
  if (!s || !sp || !sp->labels || !sp->D || !sp->SN || !sp->start) return sfail(QCBC_EINVAL, "NULL argument");
  if (sp->nifo < 1 || sp->nifo > 3 || sp->N < 8 || sp->sn_stride < sp->N / 2 || sp->n_temps < 1 ||
      sp->n_chains < 1 || sp->n_steps < 1 || sp->thin < 1 || sp->burn_in < 0 || !(sp->ladder >= 1.0))
    return sfail(QCBC_EINVAL, "bad run specification");
  if (sp->N / 2 > s->max_bins) return sfail(QCBC_EINVAL, "run has %d bins, server holds %d", sp->N / 2, s->max_bins);
  if (s->dev_steps > 0 && sp->n_temps > qcbc::kPtMaxTemps)
    return sfail(QCBC_EINVAL, "device-resident stepping takes at most %d temperatures", qcbc::kPtMaxTemps);
  Run* r = new Run();
  r->nifo = sp->nifo;
  r->N = sp->N;
  r->sn_stride = sp->sn_stride;
  for (int i = 0; i < sp->nifo; i++) r->labels[i] = sp->labels[i];
  r->Tobs = sp->Tobs;
  r->GMST = sp->GMST;
  r->fmin = sp->fmin;
  r->fmax = sp->fmax;
  r->D.assign(sp->D, sp->D + (size_t)sp->nifo * sp->N);
  r->SN.assign(sp->SN, sp->SN + (size_t)sp->nifo * sp->sn_stride);
  static const double kSig[11] = {1e-4, 1e-3, 0.02, 0.02, 0.1, 1e-4, 0.02, 0.01, 0.01, 0.02, 0.02};
  double tmin = std::max(sp->Tobs - 3.5, 1.5), tmax = sp->Tobs - 0.5;   // QuickCBC.c:178-183
  const double dmin[11] = {std::log(0.5 * kMsun), std::log(0.5 * kMsun), -0.85, -0.85, 0.0, tmin,
                           std::log(1e6 * kPc), 0.0, -1.0, 0.0, -1.0};
  const double dmax[11] = {std::log(160.0 * kMsun), std::log(300.0 * kMsun), 0.85, 0.85, kTwoPi, tmax,
                           std::log(1e10 * kPc), kTwoPi, 1.0, kPi, 1.0};
  for (int j = 0; j < 11; j++) {
    r->start[j] = sp->start[j];
    r->sigma[j] = sp->scales ? sp->scales[j] : kSig[j];
    r->pmin[j] = sp->prior_min ? sp->prior_min[j] : dmin[j];
    r->pmax[j] = sp->prior_max ? sp->prior_max[j] : dmax[j];
  }
  r->n_temps = sp->n_temps;
  r->n_chains = sp->n_chains;
  r->n_steps = sp->n_steps;
  r->burn_in = sp->burn_in;
  r->thin = sp->thin;
  r->ladder = sp->ladder;
  if (sp->likelihood != QCBC_LNL_FULL && sp->likelihood != QCBC_LNL_HET) {
    delete r;
    return sfail(QCBC_EINVAL, "likelihood %d", sp->likelihood);
  }
  if (sp->proposal != QCBC_PROPOSE_GAUSS && sp->proposal != QCBC_PROPOSE_REFERENCE) {
    delete r;
    return sfail(QCBC_EINVAL, "proposal %d", sp->proposal);
  }
  if (sp->proposal == QCBC_PROPOSE_REFERENCE && s->dev_steps == 0) {
    delete r;
    return sfail(QCBC_EINVAL, "the reference proposal runs with device-resident stepping only");
  }
  r->likelihood = sp->likelihood;
  r->proposal = sp->proposal;
  r->seed = sp->seed;
  r->rng.seed(sp->seed);
  r->bytes = estimate_bytes(*r);
  std::lock_guard<std::mutex> lk(s->mu);
  r->id = s->next_id++;
  r->t_arrival = now_s(s);
  if (r->bytes > s->budget) {
    long long need = r->bytes;
    delete r;
    return sfail(QCBC_EBUDGET, "run needs %lld B of device memory, budget is %lld B", need, s->budget);
  }
  s->runs[r->id] = r;
  s->queue.push_back(r->id);
  return r->id;
}

extern "C" int qcbc_server_cancel(qcbc_server* s, long long id) {
  if (!s) return sfail(QCBC_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->runs.find(id);
  if (it == s->runs.end()) return sfail(QCBC_EINVAL, "no run %lld", id);
  Run* r = it->second;
  if (r->state == QCBC_RUN_QUEUED) {
    for (auto q = s->queue.begin(); q != s->queue.end(); ++q)
      if (*q == id) { s->queue.erase(q); break; }
    r->state = QCBC_RUN_CANCELLED;
    r->t_done = now_s(s);
  } else if (r->state == QCBC_RUN_LIVE) {
    if (s->dev_steps > 0) {          // keep what the device sampler has so far
      int rc = dev_pull(s);
      if (rc == QCBC_OK) rc = dev_samples(r);
      if (rc != QCBC_OK) return rc;
    }
    retire(s, r, QCBC_RUN_CANCELLED);
    for (size_t k = 0; k < s->live.size(); k++)
      if (s->live[k] == id) { s->live.erase(s->live.begin() + k); break; }
  }
  return QCBC_OK;
}

// Heterodyne grid search and tables of a run's event about its starting point.
static int het_tables(Run* r) {
  int M = 0, MN = 0, MM = 0;
  int rc = qcbc_het_space(r->ev, r->start, r->pmin, r->pmax, &M, &MN, &MM);
  if (rc != QCBC_OK) return rc;
  std::vector<int> grid(M);
  if ((rc = qcbc_het_space_grid(r->ev, grid.data())) != QCBC_OK) return rc;
  return qcbc_het_setup(r->ev, r->start, grid.data(), M, MN, MM, 2);
}

// Fisher jumps of the reference proposal at the run's starting point: Fisher_Het (QuickCBC.c:5446)
// from the heterodyne tables, FisherEvec (2449) and efix with het_diff to distance 1 (4387), as
// MCMC_all prepares them (QuickCBC.c:1917-1923).
static int fisher_jumps(Run* r) {
  double F[11][11];
  int rc = qcbc_het_fisher(r->ev, r->start, 1, &F[0][0]);
  if (rc != QCBC_OK) return rc;
  qcbc::fisher_evec_11(F, r->ejump, r->evec);
  auto dist = [&](const double* px, double& z) -> int {
    if (qcbc_het_diff(r->ev, r->start, px, 1, &z) != QCBC_OK || !(z == z)) z = 1.0e20;
    return 0;
  };
  return qcbc::efix_run(r->start, r->pmin, r->pmax, r->ejump, r->evec, 1.0, dist);
}

// Admit queued runs in arrival order while a slot and the budget allow.
static void admit(qcbc_server* s) {
  while (!s->queue.empty()) {
    Run* r = s->runs[s->queue.front()];
    if (s->bytes_live + r->bytes > s->budget) break;
    int slot = -1;
    for (int k = 0; k < s->max_live; k++)
      if (s->slot_run[k] < 0) { slot = k; break; }
    if (slot < 0) break;
    s->queue.pop_front();
    r->ev = qcbc_event_open(r->nifo, r->labels, r->Tobs, r->GMST, r->N, r->D.data(), r->N, r->SN.data(),
                            r->sn_stride, r->fmin, r->fmax);
    const bool need_het = r->likelihood == QCBC_LNL_HET || r->proposal == QCBC_PROPOSE_REFERENCE;
    if (r->ev && need_het && (het_tables(r) != QCBC_OK ||
                              (r->proposal == QCBC_PROPOSE_REFERENCE && fisher_jumps(r) != QCBC_OK))) {
      qcbc_event_close(r->ev);
      r->ev = nullptr;
    }
    if (!r->ev || qcbc_batch_set_slot(s->batch, slot, r->ev) != QCBC_OK) {
      if (r->ev) qcbc_event_close(r->ev);
      r->ev = nullptr;
      r->state = QCBC_RUN_FAILED;
      r->t_done = now_s(s);
      continue;
    }
    r->bytes = qcbc_event_device_bytes(r->ev);
    s->bytes_live += r->bytes;
    r->slot = slot;
    s->slot_run[slot] = r->id;
    r->state = QCBC_RUN_LIVE;
    r->t_admit = now_s(s);
    int nc = r->n_temps * r->n_chains;
    r->x.assign((size_t)nc * 11, 0.0);
    r->lnl.assign(nc, -1e20);
    r->temp.assign(nc, 1.0);
    r->scale.assign(r->n_temps, 1.0);
    r->acc.assign(r->n_temps, 0);
    r->prop.assign(r->n_temps, 0);
    for (int c = 0; c < nc; c++) {
      int t = c % r->n_temps;
      r->temp[c] = std::pow(r->ladder, t);
      for (int j = 0; j < 11; j++) r->x[(size_t)c * 11 + j] = r->start[j];
    }
    for (int t = 0; t < r->n_temps; t++) r->scale[t] = std::sqrt(std::pow(r->ladder, t));
    if (s->dev_steps > 0) {
      if (dev_init_run(r, r->seed) != QCBC_OK) {
        retire(s, r, QCBC_RUN_FAILED);
        continue;
      }
      s->dirty = true;
    }
    s->live.push_back(r->id);
  }
}

// log prior density of update (QuickCBC.c:2352-2381) up to a constant: flat in m1, m2 and uniform
// in volume, in the sampled ln Mc, ln Mt, ln D coordinates
static double log_prior(const double* p) {
  const double leta = (5.0 / 3.0) * (p[0] - p[1]);
  const double eta = std::exp(leta);
  return 2.0 * p[1] + leta - 0.5 * std::log(std::max(1.0 - 4.0 * eta, 1e-16)) + 3.0 * p[6];
}

static bool in_prior(const Run* r, const double* y) {
  for (int j = 0; j < 11; j++)
    if (y[j] < r->pmin[j] || y[j] > r->pmax[j]) return false;
  double leta = (5.0 / 3.0) * (y[0] - y[1]);          // symmetric mass ratio (QuickCBC.c:2341-2364)
  return leta <= std::log(0.25) && leta >= std::log(0.05);
}

static void wrap(double* y) {
  y[4] = std::fmod(y[4], kTwoPi);
  if (y[4] < 0) y[4] += kTwoPi;
  y[7] = std::fmod(y[7], kTwoPi);
  if (y[7] < 0) y[7] += kTwoPi;
  y[9] = std::fmod(y[9], kPi);
  if (y[9] < 0) y[9] += kPi;
  for (int j : {8, 10}) {
    if (y[j] > 1.0) y[j] = 2.0 - y[j];
    if (y[j] < -1.0) y[j] = -2.0 - y[j];
  }
}

// ---------------------------------------------------------------- device-resident stepping
static void free_dev(qcbc_server* s) {
  qcbc::PtChains& c = s->dc;
  cudaFree(c.x); cudaFree(c.lnl); cudaFree(c.y); cudaFree(c.lnly); cudaFree(c.eo); cudaFree(c.run); cudaFree(c.rng);
  cudaFree(c.kind); cudaFree(c.jack);
  cudaFree(s->d_runs);
  c = qcbc::PtChains{};
  s->d_runs = nullptr;
  s->capB = s->capR = 0;
}

// Device view of a newly live run: starting points, per-chain generators seeded from the run's
// seed, scales sqrt(ladder^t), and the device buffer for its thinned samples.
static int dev_init_run(Run* r, unsigned long long seed) {
  qcbc::PtRun& p = r->pt;
  memset(&p, 0, sizeof(p));
  p.slot = r->slot;
  p.nc = r->n_temps * r->n_chains;
  p.n_temps = r->n_temps;
  p.n_chains = r->n_chains;
  p.burn_in = r->burn_in;
  p.thin = r->thin;
  p.n_steps = r->n_steps;
  p.ladder = r->ladder;
  for (int j = 0; j < 11; j++) { p.sigma[j] = r->sigma[j]; p.pmin[j] = r->pmin[j]; p.pmax[j] = r->pmax[j]; }
  for (int t = 0; t < r->n_temps; t++) p.scale[t] = std::sqrt(std::pow(r->ladder, t));
  p.proposal = r->proposal == QCBC_PROPOSE_REFERENCE ? qcbc::kProposeReference : qcbc::kProposeGauss;
  p.nifo = r->nifo;
  for (int i = 0; i < r->nifo; i++) p.labels[i] = r->labels[i];
  p.GMST = r->GMST;
  if (p.proposal == qcbc::kProposeReference) {
    memcpy(p.ejump, r->ejump, sizeof(p.ejump));
    memcpy(p.evec, r->evec, sizeof(p.evec));
    // the history of every temperature starts at the starting point (MCMC_all fills it with the
    // chains' states, QuickCBC.c:1944-1951)
    const size_t nh = (size_t)r->n_temps * qcbc::kPtHist;
    std::vector<double> h(nh * 11);
    for (size_t k = 0; k < nh; k++) memcpy(&h[k * 11], r->start, sizeof(double) * 11);
    if (cudaMalloc(&p.hist, sizeof(double) * h.size()) != cudaSuccess)
      return sfail(QCBC_ENOMEM, "history of %d temperatures", r->n_temps);
    if (cudaMemcpy(p.hist, h.data(), sizeof(double) * h.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return sfail(QCBC_ECUDA, "history upload failed");
  }
  int rows = r->n_steps > r->burn_in ? (r->n_steps - r->burn_in) / r->thin : 0;
  p.cap_samples = rows * r->n_chains;
  if (p.cap_samples > 0 &&
      cudaMalloc(&p.samples, sizeof(double) * 12 * (size_t)p.cap_samples) != cudaSuccess)
    return sfail(QCBC_ENOMEM, "sample buffer of %d rows", p.cap_samples);
  r->rng_chains.assign((size_t)p.nc * 4, 0);
  for (int c = 0; c < p.nc; c++) {
    uint64_t v = seed + 0x632BE59BD9B4E019ULL * (uint64_t)(c + 1);
    for (int k = 0; k < 4; k++) r->rng_chains[(size_t)c * 4 + k] = Rng::splitmix(v);
  }
  return QCBC_OK;
}

// Device state of the packed runs back into their Run objects (the device stays authoritative).
static int dev_pull(qcbc_server* s) {
  if (s->packed.empty()) return QCBC_OK;
  const int B = s->Bpk, R = (int)s->packed.size();
  std::vector<double> x((size_t)B * 11), lnl(B);
  std::vector<uint64_t> rng((size_t)B * 4);
  std::vector<qcbc::PtRun> pr(R);
  if (cudaStreamSynchronize(s->dstream) != cudaSuccess ||
      cudaMemcpy(x.data(), s->dc.x, x.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(lnl.data(), s->dc.lnl, lnl.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(rng.data(), s->dc.rng, rng.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(pr.data(), s->d_runs, sizeof(qcbc::PtRun) * R, cudaMemcpyDeviceToHost) != cudaSuccess)
    return sfail(QCBC_ECUDA, "device sampler state download failed");
  for (int k = 0; k < R; k++) {
    Run* r = s->runs[s->packed[k]];
    if (r->state != QCBC_RUN_LIVE) continue;
    const qcbc::PtRun& p = pr[k];
    r->pt = p;
    memcpy(r->x.data(), &x[(size_t)p.off * 11], sizeof(double) * 11 * p.nc);
    memcpy(r->lnl.data(), &lnl[p.off], sizeof(double) * p.nc);
    memcpy(r->rng_chains.data(), &rng[(size_t)p.off * 4], sizeof(uint64_t) * 4 * p.nc);
    r->cold_acc = (long long)p.cold_acc;
    r->cold_prop = (long long)p.cold_prop;
    r->swaps = (long long)p.swaps;
    r->swap_tries = (long long)p.swap_tries;
  }
  return QCBC_OK;
}

// The thinned samples a device run holds so far into its host copy.
static int dev_samples(Run* r) {
  r->samples.assign((size_t)r->pt.n_samples * 12, 0.0);
  if (r->pt.n_samples > 0 && r->pt.samples &&
      cudaMemcpy(r->samples.data(), r->pt.samples, r->samples.size() * 8, cudaMemcpyDeviceToHost) != cudaSuccess)
    return sfail(QCBC_ECUDA, "sample download failed");
  return QCBC_OK;
}

template <class T>
static int dev_grow(T** p, size_t n) {
  cudaFree(*p);
  *p = nullptr;
  return cudaMalloc(p, sizeof(T) * (n > 0 ? n : 1)) == cudaSuccess ? QCBC_OK : QCBC_ENOMEM;
}

// Live runs into the flat device arrays: full-likelihood runs first, then heterodyned ones.
static int dev_pack(qcbc_server* s) {
  std::vector<long long> order;
  for (int pass = 0; pass < 2; pass++)
    for (long long id : s->live)
      if ((s->runs[id]->likelihood == QCBC_LNL_HET) == (pass == 1)) order.push_back(id);
  int B = 0, Bf = 0;
  for (long long id : order) {
    Run* r = s->runs[id];
    r->pt.off = B;
    B += r->pt.nc;
    if (r->likelihood != QCBC_LNL_HET) Bf = B;
  }
  const int R = (int)order.size();
  if (B > s->capB) {
    int rc = 0;
    qcbc::PtChains& c = s->dc;
    rc |= dev_grow(&c.x, (size_t)B * 11) | dev_grow(&c.lnl, (size_t)B) | dev_grow(&c.y, (size_t)B * 11) |
          dev_grow(&c.lnly, (size_t)B) | dev_grow(&c.eo, (size_t)B) | dev_grow(&c.run, (size_t)B) |
          dev_grow(&c.rng, (size_t)B * 4) | dev_grow(&c.kind, (size_t)B) | dev_grow(&c.jack, (size_t)B);
    if (rc) return sfail(QCBC_ENOMEM, "device sampler arrays for %d chains", B);
    s->capB = B;
  }
  if (R > s->capR) {
    if (dev_grow(&s->d_runs, (size_t)R)) return sfail(QCBC_ENOMEM, "device run table");
    s->capR = R;
  }
  std::vector<double> x((size_t)B * 11), lnl(B);
  std::vector<uint64_t> rng((size_t)B * 4);
  std::vector<int> run(B);
  std::vector<qcbc::PtRun> pr(R);
  for (int k = 0; k < R; k++) {
    Run* r = s->runs[order[k]];
    const qcbc::PtRun& p = r->pt;
    pr[k] = p;
    memcpy(&x[(size_t)p.off * 11], r->x.data(), sizeof(double) * 11 * p.nc);
    memcpy(&lnl[p.off], r->lnl.data(), sizeof(double) * p.nc);
    memcpy(&rng[(size_t)p.off * 4], r->rng_chains.data(), sizeof(uint64_t) * 4 * p.nc);
    for (int c = 0; c < p.nc; c++) run[p.off + c] = k;
  }
  if (B > 0 &&
      (cudaMemcpy(s->dc.x, x.data(), x.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(s->dc.lnl, lnl.data(), lnl.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(s->dc.rng, rng.data(), rng.size() * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(s->dc.run, run.data(), run.size() * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
       cudaMemcpy(s->d_runs, pr.data(), sizeof(qcbc::PtRun) * R, cudaMemcpyHostToDevice) != cudaSuccess))
    return sfail(QCBC_ECUDA, "device sampler state upload failed");
  s->packed = order;
  s->Bpk = B;
  s->Bfpk = Bf;
  s->any_ref = false;
  for (long long id : order) s->any_ref |= s->runs[id]->proposal == QCBC_PROPOSE_REFERENCE;
  s->dirty = false;
  return QCBC_OK;
}

// Up to dev_steps steps of every live run on the device, stopping when a run finishes.
static int dev_step(qcbc_server* s) {
  double t0 = now_s(s);
  int rc;
  if (s->dirty) {
    if ((rc = dev_pull(s))) return rc;
    if ((rc = dev_pack(s))) return rc;
  }
  if (s->packed.empty()) return QCBC_OK;
  int K = s->dev_steps;
  for (long long id : s->packed) {
    Run* r = s->runs[id];
    K = std::min(K, r->n_steps - r->steps_done + (r->initialised ? 0 : 1));
  }
  const int B = s->Bpk, Bf = s->Bfpk, Bh = B - Bf, R = (int)s->packed.size();
  double t1 = now_s(s);
  qcbc::PtChains c = s->dc;
  for (int k = 0; k < K; k++) {
    qcbc::launch_pt_propose(s->d_runs, c, B, s->dstream);
    if (s->any_ref) qcbc::launch_pt_skyring(s->d_runs, c, B, s->dstream);
    if (Bf > 0 && (rc = qcbc_lnl_multi_dev(s->batch, c.eo, c.y, Bf, c.lnly, s->precision, s->dstream))) return rc;
    if (Bh > 0 &&
        (rc = qcbc_lnl_multi_het_dev(s->batch, c.eo + Bf, c.y + (size_t)Bf * 11, Bh, c.lnly + Bf, s->precision,
                                     s->dstream)))
      return rc;
    qcbc::launch_pt_accept(s->d_runs, c, B, s->dstream);
    qcbc::launch_pt_swap_finish(s->d_runs, R, 0, c, s->dstream);
  }
  cudaError_t e = cudaStreamSynchronize(s->dstream);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) return sfail(QCBC_ECUDA, "device steps: %s", cudaGetErrorString(e));
  double t2 = now_s(s);
  s->launches += (long long)K * ((Bf > 0) + (Bh > 0));
  s->evals += (long long)K * B;
  std::vector<long long> finished;
  for (long long id : s->packed) {
    Run* r = s->runs[id];
    r->evals += (long long)K * r->pt.nc;
    r->steps_done += r->initialised ? K : K - 1;
    r->initialised = true;
    if (r->steps_done >= r->n_steps) finished.push_back(id);
  }
  if (!finished.empty()) {
    if ((rc = dev_pull(s))) return rc;
    for (long long id : finished) {
      Run* r = s->runs[id];
      if ((rc = dev_samples(r))) return rc;
      retire(s, r, QCBC_RUN_DONE);
      for (size_t q = 0; q < s->live.size(); q++)
        if (s->live[q] == id) { s->live.erase(s->live.begin() + q); break; }
    }
    s->packed.clear();
    s->dirty = true;
  }
  double t3 = now_s(s);
  s->t_propose += t1 - t0;
  s->t_lnl += t2 - t1;
  s->t_update += t3 - t2;
  return QCBC_OK;
}

extern "C" int qcbc_server_set_device_steps(qcbc_server* s, int steps) {
  if (!s || steps < 0) return sfail(QCBC_EINVAL, "NULL server or negative step count");
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->live.empty() || !s->queue.empty()) return sfail(QCBC_EINVAL, "set the stepping mode before submitting runs");
  if (steps > 0 && !s->dstream && cudaStreamCreateWithFlags(&s->dstream, cudaStreamNonBlocking) != cudaSuccess)
    return sfail(QCBC_ECUDA, "stream creation failed");
  s->dev_steps = steps;
  return QCBC_OK;
}

static void step_counts(qcbc_server* s, int* n_live, int* n_queued, int* n_done) {
  if (n_live) *n_live = (int)s->live.size();
  if (n_queued) *n_queued = (int)s->queue.size();
  if (n_done) {
    int d = 0;
    for (auto& kv : s->runs) d += kv.second->state >= QCBC_RUN_DONE;
    *n_done = d;
  }
}

extern "C" int qcbc_server_step(qcbc_server* s, int* n_live, int* n_queued, int* n_done) {
  if (!s) return sfail(QCBC_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  admit(s);
  if (s->dev_steps > 0) {
    int rc = dev_step(s);
    step_counts(s, n_live, n_queued, n_done);
    return rc;
  }
  double t0 = now_s(s);
  s->eo.clear();
  s->params.clear();
  s->eo_h.clear();
  s->params_h.clear();
  // proposals (or the starting points of newly admitted runs)
  for (long long id : s->live) {
    Run* r = s->runs[id];
    const bool het = r->likelihood == QCBC_LNL_HET;
    std::vector<int>& eo = het ? s->eo_h : s->eo;
    std::vector<double>& P = het ? s->params_h : s->params;
    int nc = r->n_temps * r->n_chains;
    for (int c = 0; c < nc; c++) {
      double y[11];
      const double* x = &r->x[(size_t)c * 11];
      if (r->initialised) {
        int t = c % r->n_temps;
        for (int j = 0; j < 11; j++) y[j] = x[j] + r->scale[t] * r->sigma[j] * r->rng.step();
        wrap(y);
      } else {
        for (int j = 0; j < 11; j++) y[j] = x[j];
      }
      bool ok = in_prior(r, y);
      eo.push_back(ok ? r->slot : -1);
      P.insert(P.end(), y, y + 11);
    }
  }
  const int Bf = (int)s->eo.size(), Bh = (int)s->eo_h.size();
  double t1 = now_s(s);
  if (Bf > 0) {
    s->out.assign(Bf, -1e20);
    int rc = qcbc_lnl_multi(s->batch, s->eo.data(), s->params.data(), Bf, s->out.data(), nullptr, s->precision);
    if (rc != QCBC_OK && rc != QCBC_EDOM) return rc;   // EDOM: out-of-prior or invalid sets, lnL = -1e20
    s->launches++;
    s->evals += Bf;
  }
  if (Bh > 0) {
    s->out_h.assign(Bh, -1e20);
    int rc = qcbc_lnl_multi_het(s->batch, s->eo_h.data(), s->params_h.data(), Bh, s->out_h.data(), s->precision);
    if (rc != QCBC_OK && rc != QCBC_EDOM) return rc;
    s->launches++;
    s->evals += Bh;
  }
  double t2 = now_s(s);
  // accept / reject, swaps, adaptation, samples
  size_t kf = 0, kh = 0;
  std::vector<long long> finished;
  for (long long id : s->live) {
    Run* r = s->runs[id];
    const bool het = r->likelihood == QCBC_LNL_HET;
    const double* out = het ? s->out_h.data() : s->out.data();
    const double* P = het ? s->params_h.data() : s->params.data();
    size_t& k = het ? kh : kf;
    int nc = r->n_temps * r->n_chains;
    r->evals += nc;
    if (!r->initialised) {
      for (int c = 0; c < nc; c++, k++) r->lnl[c] = out[k];
      r->initialised = true;
      continue;
    }
    for (int c = 0; c < nc; c++, k++) {
      int t = c % r->n_temps;
      double Ly = out[k];
      r->prop[t]++;
      if (t == 0) r->cold_prop++;
      if (Ly > -1e19) {
        double la = (Ly - r->lnl[c]) / r->temp[c] + log_prior(&P[k * 11]) - log_prior(&r->x[(size_t)c * 11]);
        if (la >= 0.0 || std::log(r->rng.uniform()) < la) {
          std::memcpy(&r->x[(size_t)c * 11], &P[k * 11], 11 * sizeof(double));
          r->lnl[c] = Ly;
          r->acc[t]++;
          if (t == 0) r->cold_acc++;
        }
      }
    }
    if (r->n_temps > 1) {
      for (int ch = 0; ch < r->n_chains; ch++) {
        int t = (int)(r->rng.uniform() * (r->n_temps - 1));
        int a = ch * r->n_temps + t, b = a + 1;
        double la = (r->lnl[b] - r->lnl[a]) * (1.0 / r->temp[a] - 1.0 / r->temp[b]);
        r->swap_tries++;
        if (la >= 0.0 || std::log(r->rng.uniform()) < la) {
          for (int j = 0; j < 11; j++) std::swap(r->x[(size_t)a * 11 + j], r->x[(size_t)b * 11 + j]);
          std::swap(r->lnl[a], r->lnl[b]);
          r->swaps++;
        }
      }
    }
    r->steps_done++;
    if (r->steps_done <= r->burn_in && r->steps_done % 50 == 0) {
      for (int t = 0; t < r->n_temps; t++) {
        double rate = r->prop[t] ? (double)r->acc[t] / r->prop[t] : 0.25;
        double f = std::exp(rate - 0.25);
        r->scale[t] = std::min(std::max(r->scale[t] * f, 1e-3), 1e3);
        r->acc[t] = r->prop[t] = 0;
      }
    }
    if (r->steps_done > r->burn_in && (r->steps_done - r->burn_in) % r->thin == 0) {
      for (int ch = 0; ch < r->n_chains; ch++) {
        int c = ch * r->n_temps;   // T = 1
        r->samples.insert(r->samples.end(), &r->x[(size_t)c * 11], &r->x[(size_t)c * 11] + 11);
        r->samples.push_back(r->lnl[c]);
      }
    }
    if (r->steps_done >= r->n_steps) finished.push_back(id);
  }
  double t3 = now_s(s);
  s->t_propose += t1 - t0;
  s->t_lnl += t2 - t1;
  s->t_update += t3 - t2;
  for (long long id : finished) {
    retire(s, s->runs[id], QCBC_RUN_DONE);
    for (size_t q = 0; q < s->live.size(); q++)
      if (s->live[q] == id) { s->live.erase(s->live.begin() + q); break; }
  }
  if (n_live) *n_live = (int)s->live.size();
  if (n_queued) *n_queued = (int)s->queue.size();
  if (n_done) {
    int d = 0;
    for (auto& kv : s->runs) d += kv.second->state >= QCBC_RUN_DONE;
    *n_done = d;
  }
  return QCBC_OK;
}

extern "C" int qcbc_server_run_info(qcbc_server* s, long long id, qcbc_run_info* o) {
  if (!s || !o) return sfail(QCBC_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->runs.find(id);
  if (it == s->runs.end()) return sfail(QCBC_EINVAL, "no run %lld", id);
  Run* r = it->second;
  if (s->dev_steps > 0 && r->state == QCBC_RUN_LIVE) {   // the device holds the live counters
    int rc = dev_pull(s);
    if (rc == QCBC_OK) rc = dev_samples(r);
    if (rc != QCBC_OK) return rc;
  }
  o->state = r->state;
  o->steps_done = r->steps_done;
  o->t_arrival = r->t_arrival;
  o->t_admit = r->t_admit;
  o->t_done = r->t_done;
  o->accept_cold = r->cold_prop ? (double)r->cold_acc / r->cold_prop : 0.0;
  o->swap_rate = r->swap_tries ? (double)r->swaps / r->swap_tries : 0.0;
  o->device_bytes = r->bytes;
  o->lnl_evals = r->evals;
  o->n_samples = (int)(r->samples.size() / 12);
  return QCBC_OK;
}

extern "C" int qcbc_server_run_samples(qcbc_server* s, long long id, double* out, int max_rows, int* n_rows) {
  if (!s || !out || !n_rows) return sfail(QCBC_EINVAL, "NULL argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->runs.find(id);
  if (it == s->runs.end()) return sfail(QCBC_EINVAL, "no run %lld", id);
  if (s->dev_steps > 0 && it->second->state == QCBC_RUN_LIVE) {
    int rc = dev_pull(s);
    if (rc == QCBC_OK) rc = dev_samples(it->second);
    if (rc != QCBC_OK) return rc;
  }
  int n = (int)std::min<size_t>(it->second->samples.size() / 12, (size_t)std::max(max_rows, 0));
  std::memcpy(out, it->second->samples.data(), sizeof(double) * 12 * (size_t)n);
  *n_rows = n;
  return QCBC_OK;
}

extern "C" int qcbc_server_stats(qcbc_server* s, long long* evals, long long* launches, long long* bytes) {
  if (!s) return sfail(QCBC_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (evals) *evals = s->evals;
  if (launches) *launches = s->launches;
  if (bytes) *bytes = s->bytes_live;
  return QCBC_OK;
}

extern "C" int qcbc_server_timing(qcbc_server* s, double* propose_s, double* lnl_s, double* update_s) {
  if (!s) return sfail(QCBC_EINVAL, "NULL server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (propose_s) *propose_s = s->t_propose;
  if (lnl_s) *lnl_s = s->t_lnl;
  if (update_s) *update_s = s->t_update;
  return QCBC_OK;
}
