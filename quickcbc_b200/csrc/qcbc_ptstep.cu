// Device-resident parallel-tempering step (see qcbc_ptstep.h), after the reference's MCMC_all /
// update (QuickCBC.c:1781-2405):
//   * proposals: kProposeGauss, the host service's symmetric step with per-temperature adapted
//     scales (angles wrapped, sin/cos parameters reflected); or kProposeReference, update's mixture
//     (QuickCBC.c:2266-2333): Fisher eigen-jumps sqrt(T) ejump[i] N(0,1) along evec[i] (50 %),
//     differential evolution from the temperature's history (20 %, de_jump QuickCBC.c:2407-2425),
//     jiggles of 0.01 10^-floor(3U) sqrt(T) N(0,1) in every parameter (10 %), and the sky ring
//     (20 %; one detector: Fisher jump instead), which k_pt_skyring (qcbc_kernels.cu) completes;
//   * the prior box and symmetric-mass-ratio limits (QuickCBC.c:1871-1896, 2341-2364) and the
//     prior density of update (QuickCBC.c:2352-2381): flat in m1, m2 (2 ln Mt + ln eta
//     - ln(1 - 4 eta) / 2 in the ln Mc, ln Mt coordinates) and uniform in volume (3 ln D);
//   * Metropolis acceptance at T = ladder^t, one swap attempt between a random adjacent pair of
//     temperatures per ladder, scale adaptation towards 25 % acceptance every 50 burn-in steps
//     (Gauss proposal only), the history rows of every temperature refreshed every 20 steps, and
//     thinned samples of the T = 1 chains after burn-in.
// Every chain draws from its own xoshiro256** stream and the swap draws come from the ladder's
// coldest chain, so a run evolves the same alone, in any mix of runs and for any number of steps
// per host call.
#include "qcbc_ptstep.h"

#include <cmath>

namespace qcbc {
namespace {

constexpr double kTwoPiP = kPtTwoPi;
constexpr double kPiP = kPtPi;


__device__ void wrap(double* y) {
  y[4] = fmod(y[4], kTwoPiP);
  if (y[4] < 0) y[4] += kTwoPiP;
  y[7] = fmod(y[7], kTwoPiP);
  if (y[7] < 0) y[7] += kTwoPiP;
  y[9] = fmod(y[9], kPiP);
  if (y[9] < 0) y[9] += kPiP;
  for (int j = 8; j <= 10; j += 2) {
    if (y[j] > 1.0) y[j] = 2.0 - y[j];
    if (y[j] < -1.0) y[j] = -2.0 - y[j];
  }
}

__device__ bool in_prior(const PtRun& r, const double* y) { return pt_in_prior(r.pmin, r.pmax, y); }

__device__ double chain_temp(const PtRun& r, int t) { return pow(r.ladder, (double)t); }

__global__ void k_pt_propose(PtRun* __restrict__ runs, PtChains c, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const PtRun& r = runs[c.run[b]];
  double y[kPtNP];
  const double* x = c.x + (size_t)b * kPtNP;
  if (r.init && r.proposal == kProposeReference) {
    const int t = (b - r.off) % r.n_temps;
    const double sT = sqrt(chain_temp(r, t));
    Xoshiro g;
    g.load(c.rng + (size_t)b * 4);
    const double alpha = g.uniform();
    if (alpha > 0.3 && alpha <= 0.5) {                // differential evolution
      const double* H = r.hist + (size_t)t * kPtHist * kPtNP;
      const int i = (int)(g.uniform() * kPtHist);
      int j = (int)(g.uniform() * kPtHist);
      for (int k = 0; j == i && k < 64; k++) j = (int)(g.uniform() * kPtHist);
      const double a = g.uniform() < 0.9 ? 0.5 * g.gauss() : 1.0;
      for (int k = 0; k < kPtNP; k++) y[k] = x[k] + a * (H[(size_t)i * kPtNP + k] - H[(size_t)j * kPtNP + k]);
    } else if (alpha > 0.2 && alpha <= 0.3) {         // jiggle
      const double beta = 0.01 * exp10(-floor(3.0 * g.uniform())) * sT;
      for (int k = 0; k < kPtNP; k++) y[k] = x[k] + beta * g.gauss();
    } else if (alpha <= 0.2 && r.nifo >= 2) {         // sky ring: completed by k_pt_skyring
      g.store(c.rng + (size_t)b * 4);
      for (int j = 0; j < kPtNP; j++) c.y[(size_t)b * kPtNP + j] = x[j];
      c.kind[b] = kKindSkyRing;
      c.jack[b] = 0.0;
      c.eo[b] = -1;
      return;
    } else {                                          // Fisher eigen-jump (one detector: also the ring's share)
      const int i = min((int)(g.uniform() * kPtNP), kPtNP - 1);
      const double beta = sT * r.ejump[i] * g.gauss();
      for (int k = 0; k < kPtNP; k++) y[k] = x[k] + beta * r.evec[i][k];
    }
    g.store(c.rng + (size_t)b * 4);
    pt_wrap_angles(y);
  } else if (r.init) {
    const int t = (b - r.off) % r.n_temps;
    Xoshiro g;
    g.load(c.rng + (size_t)b * 4);
    for (int j = 0; j < kPtNP; j++) y[j] = x[j] + r.scale[t] * r.sigma[j] * g.step();
    g.store(c.rng + (size_t)b * 4);
    wrap(y);
  } else {
    for (int j = 0; j < kPtNP; j++) y[j] = x[j];
  }
  for (int j = 0; j < kPtNP; j++) c.y[(size_t)b * kPtNP + j] = y[j];
  c.eo[b] = in_prior(r, y) ? r.slot : -1;
  c.kind[b] = kKindOther;
  c.jack[b] = 0.0;
}

__global__ void k_pt_accept(PtRun* __restrict__ runs, PtChains c, int B) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  PtRun& r = runs[c.run[b]];
  const double Ly = c.lnly[b];
  if (!r.init) {                       // the starting point's lnL
    c.lnl[b] = Ly;
    return;
  }
  const int t = (b - r.off) % r.n_temps;
  atomicAdd(&r.prop[t], 1);
  if (t == 0) atomicAdd(&r.cold_prop, 1ULL);
  if (!(Ly > -1e19)) return;
  const double* x = c.x + (size_t)b * kPtNP;
  const double* y = c.y + (size_t)b * kPtNP;
  const double la = (Ly - c.lnl[b]) / chain_temp(r, t) + pt_log_prior(y) - pt_log_prior(x) + c.jack[b];
  bool ok = la >= 0.0;
  if (!ok) {
    Xoshiro g;
    g.load(c.rng + (size_t)b * 4);
    ok = log(g.uniform()) < la;
    g.store(c.rng + (size_t)b * 4);
  }
  if (ok) {
    for (int j = 0; j < kPtNP; j++) c.x[(size_t)b * kPtNP + j] = c.y[(size_t)b * kPtNP + j];
    c.lnl[b] = Ly;
    atomicAdd(&r.acc[t], 1);
    if (t == 0) atomicAdd(&r.cold_acc, 1ULL);
  }
}

// block (run): threads over the run's ladders for the swaps, then thread 0 .. n_temps-1 for the
// adaptation and the ladders again for the samples
__global__ void k_pt_swap_finish(PtRun* __restrict__ runs, PtChains c) {
  PtRun& r = runs[blockIdx.x];
  if (!r.init) {
    __syncthreads();
    if (threadIdx.x == 0) r.init = 1;
    return;
  }
  if (r.n_temps > 1) {
    for (int ch = threadIdx.x; ch < r.n_chains; ch += blockDim.x) {
      const size_t cold = (size_t)r.off + (size_t)ch * r.n_temps;
      Xoshiro g;
      g.load(c.rng + cold * 4);
      const int t = (int)(g.uniform() * (r.n_temps - 1));
      const size_t a = cold + t, b = a + 1;
      const double la = (c.lnl[b] - c.lnl[a]) * (1.0 / chain_temp(r, t) - 1.0 / chain_temp(r, t + 1));
      atomicAdd(&r.swap_tries, 1ULL);
      bool ok = la >= 0.0;
      if (!ok) ok = log(g.uniform()) < la;
      g.store(c.rng + cold * 4);
      if (ok) {
        for (int j = 0; j < kPtNP; j++) {
          const double v = c.x[a * kPtNP + j];
          c.x[a * kPtNP + j] = c.x[b * kPtNP + j];
          c.x[b * kPtNP + j] = v;
        }
        const double v = c.lnl[a];
        c.lnl[a] = c.lnl[b];
        c.lnl[b] = v;
        atomicAdd(&r.swaps, 1ULL);
      }
    }
  }
  __syncthreads();
  const int step = r.steps_done + 1;
  if (r.proposal == kProposeReference && step % 20 == 0) {   // history rows (QuickCBC.c:2068-2080)
    for (int e = threadIdx.x; e < r.n_chains * r.n_temps; e += blockDim.x) {
      const int ch = e / r.n_temps, t = e - ch * r.n_temps;
      const size_t src = (size_t)r.off + (size_t)ch * r.n_temps + t;
      double* h = r.hist + ((size_t)t * kPtHist + (size_t)((r.hist_pos + ch) % kPtHist)) * kPtNP;
      for (int j = 0; j < kPtNP; j++) h[j] = c.x[src * kPtNP + j];
    }
  }
  if (r.proposal == kProposeGauss && step <= r.burn_in && step % 50 == 0) {
    for (int t = threadIdx.x; t < r.n_temps; t += blockDim.x) {
      const double rate = r.prop[t] ? (double)r.acc[t] / r.prop[t] : 0.25;
      const double f = exp(rate - 0.25);
      r.scale[t] = fmin(fmax(r.scale[t] * f, 1e-3), 1e3);
      r.acc[t] = 0;
      r.prop[t] = 0;
    }
  }
  if (step > r.burn_in && (step - r.burn_in) % r.thin == 0) {
    for (int ch = threadIdx.x; ch < r.n_chains; ch += blockDim.x) {
      const int row = r.n_samples + ch;
      if (row < r.cap_samples) {
        const size_t cold = (size_t)r.off + (size_t)ch * r.n_temps;
        double* o = r.samples + (size_t)row * 12;
        for (int j = 0; j < kPtNP; j++) o[j] = c.x[cold * kPtNP + j];
        o[11] = c.lnl[cold];
      }
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (step > r.burn_in && (step - r.burn_in) % r.thin == 0) r.n_samples = min(r.n_samples + r.n_chains, r.cap_samples);
    if (r.proposal == kProposeReference && step % 20 == 0) r.hist_pos = (r.hist_pos + r.n_chains) % kPtHist;
    r.steps_done = step;
  }
}

}  // namespace

void launch_pt_propose(PtRun* d_runs, PtChains c, int B, cudaStream_t s) {
  if (B > 0) k_pt_propose<<<(B + 127) / 128, 128, 0, s>>>(d_runs, c, B);
}
void launch_pt_accept(PtRun* d_runs, PtChains c, int B, cudaStream_t s) {
  if (B > 0) k_pt_accept<<<(B + 127) / 128, 128, 0, s>>>(d_runs, c, B);
}
void launch_pt_swap_finish(PtRun* d_runs, int nrun, int max_ladders, PtChains c, cudaStream_t s) {
  (void)max_ladders;
  if (nrun > 0) k_pt_swap_finish<<<nrun, 64, 0, s>>>(d_runs, c);
}

}  // namespace qcbc
