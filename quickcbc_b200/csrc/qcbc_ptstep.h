// Device-resident parallel-tempering step of the continuous-batching service: proposal,
// Metropolis acceptance, adjacent-temperature swaps, scale adaptation and thinning as kernels,
// so that many steps of all live runs queue on one stream without host round trips.
// Internal interface between qcbc_ptstep.cu and qcbc_serve.cu.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

namespace qcbc {

constexpr int kPtMaxTemps = 64;
constexpr int kPtNP = 11;
constexpr int kPtHist = 1000;        // differential-evolution history per temperature (NH, ConstCBC.h:72)

enum PtProposal { kProposeGauss = 0, kProposeReference = 1 };

// One live run, as the kernels see it.  Chains of the run are [off, off + nc) of the packed chain
// arrays; chain c has temperature index c % n_temps and ladder c / n_temps.
struct PtRun {
  int slot, nc, n_temps, n_chains, off, burn_in, thin, n_steps;
  int steps_done, init;               // init: the starting point's lnL has been evaluated
  double ladder;
  double sigma[kPtNP], pmin[kPtNP], pmax[kPtNP];
  double scale[kPtMaxTemps];
  int acc[kPtMaxTemps], prop[kPtMaxTemps];
  unsigned long long cold_acc, cold_prop, swaps, swap_tries;
  double* samples;                    // device, rows of 12 (11 parameters, lnL)
  int n_samples, cap_samples;
  // kProposeReference: the reference's proposal mixture (update, QuickCBC.c:2238-2405)
  int proposal;
  int hist_pos;                       // next history row of every temperature
  double* hist;                       // device [n_temps][kPtHist][11]
  double ejump[kPtNP];                // Fisher jump sizes (FisherEvec + efix at the start point)
  double evec[kPtNP][kPtNP];          // their eigen-directions
  int nifo, labels[3];                // the run's network and GMST (sky-ring proposal)
  double GMST;
};

struct PtChains {
  double* x;              // [B][11] current points
  double* lnl;            // [B]
  double* y;              // [B][11] proposals
  double* lnly;           // [B] their lnL
  int* eo;                // [B] batch slot of the proposal (-1: outside the prior)
  int* run;               // [B] live-run index of the chain
  uint64_t* rng;          // [B][4] xoshiro256** state
  int* kind;              // [B] proposal of this step (kKindSkyRing: completed by the sky-ring kernel)
  double* jack;           // [B] log Jacobian of the proposal (sky ring), else 0
};

constexpr int kKindOther = 0;
constexpr int kKindSkyRing = 4;

// ---- shared by the step kernels (qcbc_ptstep.cu) and the sky-ring kernel (qcbc_kernels.cu)
constexpr double kPtTwoPi = 6.2831853071795862319959269370884;
constexpr double kPtPi = 3.1415926535897931159979634685442;

// xoshiro256** with splitmix64 seeding on the host side
struct Xoshiro {
  uint64_t s[4];
  __device__ static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  __device__ uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return r;
  }
  __device__ double uniform() { return (next() >> 11) * (1.0 / 9007199254740992.0); }
  // symmetric, zero-mean, unit-variance step: (u1 + u2 + u3 + u4 - 2) sqrt(3)
  __device__ double step() {
    const uint64_t a = next(), b = next();
    const double k = 1.0 / 4294967296.0;
    const double s4 = ((double)(uint32_t)a + (double)(a >> 32) + (double)(uint32_t)b + (double)(b >> 32)) * k;
    return (s4 - 2.0) * 1.7320508075688772;
  }
  // standard normal by the Box-Muller transform
  __device__ double gauss() {
    const double u1 = 1.0 - uniform(), u2 = uniform();     // u1 in (0, 1]
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  }
  __device__ void load(const uint64_t* p) { for (int i = 0; i < 4; i++) s[i] = p[i]; }
  __device__ void store(uint64_t* p) const { for (int i = 0; i < 4; i++) p[i] = s[i]; }
};

// log prior density of update (QuickCBC.c:2352-2381) up to a constant: flat in m1, m2 and uniform
// in volume, in the sampled ln Mc, ln Mt, ln D coordinates (finite at eta = 1/4)
__device__ inline double pt_log_prior(const double* p) {
  const double leta = (5.0 / 3.0) * (p[0] - p[1]);
  const double eta = exp(leta);
  return 2.0 * p[1] + leta - 0.5 * log(fmax(1.0 - 4.0 * eta, 1e-16)) + 3.0 * p[6];
}

// angles into [0, 2 pi) / [0, pi) (QuickCBC.c:2336-2341); sin/cos parameters are left to the
// prior box, as the reference does
__device__ inline void pt_wrap_angles(double* y) {
  y[4] = fmod(y[4], kPtTwoPi);
  if (y[4] < 0) y[4] += kPtTwoPi;
  y[7] = fmod(y[7], kPtTwoPi);
  if (y[7] < 0) y[7] += kPtTwoPi;
  y[9] = fmod(y[9], kPtPi);
  if (y[9] < 0) y[9] += kPtPi;
}

// the prior box of MCMC_all and the symmetric-mass-ratio limits (QuickCBC.c:1871-1896, 2341-2364)
__device__ inline bool pt_in_prior(const double* pmin, const double* pmax, const double* y) {
  for (int j = 0; j < kPtNP; j++)
    if (!(y[j] >= pmin[j] && y[j] <= pmax[j])) return false;
  const double leta = (5.0 / 3.0) * (y[0] - y[1]);
  return leta <= log(0.25) && leta >= log(0.05);
}

// One step of every live run (B chains, nrun runs) on `s`; the lnL of the proposals (y -> lnly) is
// computed between propose and accept by the caller.
void launch_pt_propose(PtRun* d_runs, PtChains c, int B, cudaStream_t s);
void launch_pt_accept(PtRun* d_runs, PtChains c, int B, cudaStream_t s);
void launch_pt_swap_finish(PtRun* d_runs, int nrun, int max_ladders, PtChains c, cudaStream_t s);
// The sky-ring proposals of this step (chains with kind == kKindSkyRing; qcbc_kernels.cu).
void launch_pt_skyring(PtRun* d_runs, PtChains c, int B, cudaStream_t s);

}  // namespace qcbc
