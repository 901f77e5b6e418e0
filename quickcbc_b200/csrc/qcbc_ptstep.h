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
};

struct PtChains {
  double* x;              // [B][11] current points
  double* lnl;            // [B]
  double* y;              // [B][11] proposals
  double* lnly;           // [B] their lnL
  int* eo;                // [B] batch slot of the proposal (-1: outside the prior)
  int* run;               // [B] live-run index of the chain
  uint64_t* rng;          // [B][4] xoshiro256** state
};

// One step of every live run (B chains, nrun runs) on `s`; the lnL of the proposals (y -> lnly) is
// computed between propose and accept by the caller.
void launch_pt_propose(PtRun* d_runs, PtChains c, int B, cudaStream_t s);
void launch_pt_accept(PtRun* d_runs, PtChains c, int B, cudaStream_t s);
void launch_pt_swap_finish(PtRun* d_runs, int nrun, int max_ladders, PtChains c, cudaStream_t s);

}  // namespace qcbc
