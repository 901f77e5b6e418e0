// Heterodyne grid search (het_space, QuickCBC.c:4570-4910): host control logic over device
// waveforms.  Internal interface between qcbc_hetspace.cu and the C ABI.
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "qcbc_kernels.cuh"

namespace qcbc {

struct HetSpaceIn {
  NetGeom g;                 // network; g.Tobs is the Tobs the waveforms use (net->Tobs)
  QnmTable qnm;
  const double* h_S;         // host PSD rows [nifo][sn_stride], entries [0, N/2)
  int sn_stride;
  const double* h_freq;      // host frequencies [N/2] (freq[0] = 1/Tobs, freq[i] = i/Tobs)
  int N;
  double Tobs;               // the Tobs argument of het_space (bin <-> frequency)
  double fmin, fmax;         // analysis band (ConstCBC.h:33-34)
  cudaStream_t stream;
};

struct HetSpaceOut {
  int MN = 0, MM = 0, J = 2, M = 0, NR = 0;
  std::vector<int> fgrid;    // bins of the M grid points
  int launches = 0;
};

// Returns 0, or -2 (bad input: empty band, runaway grid) / -3 (CUDA error) with err set.
int het_space_run(const HetSpaceIn& in, const double* params, const double* pmin, const double* pmax,
                  HetSpaceOut& out, std::string& err);

// FisherEvec (QuickCBC.c:2449-2530): 1-sigma jump sizes ej (ascending |eigenvalue|, each
// eigenvalue raised to at least 10) and eigenvectors ev[i] of an 11 x 11 Fisher matrix.
void fisher_evec_11(const double (&F)[11][11], double* ej, double (&ev)[11][11]);

// efix (QuickCBC.c:4387-4567): rescales each eval[i] so that the step eval[i] evec[i] from params
// (sign-flipped, wrapped and clamped as the reference does) has distance zs, by a doubling /
// halving bracket and a secant search on dist(px, z); a direction that misses by more than zs gets
// size 0.  Returns the first nonzero status of dist.
int efix_run(const double* params, const double* pmin, const double* pmax, double* eval, const double (&evec)[11][11],
             double zs, const std::function<int(const double*, double&)>& dist);

}  // namespace qcbc
