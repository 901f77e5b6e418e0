// Heterodyne grid search: het_space (QuickCBC.c:4570-4910) with limits (4275-4385),
// Fisher_All (2695-2817), FisherEvec (2449-2530), efix (4387-4567) and diff (4913-4964).
//
// The control logic (band limits from the SNR accumulation, the eigen-directions of the Fisher
// matrix, the bracketing/secant search of efix, the adaptive grid walk and its flattening to
// J = 2 regions) runs on the host in FP64, restated from the reference.  Every waveform it needs
// is computed on the device: the reference set and its 22 central-difference neighbours over the
// whole band for the Fisher matrix (one launch), each efix trial point, and the 12 sets of the
// grid walk, whose phase/amplitude ratios are formed on the device as well.
//
// Differences from the reference, on purpose: no diagnostic files (fspace.dat, df.dat,
// df_flat.dat, ratio.dat) and no printing; the grid is copied out before its scratch is released
// (the reference reads it after free, QuickCBC.c:4866-4893).
#include <cuda_runtime.h>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "qcbc_hetspace.h"

namespace qcbc {
namespace {

constexpr int NP = 11;
constexpr double kEtaMin = 0.05;                       // ConstCBC.h:57
constexpr double kTPIr = 6.2831853071795862319959269370884;   // TPI, ConstCBC.h:4
constexpr double kPIr = 3.1415926535897931159979634685442;    // PI, Constants.h:2
constexpr double kEps = 1.0e-5;                        // Fisher_All step, QuickCBC.c:2723

// Final-state fit of the ringdown frequency (Utilities.c:313-360), masses in seconds.
double fqnm(double m1, double m2, double chi1, double chi2) {
  const double p0 = 0.04827, p1 = 0.01707;
  const double k00 = -3.82, k01 = -1.2019, k02 = -1.20764, k10 = 3.79245, k11 = 1.18385, k12 = 4.90494;
  const double scri = 0.41616;
  double q = m1 < m2 ? m1 / m2 : m2 / m1;
  double eta = q / ((1.0 + q) * (1.0 + q));
  double atot = (chi1 + q * q * chi2) / ((1.0 + q) * (1.0 + q));
  double aeff = atot + scri * eta * (chi1 + chi2);
  double Z1 = 1.0 + pow((1.0 - aeff * aeff), (1. / 3.)) * (pow((1. + aeff), (1. / 3.)) + pow((1. - aeff), (1. / 3.)));
  double Z2 = sqrt(3.0 * aeff * aeff + Z1 * Z1);
  double risco = 3.0 + Z2 - (aeff / (fabs(aeff) + 1.0e-20)) * sqrt((3.0 - Z1) * (3.0 + Z1 + 2.0 * Z2));
  double Eisco = sqrt(1.0 - 2. / (3.0 * risco));
  double Lisco = (2. / (3.0 * sqrt(3.))) * (1. + 2.0 * sqrt(3.0 * risco - 2.0));
  double Mf = (1.0 - eta * (1.0 - Eisco) - 4.0 * eta * eta * (4.0 * p0 + 16.0 * p1 * atot * (atot + 1.0) + Eisco - 1.0)) *
              (m1 + m2);
  double af = atot + eta * (Lisco - 2 * atot * (Eisco - 1.0)) + k00 * eta * eta + k01 * eta * eta * aeff +
              k02 * eta * eta * aeff * aeff + k10 * eta * eta * eta + k11 * eta * eta * eta * aeff +
              k12 * eta * eta * eta * aeff * aeff;
  return (1.5251 - 1.1568 * pow((1.0 - af), 0.1292)) / (kTPIr * Mf);
}

// Utilities.c:567-585
double fringdown(const double* p) {
  const double Msun = 1.988546954961461467461011951140572744e30, Tsun = 4.92569043916e-6;
  double Mc = exp(p[0]) / Msun * Tsun, M = exp(p[1]) / Msun * Tsun;
  double eta = pow((Mc / M), (5.0 / 3.0));
  if (eta > 0.25) eta = 0.25;
  double dm = sqrt(1.0 - 4.0 * eta);
  return fqnm(M * (1.0 + dm) / 2.0, M * (1.0 - dm) / 2.0, p[2], p[3]);
}

// Cyclic Jacobi rotations for the symmetric eigenproblem (Golub & Van Loan, Matrix Computations
// 8.5): A is overwritten; V gets the eigenvectors as columns; eigenvalues on the diagonal.
void jacobi_eigen(double (&A)[NP][NP], double (&V)[NP][NP], double* eval) {
  for (int i = 0; i < NP; i++)
    for (int j = 0; j < NP; j++) V[i][j] = i == j ? 1.0 : 0.0;
  for (int sweep = 0; sweep < 100; sweep++) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < NP; i++)
      for (int j = 0; j < NP; j++) {
        tot += A[i][j] * A[i][j];
        if (i != j) off += A[i][j] * A[i][j];
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p + 1 < NP; p++)
      for (int q = p + 1; q < NP; q++) {
        const double apq = A[p][q];
        if (apq == 0.0) continue;
        const double theta = (A[q][q] - A[p][p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < NP; k++) {
          const double akp = A[k][p], akq = A[k][q];
          A[k][p] = c * akp - s * akq;
          A[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < NP; k++) {
          const double apk = A[p][k], aqk = A[q][k];
          A[p][k] = c * apk - s * aqk;
          A[q][k] = s * apk + c * aqk;
        }
        for (int k = 0; k < NP; k++) {
          const double vkp = V[k][p], vkq = V[k][q];
          V[k][p] = c * vkp - s * vkq;
          V[k][q] = s * vkp + c * vkq;
        }
      }
  }
  for (int i = 0; i < NP; i++) eval[i] = A[i][i];
}

// FisherEvec (QuickCBC.c:2449-2530): eigenvalues in ascending |value| as 1-sigma jump sizes
// 1/sqrt(max(value, 10)); ev[i] = eigenvector i.  A vanishing diagonal gives unit directions.
void fisher_evec(const double (&F)[NP][NP], double* ej, double (&ev)[NP][NP]) {
  bool small = false;
  for (int i = 0; i < NP; i++)
    if (fabs(F[i][i]) < 1.0e-16) small = true;
  if (small) {
    for (int i = 0; i < NP; i++) {
      ej[i] = 10000.0;
      for (int j = 0; j < NP; j++) ev[i][j] = i == j ? 1.0 : 0.0;
    }
    return;
  }
  double A[NP][NP], V[NP][NP], val[NP];
  memcpy(A, F, sizeof(A));
  jacobi_eigen(A, V, val);
  for (int i = 0; i + 1 < NP; i++) {            // ascending |value|, columns follow
    int best = i;
    for (int j = i + 1; j < NP; j++)
      if (fabs(val[j]) < fabs(val[best])) best = j;
    if (best != i) {
      std::swap(val[i], val[best]);
      for (int k = 0; k < NP; k++) std::swap(V[k][i], V[k][best]);
    }
  }
  for (int i = 0; i < NP; i++) {
    ej[i] = val[i];
    for (int j = 0; j < NP; j++) ev[i][j] = V[j][i];
  }
  for (int i = 0; i < NP; i++) {
    if (ej[i] < 10.0) ej[i] = 10.0;
    ej[i] = 1.0 / sqrt(ej[i]);
  }
}

// A step from params along direction (eval e_i): sign flipped if it leaves eta <= 1/4, angles
// wrapped, clamped to the prior box, eta kept in [etamin, 0.2499] (QuickCBC.c:4414-4450).
void step_point(const double* params, double a, const double* e, const double* pmin, const double* pmax, double* px) {
  for (int j = 0; j < NP; ++j) px[j] = params[j] + a * e[j];
  double leta = (5.0 / 3.0) * (px[0] - px[1]);
  if (exp(leta) > 0.25)
    for (int j = 0; j < NP; ++j) px[j] = params[j] - a * e[j];
  double x = px[4] / kTPIr;
  px[4] = (x - floor(x)) * kTPIr;
  if (x < 0.0) px[4] += 1.0;
  x = px[7] / kTPIr;
  px[7] = (x - floor(x)) * kTPIr;
  if (x < 0.0) px[7] += 1.0;
  x = px[9] / kPIr;
  px[9] = (x - floor(x)) * kPIr;
  if (x < 0.0) px[9] += 1.0;
  while (px[4] > kTPIr) px[4] -= kTPIr;
  while (px[4] < 0.0) px[4] += kTPIr;
  while (px[7] > kTPIr) px[7] -= kTPIr;
  while (px[7] < 0.0) px[7] += kTPIr;
  while (px[9] > kPIr) px[9] -= kPIr;
  while (px[9] < 0.0) px[9] += kPIr;
  for (int j = 0; j < NP; ++j) if (px[j] > pmax[j]) px[j] = pmax[j];
  for (int j = 0; j < NP; ++j) if (px[j] < pmin[j]) px[j] = pmin[j];
  leta = (5.0 / 3.0) * (px[0] - px[1]);
  const double eta = exp(leta);
  if (eta > 0.25) px[0] = px[1] + 3.0 / 5.0 * log(0.2499);
  if (eta < kEtaMin) px[0] = px[1] + 3.0 / 5.0 * log(kEtaMin);
}

#define HS_CU(x)                                                                   \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) {                                                       \
      err = std::string(#x) + ": " + cudaGetErrorString(e_);                       \
      return -3;                                                                   \
    }                                                                              \
  } while (0)

// Device scratch of the grid searches of one host thread, kept from call to call (grow-only, per
// device).  The Fisher waves alone are (2 NP + 1) nifo N/2 doubles twice, about 290 MB at 128 s and
// 4096 Hz, and allocating and releasing them on every call cost up to a second.  A search ends with
// its stream synchronised, so the next search of the thread may reuse the buffers.  They are
// released with the process.
struct ScratchCache {
  std::vector<void*> p[16];
  std::vector<size_t> cap[16];
};
thread_local ScratchCache tls_scratch;

// Hands out the cached buffers in the order a search asks for them; on every exit path the search's
// stream is drained before the buffers can be handed out again.
struct Scratch {
  int device = 0;
  size_t next = 0;
  cudaStream_t stream;
  explicit Scratch(cudaStream_t s) : stream(s) { cudaGetDevice(&device); }
  ~Scratch() { cudaStreamSynchronize(stream); }
  template <class T>
  cudaError_t alloc(T** out, size_t n) {
    std::vector<void*>& p = tls_scratch.p[device];
    std::vector<size_t>& cap = tls_scratch.cap[device];
    const size_t bytes = n * sizeof(T) > 0 ? n * sizeof(T) : 1;
    if (next == p.size()) {
      p.push_back(nullptr);
      cap.push_back(0);
    }
    if (cap[next] < bytes) {
      cudaFree(p[next]);
      p[next] = nullptr;
      cap[next] = 0;
      cudaError_t e = cudaMalloc(&p[next], bytes);
      if (e != cudaSuccess) return e;
      cap[next] = bytes;
    }
    *out = static_cast<T*>(p[next++]);
    return cudaSuccess;
  }
};

}  // namespace

void fisher_evec_11(const double (&F)[11][11], double* ej, double (&ev)[11][11]) { fisher_evec(F, ej, ev); }

int efix_run(const double* params, const double* pmin, const double* pmax, double* eval, const double (&evec)[11][11],
             double zs, const std::function<int(const double*, double&)>& dist) {
  const double zmx = zs * 2.0, zmn = zs / 2.0;
  double px[NP], e[NP];
  int rc;
  for (int i = 0; i < NP; ++i) {
    double dzmin = 1.0e20, alpham = 1.0, alpha0 = 1.0, z0 = 0.0, z = 0.0;
    for (int j = 0; j < NP; j++) e[j] = eval[i] * evec[i][j];
    int k = 0;
    do {
      step_point(params, alpha0, e, pmin, pmax, px);
      if ((rc = dist(px, z0))) return rc;
      double dz = fabs(z0 - zs);
      if (dz < dzmin) { dzmin = dz; alpham = alpha0; }
      if (z0 < zmn) alpha0 *= 2.0;
      if (z0 > zmx) alpha0 /= 1.9;
      k++;
    } while ((z0 > zmx || z0 < zmn) && k < 15 && fabs(alpha0 < 1.0e4));
    double alpha = alpha0 * 1.1;
    k = 0;
    do {
      step_point(params, alpha, e, pmin, pmax, px);
      if ((rc = dist(px, z))) return rc;
      double alphanew;
      if (alpha > alpha0) alphanew = alpha0 + (zs - z0) / (z - z0) * (alpha - alpha0);
      else alphanew = alpha + (zs - z) / (z0 - z) * (alpha0 - alpha);
      double dz = fabs(z - zs);
      if (dz < dzmin) { dzmin = dz; alpham = alpha; }
      z0 = z;
      alpha0 = alpha;
      alpha = alphanew;
      k++;
    } while (fabs(z - zs) > 0.2 && k < 10 && fabs(alpha < 1.0e4));
    if (dzmin / zs > 1.0) alpham = 0.0;               // kill any failed direction
    eval[i] *= alpham;
  }
  return 0;
}

int het_space_run(const HetSpaceIn& in, const double* params, const double* pmin, const double* pmax,
                  HetSpaceOut& out, std::string& err) {
  const NetGeom& g = in.g;
  const int nifo = g.nifo, N = in.N, N2 = N / 2;
  const double Tobs = in.Tobs;
  const int ss = in.sn_stride;
  cudaStream_t s = in.stream;
  Scratch sc(s);
  double *d_freq, *d_S, *d_par, *d_amp, *d_ph, *d_out;
  PhdRec* d_rec;
  int* d_st;
  const size_t wave_cap = (size_t)(2 * NP + 1) * nifo * N2;     // the Fisher waves are the largest
  HS_CU(sc.alloc(&d_freq, (size_t)N2));
  HS_CU(sc.alloc(&d_S, (size_t)nifo * ss));
  HS_CU(sc.alloc(&d_par, (size_t)(2 * NP + 1) * NP));
  HS_CU(sc.alloc(&d_rec, (size_t)(2 * NP + 1)));
  HS_CU(sc.alloc(&d_st, (size_t)(2 * NP + 1)));
  HS_CU(sc.alloc(&d_amp, wave_cap));
  HS_CU(sc.alloc(&d_ph, wave_cap));
  HS_CU(sc.alloc(&d_out, (size_t)NP * NP));
  HS_CU(cudaMemcpyAsync(d_freq, in.h_freq, sizeof(double) * N2, cudaMemcpyHostToDevice, s));
  HS_CU(cudaMemcpyAsync(d_S, in.h_S, sizeof(double) * nifo * ss, cudaMemcpyHostToDevice, s));
  int launches = 0;

  // waves of `nset` parameter sets (host rows of NP) over n bins into d_amp/d_ph
  auto waves = [&](const double* h_par, int nset, int n, double* amp, double* ph) -> int {
    HS_CU(cudaMemcpyAsync(d_par, h_par, sizeof(double) * NP * nset, cudaMemcpyHostToDevice, s));
    launch_setup(d_par, nset, g, in.qnm, d_rec, d_st, s);
    launch_waves(d_rec, nset, g, d_freq, n, amp, ph, s);
    launches += 2;
    return 0;
  };

  // ---- limits (QuickCBC.c:4275-4385)
  double fstop = 2.0 * fringdown(params);
  if (fstop < 64.0) fstop = 64.0;
  int M = (int)(fstop * Tobs);
  if (M > N2) M = N2;
  if (M < 2) { err = "het_space: signal band below two bins"; return -2; }
  int rc = waves(params, 1, M, d_amp, d_ph);        // the reference set, kept for diff
  if (rc) return rc;
  PhdRec rec0;
  std::vector<double> Ar((size_t)nifo * M);
  HS_CU(cudaMemcpyAsync(&rec0, d_rec, sizeof(PhdRec), cudaMemcpyDeviceToHost, s));
  HS_CU(cudaMemcpyAsync(Ar.data(), d_amp, sizeof(double) * nifo * M, cudaMemcpyDeviceToHost, s));
  HS_CU(cudaStreamSynchronize(s));
  const double fs = rec0.fs;                          // fbegin(params), Utilities.c:587
  const int jmin0 = (in.fmin > fs) ? (int)(Tobs * in.fmin) : (int)(Tobs * fs);
  std::vector<double> SNRsq(M, 0.0), dSNRsq(M, 0.0), ratio((size_t)N2 + 1, 1.0);
  {
    double dx = 0.0;
    for (int j = jmin0; j < M; j++) {
      for (int id = 0; id < nifo; id++) {
        const double a = Ar[(size_t)id * M + j];
        const double x = 4.0 * (a * a) / in.h_S[(size_t)id * ss + j];
        dSNRsq[j] += x;
        dx += x;
      }
      SNRsq[j] = dx;
    }
  }
  int stst0 = jmin0, stst1 = M - 1;
  {
    const double SNRsqT = SNRsq[M - 1];
    bool f1 = false, f2 = false;
    for (int j = jmin0; j < M; j++) {
      if (!f1 && SNRsq[j] > 0.001) { f1 = true; stst0 = j; }
      if (!f2 && SNRsqT - SNRsq[j] < 0.001) { f2 = true; stst1 = j; }
    }
    if (!f2) stst1 = M - 1;
    if (stst0 < jmin0) stst0 = jmin0;
    const double x = SNRsqT / (double)(stst1 - stst0);   // average contribution per significant bin
    for (int j = 1; j < M; j++) {
      const double d = dSNRsq[j] / x;
      ratio[j] = 1.0;
      if (d > 0.0) ratio[j] = 1.0 / d;
    }
  }
  const int MN = stst0, MM = stst1, J = 2;
  const double tol = 0.003;
  if (MM <= MN) { err = "het_space: empty signal band"; return -2; }

  // ---- Fisher_All (QuickCBC.c:2695-2817) and FisherEvec
  double F[NP][NP];
  for (int i = 0; i < NP; i++)
    for (int j = 0; j < NP; j++) F[i][j] = i == j ? 1.0e4 : 0.0;
  if (fabs(params[2]) < 0.9999 && fabs(params[3]) < 0.9999) {
    std::vector<double> P((size_t)(2 * NP + 1) * NP);
    for (int k = 0; k < 2 * NP + 1; k++) memcpy(&P[(size_t)k * NP], params, NP * sizeof(double));
    for (int i = 0; i < NP; i++) {
      P[(size_t)(1 + 2 * i) * NP + i] += kEps;
      P[(size_t)(2 + 2 * i) * NP + i] -= kEps;
    }
    // the reference set's waves over M bins stay in d_amp/d_ph[0..nifo*M); the Fisher waves go after
    double* fa = d_amp + (size_t)nifo * M;
    double* fp = d_ph + (size_t)nifo * M;
    if ((size_t)nifo * M + (size_t)(2 * NP + 1) * nifo * N2 > wave_cap) {
      double *a2, *p2;
      HS_CU(sc.alloc(&a2, (size_t)(2 * NP + 1) * nifo * N2));
      HS_CU(sc.alloc(&p2, (size_t)(2 * NP + 1) * nifo * N2));
      fa = a2;
      fp = p2;
    }
    if ((rc = waves(P.data(), 2 * NP + 1, N2, fa, fp))) return rc;
    int imin = (int)(Tobs * in.fmin), imax = (int)(Tobs * in.fmax);
    if (imax > N2) imax = N2;
    launch_fisher_full(fa, fp, 1, g, N2, d_S, ss, imin, imax, kEps, d_out, s);
    launches += 1;
    double G[NP * NP];
    HS_CU(cudaMemcpyAsync(G, d_out, sizeof(G), cudaMemcpyDeviceToHost, s));
    HS_CU(cudaStreamSynchronize(s));
    for (int i = 0; i < NP; i++)
      for (int j = i; j < NP; j++) F[i][j] = F[j][i] = G[i * NP + j];
  }
  double eval[NP], evec[NP][NP];
  fisher_evec(F, eval, evec);

  // ---- efix (QuickCBC.c:4387-4567), zs = 30, diff on the full grid
  const int imin_d = (in.fmin > fs) ? (int)(Tobs * in.fmin) : (int)(Tobs * fs);
  double* trial_a = d_amp + (size_t)nifo * M;        // one trial set after the reference waves
  double* trial_p = d_ph + (size_t)nifo * M;
  constexpr int kChunks = 148;
  double* d_part;
  HS_CU(sc.alloc(&d_part, (size_t)kChunks));
  auto diff = [&](const double* px, double& z) -> int {
    if ((rc = waves(px, 1, M, trial_a, trial_p))) return rc;
    launch_diff_full(d_amp, d_ph, trial_a, trial_p, 1, g, M, imin_d, M, d_S, ss, kChunks, d_part, s);
    launches += 1;
    double part[kChunks];
    HS_CU(cudaMemcpyAsync(part, d_part, sizeof(part), cudaMemcpyDeviceToHost, s));
    HS_CU(cudaStreamSynchronize(s));
    z = 0.0;
    for (int c = 0; c < kChunks; c++) z += part[c];
    return 0;
  };
  auto dist = [&](const double* px, double& z) -> int { return diff(px, z); };
  rc = efix_run(params, pmin, pmax, eval, evec, 30.0, dist);
  if (rc != 0) return rc;

  // ---- grid walk (QuickCBC.c:4624-4765): the 12 sets' waves, their ratios and the walk on the device
  std::vector<double> P((size_t)(NP + 1) * NP);
  memcpy(P.data(), params, NP * sizeof(double));
  for (int i = 0; i < NP; ++i) {
    double e[NP];
    for (int j = 0; j < NP; j++) e[j] = eval[i] * evec[i][j];
    step_point(params, 1.0, e, pmin, pmax, &P[(size_t)(1 + i) * NP]);
  }
  if ((rc = waves(P.data(), NP + 1, MM, d_amp, d_ph))) return rc;
  const int W = MM - MN, per = NP * nifo;
  double *d_Cs, *d_Sn, *d_DH, *d_ratio;
  int *d_grid, *d_count;
  HS_CU(sc.alloc(&d_Cs, (size_t)per * W));
  HS_CU(sc.alloc(&d_Sn, (size_t)per * W));
  HS_CU(sc.alloc(&d_DH, (size_t)per * W));
  HS_CU(sc.alloc(&d_ratio, ratio.size()));
  HS_CU(sc.alloc(&d_grid, (size_t)W + 2));
  HS_CU(sc.alloc(&d_count, 1));
  HS_CU(cudaMemcpyAsync(d_ratio, ratio.data(), sizeof(double) * ratio.size(), cudaMemcpyHostToDevice, s));
  launch_hs_ratios(d_amp, d_ph, NP + 1, nifo, MM, MN, MM, d_Cs, d_Sn, d_DH, s);
  const int djmax = (int)(100.0 * Tobs);                 // maximum spacing
  launch_hs_walk(d_Cs, d_Sn, d_DH, d_ratio, per, MN, MM, djmax, tol, W + 2, d_grid, d_count, s);
  launches += 2;
  int count = 0;
  HS_CU(cudaMemcpyAsync(&count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s));
  HS_CU(cudaStreamSynchronize(s));
  if (count < 1) { err = "het_space: grid walk did not finish"; return -2; }
  std::vector<int> fgrid((size_t)count);
  HS_CU(cudaMemcpy(fgrid.data(), d_grid, sizeof(int) * count, cudaMemcpyDeviceToHost));
  const int Mr = (int)fgrid.size() - 1;

  // ---- spacing per bin and the flattened grid with J = 2 points per region (QuickCBC.c:4767-4864)
  std::vector<int> dfa((size_t)N2, 100);
  for (int ii = 0; ii < Mr; ii++) {
    const int d = fgrid[ii + 1] - fgrid[ii];
    for (int i = fgrid[ii]; i < fgrid[ii + 1]; ++i) dfa[i] = d;
  }
  {
    const int d = MM - fgrid[Mr];
    for (int i = fgrid[Mr]; i < MM; ++i) dfa[i] = d;
  }
  std::vector<int> fg;
  fg.reserve(1024);
  int j = MN, k = 0, ii = 0;
  fg.push_back(j);
  do {
    int jm = dfa[j];
    bool flag;
    do {
      flag = false;
      k = j + jm * J;
      for (int i = j; i <= k; ++i) {
        if (i < N2) {
          if (dfa[i] < jm) { jm = dfa[i]; flag = true; }
        } else {
          flag = false;
        }
      }
    } while (flag);
    j = k;
    for (int i = 0; i < J; ++i) {
      ii++;
      fg.push_back(fg[ii - 1] + jm);
    }
    if (ii > N2) { err = "het_space: grid does not terminate"; return -2; }
  } while (j < MM);
  {
    const int jm = (MM - fg[ii - J]) / J;                // fix the last section so it ends at MM
    if (jm >= 1) {
      ii -= J;
      for (int i = 0; i < J; ++i) {
        ii++;
        fg[ii] = fg[ii - 1] + jm;
      }
    }
  }
  out.MN = MN;
  out.MM = MM;
  out.J = J;
  out.M = ii + 1;
  out.NR = ii / J;
  out.fgrid.assign(fg.begin(), fg.begin() + out.M);
  out.launches = launches;
  return 0;
}

}  // namespace qcbc
