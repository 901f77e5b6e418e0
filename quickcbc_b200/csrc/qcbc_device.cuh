// Device-side IMRPhenomD and detector projection for the QuickCBC likelihood.
//
// Layout of the work: everything that depends only on one parameter set is
// computed once, in FP64, by qcbc_setup_record() into a PhdRec (about 80
// doubles).  The per-bin evaluators then read the record from shared memory.
//
// Reference behaviour restated here (QuickCBC, file:line):
//   parameter mapping and projection        QuickCBC.c:3698-3771 (fulltemplates)
//                                          QuickCBC.c:3795-3866 (fullphaseamp)
//   IMRPhenomD setup                        IMRPhenomD.c:413-503
//   phenomenological fits (Table V)         IMRPhenomD_internals.c:537-1399
//   amplitude / phase evaluators            IMRPhenomD_internals.c:594-604, 715-726,
//                                           1107-1134, 1222-1240, 1299-1310, 1399-1425,
//                                           1590-1617
//   antenna patterns and geocentre delays   Utilities.c:995-1109
//   start frequency                         Utilities.c:587-629 (fbegin)
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace qcbc {

// ---- constants (IMRPhenomD_internals.h:106-136, Constants.h, ConstCBC.h) ----
constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kPi4 = 0.785398163397448309615660845819875721;
constexpr double kGammaE = 0.577215664901532860606512090082402431;
constexpr double kMsun = 1.988546954961461467461011951140572744e30;
constexpr double kMtsun = 4.925491025543575903411922162094833998e-6;
constexpr double kMrsun = 1.476625061404649406193430731479084713e3;
constexpr double kTsunCBC = 4.92569043916e-6;       // fbegin uses the QuickCBC value
constexpr double kTwoPi = 6.2831853071795862319959269370884;
constexpr double kClight = 299792458.0;
constexpr double kH22fac = 0.31539156525252;
constexpr double kFref = 100.0;
constexpr double kFcut = 0.2;
constexpr double kAmpJoin = 0.014;
constexpr double kPhiJoin = 0.018;
constexpr int kMaxIfo = 3;

// Record flags
constexpr int kRecValid = 1;

// The waveform of one parameter set as the mixed-precision kernel evaluates it at bin i,
// Mf = m i with m = Msec df: every power of m and the factor 1/(2 pi) are folded into
// per-set coefficients (computed in FP64 by the setup), so a bin needs only i, t = i^{1/3},
// u = i^{-1/3}, L = log i and s = i^{3/4} (per-device tables) and no Mf at all.
//   phase in cycles, the three pieces of IMRPhenomD.c:169-186 / internals.c:1540-1584, each
//   minus t0 (Mf - MfRef) + phi_pre, written as the ringdown's linear part R0 + i Ri plus a rest:
//     inspiral      R0 + i Ri + A0 + t (At + t Att) + L (AL + t AtL) + u (Au + u (Auu + u (Au3 + u^2 Au5)))
//                                 + i (Ai + t (Ait + t Aitt) + i Aii)
//     intermediate  R0 + i Ri + B0 + i Bi + u^9 Bu9 + L BL
//     ringdown      R0 + i Ri + Ru3 / i + Rs s + Rat atan(i D1 - D0)
//   The kernel applies R0 + i Ri through its FP64-built rotation tables. The inspiral and
//   intermediate rests are evaluated in FP64; the ringdown rest is a few cycles and is evaluated
//   in FP32, with every coefficient split into a pair hi + lo of floats so that its rounding
//   adds no error that is the same in every bin.
//   amplitude (FP32) relative to a0 (Msec df)^{-7/6} i^{-7/6}, IMRPhenomD_internals.c:576-707:
//     inspiral      1 + t^2 al0 + i (al1 + t (al2 + t al3) + i (al4 + t (al5 + t al6) + i al7))
//     intermediate  Newton form in x = m i - hx1 (nodes hx1, hx1, hx2, hx3, hx3)
//     ringdown      exp(-dfr g2/fg) fg g1 / (dfr^2 + fg^2), dfr = m i - fRD
//   with m, hx1 and fRD as float pairs.
//   iA, iF, iP, iM: first bins of the intermediate amplitude, ringdown amplitude, intermediate
//   phase and ringdown phase (Msec f_i compared with 0.014, fmax, 0.018, fRD/2 in FP64).
//   Each piece's coefficients are 16-byte aligned and ordered as the kernel uses them, so that a
//   bin reads them with 128-bit shared-memory loads: pairs of doubles, quadruples of floats.
struct alignas(16) MixPhIns { double A0, At, Att, AtL, AL, Au, Auu, Au3, Au5, Ai, Ait, Aitt, Aii, pad; };
struct alignas(16) MixPhInt { double B0, Bi, Bu9, BL; };
struct alignas(16) MixPhMrd { double R0, Ri; float Ru3[2], Rs[2], Rat[2], D1[2], D0[2], pad[2]; };
struct alignas(16) MixAmpIns { float al[8]; };
struct alignas(16) MixAmpInt { float m[2], hx1[2]; float hc[5], h21, h31, pad; };
struct alignas(16) MixAmpMrd { float m[2], fRD[2]; float g2_over_fg, fg_g1, fg2, pad; };
struct alignas(16) MixPoly {
  MixPhIns pins;
  MixPhInt pint;
  MixPhMrd pmrd;
  MixAmpIns ains;
  MixAmpInt aint;
  MixAmpMrd amrd;
  int iA, iF, iP, iM;
};

struct PhdRec {
  // dimensional scales
  double Msec, fCut, amp_scale, eta, inv_eta;
  double fRD, fDM, fmax;
  // amplitude
  double a0;           // amp0Func(eta)
  double ai[8];        // inspiral prefactors of Mf^{2/3}, Mf, 4/3, 5/3, 2, 7/3, 8/3, 3
  double g1, g2, g3;   // merger-ringdown
  double hx1, hx2, hx3, hc[5];   // intermediate amplitude, Newton form
  // phase
  double pq[13];       // inspiral phase prefactors
  double b1, b2, b3, al1, al2, al3, al4, al5;
  double C1Int, C2Int, C1MRD, C2MRD, fMRDJoin;
  double t0, MfRef, phi_pre, pi_third;
  // projection
  double fs, ts, sqT;
  double Fs[kMaxIfo], lam[kMaxIfo], td[kMaxIfo];
  // scales of Mf = (Msec df) i for the per-bin tables of the mixed kernel
  double mdf, mdf_third, mdf_rthird, mdf_log, mdf_m76, mdf_34;
  MixPoly mix;
  int i_lo, i_hi;      // bins with f > fbegin and f <= fCut (inclusive), clamped to the band
  int flags, event;    // event: index into the event table (multi-event launches)
};
static_assert(sizeof(PhdRec) % 16 == 0, "records are copied in 16-byte words");

// Table V of arXiv:1508.07253: lambda = l00 + l10 eta + (l01 + l11 eta + l21 eta^2) xi
//   + (l02 + l12 eta + l22 eta^2) xi^2 + (l03 + l13 eta + l23 eta^2) xi^3, xi = chiPN - 1.
enum FitId { F_RHO1, F_RHO2, F_RHO3, F_GAM1, F_GAM2, F_GAM3, F_V2, F_AL1, F_AL2, F_AL3, F_AL4, F_AL5,
             F_BE1, F_BE2, F_BE3, F_SI1, F_SI2, F_SI3, F_SI4, F_COUNT };

// The fit and antenna tables live in qcbc_kernels.cu's constant memory.

// QNM spline table (natural cubic spline over final spin), device global:
// x[n], fring[n], fring''[n], fdamp[n], fdamp''[n]
// bucket[k] = index of the interval holding spin -1 + k/1000 (k = 0..2000), so one or two
// comparisons find the interval instead of a binary search over the table.
struct QnmTable { const double *x, *yr, *mr, *yd, *md; const int* bucket; int n, nbucket; };

struct Pow6 { double sixth, third, two_thirds, four_thirds, five_thirds, two, seven_thirds, eight_thirds; };

// Math routines of the waveform pieces.  The per-bin kernels inline CUDA's routines; the
// setup, which evaluates each piece a few times per record in several warps, calls one
// out-of-line copy of each (MathOutline in qcbc_kernels.cu) to keep its code footprint small.
struct MathInline {
  static __device__ __forceinline__ double pow(double x, double y) { return ::pow(x, y); }
  static __device__ __forceinline__ double exp(double x) { return ::exp(x); }
  static __device__ __forceinline__ double log(double x) { return ::log(x); }
  static __device__ __forceinline__ double atan(double x) { return ::atan(x); }
};

// Powers of x from one x^{1/6} (IMRPhenomD_internals.c:515-533).
template <class M = MathInline>
__device__ __forceinline__ Pow6 pow6(double x) {
  Pow6 p;
  if (x < 0.0) x = 1.0e-10;
  p.sixth = M::pow(x, 1.0 / 6.0);
  p.third = p.sixth * p.sixth;
  p.two_thirds = x / p.third;
  p.four_thirds = x * p.third;
  p.five_thirds = p.four_thirds * p.third;
  p.two = x * x;
  p.seven_thirds = p.third * p.two;
  p.eight_thirds = p.two_thirds * p.two;
  return p;
}

__device__ __forceinline__ int qnm_interval(const QnmTable& t, double s) {
  int lo;
  if (t.bucket) {
    int k = (int)floor((s + 1.0) * 1000.0);
    k = k < 0 ? 0 : (k >= t.nbucket ? t.nbucket - 1 : k);
    lo = __ldg(t.bucket + k);
    for (int it = 0; it < 4 && lo > 0 && __ldg(t.x + lo) > s; it++) lo--;
    for (int it = 0; it < 4 && lo < t.n - 2 && __ldg(t.x + lo + 1) <= s; it++) lo++;
  } else {
    lo = 0;
    int hi = t.n - 1;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (__ldg(t.x + mid) > s) hi = mid; else lo = mid;
    }
  }
  return lo;
}

__device__ __forceinline__ double qnm_eval_at(const QnmTable& t, const double* y, const double* m2, int lo, double s) {
  double xl = __ldg(t.x + lo), h = __ldg(t.x + lo + 1) - xl, dx = s - xl;
  double Ml = __ldg(m2 + lo), Mr = __ldg(m2 + lo + 1), yl = __ldg(y + lo);
  double b = (__ldg(y + lo + 1) - yl) / h - h * (2.0 * Ml + Mr) / 6.0;
  return yl + dx * (b + dx * (0.5 * Ml + dx * (Mr - Ml) / (6.0 * h)));
}

// ------------------------------------------------------------- amplitude
template <class M = MathInline>
__device__ __forceinline__ double amp_mrd(const PhdRec& c, double f) {
  double fg = c.fDM * c.g3, df = f - c.fRD;
  return M::exp(-df * c.g2 / fg) * (fg * c.g1) / (df * df + fg * fg);
}
__device__ __forceinline__ double amp_ins(const PhdRec& c, double Mf, const Pow6& p) {
  return 1.0 + p.two_thirds * c.ai[0] + Mf * c.ai[1] + p.four_thirds * c.ai[2] + p.five_thirds * c.ai[3] +
         p.two * c.ai[4] + p.seven_thirds * c.ai[5] + p.eight_thirds * c.ai[6] + Mf * p.two * c.ai[7];
}
__device__ __forceinline__ double amp_int(const PhdRec& c, double Mf) {
  double x = Mf - c.hx1;
  return c.hc[0] + x * (c.hc[1] + x * (c.hc[2] + (Mf - c.hx2) * (c.hc[3] + (Mf - c.hx3) * c.hc[4])));
}

// ------------------------------------------------------------- phase pieces
template <class M = MathInline>
__device__ __forceinline__ double phi_ins(const PhdRec& c, double Mf, const Pow6& p) {
  double v = p.third * c.pi_third, logv = M::log(v);
  const double* q = c.pq;
  double ph = q[0];
  ph += q[1] * p.two_thirds;
  ph += q[2] * p.third;
  ph += q[3] * logv * p.third;
  ph += q[4] * logv;
  ph += q[5] / p.third;
  ph += q[6] / p.two_thirds;
  ph += q[7] / Mf;
  ph += q[8] / p.five_thirds;
  ph += (q[9] * Mf + q[10] * p.four_thirds + q[11] * p.five_thirds + q[12] * p.two) / c.eta;
  return ph;
}
template <class M = MathInline>
__device__ __forceinline__ double phi_int(const PhdRec& c, double f) {
  return c.b1 * f - c.b3 / (3. * f * f * f) + c.b2 * M::log(f);
}
__device__ __forceinline__ double dphi_int(const PhdRec& c, double f) {
  return (c.b1 + c.b3 / (f * f * f * f) + c.b2 / f) / c.eta;
}
template <class M = MathInline>
__device__ __forceinline__ double phi_mrd(const PhdRec& c, double f) {
  double sq = sqrt(f), f34 = sqrt(f * sq);
  return -(c.al2 / f) + (4.0 / 3.0) * (c.al3 * f34) + c.al1 * f + c.al4 * M::atan((f - c.al5 * c.fRD) / c.fDM);
}
template <class M = MathInline>
__device__ __forceinline__ double dphi_mrd(const PhdRec& c, double f) {
  double x = f - c.al5 * c.fRD;
  return (c.al1 + c.al2 / (f * f) + c.al3 / M::pow(f, 0.25) + c.al4 / (c.fDM * (1 + x * x / (c.fDM * c.fDM)))) / c.eta;
}

// FP64 amplitude (without amp_scale) and phase (with the fRef shift) at geometric frequency Mf.
__device__ __forceinline__ void phd_eval64(const PhdRec& c, double Mf, double& amp, double& phase) {
  Pow6 p = pow6(Mf);
  double pre = c.a0 / (Mf * p.sixth);
  if (Mf < kAmpJoin) amp = pre * amp_ins(c, Mf, p);
  else if (Mf >= c.fmax) amp = pre * amp_mrd(c, Mf);
  else amp = pre * amp_int(c, Mf);
  double ph;
  if (Mf < kPhiJoin) ph = phi_ins(c, Mf, p);
  else if (Mf >= c.fMRDJoin) ph = phi_mrd(c, Mf) * c.inv_eta + c.C1MRD + c.C2MRD * Mf;
  else ph = phi_int(c, Mf) * c.inv_eta + c.C1Int + c.C2Int * Mf;
  phase = ph - (c.t0 * (Mf - c.MfRef) + c.phi_pre);
}

// Reduce x to [-pi, pi] in FP64 with a two-constant 2 pi (|x| < 1e9 keeps it exact to ~1e-15).
__device__ __forceinline__ double reduce_2pi(double x) {
  constexpr double kInv2Pi = 0.15915494309189533577;
  constexpr double kHi = 6.28318530717958623200;      // 2 pi rounded to double
  constexpr double kLo = 2.4492935982947064e-16;      // 2 pi - kHi
  double k = rint(x * kInv2Pi);
  double r = fma(-k, kHi, x);
  return fma(-k, kLo, r);
}

}  // namespace qcbc
