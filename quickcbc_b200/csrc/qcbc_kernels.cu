// CUDA kernels of the QuickCBC likelihood hot path (sm_100a).
//
//   k_setup          one block of 4 warps per 32 parameter sets: IMRPhenomD
//                    coefficients, start/cut-off bins and detector response,
//                    all FP64, the warps working on independent pieces.
//   k_lnl_full<P>    fused waveform -> projection -> PSD-weighted inner
//                    products over one tile of bins of one parameter set; no
//                    h(f) is written to memory.  P = FP64 or mixed.
//   k_finalize_full  fixed-order sum of the tile partials -> lnL, rho.
//   k_lnl_het<P>     heterodyned likelihood, one block per parameter set.
//   waveform kernels for the reference-signature entry points and the FP64
//   heterodyne setup sums.
//
// Reference algorithm: QuickCBC.c:3683-3869 (templates), 4236-4273 (full
// lnL), 5112-5299 (heterodyne), 5303-5444 (heterodyned lnL); Utilities.c
// :587-629, 716-736, 995-1109; IMRPhenomD.c:413-563.
#include "qcbc_kernels.cuh"
#include "qcbc_ptstep.h"
#include <cmath>
#include <cstdio>

namespace qcbc {

// ---------------------------------------------------------------- tables
__constant__ double c_fits[F_COUNT][11] = {
  {3931.8979897196696, -17395.758706812805, 3132.375545898835, 343965.86092361377, -1216256.5819981997, -70698.00600428853, 1383907.177859705, -3966276.1890979446, -60017.52423652596, 803515.1181825735, -2091710.365941658},
  {-40105.47653771657, 112253.0169706701, 23561.696065836168, -3476180.699403351, 11375936.70849482, 754313.1127166454, -13084760.44625268, 36444584.853928134, 596226.612472288, -7427790.1143564405, 18928977.514040343},
  {83208.35471266537, -191237.7264145924, -210916.2454782992, 8717975.08352568, -26914942.420669552, -1988980.6527362722, 30888029.960154563, -83908702.79256162, -1453503.1953446497, 17063528.990822166, -42748659.731120914},
  {0.006927402739328343, 0.03020474290328911, 0.006308024337706171, -0.12074130661131138, 0.26271598905781324, 0.0034151773647198794, -0.10779338611188374, 0.27098966966891747, 0.0007374185938559283, -0.02749621038376281, 0.0733150789135702},
  {1.010344404799477, 0.0008993122007234548, 0.283949116804459, -4.049752962958005, 13.207828172665366, 0.10396278486805426, -7.025059158961947, 24.784892370130475, 0.03093202475605892, -2.6924023896851663, 9.609374464684983},
  {1.3081615607036106, -0.005537729694807678, -0.06782917938621007, -0.6689834970767117, 3.403147966134083, -0.05296577374411866, -0.9923793203111362, 4.820681208409587, -0.006134139870393713, -0.38429253308696365, 1.7561754421985984},
  {0.8149838730507785, 2.5747553517454658, 1.1610198035496786, -2.3627771785551537, 6.771038707057573, 0.7570782938606834, -2.7256896890432474, 7.1140380397149965, 0.1766934149293479, -0.7978690983168183, 2.1162391502005153},
  {43.31514709695348, 638.6332679188081, -32.85768747216059, 2415.8938269370315, -5766.875169379177, -61.85459307173841, 2953.967762459948, -8986.29057591497, -21.571435779762044, 981.2158224673428, -3239.5664895930286},
  {-0.07020209449091723, -0.16269798450687084, -0.1872514685185499, 1.138313650449945, -2.8334196304430046, -0.17137955686840617, 1.7197549338119527, -4.539717148261272, -0.049983437357548705, 0.6062072055948309, -1.682769616644546},
  {9.5988072383479, -397.05438595557433, 16.202126189517813, -1574.8286986717037, 3600.3410843831093, 27.092429659075467, -1786.482357315139, 5152.919378666511, 11.175710130033895, -577.7999423177481, 1808.730762932043},
  {-0.02989487384493607, 1.4022106448583738, -0.07356049468633846, 0.8337006542278661, 0.2240008282397391, -0.055202870001177226, 0.5667186343606578, 0.7186931973380503, -0.015507437354325743, 0.15750322779277187, 0.21076815715176228},
  {0.9974408278363099, -0.007884449714907203, -0.059046901195591035, 1.3958712396764088, -4.516631601676276, -0.05585343136869692, 1.7516580039343603, -5.990208965347804, -0.017945336522161195, 0.5965097794825992, -2.0608879367971804},
  {97.89747327985583, -42.659730877489224, 153.48421037904913, -1417.0620760768954, 2752.8614143665027, 138.7406469558649, -1433.6585075135881, 2857.7418952430758, 41.025109467376126, -423.680737974639, 850.3594335657173},
  {-3.282701958759534, -9.051384468245866, -12.415449742258042, 55.4716447709787, -106.05109938966335, -11.953044553690658, 76.80704618365418, -155.33172948098394, -3.4129261592393263, 25.572377569952536, -54.408036707740465},
  {-2.5156429818799565e-05, 1.9750256942201327e-05, -1.8370671469295915e-05, 2.1886317041311973e-05, 8.250240316860033e-05, 7.157371250566708e-06, -5.5780000112270685e-05, 0.00019142082884072178, 5.447166261464217e-06, -3.220610095021982e-05, 7.974016714984341e-05},
  {2096.551999295543, 1463.7493168261553, 1312.5493286098522, 18307.330017082117, -43534.1440746107, -833.2889543511114, 32047.31997183187, -108609.45037520859, 452.25136398112204, 8353.439546391714, -44531.3250037322},
  {-10114.056472621156, -44631.01109458185, -6541.308761668722, -266959.23419307504, 686328.3229317984, 3405.6372187679685, -437507.7208209015, 1631817.1307344697, -7462.648563007646, -114585.25177153319, 674402.4689098676},
  {22933.658273436497, 230960.00814979506, 14961.083974183695, 1194018.1342318142, -3104223.9693052764, -3038.166617199259, 1872032.2849093592, -7309145.012085539, 42738.22871475411, 467502.018616601, -3064853.498512499},
  {-14621.71522218357, -377812.8579387104, -9608.682631509726, -1710892.5257214056, 4332924.601416521, -22366.683262266528, -2501971.6386377467, 10274495.902259542, -85360.30079034246, -570025.3441737515, 4396844.346849777},
};

// F+ / Fx of H1, L1, V1: the reference's polynomials in cos/sin of psi, delta and
// (alpha - GMST) with its rounded coefficients (Utilities.c:1004-1076), rearranged as dense
// rows over one basis of 21 (F+) and 18 (Fx) monomials shared by the three detectors.
__constant__ double c_antP[3][21] = {
  {0.3104536562, 0.494778091, 1.424276331, -0.4559956644, -0.1552268274, 0.3104536562, -0.1552268276, -0.4928680677, 1.424276334, 0.3104536558, -0.9119913289, -0.9314082637, -0.712138166, 0.9119913288, -0.6209073089, 2.848552667, -0.9895561804, 0.2464340337, -0.9895561811, -0.7121381653, 0.4657041323},
  {-0.5608410611, -0.4945891833, -1.040573095, 0.363231261, 0.2804205304, -0.5608410611, 0.2804205305, -0.3865389475, -1.040573095, -0.5608410611, 0.7264625218, 1.427112041, 0.5202865467, -0.7264625224, 1.121682123, -2.081146187, 0.9891783667, 0.1932694762, 0.9891783666, 0.5202865474, -0.7135560209},
  {0.3963351156, 0.465152434, -1.383399753, -0.3756662059, -0.1981675579, 0.3963351153, -0.1981675578, 1.303555289, -1.383399752, 0.3963351158, -0.7513324118, 0.0798444642, 0.6916998761, 0.7513324118, -0.792670233, -2.766799504, -0.9303048681, -0.6517776444, -0.9303048681, 0.6916998765, -0.039922232}
};
__constant__ double c_antX[3][18] = {
  {-1.424276332, -0.3104536551, -0.6209073087, -0.989556182, 0.3104536561, 0.9895561812, -1.424276332, -0.9119913298, 2.848552668, -0.911991329, 0.9314082638, -1.424276333, -0.1552268276, 0.3104536564, 0.4947780906, -0.3104536556, 0.4928680679, 0.4559956636},
  {1.040573095, 0.5608410611, 1.121682122, 0.9891783668, -0.5608410611, -0.9891783668, 1.040573095, 0.7264625222, -2.081146187, 0.7264625218, -1.427112042, 1.040573094, 0.2804205304, -0.560841061, -0.4945891833, 0.5608410611, 0.3865389466, -0.3632312614},
  {1.383399753, -0.396335116, -0.7926702326, -0.9303048681, 0.3963351158, 0.9303048686, 1.383399752, -0.7513324118, -2.766799505, -0.7513324118, -0.0798444646, 1.383399752, -0.1981675579, 0.3963351158, 0.465152434, -0.3963351158, -1.303555288, 0.3756662059}
};

// detector vertices, metres (Utilities.c:1078-1109)
__constant__ double c_detpos[3][3] = {
  {-2.161414928e6, 3.834695183e6, 4.600350224e6},
  {-74276.04192, 5.496283721e6, 3.224257016e6},
  {4546374.098, -842989.6972, 4378576.963},
};

__device__ __forceinline__ double fit_eval(int k, double eta, double chi) {
  const double* c = c_fits[k];
  double xi = -1 + chi, xi2 = xi * xi, xi3 = xi2 * xi, eta2 = eta * eta;
  return c[0] + c[1] * eta + (c[2] + c[3] * eta + c[4] * eta2) * xi + (c[5] + c[6] * eta + c[7] * eta2) * xi2 +
         (c[8] + c[9] * eta + c[10] * eta2) * xi3;
}

// Frequency-independent constants of the setup: x^{1/6}-powers of pi and of the two fixed join
// frequencies, and the PN quantities at the phase join, computed once on the host with the C
// library exactly as the reference computes them (IMRPhenomD_internals.c:515-533, 1455-1493).
struct SetupConst {
  Pow6 pi6, f1p, fjp;
  double vj[9];        // v^k at v = cbrt(pi * 0.018), k = 0..8
  double logvj;        // log v there
  double log_fj;       // log 0.018
};
__constant__ SetupConst c_setup;

static Pow6 host_pow6(double x) {
  Pow6 p;
  p.sixth = std::pow(x, 1.0 / 6.0);
  p.third = p.sixth * p.sixth;
  p.two_thirds = x / p.third;
  p.four_thirds = x * p.third;
  p.five_thirds = p.four_thirds * p.third;
  p.two = x * x;
  p.seven_thirds = p.third * p.two;
  p.eight_thirds = p.two_thirds * p.two;
  return p;
}

void upload_tables() {
  SetupConst h;
  h.pi6 = host_pow6(kPi);
  h.f1p = host_pow6(kAmpJoin);
  h.fjp = host_pow6(kPhiJoin);
  double v = std::cbrt(kPi * kPhiJoin);
  h.vj[0] = 1.0;
  for (int k = 1; k < 9; k++) h.vj[k] = v * h.vj[k - 1];
  h.logvj = std::log(v);
  h.log_fj = std::log(kPhiJoin);
  cudaMemcpyToSymbol(c_setup, &h, sizeof(h));
}   // tables are statically initialised __constant__ data

// ---------------------------------------------------------------- setup
// The 39 antenna monomials for one sky position / polarisation (straight-line code).
__device__ __forceinline__ void antenna_basis(double cp, double sp, double cd, double sd, double ca, double sa,
                                              double* mp, double* mx) {
  const double cp2 = cp * cp, sd2 = sd * sd, ca2 = ca * ca;
  mp[0] = cp2*ca*sa;
  mp[1] = cd*sd*ca;
  mp[2] = cp2*sd2*ca2;
  mp[3] = cd*sd*sa;
  mp[4] = sd2*ca*sa;
  mp[5] = cp*sp*sd;
  mp[6] = ca*sa;
  mp[7] = cp2*sd2;
  mp[8] = cp2*ca2;
  mp[9] = cp2*sd2*ca*sa;
  mp[10] = cp*sp*cd*ca;
  mp[11] = cp2;
  mp[12] = ca2;
  mp[13] = cp2*cd*sd*sa;
  mp[14] = cp*sp*sd*ca2;
  mp[15] = cp*sp*sd*ca*sa;
  mp[16] = cp2*cd*sd*ca;
  mp[17] = sd2;
  mp[18] = cp*sp*cd*sa;
  mp[19] = sd2*ca2;
  mp[20] = 1.0;
  mx[0] = cp*sp*sd2*ca2;
  mx[1] = cp*sp*ca*sa;
  mx[2] = cp2*sd*ca2;
  mx[3] = cp2*cd*sa;
  mx[4] = sd*ca2;
  mx[5] = cp*sp*cd*sd*ca;
  mx[6] = sd*ca*sa;
  mx[7] = cp2*cd*ca;
  mx[8] = cp2*sd*ca*sa;
  mx[9] = cp*sp*cd*sd*sa;
  mx[10] = cp*sp;
  mx[11] = cp*sp*ca2;
  mx[12] = sd;
  mx[13] = cp2*sd;
  mx[14] = cd*sa;
  mx[15] = cp*sp*sd2*ca*sa;
  mx[16] = cp*sp*sd2;
  mx[17] = cd*ca;
}

// final spin, eq. 3.6 of arXiv:1508.07250
__device__ double final_spin(double eta, double chi1, double chi2) {
  double Seta = sqrt(1.0 - 4.0 * eta), m1 = 0.5 * (1.0 + Seta), m2 = 0.5 * (1.0 - Seta);
  double s = m1 * m1 * chi1 + m2 * m2 * chi2;
  double e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta, s2 = s * s, s3 = s2 * s, s4 = s3 * s;
  return 3.4641016151377544 * eta - 4.399247300629289 * e2 + 9.397292189321194 * e3 - 13.180949901606242 * e4 +
         (1 - 0.0850917821418767 * eta - 5.837029316602263 * e2) * s +
         (0.1014665242971878 * eta - 2.0967746996832157 * e2) * s2 +
         (-1.3546806617824356 * eta + 4.108962025369336 * e2) * s3 +
         (-0.8676969352555539 * eta + 2.064046835273906 * e2) * s4;
}
// radiated energy, eqs. 3.7-3.8 of arXiv:1508.07250
__device__ double erad(double eta, double chi1, double chi2) {
  double Seta = sqrt(1.0 - 4.0 * eta), m1 = 0.5 * (1.0 + Seta), m2 = 0.5 * (1.0 - Seta);
  double m1s = m1 * m1, m2s = m2 * m2, s = (m1s * chi1 + m2s * chi2) / (m1s + m2s);
  double e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta;
  return ((0.055974469826360077 * eta + 0.5809510763115132 * e2 - 0.9606726679372312 * e3 + 3.352411249771192 * e4) *
          (1. + (-0.0030302335878845507 - 2.0066110851351073 * eta + 7.7050567802399215 * e2) * s)) /
         (1. + (-0.6714403054720589 - 1.4756929437702908 * eta + 7.304676214885011 * e2) * s);
}

__device__ double damp_ins_p(const PhdRec& c, double Mf, const Pow6& p) {
  return (2.0 / 3.0) * c.ai[0] / p.third + c.ai[1] + (4.0 / 3.0) * c.ai[2] * p.third +
         (5.0 / 3.0) * c.ai[3] * p.two_thirds + 2.0 * c.ai[4] * Mf + (7.0 / 3.0) * c.ai[5] * p.four_thirds +
         (8.0 / 3.0) * c.ai[6] * p.five_thirds + 3.0 * c.ai[7] * p.two;
}
// d(phi_ins)/dMf at the join Mf = 0.018 from the host-computed powers of v there
__device__ double dphi_ins_join(const PhdRec& c, const double* pv, const double* pvl, double s1, double s2, double s3,
                                double s4, double pi_third, double pi_two_thirds) {
  const double* v = c_setup.vj;
  double logv = c_setup.logvj;
  double D = 0.0;
  D += 2.0 * pv[7] * v[7];
  D += (pv[6] + pvl[6] * (1.0 + logv)) * v[6];
  D += pvl[5] * v[5];
  D += -1.0 * pv[4] * v[4];
  D += -2.0 * pv[3] * v[3];
  D += -3.0 * pv[2] * v[2];
  D += -4.0 * pv[1] * v[1];
  D += -5.0 * pv[0];
  D /= v[8] * 3.0 / kPi;
  D += (s1 + s2 * v[1] / pi_third + s3 * v[2] / pi_two_thirds + (s4 / kPi) * v[3]) / c.eta;
  return D;
}
// phi_ins with log v supplied
__device__ double phi_ins_logv(const PhdRec& c, double Mf, const Pow6& p, double logv) {
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

// One out-of-line copy of each math routine for the setup code (see MathInline).
struct MathOutline {
  static __device__ __noinline__ double pow(double x, double y) { return ::pow(x, y); }
  static __device__ __noinline__ double exp(double x) { return ::exp(x); }
  static __device__ __noinline__ double log(double x) { return ::log(x); }
  static __device__ __noinline__ double atan(double x) { return ::atan(x); }
  static __device__ __noinline__ double atan2(double y, double x) { return ::atan2(y, x); }
  static __device__ __noinline__ double cbrt(double x) { return ::cbrt(x); }
  static __device__ __noinline__ void sincos(double x, double* sv, double* cv) { ::sincos(x, sv, cv); }
};
using MO = MathOutline;

// ---- IMRPhenomD coefficient setup (IMRPhenomD.c:413-503), in pieces.  The serial
// phd_setup below and the cooperative k_setup (four warps per 32 parameter sets) evaluate
// the same expressions; only the compiler's contraction of them may differ (last-bit).

// Validity bits, mass ordering (m1 >= m2), scales.  Masses in Msun.
struct PhdMass { double m1, m2, chi1, chi2, eta, Seta, chi; int st; };
__device__ __forceinline__ PhdMass phd_masses(PhdRec& c, double m1_in, double m2_in, double chi1_in, double chi2_in,
                                              double dist) {
  PhdMass m;
  m.st = kStOK;
  if (!(m1_in > 0.0) || !(m2_in > 0.0)) m.st |= kStBadMass;
  if (!(dist > 0.0)) m.st |= kStBadDist;
  if (!(chi1_in <= 1.0 && chi1_in >= -1.0 && chi2_in <= 1.0 && chi2_in >= -1.0)) m.st |= kStBadSpin;
  m.m1 = m1_in; m.m2 = m2_in; m.chi1 = chi1_in; m.chi2 = chi2_in;
  if (!(m1_in > m2_in)) { m.m1 = m2_in; m.m2 = m1_in; m.chi1 = chi2_in; m.chi2 = chi1_in; }
  c.pi_third = c_setup.pi6.third;
  double M = m.m1 + m.m2, eta = m.m1 * m.m2 / (M * M);
  c.eta = eta; c.inv_eta = 1.0 / eta;
  c.Msec = M * kMtsun;
  c.amp_scale = M * kMrsun * M * kMtsun / dist;
  c.fCut = kFcut / c.Msec;
  m.eta = eta;
  m.Seta = sqrt(1.0 - 4.0 * eta);
  m.chi = (m.chi1 + m.chi2) / 2.0 * (1.0 - eta * 76.0 / 113.0) + m.Seta * ((m.chi1 - m.chi2) / 2.0);
  return m;
}

// Ringdown and damping frequencies from the final spin and radiated energy; returns status bits.
__device__ __forceinline__ int phd_ringdown(PhdRec& c, const PhdMass& m, const QnmTable& q) {
  int st = 0;
  double fsp = final_spin(m.eta, m.chi1, m.chi2);
  if (!(fsp <= 1.0)) { st |= kStBadSpinFinal; fsp = 1.0; }
  if (!(fsp >= -1.0)) fsp = -1.0;
  double er = erad(m.eta, m.chi1, m.chi2);
  int qi = qnm_interval(q, fsp);
  c.fRD = qnm_eval_at(q, q.yr, q.mr, qi, fsp) / (1.0 - er);
  c.fDM = qnm_eval_at(q, q.yd, q.md, qi, fsp) / (1.0 - er);
  return st;
}

// The Table V fits: merger-ringdown amplitude, inspiral amplitude rho_1..3, phase alpha/beta
// into the record; the collocation value v2 and the sigma_1..4 into the outputs.
__device__ __forceinline__ void phd_fits(PhdRec& c, double eta, double chi, double& v2, double* s) {
  c.g1 = fit_eval(F_GAM1, eta, chi); c.g2 = fit_eval(F_GAM2, eta, chi); c.g3 = fit_eval(F_GAM3, eta, chi);
  c.ai[5] = fit_eval(F_RHO1, eta, chi);
  c.ai[6] = fit_eval(F_RHO2, eta, chi);
  c.ai[7] = fit_eval(F_RHO3, eta, chi);
  v2 = fit_eval(F_V2, eta, chi);
  s[0] = fit_eval(F_SI1, eta, chi); s[1] = fit_eval(F_SI2, eta, chi); s[2] = fit_eval(F_SI3, eta, chi);
  s[3] = fit_eval(F_SI4, eta, chi);
  c.b1 = fit_eval(F_BE1, eta, chi); c.b2 = fit_eval(F_BE2, eta, chi); c.b3 = fit_eval(F_BE3, eta, chi);
  c.al1 = fit_eval(F_AL1, eta, chi); c.al2 = fit_eval(F_AL2, eta, chi); c.al3 = fit_eval(F_AL3, eta, chi);
  c.al4 = fit_eval(F_AL4, eta, chi); c.al5 = fit_eval(F_AL5, eta, chi);
}

// a0 and the analytic inspiral amplitude prefactors, Appendix B of arXiv:1508.07253.
__device__ __forceinline__ void phd_amp_prefactors(PhdRec& c, const PhdMass& m) {
  const Pow6 pip = c_setup.pi6;
  double eta = m.eta, Seta = m.Seta;
  c.a0 = (sqrt(2.0 / 3.0) * sqrt(eta)) / pip.sixth;
  double x1 = m.chi1, x2 = m.chi2, x1s = x1 * x1, x2s = x2 * x2, e2 = eta * eta, e3 = eta * e2, Pi = kPi;
  double Pi2 = pip.two;
  c.ai[0] = ((-969 + 1804 * eta) * pip.two_thirds) / 672.;
  c.ai[1] = ((x1 * (81 * (1 + Seta) - 44 * eta) + x2 * (81 - 81 * Seta - 44 * eta)) * Pi) / 48.;
  c.ai[2] = ((-27312085.0 - 10287648 * x2s - 10287648 * x1s * (1 + Seta) + 10287648 * x2s * Seta +
              24 * (-1975055 + 857304 * x1s - 994896 * x1 * x2 + 857304 * x2s) * eta + 35371056 * e2) *
             pip.four_thirds) / 8.128512e6;
  c.ai[3] = (pip.five_thirds * (x2 * (-285197 * (-1 + Seta) + 4 * (-91902 + 1579 * Seta) * eta - 35632 * e2) +
                                x1 * (285197 * (1 + Seta) - 4 * (91902 + 1579 * Seta) * eta - 35632 * e2) +
                                42840 * (-1.0 + 4 * eta) * Pi)) / 32256.;
  c.ai[4] = -(Pi2 * (-336 * (-3248849057.0 + 2943675504 * x1s - 3339284256 * x1 * x2 + 2943675504 * x2s) * e2 -
                     324322727232 * e3 -
                     7 * (-177520268561 + 107414046432 * x2s + 107414046432 * x1s * (1 + Seta) -
                          107414046432 * x2s * Seta + 11087290368 * (x1 + x2 + x1 * Seta - x2 * Seta) * Pi) +
                     12 * eta * (-545384828789 - 176491177632 * x1 * x2 + 202603761360 * x2s +
                                 77616 * x1s * (2610335 + 995766 * Seta) - 77287373856 * x2s * Seta +
                                 5841690624 * (x1 + x2) * Pi + 21384760320 * Pi2))) / 6.0085960704e10;
}

// TaylorF2 phasing incl. aligned-spin terms (IMRPhenomD_internals.c:244-365), minus the 3PN
// spin-spin term PhenomD was not tuned with (IMRPhenomD.c:478); the inspiral phase prefactors
// pq[0..8] follow from it.
__device__ __forceinline__ void phd_taylorf2(PhdRec& c, const PhdMass& m, double* pv, double* pvl) {
  const Pow6 pip = c_setup.pi6;
  double m1 = m.m1, m2 = m.m2, chi1 = m.chi1, chi2 = m.chi2;
  double mt = m1 + m2, d = (m1 - m2) / mt, et = m1 * m2 / mt / mt, m1M = m1 / mt, m2M = m2 / mt;
  double SL = m1M * m1M * chi1 + m2M * m2M * chi2, dSigmaL = d * (m2M * chi2 - m1M * chi1);
  double pfaN = 3.0 / (128.0 * et);
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0}, vl[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  v[0] = 1.0;
  v[2] = 5.0 * (743.0 / 84.0 + 11.0 * et) / 9.0;
  v[3] = -16.0 * kPi;
  v[4] = 5.0 * (3058.673 / 7.056 + 5429.0 / 7.0 * et + 617.0 * et * et) / 72.0;
  v[5] = 5.0 / 9.0 * (7729.0 / 84.0 - 13.0 * et) * kPi;
  vl[5] = 5.0 / 3.0 * (7729.0 / 84.0 - 13.0 * et) * kPi;
  v[6] = (11583.231236531 / 4.694215680 - 640.0 / 3.0 * kPi * kPi - 6848.0 / 21.0 * kGammaE) +
         et * (-15737.765635 / 3.048192 + 2255. / 12. * kPi * kPi) + et * et * 76055.0 / 1728.0 -
         et * et * et * 127825.0 / 1296.0;
  v[6] += (-6848.0 / 21.0) * 1.3862943611198906;     // log 4
  vl[6] = -6848.0 / 21.0;
  v[7] = kPi * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * et - 74045.0 / 756.0 * et * et);
  double sig = et * (721.0 / 48.0 * chi1 * chi2 - 247.0 / 48.0 * chi1 * chi2);
  sig += (720.0 - 1.0) / 96.0 * m1M * m1M * chi1 * chi1;
  sig += (720.0 - 1.0) / 96.0 * m2M * m2M * chi2 * chi2;
  sig -= (240.0 - 7.0) / 96.0 * m1M * m1M * chi1 * chi1;
  sig -= (240.0 - 7.0) / 96.0 * m2M * m2M * chi2 * chi2;
  double ss3 = (326.75 / 1.12 + 557.5 / 1.8 * et) * et * chi1 * chi2;
  ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m1M - 120.0 * m1M * m1M) +
          (-4108.25 / 6.72 - 108.5 / 1.2 * m1M + 125.5 / 3.6 * m1M * m1M)) * m1M * m1M * chi1 * chi1;
  ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m2M - 120.0 * m2M * m2M) +
          (-4108.25 / 6.72 - 108.5 / 1.2 * m2M + 125.5 / 3.6 * m2M * m2M)) * m2M * m2M * chi2 * chi2;
  double gam = (554345.0 / 1134.0 + 110.0 * et / 9.0) * SL + (13915.0 / 84.0 - 10.0 * et / 3.0) * dSigmaL;
  v[7] += (-8980424995.0 / 762048.0 + 6586595.0 * et / 756.0 - 305.0 * et * et / 36.0) * SL -
          (170978035.0 / 48384.0 - 2876425.0 * et / 672.0 - 4735.0 * et * et / 144.0) * dSigmaL;
  v[6] += kPi * (3760.0 * SL + 1490.0 * dSigmaL) / 3.0 + ss3;
  v[5] += -1.0 * gam;
  vl[5] += -3.0 * gam;
  v[4] += -10.0 * sig;
  v[3] += 188.0 * SL / 3.0 + 25.0 * dSigmaL;
  for (int k = 0; k < 8; k++) { pv[k] = v[k] * pfaN; pvl[k] = vl[k] * pfaN; }
  pv[6] -= ss3 * pv[0];
  c.pq[0] = pv[5] - kPi4;
  c.pq[1] = pv[7] * pip.two_thirds;
  c.pq[2] = pv[6] * pip.third;
  c.pq[3] = pvl[6] * pip.third;
  c.pq[4] = pvl[5];
  c.pq[5] = pv[4] / pip.third;
  c.pq[6] = pv[3] / pip.two_thirds;
  c.pq[7] = pv[2] / kPi;
  c.pq[8] = pv[0] / pip.five_thirds;
}
__device__ __forceinline__ void phd_pq_sigma(PhdRec& c, const double* s) {
  c.pq[9] = s[0];
  c.pq[10] = s[1] * 3.0 / 4.0;
  c.pq[11] = s[2] * 3.0 / 5.0;
  c.pq[12] = s[3] / 2.0;
}

// Peak frequency of the merger-ringdown amplitude (needs g1..g3, fRD, fDM).
__device__ __forceinline__ double phd_fmax(const PhdRec& c) {
  if (c.g2 <= 1) return fabs(c.fRD + (c.fDM * (-1 + sqrt(1 - c.g2 * c.g2)) * c.g3) / c.g2);
  return fabs(c.fRD + (c.fDM * (-1) * c.g3) / c.g2);
}

// Intermediate amplitude: quartic with value and slope at f1, value at f2, value and slope at
// f3 (eqs. 21-26 of arXiv:1508.07253), kept in Newton form on nodes f1,f1,f2,f3,f3.
__device__ __forceinline__ void phd_amp_int(PhdRec& c, double v2) {
  double f1 = kAmpJoin, f3 = c.fmax, f2 = f1 + (f3 - f1) / 2.0;
  const Pow6 p1 = c_setup.f1p;
  double v1 = amp_ins(c, f1, p1), d1 = damp_ins_p(c, f1, p1);
  double v3 = amp_mrd<MO>(c, f3);
  double fg3 = c.fDM * c.g3, df3 = f3 - c.fRD;
  double d2 = v3 * (-c.g2 / fg3 - 2.0 * df3 / (df3 * df3 + fg3 * fg3));
  double q01 = d1, q12 = (v2 - v1) / (f2 - f1), q23 = (v3 - v2) / (f3 - f2), q34 = d2;
  double q012 = (q12 - q01) / (f2 - f1), q123 = (q23 - q12) / (f3 - f1), q234 = (q34 - q23) / (f3 - f2);
  double q0123 = (q123 - q012) / (f3 - f1), q1234 = (q234 - q123) / (f3 - f1);
  c.hx1 = f1; c.hx2 = f2; c.hx3 = f3;
  c.hc[0] = v1; c.hc[1] = q01; c.hc[2] = q012; c.hc[3] = q0123; c.hc[4] = (q1234 - q0123) / (f3 - f1);
}

// C^1 join inspiral -> intermediate at Mf = 0.018 (IMRPhenomD_internals.c:1547-1566).
__device__ __forceinline__ void phd_join_int(PhdRec& c, const double* pv, const double* pvl, const double* s) {
  const Pow6 pip = c_setup.pi6;
  double fj = kPhiJoin;
  c.C2Int = dphi_ins_join(c, pv, pvl, s[0], s[1], s[2], s[3], pip.third, pip.two_thirds) - dphi_int(c, fj);
  const Pow6 pj = c_setup.fjp;
  double phi_int_fj = c.b1 * fj - c.b3 / (3. * fj * fj * fj) + c.b2 * c_setup.log_fj;
  c.C1Int = phi_ins_logv(c, fj, pj, c_setup.logvj) - 1.0 / c.eta * phi_int_fj - c.C2Int * fj;
}

// The four phase pieces at the intermediate -> merger-ringdown join Mf = fRD/2.
struct MrdJoin { double phi_int, dphi_int, phi_mrd, dphi_mrd; };
__device__ __forceinline__ MrdJoin phd_mrd_pieces(const PhdRec& c) {
  double fm = 0.5 * c.fRD;
  MrdJoin j;
  j.phi_int = phi_int<MO>(c, fm);
  j.dphi_int = dphi_int(c, fm);
  j.phi_mrd = phi_mrd<MO>(c, fm);
  j.dphi_mrd = dphi_mrd<MO>(c, fm);
  return j;
}
// C^1 join intermediate -> merger-ringdown (IMRPhenomD_internals.c:1568-1584).
__device__ __forceinline__ void phd_join_mrd(PhdRec& c, const MrdJoin& j) {
  double eta = c.eta;
  c.fMRDJoin = 0.5 * c.fRD;
  double fm = c.fMRDJoin;
  double phiT = 1.0 / eta * j.phi_int + c.C1Int + c.C2Int * fm;
  double dphiT = c.C2Int + j.dphi_int;
  c.C2MRD = dphiT - j.dphi_mrd;
  c.C1MRD = phiT - 1.0 / eta * j.phi_mrd - c.C2MRD * fm;
}

// Phase at the reference frequency (IMRPhenomD.c:497-503): the piece that depends on the
// coefficients alone (needs pq, alpha/beta, fRD, fDM), then the join constants added.
__device__ __forceinline__ double phd_phi_ref_raw(const PhdRec& c, int& branch) {
  double Mf = c.MfRef;
  if (Mf < kPhiJoin) { branch = 0; Pow6 pr = pow6<MO>(Mf); return phi_ins<MO>(c, Mf, pr); }
  if (Mf >= 0.5 * c.fRD) { branch = 1; return phi_mrd<MO>(c, Mf); }
  branch = 2;
  return phi_int<MO>(c, Mf);
}
__device__ __forceinline__ void phd_phi_ref(PhdRec& c, double phi0, double raw, int branch) {
  double Mf = c.MfRef, phr;
  if (branch == 0) phr = raw;
  else if (branch == 1) phr = 1.0 / c.eta * raw + c.C1MRD + c.C2MRD * Mf;
  else phr = 1.0 / c.eta * raw + c.C1Int + c.C2Int * Mf;
  c.phi_pre = 2. * phi0 + phr;
}

// Serial setup of one system (used by the amplitude/phase entry point).
__device__ int phd_setup(PhdRec& c, double phi0, double fRef, double m1_in, double m2_in, double chi1_in,
                         double chi2_in, double dist, const QnmTable& q) {
  PhdMass m = phd_masses(c, m1_in, m2_in, chi1_in, chi2_in, dist);
  int st = m.st | phd_ringdown(c, m, q);
  double v2, s[4], pv[8], pvl[8];
  phd_fits(c, m.eta, m.chi, v2, s);
  c.fmax = phd_fmax(c);
  phd_amp_prefactors(c, m);
  phd_amp_int(c, v2);
  phd_taylorf2(c, m, pv, pvl);
  phd_pq_sigma(c, s);
  phd_join_int(c, pv, pvl, s);
  phd_join_mrd(c, phd_mrd_pieces(c));
  c.t0 = dphi_mrd<MO>(c, c.fmax);
  c.MfRef = c.Msec * fRef;
  int br;
  double raw = phd_phi_ref_raw(c, br);
  phd_phi_ref(c, phi0, raw, br);
  c.flags = (st == kStOK) ? kRecValid : 0;
  return st;
}

// ---- parameter set -> record (QuickCBC.c:3698-3755 / 3795-3850)

// start frequency: 3PN inversion of t(f) for time params[5] before merger (Utilities.c:587-629),
// split into the part before and after the log of theta.
struct FbeginHead { double M, eta, chi, th; };
__device__ __forceinline__ FbeginHead fbegin_head(const double* p) {
  FbeginHead h;
  double Mc = MO::exp(p[0]) / kMsun * kTsunCBC, M = MO::exp(p[1]) / kMsun * kTsunCBC;
  double eta = MO::pow(Mc / M, 5.0 / 3.0);
  if (eta > 0.25) eta = 0.25;
  double dm = sqrt(1.0 - 4.0 * eta), m1 = M * (1.0 + dm) / 2.0, m2 = M * (1.0 - dm) / 2.0;
  h.M = M;
  h.eta = eta;
  h.chi = (m1 * p[2] + m2 * p[3]) / M;
  h.th = MO::pow(eta * p[5] / (5.0 * M), -1.0 / 8.0);
  return h;
}
__device__ __forceinline__ double fbegin_tail(const FbeginHead& h, double c1, double c2) {
  const double gE = 0.5772156649;
  double M = h.M, eta = h.eta, chi = h.chi, th = h.th;
  double t2 = th * th, t3 = t2 * th, t4 = t2 * t2, t5 = t2 * t3, t6 = t3 * t3;
  double PN1 = (11.0 / 32.0 * eta + 743.0 / 2688.0) * t2;
  double PN15 = -3.0 * kPi / 10.0 * t3 + (1.0 / 160.0) * (113.0 * chi - 38.0 * eta * (c1 + c2)) * t3;
  double PN2 = (1855099.0 / 14450688.0 + 56975.0 / 258048.0 * eta + 371.0 / 2048.0 * eta * eta) * t4 +
               (1.0 / 14450688.0) * (-3386880.0 * chi * chi + 1512.0 * c1 * c2) * t4;
  double PN25 = -(7729.0 / 21504.0 - 13.0 / 256.0 * eta) * kPi * t5;
  double PN3 = (-720817631400877.0 / 288412611379200.0 + 53.0 / 200.0 * kPi * kPi + 107.0 / 280.0 * gE +
                (25302017977.0 / 4161798144.0 - 451.0 / 2048.0 * kPi * kPi) * eta - 30913.0 / 1835008.0 * eta * eta +
                235925.0 / 1769472.0 * eta * eta * eta + 107.0 / 280.0 * MO::log(2.0 * th)) * t6;
  return t3 / (8.0 * M * kPi) * (1.0 + PN1 + PN15 + PN2 + PN25 + PN3);
}

__device__ __forceinline__ double bin_freq(const NetGeom& g, int i) {
  return g.div_exact ? (double)i * g.df : (double)i / g.Tobs;
}

// Physical inputs of phd_setup from a parameter set (QuickCBC.c:3702-3712).
struct SetPhys { double m1, m2, dist; };
__device__ __forceinline__ SetPhys set_phys(const double* p) {
  double mc = MO::exp(p[0]), mt = MO::exp(p[1]);
  double eta = MO::pow((mc / mt), (5.0 / 3.0));
  double dm = eta > 0.25 ? 0.0 : sqrt(1.0 - 4.0 * eta);
  double m1 = mt * (1.0 + dm) / 2.0, m2 = mt * (1.0 - dm) / 2.0;
  SetPhys s;
  s.m1 = m1 / kMsun;
  s.m2 = m2 / kMsun;
  s.dist = MO::exp(p[6]);
  return s;
}

// Per-detector projection: |F|, polarisation phase lambda, geocentre delay (QuickCBC.c:3724-3750),
// for detectors [id0, id1) of the network.
__device__ __forceinline__ void set_projection(PhdRec& c, const double* p, const NetGeom& g, int id0 = 0,
                                               int id1 = kMaxIfo) {
  double Ap = (1.0 + p[10] * p[10]) / 2.0, Ac = -p[10];
  double cd = sqrt(1.0 - p[8] * p[8]);
  double sa, ca, sps, cps;
  MO::sincos(g.GMST - p[7], &sa, &ca);      // Times() angle; F_ant uses alpha - GMST = -(GMST - alpha)
  MO::sincos(p[9], &sps, &cps);
  double mp[21], mx[18];
  antenna_basis(cps, sps, cd, p[8], ca, -sa, mp, mx);
  for (int id = id0; id < min(id1, g.nifo); id++) {
    int l = g.labels[id];
    double fp = 0.0, fx = 0.0;
#pragma unroll
    for (int k = 0; k < 21; k++) fp += c_antP[l][k] * mp[k];
#pragma unroll
    for (int k = 0; k < 18; k++) fx += c_antX[l][k] * mx[k];
    c.Fs[id] = sqrt(Ap * Ap * fp * fp + Ac * Ac * fx * fx);
    double lam = MO::atan2(Ac * fx, Ap * fp);
    if (lam < 0.0) lam += kTwoPi;
    c.lam[id] = lam;
    double r = c_detpos[l][0] * cd * ca + c_detpos[l][1] * cd * sa + c_detpos[l][2] * p[8];
    c.td[id] = -r / kClight;
  }
}

// Per-detector offsets of the intrinsic parametrisation (QuickCBC.c:3570-3598): detector 0 is
// the reference; detector j > 0 has phase offset p[NX+3(j-1)], time offset p[NX+3(j-1)+1] and
// amplitude ratio p[NX+3(j-1)+2], entering the template x = 2 pi f (ts - td) + pd - phi with
// amplitude Ar h22fac A / sqrt(T) exactly where lambda, td and |F| enter the full template.
__device__ __forceinline__ void set_offsets(PhdRec& c, const double* p, int nifo) {
  c.Fs[0] = 1.0;
  c.lam[0] = 0.0;
  c.td[0] = 0.0;
  for (int j = 1; j < nifo; j++) {
    c.lam[j] = p[kNX + 3 * (j - 1)];
    c.td[j] = p[kNX + 3 * (j - 1) + 1];
    c.Fs[j] = p[kNX + 3 * (j - 1) + 2];
  }
}

// Bins that carry signal: f > fbegin (QuickCBC.c:3758) and f <= fCut (IMRPhenomD.c:530), inside
// the band and inside [1, N/2) (bin N/2 of the template is zero, QuickCBC.c:3754).  The two ends
// are found independently from the band limits.
__device__ __forceinline__ int band_lo(const NetGeom& g) { return g.imin > 1 ? g.imin : 1; }
__device__ __forceinline__ int band_hi(const NetGeom& g) {
  int hi = g.imax - 1;
  if (hi > g.N / 2 - 1) hi = g.N / 2 - 1;
  return hi;
}
__device__ __forceinline__ int first_bin_above(const NetGeom& g, double fs) {
  int lo = band_lo(g), hi = band_hi(g);
  if (fs == fs) {
    double x = fs * g.Tobs;
    if (x >= (double)hi + 1.0) lo = hi + 1;
    else if (x >= (double)lo) {
      int c0 = (int)floor(x) + 1;
      for (int k = 0; k < 3 && c0 - 1 >= lo && bin_freq(g, c0 - 1) > fs; k++) c0--;
      for (int k = 0; k < 3 && c0 <= hi && !(bin_freq(g, c0) > fs); k++) c0++;
      if (c0 > lo) lo = c0;
    }
  } else {
    lo = hi + 1;                                   // NaN start frequency: template is zero
  }
  return lo;
}
__device__ __forceinline__ int last_bin_below(const NetGeom& g, double fCut) {
  int hi = band_hi(g);
  double x = fCut * g.Tobs;
  if (x < (double)hi) {
    int c1 = x < 0.0 ? -1 : (int)floor(x);
    for (int k = 0; k < 3 && c1 + 1 <= hi && bin_freq(g, c1 + 1) <= fCut; k++) c1++;
    for (int k = 0; k < 3 && c1 >= 0 && bin_freq(g, c1) > fCut; k++) c1--;
    if (c1 < hi) hi = c1;
  }
  return hi;
}

// Scales of Mf = (Msec df) i for the per-bin tables of the mixed kernel.
__device__ __forceinline__ void set_mdf(PhdRec& c, const NetGeom& g) {
  c.mdf = c.Msec * g.df;
  c.mdf_third = MO::cbrt(c.mdf);
  c.mdf_rthird = 1.0 / c.mdf_third;
  c.mdf_log = MO::log(c.mdf);
  double sixth = sqrt(c.mdf_third), sq = sqrt(c.mdf);
  c.mdf_m76 = 1.0 / (c.mdf * sixth);
  c.mdf_34 = sqrt(c.mdf * sq);
}

// ---- coefficients of the mixed-precision kernel (MixPoly), from the finished FP64 record
constexpr double kInv2PiD = 0.15915494309189533577;
constexpr double kLnPi = 1.1447298858494002;

// smallest bin i >= 0 with Msec f_i >= X (the comparison the FP64 evaluation makes)
__device__ __forceinline__ int first_bin_mf_at_least(const NetGeom& g, double Msec, double X) {
  double x = X / Msec * g.Tobs;
  if (!(x < 2.0e9)) return 2000000000;
  int i = x <= 0.0 ? 0 : (int)ceil(x);
  for (int k = 0; k < 3 && i > 0 && Msec * bin_freq(g, i - 1) >= X; k++) i--;
  for (int k = 0; k < 3 && !(Msec * bin_freq(g, i) >= X); k++) i++;
  return i;
}

// v as a pair of floats hi + lo (hi = v rounded, lo = the remainder rounded)
__device__ __forceinline__ void split_f2(double v, float (&p)[2]) {
  p[0] = (float)v;
  p[1] = (float)(v - (double)p[0]);
}

// inspiral phase but its constant, and the intermediate / ringdown pieces but the parts that
// need the ringdown join (needs pq, alpha/beta, the intermediate join, t0, the mdf scales)
__device__ __forceinline__ void mix_phase_main(PhdRec& c) {
  MixPoly& P = c.mix;
  const double* q = c.pq;
  const double K = kInv2PiD, T = c.mdf_third, U = c.mdf_rthird, m = c.mdf, ie = c.inv_eta;
  const double third = 1.0 / 3.0, lam3 = (c.mdf_log + kLnPi) * third;
  const double T2 = T * T, U2 = U * U, U3 = U2 * U, U5 = U3 * U2, U9 = U3 * U3 * U3;
  P.pins.At = K * (q[2] * T + q[3] * T * lam3);
  P.pins.Att = K * (q[1] * T2);
  P.pins.AtL = K * (q[3] * T * third);
  P.pins.AL = K * (q[4] * third);
  P.pins.Au = K * (q[5] * U);
  P.pins.Auu = K * (q[6] * U2);
  P.pins.Au3 = K * (q[7] * U3);
  P.pins.Au5 = K * (q[8] * U5);
  P.pins.Ai = K * (ie * q[9] * m - c.t0 * m);
  P.pins.Ait = K * (ie * q[10] * T * m);
  P.pins.Aitt = K * (ie * q[11] * T2 * m);
  P.pins.Aii = K * (ie * q[12] * m * m);
  P.pint.Bi = K * (c.b1 * m * ie + c.C2Int * m - c.t0 * m);
  P.pint.Bu9 = K * (-(c.b3 * third) * U9 * ie);
  P.pint.BL = K * (c.b2 * ie);
  split_f2(K * (-c.al2 * U3 * ie), P.pmrd.Ru3);
  split_f2(K * ((4.0 / 3.0) * c.al3 * c.mdf_34 * ie), P.pmrd.Rs);
  split_f2(K * (c.al4 * ie), P.pmrd.Rat);
  const double rdm = 1.0 / c.fDM;
  split_f2(m * rdm, P.pmrd.D1);
  split_f2(c.al5 * c.fRD * rdm, P.pmrd.D0);
}

// the rest of the phase pieces: constants (phi_pre) and the ringdown slope (C2MRD)
__device__ __forceinline__ void mix_phase_join(PhdRec& c) {
  MixPoly& P = c.mix;
  const double K = kInv2PiD, m = c.mdf, ie = c.inv_eta;
  const double shift = c.t0 * c.MfRef - c.phi_pre;
  P.pmrd.R0 = K * (c.C1MRD + shift);
  P.pmrd.Ri = K * (c.al1 * m * ie + c.C2MRD * m - c.t0 * m);
  P.pins.A0 = K * (c.pq[0] + c.pq[4] * ((c.mdf_log + kLnPi) * (1.0 / 3.0)) + shift) - P.pmrd.R0;
  P.pint.B0 = K * (c.b2 * ie * c.mdf_log + c.C1Int + shift) - P.pmrd.R0;
}

// the inspiral and intermediate slopes relative to the ringdown's (after mix_phase_main and
// mix_phase_join)
__device__ __forceinline__ void mix_phase_slopes(PhdRec& c) {
  c.mix.pins.Ai -= c.mix.pmrd.Ri;
  c.mix.pint.Bi -= c.mix.pmrd.Ri;
}

// FP32 amplitude coefficients (needs ai, the intermediate Newton form, g1..g3, fDM)
__device__ __forceinline__ void mix_amp(PhdRec& c) {
  MixPoly& P = c.mix;
  const double T = c.mdf_third, m = c.mdf, T2 = T * T, m2 = m * m;
  float* al = P.ains.al;
  al[0] = (float)(c.ai[0] * T2);
  al[1] = (float)(c.ai[1] * m);
  al[2] = (float)(c.ai[2] * m * T);
  al[3] = (float)(c.ai[3] * m * T2);
  al[4] = (float)(c.ai[4] * m2);
  al[5] = (float)(c.ai[5] * m2 * T);
  al[6] = (float)(c.ai[6] * m2 * T2);
  al[7] = (float)(c.ai[7] * m2 * m);
  split_f2(m, P.aint.m);
  split_f2(c.hx1, P.aint.hx1);
  P.aint.h21 = (float)(c.hx2 - c.hx1);
  P.aint.h31 = (float)(c.hx3 - c.hx1);
  for (int k = 0; k < 5; k++) P.aint.hc[k] = (float)c.hc[k];
  const double fg = c.fDM * c.g3;
  split_f2(m, P.amrd.m);
  split_f2(c.fRD, P.amrd.fRD);
  P.amrd.g2_over_fg = (float)(c.g2 / fg);
  P.amrd.fg_g1 = (float)(fg * c.g1);
  P.amrd.fg2 = (float)(fg * fg);
}

// ---- cooperative setup: a block of 4 warps builds the records of 32 parameter sets, lane l
// of every warp working on set l.  Each warp takes a different independent piece of the
// record in each of four phases, so the dependency chain of one record is about a third of
// the serial one and the lanes of a warp still run the same code:
//   phase 1  w0 masses/scales        w1 fbegin head, ts      w2 projection, det 0-1   w3 projection, det 2
//                                                            (or detector offsets)
//   phase 2  w0 fRD, fDM             w1 fits, fbegin tail    w2 a0, ai[0..4], mdf, hi w3 TaylorF2, MfRef
//   phase 3  w0 fmax, intermediate,  w1 join int, phi(fRef)  w2 MRD join pieces       w3 t0, bin iP
//            bin iA
//   phase 4  w0 MRD join, phi_pre,   w1 mixed-kernel phase,   w2 mixed-kernel          w3 first bin lo
//            mixed-kernel constants      bin iM                  amplitude, bin iF
// Each piece runs in the first phase whose inputs exist, spread so that the longest warp of each
// phase is as short as the dependencies allow (measured per warp with clock64: the four phases'
// longest pieces went from 7.1k + 11.5k + 7.1k + 7.5k to 6.2k + 8.0k + 7.6k + 4.3k cycles).
struct SetupScratch {
  double p[kMaxParams];
  PhdMass m;
  FbeginHead fb;
  double v2, s[4], pv[8], pvl[8];
  MrdJoin mj;
  double phr_raw;
  int phr_branch, st, hi, live;
};

constexpr int kSetupSets = 32;
constexpr int kSetupThreads = 128;

// geometry of set b: one shared NetGeom, or the event table of a multi-event launch
// stride(model): doubles per parameter set in the launch's parameter array (the same for every set)
struct GeomOne {
  NetGeom g;
  __device__ bool get(int, NetGeom& out, int& e) const { out = g; e = 0; return true; }
  __device__ int stride(int model) const { return param_stride(model, g.nifo); }
};
struct GeomTable {            // multi-event launches: full model only
  const int* event_of;
  const EventDesc* events;
  int n_events;
  __device__ int stride(int) const { return param_stride(kModelFull, kMaxIfo); }
  __device__ bool get(int b, NetGeom& out, int& e) const {
    e = event_of[b];
    if (e < 0 || e >= n_events || events[e].g.nifo == 0) return false;     // out of range or an empty slot
    out = events[e].g;
    return true;
  }
};

// length class of a set of `bins` bins in a band of `band` bins, 0 .. kOrderClasses - 1 (it only
// orders the launch, so its rounding does not matter)
__device__ __forceinline__ int length_class(int bins, int band) {
  return min(kOrderClasses - 1, __float2int_rz((float)bins * ((float)kOrderClasses / (float)max(band, 1))));
}

// ocnt / olist non-null: each set is filed under its length class (SetOrder)
template <class Geom>
__device__ __forceinline__ void setup_coop_block(const double* __restrict__ params, int B, const Geom& geo,
                                                 const QnmTable& q, int tile_bins, PhdRec* __restrict__ recs,
                                                 int* __restrict__ status, int* __restrict__ ntile, int model,
                                                 int* __restrict__ ocnt = nullptr, int* __restrict__ olist = nullptr) {
  __shared__ __align__(16) PhdRec s_rec[kSetupSets];
  __shared__ SetupScratch s_x[kSetupSets];
  __shared__ NetGeom s_g[kSetupSets];
  __shared__ int s_ev[kSetupSets];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int b0 = blockIdx.x * kSetupSets, nb = min(kSetupSets, B - b0);
  const int b = b0 + lane;
  PhdRec& c = s_rec[lane];
  SetupScratch& x = s_x[lane];
  if (w == 0 && lane < nb) {
    NetGeom g;
    int e;
    x.live = geo.get(b, g, e);
    s_g[lane] = g;
    s_ev[lane] = e;
  }
  {
    // The block's parameters are contiguous: every thread loads its share with independent loads
    // (one round trip, also when they are read from mapped host memory), then stores them.
    constexpr int kPer = (kSetupSets * kMaxParams + kSetupThreads - 1) / kSetupThreads;
    const int ps = geo.stride(model), n = nb * ps;
    const double* src = params + (size_t)b0 * ps;
    double v[kPer];
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int i = threadIdx.x + j * kSetupThreads;
      v[j] = i < n ? src[i] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < kPer; j++) {
      const int i = threadIdx.x + j * kSetupThreads;
      if (i < n) s_x[i / ps].p[i - (i / ps) * ps] = v[j];
    }
  }
  __syncthreads();
  const bool on = lane < nb && x.live;
  // phase 1
  if (on) {
    const double* p = x.p;
    if (w == 0) {
      SetPhys ph = set_phys(p);
      x.m = phd_masses(c, ph.m1, ph.m2, p[2], p[3], ph.dist);
    } else if (w == 1) {
      x.fb = fbegin_head(p);
      c.ts = s_g[lane].Tobs - p[5];
      c.sqT = sqrt(s_g[lane].Tobs);
    } else if (w == 2) {
      if (model == kModelIntrinsic) set_offsets(c, p, s_g[lane].nifo);
      else set_projection(c, p, s_g[lane], 0, 2);
    } else if (model != kModelIntrinsic) {
      set_projection(c, p, s_g[lane], 2, kMaxIfo);     // the third detector, if any
    }
  }
  __syncthreads();
  // phase 2
  if (on) {
    const NetGeom& g = s_g[lane];
    if (w == 0) {
      x.st = x.m.st | phd_ringdown(c, x.m, q);
    } else if (w == 1) {
      phd_fits(c, x.m.eta, x.m.chi, x.v2, x.s);
      c.fs = fbegin_tail(x.fb, x.p[2], x.p[3]);
    } else if (w == 2) {
      phd_amp_prefactors(c, x.m);
      set_mdf(c, g);
      x.hi = last_bin_below(g, c.fCut);
    } else {
      phd_taylorf2(c, x.m, x.pv, x.pvl);
      c.MfRef = c.Msec * kFref;
    }
  }
  __syncthreads();
  // phase 3
  if (on) {
    if (w == 0) {
      c.fmax = phd_fmax(c);
      phd_amp_int(c, x.v2);
      c.mix.iA = first_bin_mf_at_least(s_g[lane], c.Msec, kAmpJoin);
    } else if (w == 1) {
      phd_pq_sigma(c, x.s);
      phd_join_int(c, x.pv, x.pvl, x.s);
      x.phr_raw = phd_phi_ref_raw(c, x.phr_branch);
    } else if (w == 2) {
      x.mj = phd_mrd_pieces(c);
    } else {
      c.t0 = dphi_mrd<MO>(c, phd_fmax(c));
      c.mix.iP = first_bin_mf_at_least(s_g[lane], c.Msec, kPhiJoin);
    }
  }
  __syncthreads();
  // phase 4
  if (on && w != 0) {
    if (w == 1) {
      mix_phase_main(c);
      c.mix.iM = first_bin_mf_at_least(s_g[lane], c.Msec, 0.5 * c.fRD);
    } else if (w == 2) {
      mix_amp(c);
      c.mix.iF = first_bin_mf_at_least(s_g[lane], c.Msec, c.fmax);
    } else {
      c.i_lo = first_bin_above(s_g[lane], c.fs);
    }
  }
  if (w == 0 && lane < nb) {
    int st;
    if (on) {
      phd_join_mrd(c, x.mj);
      phd_phi_ref(c, model == kModelIntrinsic ? x.p[4] : 0.5 * x.p[4], x.phr_raw, x.phr_branch);
      mix_phase_join(c);
      st = x.st;
      c.flags = (st == kStOK) ? kRecValid : 0;
      c.i_hi = x.hi;
      c.event = s_ev[lane];
    } else {
      st = kStNoEvent;
      c.flags = 0;
      c.event = -1;
      c.i_lo = 1;
      c.i_hi = 0;
    }
    status[b] = st;
  }
  __syncthreads();
  if (ntile && w == 0 && lane < nb) {  // needs i_lo from warp 3
    const int bins = (c.flags & kRecValid) ? c.i_hi - c.i_lo + 1 : 0;
    ntile[b] = bins > 0 ? (bins + tile_bins - 1) / tile_bins : 0;
  }
  if (ocnt && w == 0) {                // all lanes of warp 0: one global atomic per class present
    int cl = -1;
    if (lane < nb) cl = length_class((c.flags & kRecValid) ? max(0, c.i_hi - c.i_lo + 1) : 0,
                                     s_g[lane].imax - s_g[lane].imin);
    const unsigned peers = __match_any_sync(0xffffffffu, cl);
    const int leader = __ffs(peers) - 1;
    int first = 0;
    if (lane == leader && cl >= 0) first = atomicAdd(ocnt + cl, __popc(peers));
    first = __shfl_sync(0xffffffffu, first, leader);
    const int r = first + __popc(peers & ((1u << lane) - 1u));
    if (cl >= 0 && r < B) olist[(size_t)cl * B + r] = b;   // r >= B only if the counts were not cleared
  }
  if (on && w == 1) mix_phase_slopes(c);   // needs Ri from warp 0
  __syncthreads();
  // the block's records are contiguous in shared and in global memory
  const int4* src = reinterpret_cast<const int4*>(s_rec);
  int4* dst = reinterpret_cast<int4*>(recs + b0);
  const int words = nb * (int)(sizeof(PhdRec) / 16);
  for (int i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
}

// Programmatic dependent launch: a kernel launched with launch_pdl may be scheduled while the
// previous kernel of its stream still runs; pdl_wait() returns once that kernel has finished and
// its writes are visible (immediately for a kernel launched the ordinary way).  A kernel that
// calls pdl_trigger() lets its dependent be scheduled from then on.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <class... KArgs, class... Args>
static void launch_pdl(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, k, args...);
}

__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// One line of the following launch's tables per thread (SetupPrefetch); every address lies inside
// its array.
__device__ __forceinline__ void setup_prefetch(const SetupPrefetch& pf) {
  size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t lines = (pf.bytes + 127) / 128;
  if (t < lines) {
    prefetch_l2(static_cast<const char*>(pf.buf) + t * 128);
    return;
  }
  t -= lines;
  if (t < (size_t)pf.nbins) {
    const int i = pf.bins[t];
    if (i < 0 || i >= pf.tab_n) return;
    if (pf.tabA) prefetch_l2(pf.tabA + i);
    if (pf.tabB) prefetch_l2(pf.tabB + i);
    if (pf.tabC) prefetch_l2(pf.tabC + i);
  }
}

__global__ void __launch_bounds__(kSetupThreads) k_setup(const double* __restrict__ params, int B, NetGeom g,
                                                         QnmTable q, PhdRec* __restrict__ recs,
                                                         int* __restrict__ status, int model, SetOrder o,
                                                         SetupPrefetch pf) {
  pdl_trigger();       // a dependent launch (the lnL kernel) may be scheduled; it waits for this grid
  setup_prefetch(pf);
  GeomOne geo{g};
  setup_coop_block(params, B, geo, q, 1, recs, status, nullptr, model, o.cnt, o.list);
}

void launch_setup(const double* d_params, int B, const NetGeom& g, const QnmTable& q, PhdRec* d_recs,
                  int* d_status, cudaStream_t s, int model, const SetupPrefetch& pf) {
  if (B <= 0) return;
  k_setup<<<(B + kSetupSets - 1) / kSetupSets, kSetupThreads, 0, s>>>(d_params, B, g, q, d_recs, d_status, model,
                                                                      SetOrder{nullptr, nullptr}, pf);
}

void launch_setup_ordered(const double* d_params, int B, const NetGeom& g, const QnmTable& q, PhdRec* d_recs,
                          int* d_status, const SetOrder& o, cudaStream_t s, int model) {
  if (B <= 0) return;
  k_setup<<<(B + kSetupSets - 1) / kSetupSets, kSetupThreads, 0, s>>>(d_params, B, g, q, d_recs, d_status, model, o,
                                                                      SetupPrefetch{});
}

// ---------------------------------------------------------------- reductions
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* [32][NV] */) {
#pragma unroll
  for (int k = 0; k < NV; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  if (lane == 0)
    for (int k = 0; k < NV; k++) smem[w * NV + k] = v[k];
  __syncthreads();
  if (w == 0) {
    for (int k = 0; k < NV; k++) {
      double x = lane < nw ? smem[lane * NV + k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
      v[k] = x;
    }
  }
}

__device__ __forceinline__ void kahan_add(float& s, float& comp, float x) {
  float y = x - comp;
  float t = s + y;
  comp = (t - s) - y;
  s = t;
}

// ---------------------------------------------------------------- full lnL: one tile of bins
// A block accumulates, per detector, SD = sum amp (wr cos x + wi sin x) and SH = sum amp^2 ws over
// bins [i0, i1] of one parameter set (wr/wi/ws carry 4/S and the event scale sigma); the finaliser
// applies the per-detector factor K = Fs h22fac amp_scale / sqrt(T) / sigma:
//   <d|h> = K SD,  <h|h> = K^2 SH   (QuickCBC.c:4258-4266, Utilities.c:716-736).
// Results land in acc[2*NIFO] of every thread (summed over the block by the caller).

// FP64 form: IMRPhenomD evaluated bin by bin as the reference does.
template <int NIFO>
__device__ __forceinline__ void tile_fp64(const PhdRec& c, const NetGeom& g, const EventData& ev, int i0, int i1,
                                          double* acc) {
  const size_t nh = (size_t)ev.nh;
  for (int i = i0 + threadIdx.x; i <= i1; i += blockDim.x) {
    double f = bin_freq(g, i);
    double Mf = c.Msec * f;
    double amp, ph;
    phd_eval64(c, Mf, amp, ph);
#pragma unroll
    for (int id = 0; id < NIFO; id++) {
      // x = 2 pi f (ts - td) + lambda - phi, evaluated in the reference's order
      double x = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, f), c.ts - c.td[id]), c.lam[id]), -ph);
      double sx, cx;
      sincos(reduce_2pi(x), &sx, &cx);
      const double* w = ev.w64 + (size_t)id * 3 * nh;
      double wr = __ldg(w + i), wi = __ldg(w + nh + i), ws = __ldg(w + 2 * nh + i);
      acc[2 * id] += amp * (wr * cx + wi * sx);
      acc[2 * id + 1] += amp * amp * ws;
    }
  }
}

// Mixed form.  Per bin i (f = i df, Mf = Msec f), with the phase written as the ringdown's linear
// part R0 + i Ri plus a rest (MixPoly):
//  * the rest of the inspiral and intermediate pieces in FP64 from per-bin tables:
//    Mf^{1/3} = (Msec df)^{1/3} i^{1/3}, Mf^{-1/3} likewise, log Mf = log(Msec df) + log i,
//    reduced to one cycle in FP64; the rest of the ringdown piece (a few cycles) in FP32 from
//    1/i and i^{3/4}; then one FP32 sincos gives e^{-2 pi i rest};
//  * detector rotation and linear phase e^{2 pi i (f (ts - td) + lambda/2pi - R0 - i Ri)}
//    = base(thread) x R[k] with a per-tile FP32 table R[k] = e^{2 pi i k blockDim (df (ts - td) - Ri)},
//    both built in FP64;
//  * amplitude in FP32 without the constant a0 (Msec df)^{-7/6} (applied in FP64 by the finaliser);
//  * FP32 partial sums over 16 bins, accumulated in FP64.
// ---- mixed-precision tile body (coefficients: MixPoly in the record)

// The piece coefficients of a parameter set stay in shared memory (the block's record) and are
// re-read at every use, 128 bits at a time: asm volatile keeps each load in the bin loop, so the
// coefficients pin no registers and three blocks of 256 threads fit an SM (80 registers per
// thread).  Every address is 16-byte aligned (the MixPoly pieces are).
__device__ __forceinline__ double2 sld2(const double* x) {
  double2 v;
  asm volatile("ld.shared.v2.f64 {%0, %1}, [%2];" : "=d"(v.x), "=d"(v.y) : "r"((uint32_t)__cvta_generic_to_shared(x)));
  return v;
}
__device__ __forceinline__ float4 sld4(const float* x) {
  float4 v;
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "r"((uint32_t)__cvta_generic_to_shared(x)));
  return v;
}

// the three phase pieces in cycles (FP64) and the three amplitude pieces (FP32) at bin xi
__device__ __forceinline__ double mph_ins(const MixPhIns& q, double xi, double t, double u, double L) {
  const double2 c0 = sld2(&q.A0), c1 = sld2(&q.Att), c2 = sld2(&q.AL), c3 = sld2(&q.Auu), c4 = sld2(&q.Au5),
                c5 = sld2(&q.Ait), c6 = sld2(&q.Aii);
  // c0 = (A0, At), c1 = (Att, AtL), c2 = (AL, Au), c3 = (Auu, Au3), c4 = (Au5, Ai), c5 = (Ait, Aitt), c6 = (Aii, -)
  double ph = fma(t, fma(t, c1.x, c0.y), c0.x);
  ph = fma(L, fma(t, c1.y, c2.x), ph);
  double pu = fma(u * u, c4.x, c3.y);
  pu = fma(u, pu, c3.x);
  pu = fma(u, pu, c2.y);
  ph = fma(u, pu, ph);
  const double pi = fma(xi, c6.x, fma(t, fma(t, c5.y, c5.x), c4.y));
  return fma(xi, pi, ph);
}
__device__ __forceinline__ double mph_int(const MixPhInt& q, double xi, double u, double L) {
  const double2 c0 = sld2(&q.B0), c1 = sld2(&q.Bu9);     // (B0, Bi), (Bu9, BL)
  const double u3 = u * u * u;
  return fma(xi, c0.y, c0.x) + fma(L, c1.y, (u3 * u3 * u3) * c1.x);
}
// the ringdown rest in FP32 (cycles, a few at most): Ru3 / i + Rs s + Rat atan(i D1 - D0) with
// tc = (1/i, s = i^{3/4}); each coefficient is a float pair applied hi after lo
__device__ __forceinline__ float mph_mrd(const MixPhMrd& q, float xf, float2 tc) {
  const float4 a = sld4(q.Ru3), b = sld4(q.Rat), d = sld4(q.D0);   // (Ru3, Rs), (Rat, D1), (D0, -)
  const float z = fmaf(xf, b.z, fmaf(xf, b.w, -d.x)) - d.y;
  const float at = atanf(z);
  float ph = fmaf(at, b.x, at * b.y);
  ph = fmaf(tc.y, a.z, fmaf(tc.y, a.w, ph));
  return fmaf(tc.x, a.x, fmaf(tc.x, a.y, ph));
}
// x minus the nearest integer, for |x| < 2^22, in FP32 adds
__device__ __forceinline__ float frac_cyc(float x) {
  return __fsub_rn(x, __fsub_rn(__fadd_rn(x, 12582912.0f), 12582912.0f));
}
__device__ __forceinline__ float mamp_ins(const MixAmpIns& a, float xf, float tf) {
  const float4 l = sld4(a.al), h = sld4(a.al + 4);
  const float inner = fmaf(xf, h.w, fmaf(tf, fmaf(tf, h.z, h.y), h.x));
  const float mid = fmaf(xf, inner, fmaf(tf, fmaf(tf, l.w, l.z), l.y));
  return fmaf(xf, mid, fmaf(tf * tf, l.x, 1.0f));
}
__device__ __forceinline__ float mamp_int(const MixAmpInt& a, float xf) {
  const float4 s = sld4(a.m), c = sld4(a.hc), e = sld4(a.hc + 4);   // (m, hx1), hc[0..3], (hc[4], h21, h31, -)
  const float x = fmaf(xf, s.x, fmaf(xf, s.y, -s.z)) - s.w;
  return c.x + x * (c.y + x * (c.z + (x - e.y) * (c.w + (x - e.z) * e.x)));
}
__device__ __forceinline__ float mamp_mrd(const MixAmpMrd& a, float xf) {
  const float4 s = sld4(a.m), g = sld4(&a.g2_over_fg);   // (m, fRD), (g2/fg, fg g1, fg^2, -)
  const float dfr = fmaf(xf, s.x, fmaf(xf, s.y, -s.z)) - s.w;
  return __fdividef(__expf(-dfr * g.x) * g.y, dfr * dfr + g.z);
}

// piece of bin i: 0 inspiral, 1 intermediate, 2 merger-ringdown
__device__ __forceinline__ int amp_piece(const MixPoly& P, int i) { return i < P.iA ? 0 : (i >= P.iF ? 2 : 1); }
__device__ __forceinline__ int ph_piece(const MixPoly& P, int i) { return i < P.iP ? 0 : (i >= P.iM ? 2 : 1); }

// The FP32 weighted data (wr', wi', ws') of NIFO detectors at bin b from the event's planes
// (EventData::wm): three loads for three detectors, two for one or two.
template <int NIFO>
struct MixW {
  float r[NIFO], i[NIFO], s[NIFO];
  __device__ __forceinline__ void load(const float* __restrict__ wm, size_t nh, int b) {
    if (NIFO == 3) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(wm) + b);
      const float4 c = __ldg(reinterpret_cast<const float4*>(wm + 4 * nh) + b);
      const float d = __ldg(wm + 8 * nh + b);
      r[0] = a.x; i[0] = a.y; r[1 % NIFO] = a.z; i[1 % NIFO] = a.w;
      r[2 % NIFO] = c.x; i[2 % NIFO] = c.y; s[0] = c.z; s[1 % NIFO] = c.w; s[2 % NIFO] = d;
    } else if (NIFO == 2) {
      const float4 a = __ldg(reinterpret_cast<const float4*>(wm) + b);
      const float2 c = __ldg(reinterpret_cast<const float2*>(wm + 4 * nh) + b);
      r[0] = a.x; i[0] = a.y; r[1 % NIFO] = a.z; i[1 % NIFO] = a.w; s[0] = c.x; s[1 % NIFO] = c.y;
    } else {
      const float2 a = __ldg(reinterpret_cast<const float2*>(wm) + b);
      r[0] = a.x; i[0] = a.y; s[0] = __ldg(wm + 2 * nh + b);
    }
  }
};

// FP32 partial sums of up to 16 bins per detector: S = sum (wr' - i wi') R_k a e^{-i phi} and
// sum a^2 ws' (a the amplitude without its bin factor i^{-7/6}, which the weighted data carry);
// flushed into the FP64 accumulators with the thread's rotation base applied, so that
// acc[2 id] = sum amp (wr cos x + wi sin x), x = 2 pi f (ts - td) + lambda - phi.
// bins of one thread summed in FP32 between flushes into its FP64 sums
constexpr int kMixFlushBins = 16;

// Row stride (float2 entries) of the rotation table, whose row k holds R_k of every detector:
// padded to 4 at three detectors so that a row is two aligned loads.
__host__ __device__ constexpr int mix_rs(int nifo) { return nifo == 1 ? 1 : (nifo == 2 ? 2 : 4); }

template <int NIFO>
struct MixAcc {
  float sx[NIFO], sy[NIFO], sh[NIFO];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int id = 0; id < NIFO; id++) { sx[id] = 0.f; sy[id] = 0.f; sh[id] = 0.f; }
  }
  __device__ __forceinline__ void add(float amp, float cyc, const MixW<NIFO>& w, const float2* rot) {
    float sw, cw;
    __sincosf(6.28318530717958648f * cyc, &sw, &cw);     // |argument| <= pi
    const float ex = amp * cw, ey = -amp * sw, amp2 = amp * amp;
    float2 Rr[NIFO];                 // this row's rotations: one 128-bit load for detectors 0 and 1
    if (NIFO >= 2) {
      const float4 q = *reinterpret_cast<const float4*>(rot);
      Rr[0] = make_float2(q.x, q.y);
      Rr[1 % NIFO] = make_float2(q.z, q.w);
      if (NIFO == 3) Rr[2 % NIFO] = rot[2];
    } else {
      Rr[0] = rot[0];
    }
#pragma unroll
    for (int id = 0; id < NIFO; id++) {
      const float2 R = Rr[id];
      const float qx = fmaf(R.x, ex, -R.y * ey), qy = fmaf(R.x, ey, R.y * ex);
      sx[id] = fmaf(w.r[id], qx, fmaf(w.i[id], qy, sx[id]));
      sy[id] = fmaf(w.r[id], qy, fmaf(-w.i[id], qx, sy[id]));
      sh[id] = fmaf(amp2, w.s[id], sh[id]);
    }
  }
  template <class State>
  __device__ __forceinline__ void flush(State& S) {
#pragma unroll
    for (int id = 0; id < NIFO; id++) {
      const float2 bs = S.base(id);
      S.acc(2 * id) += (double)(bs.x * sx[id] - bs.y * sy[id]);
      S.acc(2 * id + 1) += (double)sh[id];
    }
  }
};

// The mixed kernels keep a thread's rotation base and FP64 sums in its column of two shared-memory
// arrays rather than in registers: 18 registers fewer at three detectors, so that four blocks of
// 256 threads fit an SM (64 registers; 157.7 us against 165.9 us at three blocks for the config-2
// launch).
struct MixSmemState {
  float2* b;     // [NIFO][st], this thread's column
  double* a;     // [2 NIFO][st]
  int st;
  __device__ __forceinline__ float2& base(int id) { return b[id * st]; }
  __device__ __forceinline__ double& acc(int k) { return a[k * st]; }
};

// Rows [k, k_end) of the thread's bins i = i0 + tid + k bs, all in amplitude piece AP and
// phase piece PP (-1: decided per bin).  The pieces' coefficients are read from the block's
// record in shared memory at each use.
template <int NIFO, int AP, int PP, class State>
__device__ __forceinline__ void mixed_rows(const MixPoly& P, const EventData& ev, const float2* s_rot,
                                           State& S, int k, int k_end, int i, int i1, int bs) {
  if (i > i1) return;
  const int n = min(k_end - k, (i1 - i) / bs + 1);     // rows of this thread in the run
  const MixPhIns& qi = P.pins;      // in shared memory, read per use (sld)
  const MixPhInt& qn = P.pint;
  const MixPhMrd& qm = P.pmrd;
  const MixAmpIns& ai = P.ains;
  const MixAmpInt& an = P.aint;
  const MixAmpMrd& am = P.amrd;
  const size_t nh = (size_t)ev.nh;
  constexpr int RS = mix_rs(NIFO);
  const float2* pr = s_rot + (size_t)k * RS;
  const double dbs = (double)bs;
  const float fbs = (float)bs;
  double xi = (double)i;
  float xf = (float)i;
  int b = i;
  // tables a row needs: tabA for the inspiral amplitude and the FP64 phase pieces, tabB for the
  // FP64 phase pieces, tabC for the ringdown phase
  constexpr bool kTabA = AP <= 0 || PP != 2, kTabB = PP != 2, kTabC = PP == 2 || PP < 0;
  for (int r = 0; r < n; r += kMixFlushBins) {
    const int m = min(kMixFlushBins, n - r);
    MixAcc<NIFO> A;
    A.zero();
#pragma unroll 1
    for (int j = 0; j < m; j++) {
      double2 tA = make_double2(0.0, 0.0), tB = make_double2(0.0, 0.0);
      float2 tC = make_float2(0.f, 0.f);
      if (kTabA) tA = __ldg(ev.tabA + b);
      if (kTabB) tB = __ldg(ev.tabB + b);
      if (kTabC) tC = __ldg(ev.tabC + b);
      MixW<NIFO> w;
      w.load(ev.wm, nh, b);
      float cyc, a;
      if (PP == 2) {
        cyc = frac_cyc(mph_mrd(qm, xf, tC));
      } else if (PP >= 0) {
        const double ph = PP == 0 ? mph_ins(qi, xi, tA.x, tA.y, tB.x) : mph_int(qn, xi, tA.y, tB.x);
        cyc = (float)(ph - rint(ph));
      } else {
        const int pp = ph_piece(P, b);
        if (pp == 2) {
          cyc = frac_cyc(mph_mrd(P.pmrd, xf, tC));
        } else {
          const double ph = pp == 0 ? mph_ins(P.pins, xi, tA.x, tA.y, tB.x) : mph_int(P.pint, xi, tA.y, tB.x);
          cyc = (float)(ph - rint(ph));
        }
      }
      if (AP == 0) a = mamp_ins(ai, xf, (float)tA.x);
      else if (AP == 1) a = mamp_int(an, xf);
      else if (AP == 2) a = mamp_mrd(am, xf);
      else {
        const int ap = amp_piece(P, b);
        a = ap == 0 ? mamp_ins(P.ains, xf, (float)tA.x)
                    : (ap == 1 ? mamp_int(P.aint, xf) : mamp_mrd(P.amrd, xf));
      }
      A.add(a, cyc, w, pr);
      b += bs;
      pr += RS;
      xi += dbs;
      xf += fbs;
    }
    A.flush(S);
  }
}

__device__ __forceinline__ int mixed_table_len(int i0, int i1, int bs) {
  return i1 >= i0 ? (i1 - i0 + bs) / bs : 0;
}

// Builds the rotation table (shared), then runs the bin loop in runs of rows that share their
// waveform pieces.  The tile is walked by bs threads (tid = 0..bs-1).  Contains
// __syncthreads(): every thread of the block must call it.
template <int NIFO, class State>
__device__ __forceinline__ void tile_mixed(const PhdRec& c, const NetGeom& g, const EventData& ev, int i0, int i1,
                                           int tid, int bs, float2* s_rot, State& S) {
  const int nk = mixed_table_len(i0, i1, bs);
  constexpr double kInv2Pi = 0.15915494309189533577;
  const double Dstep = (double)bs * g.df;
  const double Ri = c.mix.pmrd.Ri, R0 = c.mix.pmrd.R0;    // the phase's linear part R0 + i Ri
  for (int k = tid; k < nk; k += bs) {
#pragma unroll
    for (int id = 0; id < NIFO; id++) {
      double cyc = (double)k * (Dstep * (c.ts - c.td[id]) - (double)bs * Ri);
      float sv, cv;                  // reduced to one cycle in FP64, the rotation itself in FP32
      sincospif(2.0f * (float)(cyc - rint(cyc)), &sv, &cv);
      s_rot[k * mix_rs(NIFO) + id] = make_float2(cv, sv);
    }
  }
  __syncthreads();
  int i = i0 + tid;
  if (i > i1) return;
  double f = g.div_exact ? (double)i * g.df : (double)i / g.Tobs;
#pragma unroll
  for (int id = 0; id < NIFO; id++) {
    double cyc = f * (c.ts - c.td[id]) + c.lam[id] * kInv2Pi - fma((double)i, Ri, R0);
    float sv, cv;
    sincospif(2.0f * (float)(cyc - rint(cyc)), &sv, &cv);
    S.base(id) = make_float2(cv, sv);
  }
  const MixPoly& P = c.mix;
  int k = 0;
  while (k < nk) {                 // block-uniform: depends on k only
    const int r0 = i0 + k * bs, r1 = min(r0 + bs - 1, i1);
    if (r0 > i1) break;
    const int a0 = amp_piece(P, r0), p0 = ph_piece(P, r0);
    int k_end;
    if (a0 != amp_piece(P, r1) || p0 != ph_piece(P, r1)) {
      k_end = k + 1;
      mixed_rows<NIFO, -1, -1>(P, ev, s_rot, S, k, k_end, i, i1, bs);
    } else {
      int nxt = i1 + 1;              // the pieces can only change at a threshold
      if (P.iA > r0 && P.iA < nxt) nxt = P.iA;
      if (P.iF > r0 && P.iF < nxt) nxt = P.iF;
      if (P.iP > r0 && P.iP < nxt) nxt = P.iP;
      if (P.iM > r0 && P.iM < nxt) nxt = P.iM;
      k_end = nxt > i1 ? nk : max(k + 1, (nxt - i0 - bs) / bs + 1);
      switch (a0 * 3 + p0) {
        case 0: mixed_rows<NIFO, 0, 0>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 1: mixed_rows<NIFO, 0, 1>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 2: mixed_rows<NIFO, 0, 2>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 3: mixed_rows<NIFO, 1, 0>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 4: mixed_rows<NIFO, 1, 1>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 5: mixed_rows<NIFO, 1, 2>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 6: mixed_rows<NIFO, 2, 0>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        case 7: mixed_rows<NIFO, 2, 1>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
        default: mixed_rows<NIFO, 2, 2>(P, ev, s_rot, S, k, k_end, i, i1, bs); break;
      }
    }
    k = k_end;
    i = i0 + tid + k * bs;
  }
}

// rotation-table entries per detector that a block of a launch needs: ceil(max bins per tile /
// threads) + 1
__host__ __device__ __forceinline__ int mixed_nk_cap(int band, int tiles, int threads) {
  const int bins = band > 1 ? band : 1;
  const int chunk = (bins + tiles - 1) / tiles;
  return (chunk + threads - 1) / threads + 1;
}

// tile_mixed with the thread's state in shared memory after the rotation table (nk_cap entries for
// each of nifo_cap detectors): the thread's column of base [nifo_cap][threads] float2 and of
// sums [2 nifo_cap][threads] double (threads x nifo_cap x 24 bytes).  acc[0 .. 2 NIFO) receives
// the thread's FP64 sums.
template <int NIFO>
__device__ __forceinline__ void tile_mixed_smem(const PhdRec& c, const NetGeom& g, const EventData& ev, int i0, int i1,
                                                float2* s_rot, int nk_cap, int nifo_cap, double* acc) {
  float2* s_base = s_rot + (size_t)mix_rs(nifo_cap) * nk_cap;
  double* s_acc = reinterpret_cast<double*>(s_base + (size_t)nifo_cap * blockDim.x);
  MixSmemState S{s_base + threadIdx.x, s_acc + threadIdx.x, (int)blockDim.x};
#pragma unroll
  for (int k = 0; k < 2 * NIFO; k++) S.acc(k) = 0.0;
  tile_mixed<NIFO>(c, g, ev, i0, i1, threadIdx.x, blockDim.x, s_rot, S);
#pragma unroll
  for (int k = 0; k < 2 * NIFO; k++) acc[k] = S.acc(k);
}

// bytes of shared memory a mixed block keeps its threads' state in (tile_mixed_smem)
__host__ __device__ __forceinline__ size_t mixed_state_bytes(int threads, int nifo) {
  return (size_t)threads * nifo * (sizeof(float2) + 2 * sizeof(double));
}

__device__ __forceinline__ void load_record(PhdRec& dst, const PhdRec* src) {
  const int nw = sizeof(PhdRec) / 8;
  const double* s = reinterpret_cast<const double*>(src);
  double* d = reinterpret_cast<double*>(&dst);
  for (int k = threadIdx.x; k < nw; k += blockDim.x) d[k] = s[k];
}

__device__ __forceinline__ void tile_range(const PhdRec& c, int tiles, int t, int& i0, int& i1) {
  i0 = 0;
  i1 = -1;
  if (c.flags & kRecValid) {
    int n = c.i_hi - c.i_lo + 1;
    if (n > 0) {
      int chunk = (n + tiles - 1) / tiles;
      i0 = c.i_lo + t * chunk;
      i1 = min(i0 + chunk - 1, c.i_hi);
    }
  }
}

// lnL (and rho, or the per-detector SNR^2 of the intrinsic model) of one set from its per-detector
// sums sd[id] = S[2 id], sh[id] = S[2 id + 1]; rho_b may be null
__device__ __noinline__ void finalize_set(const PhdRec& c, const double* S, const NetGeom& g, const EventData& ev, int mixed,
                             int model, double* lnl_b, double* rho_b) {
  double L = 0.0;
  int loud = 0;
  for (int id = 0; id < g.nifo; id++) {
    const double sd = S[2 * id], sh = S[2 * id + 1];
    double K = c.Fs[id] * kH22fac * c.amp_scale / c.sqT * ev.inv_sigma[id];
    if (mixed) K *= c.a0 * c.mdf_m76;       // the mixed kernel sums the amplitude without this factor
    double HD = K * sd, HH = K * K * sh;
    double x = HD - 0.5 * HH;
    if (model == kModelIntrinsic) {
      if (rho_b) rho_b[id] = 2.0 * x;
      loud += 2.0 * x > 25.0;
    } else if (rho_b) {
      rho_b[id] = HD / sqrt(HH);
    }
    L += x;
  }
  if (model == kModelIntrinsic && g.nifo > 1 && loud < 2) L = 0.0;   // a signal in at least two detectors
  *lnl_b = L;
}

// the lnL of a set whose record failed the setup: the reference's rejected-sample value
// (QuickCBC.c:2366), rho 0
__device__ void reject_set(const NetGeom& g, double* lnl_b, double* rho_b) {
  *lnl_b = -1.0e20;
  if (rho_b)
    for (int id = 0; id < g.nifo; id++) rho_b[id] = 0.0;
}

// Where a launch writes its results itself: lnl != null makes the set's last tile finalise it
// (finalize_set).  At one tile per set that tile's thread 0 does so from its block sums; at several
// tiles each tile writes its partial sums and counts itself in done[b], and the block that counts
// last sums the set's partials in tile order and finalises it (then clears done[b] for the next
// launch).  lnl == null: every tile writes its partials for k_finalize_full.
struct FinalOut {
  double* lnl;
  double* rho;
  int mixed, model;
  SetOrder order;      // order.cnt non-null: block k evaluates the k-th set longest first (one tile per set)
  int B;
  int* done;           // several tiles per set: per-set tile counts, zero before the launch
};

// The set that block k of a one-tile launch evaluates: the k-th with the classes longest first
// (SetOrder).  Warp 0 scans the class counts, two classes per lane, and the lane whose class holds
// position k reads the set from the class's list.  Returns -1 when the counts do not place a set
// in [0, B) at position k (counts that were not cleared before the setup); the caller's block then
// does nothing.  Contains __syncthreads(): every thread of the block calls it.
__device__ int ordered_set(const FinalOut& fo, int k) {
  __shared__ int s_set;
  static_assert(kOrderClasses == 64, "two classes per lane of one warp");
  if (threadIdx.x < 32) {
    const int l = threadIdx.x, c0 = kOrderClasses - 1 - 2 * l, c1 = c0 - 1;
    if (l == 0) s_set = -1;
    __syncwarp();
    const int v0 = fo.order.cnt[c0], v1 = fo.order.cnt[c1];
    int x = v0 + v1;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, off);
      if (l >= off) x += y;
    }
    const int s0 = x - v0 - v1, s1 = s0 + v0;
    int b = -1;
    if (k >= s0 && k < s1 && k - s0 < fo.B) b = fo.order.list[(size_t)c0 * fo.B + (k - s0)];
    if (k >= s1 && k < s1 + v1 && k - s1 < fo.B) b = fo.order.list[(size_t)c1 * fo.B + (k - s1)];
    if (b >= 0 && b < fo.B) s_set = b;
  }
  __syncthreads();
  return s_set;
}

// thread 0's block sums of tile t of set b: the set's lnL (its only tile, or its last to finish), or
// the tile's partials (FinalOut)
template <int NIFO>
__device__ __forceinline__ void finish_tile(const PhdRec& rec, const double* acc, const NetGeom& g,
                                            const EventData& ev, const FinalOut& fo, int b, int tiles, int t,
                                            double* partials) {
  double* rho_b = fo.rho ? fo.rho + (size_t)b * g.nifo : nullptr;
  if (fo.lnl && tiles == 1) {
    if (!(rec.flags & kRecValid)) {
      reject_set(g, fo.lnl + b, rho_b);
      return;
    }
    double S[2 * kMaxIfo];
#pragma unroll
    for (int k = 0; k < 2 * kMaxIfo; k++) S[k] = k < 2 * NIFO ? acc[k] : 0.0;
    finalize_set(rec, S, g, ev, fo.mixed, fo.model, fo.lnl + b, rho_b);
    return;
  }
  double* out = partials + ((size_t)b * tiles + t) * (2 * kMaxIfo);
#pragma unroll
  for (int k = 0; k < 2 * NIFO; k++) out[k] = acc[k];
  if (!fo.lnl || !fo.done) return;
  __threadfence();                               // the partials before the count
  if (atomicAdd(fo.done + b, 1) != tiles - 1) return;
  __threadfence();                               // every tile's partials after the count
  fo.done[b] = 0;
  if (!(rec.flags & kRecValid)) {
    reject_set(g, fo.lnl + b, rho_b);
    return;
  }
  // the same sum in the same order as k_finalize_full
  double S[2 * kMaxIfo];
#pragma unroll
  for (int k = 0; k < 2 * kMaxIfo; k++) S[k] = 0.0;
  for (int u = 0; u < tiles; u++) {
    const double* p = partials + ((size_t)b * tiles + u) * (2 * kMaxIfo);
#pragma unroll
    for (int k = 0; k < 2 * NIFO; k++) S[k] += __ldcg(p + k);
  }
  finalize_set(rec, S, g, ev, fo.mixed, fo.model, fo.lnl + b, rho_b);
}

template <int PREC, int NIFO>
__global__ void __launch_bounds__(256) k_lnl_full(const PhdRec* __restrict__ recs, NetGeom g, EventData ev, int tiles,
                                                  double* __restrict__ partials, FinalOut fo) {
  __shared__ PhdRec rec;
  __shared__ double red[32 * 2 * kMaxIfo];
  pdl_wait();          // records (and class lists) of the setup
  const int bi = blockIdx.x / tiles, t = blockIdx.x - bi * tiles;
  const int b = fo.order.cnt ? ordered_set(fo, bi) : bi;
  if (b < 0) return;   // whole block
  load_record(rec, recs + b);
  __syncthreads();
  int i0, i1;
  tile_range(rec, tiles, t, i0, i1);
  double acc[2 * NIFO];
#pragma unroll
  for (int k = 0; k < 2 * NIFO; k++) acc[k] = 0.0;
  tile_fp64<NIFO>(rec, g, ev, i0, i1, acc);
  block_sum<2 * NIFO>(acc, red);
  if (threadIdx.x == 0) finish_tile<NIFO>(rec, acc, g, ev, fo, b, tiles, t, partials);
}

#ifndef QCBC_MIXED_MINBLOCKS
#define QCBC_MIXED_MINBLOCKS 4     // 64 registers: coefficients and the thread's sums in shared memory
#endif
// Sums over the threads of each group of gs threads (gs a multiple of 32) in a fixed order;
// the first thread of each group holds its group's sums.
template <int NV>
__device__ __forceinline__ void group_sum(double (&v)[NV], double* smem /* [32][NV] */, int gs) {
#pragma unroll
  for (int k = 0; k < NV; k++)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0)
    for (int k = 0; k < NV; k++) smem[w * NV + k] = v[k];
  __syncthreads();
  if (threadIdx.x % gs == 0) {
    const int w0 = w, nw = gs >> 5;
    for (int k = 0; k < NV; k++) {
      double x = smem[w0 * NV + k];
      for (int j = 1; j < nw; j++) x += smem[(w0 + j) * NV + k];
      v[k] = x;
    }
  }
}

// While the setup runs (before pdl_wait), the first blocks of the lnL launch pull the band's FP32
// planes and bin tables into L2, one 128-byte line per thread, so that the first rows of every
// block find them there instead of in HBM.
template <int NIFO>
__device__ __forceinline__ void mixed_prefetch(const NetGeom& g, const EventData& ev) {
  const size_t nh = (size_t)ev.nh, lo = (size_t)max(g.imin, 0), n = (size_t)max(g.imax - g.imin, 0);
  const char* base[6];
  size_t len[6];
  int ns = 0;
  auto seg = [&](const void* p, size_t elem) {
    base[ns] = static_cast<const char*>(p) + lo * elem;
    len[ns++] = n * elem;
  };
  if (NIFO == 3) {
    seg(ev.wm, 16); seg(ev.wm + 4 * nh, 16); seg(ev.wm + 8 * nh, 4);
  } else if (NIFO == 2) {
    seg(ev.wm, 16); seg(ev.wm + 4 * nh, 8);
  } else {
    seg(ev.wm, 8); seg(ev.wm + 2 * nh, 4);
  }
  seg(ev.tabA, 16); seg(ev.tabB, 16); seg(ev.tabC, 8);
  size_t line = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int k = 0; k < ns; k++) {
    const size_t lines = (len[k] + 127) / 128;
    if (line < lines) {
      prefetch_l2(base[k] + line * 128);
      return;
    }
    line -= lines;
  }
}

// Mixed-precision full lnL over one tile of bins of one parameter set.
template <int NIFO>
__global__ void __launch_bounds__(256, QCBC_MIXED_MINBLOCKS) k_lnl_full_mixed(const PhdRec* __restrict__ recs, NetGeom g,
                                                                               EventData ev, int tiles,
                                                                               double* __restrict__ partials,
                                                                               FinalOut fo) {
  __shared__ PhdRec rec;
  __shared__ double red[32 * 2 * kMaxIfo];
  extern __shared__ __align__(16) float2 s_rot[];   // [nk][mix_rs(NIFO)], then the threads' state
  mixed_prefetch<NIFO>(g, ev);
  pdl_wait();          // records (and class lists) of the setup
  const int bi = blockIdx.x / tiles, t = blockIdx.x - bi * tiles;
  const int b = fo.order.cnt ? ordered_set(fo, bi) : bi;
  if (b < 0) return;   // whole block
  load_record(rec, recs + b);
  __syncthreads();
  int i0, i1;
  tile_range(rec, tiles, t, i0, i1);
  double acc[2 * NIFO];
  tile_mixed_smem<NIFO>(rec, g, ev, i0, i1, s_rot, mixed_nk_cap(g.imax - g.imin, tiles, blockDim.x), NIFO, acc);
  group_sum<2 * NIFO>(acc, red, blockDim.x);
  if (threadIdx.x == 0) finish_tile<NIFO>(rec, acc, g, ev, fo, b, tiles, t, partials);
}

// rotation-table length per block for a launch: ceil(max bins per tile / threads)
static int mixed_nk(const NetGeom& g, const FullLaunch& L) { return mixed_nk_cap(g.imax - g.imin, L.tiles, L.threads); }

template <int NIFO>
static void launch_mixed_n(const PhdRec* r, int B, const NetGeom& g, const EventData& ev, const FullLaunch& L,
                           double* part, const FinalOut& fo, cudaStream_t s) {
  dim3 grid((unsigned)(B * L.tiles)), block(L.threads);
  size_t smem = (size_t)mixed_nk(g, L) * mix_rs(NIFO) * sizeof(float2);
  smem += mixed_state_bytes(L.threads, NIFO);
  if (fo.order.cnt || fo.done) launch_pdl(k_lnl_full_mixed<NIFO>, grid, block, smem, s, r, g, ev, L.tiles, part, fo);
  else k_lnl_full_mixed<NIFO><<<grid, block, smem, s>>>(r, g, ev, L.tiles, part, fo);
}

static void launch_full_mixed(const PhdRec* r, int B, const NetGeom& g, const EventData& ev, const FullLaunch& L,
                              double* part, const FinalOut& fo, cudaStream_t s) {
  switch (g.nifo) {
    case 1: launch_mixed_n<1>(r, B, g, ev, L, part, fo, s); break;
    case 2: launch_mixed_n<2>(r, B, g, ev, L, part, fo, s); break;
    default: launch_mixed_n<3>(r, B, g, ev, L, part, fo, s); break;
  }
}

template <int PREC>
static void launch_full_prec(const PhdRec* r, int B, const NetGeom& g, const EventData& ev, const FullLaunch& L,
                             double* part, const FinalOut& fo, cudaStream_t s) {
  dim3 grid((unsigned)(B * L.tiles)), block(L.threads);
  auto k = g.nifo == 1 ? k_lnl_full<PREC, 1> : (g.nifo == 2 ? k_lnl_full<PREC, 2> : k_lnl_full<PREC, 3>);
  if (fo.order.cnt || fo.done) launch_pdl(k, grid, block, 0, s, r, g, ev, L.tiles, part, fo);
  else k<<<grid, block, 0, s>>>(r, g, ev, L.tiles, part, fo);
}

void launch_lnl_full(const PhdRec* d_recs, int B, const NetGeom& g, const EventData& ev, Precision prec,
                     const FullLaunch& L, double* d_partials, cudaStream_t s) {
  if (B <= 0) return;
  const FinalOut none{nullptr, nullptr, 0, 0, SetOrder{nullptr, nullptr}, B, nullptr};
  if (prec == kFP64) launch_full_prec<kFP64>(d_recs, B, g, ev, L, d_partials, none, s);
  else launch_full_mixed(d_recs, B, g, ev, L, d_partials, none, s);
}

bool launch_lnl_full_final(const PhdRec* d_recs, const int* d_status, int B, const NetGeom& g, const EventData& ev,
                           Precision prec, const FullLaunch& L, double* d_partials, double* d_lnl, double* d_rho,
                           int model, const SetOrder* order, cudaStream_t s, int* d_done) {
  if (B <= 0) return true;
  if (L.tiles != 1 && !d_done) {
    launch_lnl_full(d_recs, B, g, ev, prec, L, d_partials, s);
    launch_finalize_full(d_partials, d_recs, d_status, B, L.tiles, g, ev, prec, d_lnl, d_rho, s, model);
    return false;
  }
  const FinalOut fo{d_lnl, d_rho, prec == kMixed ? 1 : 0, model,
                    (order && L.tiles == 1) ? *order : SetOrder{nullptr, nullptr}, B,
                    L.tiles == 1 ? nullptr : d_done};
  if (prec == kFP64) launch_full_prec<kFP64>(d_recs, B, g, ev, L, d_partials, fo, s);
  else launch_full_mixed(d_recs, B, g, ev, L, d_partials, fo, s);
  return true;
}

__global__ void k_finalize_full(const double* __restrict__ partials, const PhdRec* __restrict__ recs,
                                const int* __restrict__ status, int B, int tiles, NetGeom g, EventData ev,
                                int mixed, int model, double* __restrict__ lnl, double* __restrict__ rho) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double* rho_b = rho ? rho + (size_t)b * g.nifo : nullptr;
  if (status[b] != kStOK) {
    reject_set(g, lnl + b, rho_b);
    return;
  }
  double S[2 * kMaxIfo];
  for (int k = 0; k < 2 * kMaxIfo; k++) S[k] = 0.0;
  for (int t = 0; t < tiles; t++) {
    const double* p = partials + ((size_t)b * tiles + t) * (2 * kMaxIfo);
    for (int k = 0; k < 2 * g.nifo; k++) S[k] += p[k];
  }
  finalize_set(recs[b], S, g, ev, mixed, model, lnl + b, rho_b);
}

void launch_finalize_full(const double* d_partials, const PhdRec* d_recs, const int* d_status, int B, int tiles,
                          const NetGeom& g, const EventData& ev, Precision prec, double* d_lnl, double* d_rho,
                          cudaStream_t s, int model) {
  if (B <= 0) return;
  k_finalize_full<<<(B + 127) / 128, 128, 0, s>>>(d_partials, d_recs, d_status, B, tiles, g, ev,
                                                  prec == kMixed ? 1 : 0, model, d_lnl, d_rho);
}

__global__ void k_fill_bin_tables(double2* __restrict__ A, double2* __restrict__ Bt, float2* __restrict__ C, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double x = (double)(i > 0 ? i : 1);
    double c3 = cbrt(x), s = pow(x, 0.75);
    A[i] = make_double2(c3, 1.0 / c3);
    Bt[i] = make_double2(log(x), s);
    C[i] = make_float2((float)(1.0 / x), (float)s);
  }
}

void launch_fill_bin_tables(double2* d_tabA, double2* d_tabB, float2* d_tabC, int n, cudaStream_t s) {
  k_fill_bin_tables<<<(n + 255) / 256, 256, 0, s>>>(d_tabA, d_tabB, d_tabC, n);
}

// ---------------------------------------------------------------- multi-event launches
__global__ void __launch_bounds__(kSetupThreads) k_setup_multi(const double* __restrict__ params,
                                                               const int* __restrict__ event_of, int B,
                                                               const EventDesc* __restrict__ events, int n_events,
                                                               QnmTable q, int tile_bins, PhdRec* __restrict__ recs,
                                                               int* __restrict__ status, int* __restrict__ ntile) {
  GeomTable geo{event_of, events, n_events};
  setup_coop_block(params, B, geo, q, tile_bins, recs, status, ntile, kModelFull);
}

void launch_setup_multi(const double* d_params, const int* d_event_of, int B, const EventDesc* d_events, int n_events,
                        const QnmTable& q, int tile_bins, PhdRec* d_recs, int* d_status, int* d_ntile, cudaStream_t s) {
  if (B <= 0) return;
  k_setup_multi<<<(B + kSetupSets - 1) / kSetupSets, kSetupThreads, 0, s>>>(d_params, d_event_of, B, d_events,
                                                                           n_events, q, tile_bins, d_recs, d_status,
                                                                           d_ntile);
}

// One block: exclusive scan of ntile into off[0..B], then expansion into items (bounded by items_cap).
__global__ void k_scan_expand(const int* __restrict__ ntile, int B, int* __restrict__ off, int* __restrict__ items,
                              int items_cap) {
  __shared__ int wsum[32];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int per = (B + nt - 1) / nt;
  const int lo = tid * per, hi = min(lo + per, B);
  int local = 0;
  for (int b = lo; b < hi; b++) local += ntile[b];
  // inclusive scan of thread totals
  int lane = tid & 31, w = tid >> 5;
  int x = local;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = lane < (nt >> 5) ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += y;
    }
    wsum[lane] = v;
  }
  __syncthreads();
  int run = x - local + (w > 0 ? wsum[w - 1] : 0);
  if (tid == 0) off[0] = 0;
  for (int b = lo; b < hi; b++) {
    int n = ntile[b];
    for (int t = 0; t < n; t++)
      if (run + t < items_cap) items[run + t] = b;
    run += n;
    off[b + 1] = run;
  }
}

void launch_scan_expand(const int* d_ntile, int B, int* d_off, int* d_items, int items_cap, cudaStream_t s) {
  k_scan_expand<<<1, 1024, 0, s>>>(d_ntile, B, d_off, d_items, items_cap);
}

#ifndef QCBC_MULTI_MINBLOCKS
#define QCBC_MULTI_MINBLOCKS 4
#endif
// Both bodies are held to the register budget of four blocks per SM: the FP64 body is light on
// registers, the mixed body reads its piece coefficients from shared memory and keeps each
// thread's sums there (tile_mixed_smem).
template <int PREC>
__global__ void __launch_bounds__(256, PREC == kFP64 ? 4 : QCBC_MULTI_MINBLOCKS) k_lnl_multi(const PhdRec* __restrict__ recs,
                                                      const EventDesc* __restrict__ events,
                                                      const int* __restrict__ off, const int* __restrict__ items,
                                                      int B, int tile_bins, int items_cap, int* __restrict__ counter,
                                                      double* __restrict__ partials) {
  __shared__ PhdRec rec;
  __shared__ EventDesc evd;
  __shared__ int s_item, s_b;
  __shared__ double red[32 * 2 * kMaxIfo];
  extern __shared__ __align__(16) float2 s_rot[];   // mixed: rotation table [nk][4], then the threads' state
  int total = off[B];
  if (total > items_cap) total = items_cap;
  for (;;) {
    if (threadIdx.x == 0) {
      int it = atomicAdd(counter, 1);
      s_item = it;
      s_b = it < total ? items[it] : -1;
    }
    __syncthreads();
    const int item = s_item, b = s_b;
    if (item >= total) break;
    load_record(rec, recs + b);
    __syncthreads();
    if (threadIdx.x == 0) evd = events[rec.event];
    __syncthreads();
    const int t = item - off[b];
    const int i0 = rec.i_lo + t * tile_bins;
    const int i1 = min(i0 + tile_bins - 1, rec.i_hi);
    double acc[2 * kMaxIfo];
#pragma unroll
    for (int k = 0; k < 2 * kMaxIfo; k++) acc[k] = 0.0;
    const int nifo = evd.g.nifo;
    if (PREC == kFP64) {
      if (nifo == 1) tile_fp64<1>(rec, evd.g, evd.ev, i0, i1, acc);
      else if (nifo == 2) tile_fp64<2>(rec, evd.g, evd.ev, i0, i1, acc);
      else tile_fp64<3>(rec, evd.g, evd.ev, i0, i1, acc);
    } else {
      const int nk = (tile_bins + blockDim.x - 1) / blockDim.x + 1;
      if (nifo == 1) tile_mixed_smem<1>(rec, evd.g, evd.ev, i0, i1, s_rot, nk, kMaxIfo, acc);
      else if (nifo == 2) tile_mixed_smem<2>(rec, evd.g, evd.ev, i0, i1, s_rot, nk, kMaxIfo, acc);
      else tile_mixed_smem<3>(rec, evd.g, evd.ev, i0, i1, s_rot, nk, kMaxIfo, acc);
    }
    block_sum<2 * kMaxIfo>(acc, red);
    if (threadIdx.x == 0) {
      double* out = partials + (size_t)item * (2 * kMaxIfo);
#pragma unroll
      for (int k = 0; k < 2 * kMaxIfo; k++) out[k] = acc[k];
    }
    __syncthreads();
  }
}

static size_t multi_smem(Precision prec, int threads, int tile_bins) {
  if (prec == kFP64) return 0;
  int nk = (tile_bins + threads - 1) / threads + 1;
  return (size_t)nk * mix_rs(kMaxIfo) * sizeof(float2) + mixed_state_bytes(threads, kMaxIfo);
}

int multi_blocks_per_sm(Precision prec, int threads, int tile_bins) {
  int n = 0;
  size_t smem = multi_smem(prec, threads, tile_bins);
  if (prec == kFP64) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lnl_multi<kFP64>, threads, smem);
  else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_lnl_multi<kMixed>, threads, smem);
  return n > 0 ? n : 1;
}

void launch_lnl_multi(const PhdRec* d_recs, const EventDesc* d_events, const int* d_off, const int* d_items, int B,
                      int tile_bins, int items_cap, Precision prec, int threads, int blocks, int* d_counter,
                      double* d_partials, cudaStream_t s) {
  if (B <= 0) return;
  size_t smem = multi_smem(prec, threads, tile_bins);
  const int cap = items_cap;
  if (prec == kFP64) {
    k_lnl_multi<kFP64><<<blocks, threads, smem, s>>>(d_recs, d_events, d_off, d_items, B, tile_bins, cap, d_counter,
                                                     d_partials);
  } else {
    k_lnl_multi<kMixed><<<blocks, threads, smem, s>>>(d_recs, d_events, d_off, d_items, B, tile_bins, cap, d_counter,
                                                      d_partials);
  }
}



__global__ void k_finalize_multi(const double* __restrict__ partials, const PhdRec* __restrict__ recs,
                                 const int* __restrict__ status, const int* __restrict__ off,
                                 const EventDesc* __restrict__ events, int B, int items_cap, int mixed,
                                 double* __restrict__ lnl, double* __restrict__ rho) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const PhdRec& c = recs[b];
  if (status[b] != kStOK) {
    lnl[b] = -1.0e20;
    if (rho) for (int id = 0; id < kMaxIfo; id++) rho[(size_t)b * kMaxIfo + id] = 0.0;
    return;
  }
  const EventDesc& e = events[c.event];
  double L = 0.0;
  for (int id = 0; id < kMaxIfo; id++) {
    if (id >= e.g.nifo) {
      if (rho) rho[(size_t)b * kMaxIfo + id] = 0.0;
      continue;
    }
    double sd = 0.0, sh = 0.0;
    const int it_end = min(off[b + 1], items_cap);
    for (int it = off[b]; it < it_end; it++) {
      sd += partials[(size_t)it * (2 * kMaxIfo) + 2 * id];
      sh += partials[(size_t)it * (2 * kMaxIfo) + 2 * id + 1];
    }
    double K = c.Fs[id] * kH22fac * c.amp_scale / c.sqT * e.ev.inv_sigma[id];
    if (mixed) K *= c.a0 * c.mdf_m76;
    double HD = K * sd, HH = K * K * sh;
    if (rho) rho[(size_t)b * kMaxIfo + id] = HD / sqrt(HH);
    L += HD - 0.5 * HH;
  }
  lnl[b] = L;
}

void launch_finalize_multi(const double* d_partials, const PhdRec* d_recs, const int* d_status, const int* d_off,
                           const EventDesc* d_events, int B, int items_cap, Precision prec, double* d_lnl,
                           double* d_rho, cudaStream_t s) {
  if (B <= 0) return;
  k_finalize_multi<<<(B + 127) / 128, 128, 0, s>>>(d_partials, d_recs, d_status, d_off, d_events, B, items_cap,
                                                   prec == kMixed ? 1 : 0, d_lnl, d_rho);
}

// ---------------------------------------------------------------- heterodyned lnL
// One warp per parameter set, several sets per block, no block-wide barrier.  Phase 1: waveform at
// the M grid points and the per-detector ratios hc, hs, cc to the reference (QuickCBC.c:5332-5345)
// into the warp's shared memory.  Phase 2: per region r, uu = IP[r] v for v in {cc, hc, hs},
// contracted with SL / lc / ls and the edge over-count correction (QuickCBC.c:5347-5425); warp sum;
// lnL = logLb - sum (HR + HH/2).  The warp's shared memory: the record, then [3][nifo][M] doubles.
constexpr int kRecDoubles = (int)(sizeof(PhdRec) / 8);
#ifndef QCBC_HET_MINBLOCKS
#define QCBC_HET_MINBLOCKS 8     // 64 registers: 32 sets in flight per SM, 4096 sets in one wave
#endif

// doubles of shared memory one set's warp uses (a multiple of 2, so the next record stays 16-B aligned)
__host__ __device__ inline int het_warp_doubles(int nifo, int M) { return kRecDoubles + (3 * nifo * M + 1) / 2 * 2; }

// The mixed-precision waveform at bin i of the event (a heterodyne grid point, f = i/Tobs) from
// the folded polynomials of the mixed full-likelihood kernel (MixPoly) and the per-bin tables:
// phc = phase / 2 pi = R0 + i Ri + the piece's rest (FP64 for the inspiral and intermediate
// rests, FP32 for the ringdown's few cycles), amp = a0 Mf^{-7/6} A(Mf) in FP32 (the piece's
// amplitude times a0 (Msec df)^{-7/6} i^{-7/6}).  No log, cube root or FP64 division per point.
// The record must be in shared memory (its coefficients are read with shared loads).
__device__ __forceinline__ void mixed_point(const PhdRec& c, const HetData& h, int i, float& amp, double& phc) {
  const MixPoly& P = c.mix;
  const double2 tA = __ldg(h.tabA + i), tB = __ldg(h.tabB + i);
  const float2 tC = __ldg(h.tabC + i);
  const double xi = (double)i;
  const float xf = (float)i;
  const int pp = ph_piece(P, i), ap = amp_piece(P, i);
  double rest;
  if (pp == 0) rest = mph_ins(P.pins, xi, tA.x, tA.y, tB.x);
  else if (pp == 1) rest = mph_int(P.pint, xi, tA.y, tB.x);
  else rest = (double)mph_mrd(P.pmrd, xf, tC);
  const double2 r = sld2(&P.pmrd.R0);                          // (R0, Ri)
  phc = fma(xi, r.y, r.x) + rest;
  const float a = ap == 0 ? mamp_ins(P.ains, xf, (float)tA.x) : (ap == 1 ? mamp_int(P.aint, xf) : mamp_mrd(P.amrd, xf));
  const float u = (float)tA.y;                                // i^{-1/3}
  amp = a * (u * u * u) * sqrtf(u) * (float)(c.a0 * c.mdf_m76);
}

// Phase 1 of a set: the waveform at grid points j0, j0 + jstep, ... and the per-detector ratios
// to the reference into the set's shared memory sm ([3][nifo][M]: hc, hs, cc).
template <int PREC>
__device__ __forceinline__ void het_points(const PhdRec& c, const NetGeom& g, const HetData& h, double* sm, int j0,
                                           int jstep) {
  const int M = h.M, nifo = g.nifo;
  double* s_hc = sm;                 // [nifo][M]
  double* s_hs = sm + nifo * M;
  double* s_cc = sm + 2 * nifo * M;
  constexpr double kInv2Pi = 0.15915494309189533577;
  for (int j = j0; j < M; j += jstep) {
    double f = __ldg(h.freq + j);
    double y = 1.0;
    if (f < c.fs) y = exp(10.0 * (f - c.fs) / c.fs);          // taper below fbegin (QuickCBC.c:3859)
    if (PREC == kFP64) {
      double amp = 0.0, ph = 0.0;
      if (!(f > c.fCut)) { phd_eval64(c, c.Msec * f, amp, ph); amp *= c.amp_scale; }
      for (int id = 0; id < nifo; id++) {
        double A = c.Fs[id] * kH22fac * amp / c.sqT * y;
        double x = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, f), c.ts - c.td[id]), c.lam[id]), -ph);
        double aref = __ldg(h.amp + id * M + j), pref = __ldg(h.phase + id * M + j);
        double sx, cx;
        sincos(reduce_2pi(pref - x), &sx, &cx);
        double cc = 2.0 * (aref - A * cx), ss = 2.0 * A * sx;
        double hc = cc / aref, hs = ss / aref;
        s_hc[id * M + j] = hc;
        s_hs[id * M + j] = hs;
        s_cc[id * M + j] = hc * hc + hs * hs;
      }
    } else {
      float amp = 0.f;
      double phc = 0.0;
      if (!(f > c.fCut)) mixed_point(c, h, (int)rint(f * g.Tobs), amp, phc);
      for (int id = 0; id < nifo; id++) {
        double aref = __ldg(h.amp + id * M + j), pref = __ldg(h.phase + id * M + j);
        float ratio = amp * (float)(c.Fs[id] * kH22fac * c.amp_scale / c.sqT * y / aref);
        double cyc = pref * kInv2Pi - fma(f, c.ts - c.td[id], c.lam[id] * kInv2Pi - phc);
        float r = (float)(cyc - rint(cyc));
        float sx, cx;
        sincospif(2.0f * r, &sx, &cx);
        float hc = 2.0f * (1.0f - ratio * cx), hs = 2.0f * ratio * sx;
        s_hc[id * M + j] = (double)hc;
        s_hs[id * M + j] = (double)hs;
        s_cc[id * M + j] = (double)hc * (double)hc + (double)hs * (double)hs;
      }
    }
  }
}

// Phase 2 of a set, by one warp once phase 1 is in sm: the region contractions (lane r takes
// regions r, r + 32, ...), a butterfly warp sum, and lane 0 writes lnL to *out.
__device__ __forceinline__ void het_regions(const NetGeom& g, const HetData& h, const double* sm, double* out) {
  const int lane = threadIdx.x & 31;
  const int M = h.M, nifo = g.nifo;
  const double* s_hc = sm;
  const double* s_hs = sm + nifo * M;
  const double* s_cc = sm + 2 * nifo * M;
  const int J = h.J, J1 = J + 1, NR = h.NR;
  double acc[4 * kMaxIfo];           // per detector: HH, HR, x, y
#pragma unroll
  for (int k = 0; k < 4 * kMaxIfo; k++) acc[k] = 0.0;
  for (int r = lane; r < NR; r += 32) {
    const double* ip = h.IP + (size_t)r * J1 * J1;
#pragma unroll
    for (int id = 0; id < kMaxIfo; id++) {     // unrolled: acc stays in registers
      if (id >= nifo) break;
      const double* sl = h.SL + ((size_t)r * nifo + id) * J1;
      const double* lc = h.lc + ((size_t)r * nifo + id) * J1;
      const double* ls = h.ls + ((size_t)r * nifo + id) * J1;
      const double* vc = s_cc + id * M + r * J;
      const double* vh = s_hc + id * M + r * J;
      const double* vs = s_hs + id * M + r * J;
      double HH = 0.0, HR = 0.0;
      for (int a = 0; a < J1; a++) {
        double u1 = 0.0, u2 = 0.0, u3 = 0.0;
        for (int k = 0; k < J1; k++) {
          double w = __ldg(ip + a * J1 + k);
          u1 += w * vc[k];
          u2 += w * vh[k];
          u3 += w * vs[k];
        }
        HH += u1 * __ldg(sl + a);
        HR += u2 * __ldg(lc + a) + u3 * __ldg(ls + a);
      }
      acc[4 * id] += HH;
      acc[4 * id + 1] += HR;
      if (r < NR - 2) {
        acc[4 * id + 2] += __ldg(h.aa + id * NR + r + 1) * vc[J];
        acc[4 * id + 3] += __ldg(h.rc + id * NR + r + 1) * vh[J] + __ldg(h.rs + id * NR + r + 1) * vs[J];
      }
    }
  }
#pragma unroll
  for (int k = 0; k < 4 * kMaxIfo; k++)
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  if (lane == 0) {
    double L = h.logLb;
    for (int id = 0; id < nifo; id++) {
      double HH = acc[4 * id] - acc[4 * id + 2], HR = acc[4 * id + 1] - acc[4 * id + 3];
      L -= (HR + 0.5 * HH);
    }
    *out = L;
  }
}

// lnL of one set by one warp: phase 1 over the warp's lanes, then phase 2
template <int PREC>
__device__ __forceinline__ void het_warp(const PhdRec& c, const NetGeom& g, const HetData& h, double* sm,
                                         double* out) {
  het_points<PREC>(c, g, h, sm, threadIdx.x & 31, 32);
  __syncwarp();
  het_regions(g, h, sm, out);
}

// the warp's record into its shared memory
__device__ __forceinline__ void warp_load_record(double* dst, const PhdRec* src) {
  const double* s = reinterpret_cast<const double*>(src);
  for (int k = threadIdx.x & 31; k < kRecDoubles; k += 32) dst[k] = s[k];
  __syncwarp();
}

template <int PREC>
__global__ void __launch_bounds__(128, QCBC_HET_MINBLOCKS) k_lnl_het(const PhdRec* __restrict__ recs, const int* __restrict__ status,
                                                 NetGeom g, HetData h, int B, int warp_doubles,
                                                 double* __restrict__ lnl) {
  extern __shared__ __align__(16) double sm[];
  pdl_wait();          // records of the setup (immediate when launched the ordinary way)
  const int w = threadIdx.x >> 5;
  const int b = blockIdx.x * (blockDim.x >> 5) + w;
  if (b >= B) return;                // the whole warp leaves; no block barrier follows
  double* base = sm + (size_t)w * warp_doubles;
  if (status[b] != kStOK) {
    if ((threadIdx.x & 31) == 0) lnl[b] = -1.0e20;
    return;
  }
  warp_load_record(base, recs + b);
  het_warp<PREC>(*reinterpret_cast<const PhdRec*>(base), g, h, base + kRecDoubles, lnl + b);
}

// Heterodyned lnL of sets of many events: set b uses the geometry and heterodyne tables of its
// record's event (het[e].M == 0: the event has no tables, lnL = -1e20).
template <int PREC>
__global__ void __launch_bounds__(128, QCBC_HET_MINBLOCKS) k_lnl_het_multi(const PhdRec* __restrict__ recs, const int* __restrict__ status,
                                                       const EventDesc* __restrict__ events,
                                                       const HetData* __restrict__ het, int B, int warp_doubles,
                                                       double* __restrict__ lnl) {
  extern __shared__ __align__(16) double sm[];
  const int w = threadIdx.x >> 5;
  const int b = blockIdx.x * (blockDim.x >> 5) + w;
  if (b >= B) return;
  double* base = sm + (size_t)w * warp_doubles;
  if (status[b] != kStOK) {
    if ((threadIdx.x & 31) == 0) lnl[b] = -1.0e20;
    return;
  }
  warp_load_record(base, recs + b);
  const PhdRec& rec = *reinterpret_cast<const PhdRec*>(base);
  const int e = rec.event;
  if (e < 0 || het[e].M == 0) {
    if ((threadIdx.x & 31) == 0) lnl[b] = -1.0e20;
    return;
  }
  het_warp<PREC>(rec, events[e].g, het[e], base + kRecDoubles, lnl + b);
}

size_t het_smem_bytes(const NetGeom& g, const HetData& h) {
  return (size_t)het_warp_doubles(g.nifo, h.M) * sizeof(double);
}

// Heterodyned lnL of a few sets (the reference-signature calls, alone or merged): one block per
// set, phase 1 over all the block's threads (one grid point each while M <= blockDim), then phase 2
// by warp 0 exactly as k_lnl_het's warp does it, so both kernels give the same bits.  The block's
// shared memory: the record, then [3][nifo][M] doubles.
template <int PREC>
__global__ void __launch_bounds__(128) k_lnl_het_wide(const PhdRec* __restrict__ recs, const int* __restrict__ status,
                                                     NetGeom g, HetData h, int B, double* __restrict__ lnl) {
  extern __shared__ __align__(16) double sm[];
  pdl_wait();          // records of the setup
  const int b = blockIdx.x;
  if (b >= B) return;
  if (status[b] != kStOK) {
    if (threadIdx.x == 0) lnl[b] = -1.0e20;
    return;
  }
  const double* src = reinterpret_cast<const double*>(recs + b);
  for (int k = threadIdx.x; k < kRecDoubles; k += blockDim.x) sm[k] = src[k];
  __syncthreads();
  het_points<PREC>(*reinterpret_cast<const PhdRec*>(sm), g, h, sm + kRecDoubles, threadIdx.x, blockDim.x);
  __syncthreads();
  if (threadIdx.x < 32) het_regions(g, h, sm + kRecDoubles, lnl + b);
}

// batches up to this size take k_lnl_het_wide
constexpr int kHetWideMaxSets = 128;

// sets per block: four warps while their shared memory stays within 96 KB
static int het_sets_per_block(size_t warp_bytes) {
  int n = 4;
  while (n > 1 && (size_t)n * warp_bytes > 96 * 1024) n >>= 1;
  return n;
}

void launch_lnl_het_multi(const PhdRec* d_recs, const int* d_status, int B, const EventDesc* d_events,
                          const HetData* d_het, size_t smem, Precision prec, double* d_lnl, cudaStream_t s) {
  if (B <= 0) return;
  const int spb = het_sets_per_block(smem);
  const int wd = (int)(smem / sizeof(double));
  const unsigned grid = (unsigned)((B + spb - 1) / spb);
  if (prec == kFP64)
    k_lnl_het_multi<kFP64><<<grid, 32 * spb, spb * smem, s>>>(d_recs, d_status, d_events, d_het, B, wd, d_lnl);
  else
    k_lnl_het_multi<kMixed><<<grid, 32 * spb, spb * smem, s>>>(d_recs, d_status, d_events, d_het, B, wd, d_lnl);
}

void launch_lnl_het(const PhdRec* d_recs, const int* d_status, int B, const NetGeom& g, const HetData& h,
                    Precision prec, double* d_lnl, cudaStream_t s) {
  if (B <= 0) return;
  const size_t smem = het_smem_bytes(g, h);
  const int spb = het_sets_per_block(smem);
  const int wd = het_warp_doubles(g.nifo, h.M);
  const unsigned grid = (unsigned)((B + spb - 1) / spb);
  // A small batch (the reference-signature calls, merged or not) takes a block per set and is
  // launched with programmatic dependent launch after the setup, so its blocks wait on the SMs
  // instead of behind a launch gap; a large one takes a warp per set, launched the ordinary way
  // (early blocks holding SMs slowed it).
  if (B <= kHetWideMaxSets) {
    auto kw = prec == kFP64 ? k_lnl_het_wide<kFP64> : k_lnl_het_wide<kMixed>;
    const int threads = std::min(128, std::max(32, (h.M + 31) / 32 * 32));
    launch_pdl(kw, dim3((unsigned)B), dim3(threads), smem, s, d_recs, d_status, g, h, B, d_lnl);
    return;
  }
  auto k = prec == kFP64 ? k_lnl_het<kFP64> : k_lnl_het<kMixed>;
  k<<<grid, 32 * spb, spb * smem, s>>>(d_recs, d_status, g, h, B, wd, d_lnl);
}

// ---------------------------------------------------------------- heterodyne-grid waveforms, het_diff, Fisher_Het
constexpr int kNP = 11;                       // parameters of a full set (NP, ConstCBC.h:68)
constexpr int kFisherSets = 2 * kNP + 1;      // the point and +/- eps along each parameter
// fullphaseamp (QuickCBC.c:3850-3866), FP64, for B records on the frequencies freq[0..M):
// A = |F| h22fac amp / sqrt(T) x taper, x = 2 pi f (ts - td) + lambda - phi; out [B][nifo][M].
__global__ void k_waves(const PhdRec* __restrict__ recs, NetGeom g, const double* __restrict__ freq, int M,
                        double* __restrict__ amp_out, double* __restrict__ ph_out) {
  __shared__ PhdRec rec;
  const int b = blockIdx.y;
  load_record(rec, recs + b);
  __syncthreads();
  const PhdRec& c = rec;
  const int nifo = g.nifo;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < M; j += gridDim.x * blockDim.x) {
    const double f = __ldg(freq + j);
    double y = 1.0;
    if (f < c.fs) y = exp(10.0 * (f - c.fs) / c.fs);
    double amp = 0.0, ph = 0.0;
    if (!(f > c.fCut)) { phd_eval64(c, c.Msec * f, amp, ph); amp *= c.amp_scale; }
    for (int id = 0; id < nifo; id++) {
      const size_t o = ((size_t)b * nifo + id) * M + j;
      amp_out[o] = c.Fs[id] * kH22fac * amp / c.sqT * y;
      ph_out[o] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, f), c.ts - c.td[id]), c.lam[id]), -ph);
    }
  }
}

void launch_waves(const PhdRec* d_recs, int B, const NetGeom& g, const double* d_freq, int M, double* d_amp,
                  double* d_phase, cudaStream_t s) {
  if (B <= 0 || M <= 0) return;
  int bx = (M + 255) / 256;
  if (bx > 296) bx = 296;
  dim3 grid((unsigned)bx, (unsigned)B);
  k_waves<<<grid, 256, 0, s>>>(d_recs, g, d_freq, M, d_amp, d_phase);
}

void launch_het_waves(const PhdRec* d_recs, int B, const NetGeom& g, const HetData& h, double* d_amp,
                      double* d_phase, cudaStream_t s) {
  launch_waves(d_recs, B, g, h.freq, h.M, d_amp, d_phase, s);
}

// Fisher_All (QuickCBC.c:2695-2817): one block per (matrix f, pair i <= j) over the full band:
// sum over detectors and bins k in [imin, imax) of 4 (dA_i dA_j + A^2 dphi_i dphi_j) / S, with
// the central differences of the 23 wave sets of matrix f (as k_het_fisher) on n bins.
__global__ void __launch_bounds__(256) k_fisher_full(const double* __restrict__ amp, const double* __restrict__ ph,
                                                     NetGeom g, int n, const double* __restrict__ S, int sn_stride,
                                                     int imin, int imax, double eps, double* __restrict__ fish) {
  __shared__ double red[32];
  __shared__ int s_ij[2];
  const int f = blockIdx.y, nifo = g.nifo;
  if (threadIdx.x == 0) {
    int q = blockIdx.x, i = 0;
    while (q >= kNP - i) { q -= kNP - i; i++; }
    s_ij[0] = i;
    s_ij[1] = i + q;
  }
  __syncthreads();
  const int i = s_ij[0], j = s_ij[1];
  const size_t set0 = (size_t)f * kFisherSets;
  double acc[1] = {0.0};
  for (int id = 0; id < nifo; id++) {
    const double* A0 = amp + (set0 * nifo + id) * n;
    const double* Api = amp + ((set0 + 1 + 2 * i) * nifo + id) * n;
    const double* Ami = amp + ((set0 + 2 + 2 * i) * nifo + id) * n;
    const double* Apj = amp + ((set0 + 1 + 2 * j) * nifo + id) * n;
    const double* Amj = amp + ((set0 + 2 + 2 * j) * nifo + id) * n;
    const double* Ppi = ph + ((set0 + 1 + 2 * i) * nifo + id) * n;
    const double* Pmi = ph + ((set0 + 2 + 2 * i) * nifo + id) * n;
    const double* Ppj = ph + ((set0 + 1 + 2 * j) * nifo + id) * n;
    const double* Pmj = ph + ((set0 + 2 + 2 * j) * nifo + id) * n;
    const double* Sd = S + (size_t)id * sn_stride;
    for (int k = imin + threadIdx.x; k < imax; k += blockDim.x) {
      const double dAi = (Api[k] - Ami[k]) / (2.0 * eps), dAj = (Apj[k] - Amj[k]) / (2.0 * eps);
      const double dPi = (Ppi[k] - Pmi[k]) / (2.0 * eps), dPj = (Ppj[k] - Pmj[k]) / (2.0 * eps);
      acc[0] += 4.0 * (dAi * dAj + A0[k] * A0[k] * dPi * dPj) / Sd[k];
    }
  }
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) fish[((size_t)f * kNP + i) * kNP + j] = acc[0];
}

void launch_fisher_full(const double* d_amp, const double* d_phase, int nmat, const NetGeom& g, int n,
                        const double* d_S, int sn_stride, int imin, int imax, double eps, double* d_fish,
                        cudaStream_t s) {
  if (nmat <= 0) return;
  dim3 grid(kNP * (kNP + 1) / 2, (unsigned)nmat);
  k_fisher_full<<<grid, 256, 0, s>>>(d_amp, d_phase, g, n, d_S, sn_stride, imin, imax, eps, d_fish);
}

// diff (QuickCBC.c:4913-4964): partial sums over detectors and bins j in [imin, m) of
// 4 |h_ref - h_b|^2 / S for the reference waves (one set) and B other wave sets on n bins; block
// (c, b) covers chunk c of the bins of set b and writes out[b * gridDim.x + c].
__global__ void __launch_bounds__(256) k_diff_full(const double* __restrict__ amp_ref, const double* __restrict__ ph_ref,
                                                   const double* __restrict__ amp, const double* __restrict__ ph,
                                                   NetGeom g, int n, int imin, int m, const double* __restrict__ S,
                                                   int sn_stride, double* __restrict__ out) {
  __shared__ double red[32];
  const int b = blockIdx.y, nifo = g.nifo;
  const int span = (m - imin + gridDim.x - 1) / gridDim.x;
  const int j0 = imin + blockIdx.x * span, j1 = min(m, j0 + span);
  double acc[1] = {0.0};
  for (int id = 0; id < nifo; id++) {
    const double* Ar = amp_ref + (size_t)id * n;
    const double* Pr = ph_ref + (size_t)id * n;
    const double* Ap = amp + ((size_t)b * nifo + id) * n;
    const double* Pp = ph + ((size_t)b * nifo + id) * n;
    const double* Sd = S + (size_t)id * sn_stride;
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      const double d = Pr[j] - Pp[j];
      const double re = Ar[j] - Ap[j] * cos(d), im = Ap[j] * sin(d);
      acc[0] += 4.0 * (re * re + im * im) / Sd[j];
    }
  }
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) out[(size_t)b * gridDim.x + blockIdx.x] = acc[0];
}

void launch_diff_full(const double* d_amp_ref, const double* d_ph_ref, const double* d_amp, const double* d_ph, int B,
                      const NetGeom& g, int n, int imin, int m, const double* d_S, int sn_stride, int chunks,
                      double* d_out, cudaStream_t s) {
  if (B <= 0 || chunks <= 0) return;
  dim3 grid((unsigned)chunks, (unsigned)B);
  k_diff_full<<<grid, 256, 0, s>>>(d_amp_ref, d_ph_ref, d_amp, d_ph, g, n, imin, m, d_S, sn_stride, d_out);
}

// het_space's ratios to the reference waveform (QuickCBC.c:4688-4702) for the wave sets
// 1..nset-1 against set 0, bins [j0, j1) of n: Cs = 1 - Ap/Ar cos(Pr - Pp), Sn = Ap/Ar sin(Pr - Pp),
// DH = Cs^2 + Sn^2, each [j1-j0][nset-1][nifo] (bin-major, as the grid walk reads them).
__global__ void k_hs_ratios(const double* __restrict__ amp, const double* __restrict__ ph, int nset, int nifo, int n,
                            int j0, int j1, double* __restrict__ Cs, double* __restrict__ Sn,
                            double* __restrict__ DH) {
  const int per = (nset - 1) * nifo;
  const long long total = (long long)per * (j1 - j0);
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(t % per);
    const int j = j0 + (int)(t / per);
    const int id = r % nifo, i = r / nifo;
    const double Ar = amp[(size_t)id * n + j], Pr = ph[(size_t)id * n + j];
    const double Ap = amp[((size_t)(i + 1) * nifo + id) * n + j], Pp = ph[((size_t)(i + 1) * nifo + id) * n + j];
    const double c = 1.0 - Ap / Ar * cos(Pr - Pp);
    const double sv = Ap / Ar * sin(Pr - Pp);
    Cs[t] = c;
    Sn[t] = sv;
    DH[t] = c * c + sv * sv;
  }
}

void launch_hs_ratios(const double* d_amp, const double* d_ph, int nset, int nifo, int n, int j0, int j1,
                      double* d_Cs, double* d_Sn, double* d_DH, cudaStream_t s) {
  long long total = (long long)(nset - 1) * nifo * (j1 - j0);
  if (total <= 0) return;
  long long blocks = (total + 255) / 256;
  if (blocks > 4736) blocks = 4736;
  k_hs_ratios<<<(unsigned)blocks, 256, 0, s>>>(d_amp, d_ph, nset, nifo, n, j0, j1, d_Cs, d_Sn, d_DH);
}

// het_space's grid walk (QuickCBC.c:4720-4765) in one block: from the current grid point jmin,
// the next one is the first bin j > jmin at which the linear interpolation between jmin and j of
// any ratio (Cs, Sn, DH of any direction and detector) misses its value at the mid-point by more
// than tl = max(tol ratio[j], tol), or at which j - jmin exceeds djmax.  The block tests 1024
// consecutive bins at a time and keeps the first hit.  grid[0..*count) gets the points; the walk
// stops at the cap (*count = -1 then).
__global__ void __launch_bounds__(1024) k_hs_walk(const double* __restrict__ Cs, const double* __restrict__ Sn,
                                                  const double* __restrict__ DH, const double* __restrict__ ratio,
                                                  int per, int MN, int MM, int djmax, double tol, int cap,
                                                  int* __restrict__ grid, int* __restrict__ count) {
  __shared__ int s_first;
  int jmin = MN, nout = 0;
  if (threadIdx.x == 0) grid[nout] = jmin;
  nout++;
  for (;;) {
    int found = MM;
    for (int base = jmin + 1; base < MM && found == MM; base += blockDim.x) {
      if (threadIdx.x == 0) s_first = MM;
      __syncthreads();
      const int j = base + threadIdx.x;
      bool flag = false;
      if (j < MM) {
        double tl = tol * ratio[j];
        if (tl < tol) tl = tol;
        const int jmid = (j + jmin) / 2;
        const double w0 = (double)(j - jmid), w1 = (double)(jmid - jmin), dw = (double)(j - jmin);
        const size_t oa = (size_t)(jmin - MN) * per, ob = (size_t)(j - MN) * per, om = (size_t)(jmid - MN) * per;
        for (int r = 0; r < per && !flag; r++) {
          const double cmid = (Cs[oa + r] * w0 + Cs[ob + r] * w1) / dw;
          const double smid = (Sn[oa + r] * w0 + Sn[ob + r] * w1) / dw;
          const double dmid = (DH[oa + r] * w0 + DH[ob + r] * w1) / dw;
          if (fabs(Cs[om + r] - cmid) > tl || fabs(Sn[om + r] - smid) > tl || fabs(DH[om + r] - dmid) > tl)
            flag = true;
        }
        if (j - jmin > djmax) flag = true;
      }
      if (flag) atomicMin(&s_first, j);
      __syncthreads();
      found = s_first;
      __syncthreads();
    }
    if (found >= MM) break;
    jmin = found;
    if (nout >= cap) {
      if (threadIdx.x == 0) *count = -1;
      return;
    }
    if (threadIdx.x == 0) grid[nout] = jmin;
    nout++;
  }
  if (threadIdx.x == 0) *count = nout;
}

void launch_hs_walk(const double* d_Cs, const double* d_Sn, const double* d_DH, const double* d_ratio, int per, int MN,
                    int MM, int djmax, double tol, int cap, int* d_grid, int* d_count, cudaStream_t s) {
  k_hs_walk<<<1, 1024, 0, s>>>(d_Cs, d_Sn, d_DH, d_ratio, per, MN, MM, djmax, tol, cap, d_grid, d_count);
}

// The slow-term quadrature of the heterodyne summary for one detector and the regions
// r = r0, r0 + rstep, ...: sum_r (IP[r] v_r) . SL[r][id], and separately the over-counted edge
// values sum_{r < NR-2} aa[id][r+1] v[rJ + J] (QuickCBC.c:5005-5035, 5571-5597).
__device__ __forceinline__ void het_slow_terms(const HetData& h, int nifo, int id, const double* v, int r0, int rstep,
                                               double& hh, double& edge) {
  const int J = h.J, J1 = J + 1, NR = h.NR;
  for (int r = r0; r < NR; r += rstep) {
    const double* ip = h.IP + (size_t)r * J1 * J1;
    const double* sl = h.SL + ((size_t)r * nifo + id) * J1;
    const double* vv = v + r * J;
    for (int a = 0; a < J1; a++) {
      double u = 0.0;
      for (int k = 0; k < J1; k++) u += __ldg(ip + a * J1 + k) * vv[k];
      hh += u * __ldg(sl + a);
    }
    if (r < NR - 2) edge += __ldg(h.aa + id * NR + r + 1) * vv[J];
  }
}

// het_diff: one block per pair p of wave sets (2p, 2p+1); d_out[p] = sum over detectors of the
// slow-term quadrature of cc = 4 |h_2p - h_2p+1|^2 / Aref^2 (QuickCBC.c:4995-5040).
__global__ void __launch_bounds__(256) k_het_diff(const double* __restrict__ amp, const double* __restrict__ ph,
                                                  NetGeom g, HetData h, double* __restrict__ out) {
  extern __shared__ double s_cc[];   // [M]
  __shared__ double red[32 * 2];
  const int p = blockIdx.x, M = h.M, nifo = g.nifo;
  double tot = 0.0;
  for (int id = 0; id < nifo; id++) {
    const double* Ar = amp + ((size_t)(2 * p) * nifo + id) * M;
    const double* Ap = amp + ((size_t)(2 * p + 1) * nifo + id) * M;
    const double* Pr = ph + ((size_t)(2 * p) * nifo + id) * M;
    const double* Pp = ph + ((size_t)(2 * p + 1) * nifo + id) * M;
    for (int j = threadIdx.x; j < M; j += blockDim.x) {
      const double d = Pr[j] - Pp[j];
      const double re = Ar[j] - Ap[j] * cos(d), im = Ap[j] * sin(d);
      const double aref = __ldg(h.amp + id * M + j);
      s_cc[j] = 4.0 * (re * re + im * im) / (aref * aref);
    }
    __syncthreads();
    double v[2] = {0.0, 0.0};
    het_slow_terms(h, nifo, id, s_cc, threadIdx.x, blockDim.x, v[0], v[1]);
    block_sum<2>(v, red);
    if (threadIdx.x == 0) tot += v[0] - v[1];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[p] = tot;
}

void launch_het_diff(const double* d_amp, const double* d_phase, int npair, const NetGeom& g, const HetData& h,
                     double* d_out, cudaStream_t s) {
  if (npair <= 0) return;
  k_het_diff<<<npair, 256, (size_t)h.M * sizeof(double), s>>>(d_amp, d_phase, g, h, d_out);
}

// Fisher_Het: one block per (matrix f, pair i <= j).  Central differences of the amplitude and
// phase (wave sets 23 f + 1 + 2 i and 23 f + 2 + 2 i, step eps), then per detector the slow-term
// quadrature of cc = 4 (dA_i dA_j + A^2 dphi_i dphi_j) / Aref^2 (QuickCBC.c:5503-5600).
__global__ void __launch_bounds__(256) k_het_fisher(const double* __restrict__ amp, const double* __restrict__ ph,
                                                    NetGeom g, HetData h, double eps, double* __restrict__ fish) {
  extern __shared__ double s_cc[];   // [M]
  __shared__ double red[32 * 2];
  __shared__ int s_ij[2];
  const int f = blockIdx.y, M = h.M, nifo = g.nifo;
  if (threadIdx.x == 0) {           // pair index -> (i, j >= i) in row-major order of the upper triangle
    int q = blockIdx.x, i = 0;
    while (q >= kNP - i) { q -= kNP - i; i++; }
    s_ij[0] = i;
    s_ij[1] = i + q;
  }
  __syncthreads();
  const int i = s_ij[0], j = s_ij[1];
  const size_t set0 = (size_t)f * kFisherSets;
  double tot = 0.0;
  for (int id = 0; id < nifo; id++) {
    const double* A0 = amp + (set0 * nifo + id) * M;
    const double* Api = amp + ((set0 + 1 + 2 * i) * nifo + id) * M;
    const double* Ami = amp + ((set0 + 2 + 2 * i) * nifo + id) * M;
    const double* Apj = amp + ((set0 + 1 + 2 * j) * nifo + id) * M;
    const double* Amj = amp + ((set0 + 2 + 2 * j) * nifo + id) * M;
    const double* Ppi = ph + ((set0 + 1 + 2 * i) * nifo + id) * M;
    const double* Pmi = ph + ((set0 + 2 + 2 * i) * nifo + id) * M;
    const double* Ppj = ph + ((set0 + 1 + 2 * j) * nifo + id) * M;
    const double* Pmj = ph + ((set0 + 2 + 2 * j) * nifo + id) * M;
    for (int k = threadIdx.x; k < M; k += blockDim.x) {
      const double dAi = (Api[k] - Ami[k]) / (2.0 * eps), dAj = (Apj[k] - Amj[k]) / (2.0 * eps);
      const double dPi = (Ppi[k] - Pmi[k]) / (2.0 * eps), dPj = (Ppj[k] - Pmj[k]) / (2.0 * eps);
      const double aref = __ldg(h.amp + id * M + k);
      s_cc[k] = 4.0 * (dAi * dAj + A0[k] * A0[k] * dPi * dPj) / (aref * aref);
    }
    __syncthreads();
    double v[2] = {0.0, 0.0};
    het_slow_terms(h, nifo, id, s_cc, threadIdx.x, blockDim.x, v[0], v[1]);
    block_sum<2>(v, red);
    if (threadIdx.x == 0) tot += v[0] - v[1];
    __syncthreads();
  }
  if (threadIdx.x == 0) fish[((size_t)f * kNP + i) * kNP + j] = tot;
}

void launch_het_fisher(const double* d_amp, const double* d_phase, int nmat, const NetGeom& g, const HetData& h,
                       double eps, double* d_fish, cudaStream_t s) {
  if (nmat <= 0) return;
  dim3 grid(kNP * (kNP + 1) / 2, (unsigned)nmat);
  k_het_fisher<<<grid, 256, (size_t)h.M * sizeof(double), s>>>(d_amp, d_phase, g, h, eps, d_fish);
}

// AmpPhase outputs for bins [1, n) (QuickCBC.c:3435-3440)
__global__ void k_ampphase_out(const double* __restrict__ freq, const double* __restrict__ amp,
                               const double* __restrict__ phase, int n, double ts, double* __restrict__ Af,
                               double* __restrict__ Pf) {
  for (int i = 1 + blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    Pf[i] = __dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, freq[i]), ts), -phase[i]);
    Af[i] = kH22fac * amp[i];
  }
}

void launch_ampphase_out(const double* d_freq, const double* d_amp, const double* d_phase, int n, double ts,
                         double* d_Af, double* d_Pf, cudaStream_t s) {
  int blocks = (n + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  k_ampphase_out<<<blocks, 256, 0, s>>>(d_freq, d_amp, d_phase, n, ts, d_Af, d_Pf);
}

// ---------------------------------------------------------------- waveform outputs
__global__ void k_setup_phys(double phi0, double fRef, double m1, double m2, double chi1, double chi2, double dist,
                             QnmTable q, PhdRec* rec, int* status) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    PhdRec c;
    status[0] = phd_setup(c, phi0, fRef, m1, m2, chi1, chi2, dist, q);
    *rec = c;
  }
}

// IMRPhenomDGenerateh22FDAmpPhase on an arbitrary frequency list (IMRPhenomD.c:527-556)
__global__ void k_amp_phase(const PhdRec* __restrict__ recp, const double* __restrict__ freq, int n,
                            double* __restrict__ amp, double* __restrict__ phase) {
  __shared__ PhdRec c;
  if (threadIdx.x == 0) c = *recp;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double f = freq[i];
    if (f > c.fCut) { amp[i] = 0.0; phase[i] = 0.0; continue; }
    double a, p;
    phd_eval64(c, c.Msec * f, a, p);
    amp[i] = c.amp_scale * a;
    phase[i] = p;
  }
}

void launch_amp_phase(const double* d_freq, int n, double phi0, double fRef, double m1, double m2, double chi1,
                      double chi2, double dist, const QnmTable& q, PhdRec* d_rec, double* d_amp, double* d_phase,
                      int* d_status, cudaStream_t s) {
  k_setup_phys<<<1, 32, 0, s>>>(phi0, fRef, m1, m2, chi1, chi2, dist, q, d_rec, d_status);
  int blocks = (n + 255) / 256;
  if (blocks > 1184) blocks = 1184;
  if (blocks < 1) blocks = 1;
  k_amp_phase<<<blocks, 256, 0, s>>>(d_rec, d_freq, n, d_amp, d_phase);
}

// fulltemplates: h[id][i] = A cos x, h[id][N-i] = A sin x for f > fbegin, else 0 (QuickCBC.c:3752-3772)
__global__ void k_fulltemplates(const PhdRec* __restrict__ recp, NetGeom g, const double* __restrict__ freq,
                                double* __restrict__ h) {
  __shared__ PhdRec c;
  if (threadIdx.x == 0) c = *recp;
  __syncthreads();
  const int N = g.N, half = N / 2;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i <= half; i += gridDim.x * blockDim.x) {
    if (i == 0 || i == half) {
      for (int id = 0; id < g.nifo; id++) h[(size_t)id * N + i] = 0.0;
      continue;
    }
    double f = freq[i];
    if (!(f > c.fs)) {
      for (int id = 0; id < g.nifo; id++) { h[(size_t)id * N + i] = 0.0; h[(size_t)id * N + N - i] = 0.0; }
      continue;
    }
    double amp = 0.0, ph = 0.0;
    if (!(f > c.fCut)) { phd_eval64(c, c.Msec * f, amp, ph); amp *= c.amp_scale; }
    for (int id = 0; id < g.nifo; id++) {
      double A = c.Fs[id] * kH22fac * amp / c.sqT;
      double x = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, f), c.ts - c.td[id]), c.lam[id]), -ph);
      double sx, cx;
      sincos(reduce_2pi(x), &sx, &cx);
      h[(size_t)id * N + i] = A * cx;
      h[(size_t)id * N + N - i] = A * sx;
    }
  }
}

void launch_fulltemplates(const double* d_params, const NetGeom& g, const QnmTable& q, const double* d_freq,
                          PhdRec* d_rec, int* d_status, double* d_h, cudaStream_t s, int model) {
  launch_setup(d_params, 1, g, q, d_rec, d_status, s, model);
  int blocks = (g.N / 2 + 256) / 256;
  if (blocks > 2368) blocks = 2368;
  k_fulltemplates<<<blocks, 256, 0, s>>>(d_rec, g, d_freq, d_h);
}

// fullphaseamp: amp = A * taper, phase = x on freq[0..n) (QuickCBC.c:3850-3866)
__global__ void k_fullphaseamp(const PhdRec* __restrict__ recp, NetGeom g, const double* __restrict__ freq, int n,
                               double* __restrict__ amp_out, double* __restrict__ ph_out) {
  __shared__ PhdRec c;
  if (threadIdx.x == 0) c = *recp;
  __syncthreads();
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double f = freq[i];
    double amp = 0.0, ph = 0.0;
    if (!(f > c.fCut)) { phd_eval64(c, c.Msec * f, amp, ph); amp *= c.amp_scale; }
    double y = 1.0;
    if (f < c.fs) y = exp(10.0 * (f - c.fs) / c.fs);
    for (int id = 0; id < g.nifo; id++) {
      double A = c.Fs[id] * kH22fac * amp / c.sqT;
      amp_out[(size_t)id * n + i] = A * y;
      ph_out[(size_t)id * n + i] = __dadd_rn(__dadd_rn(__dmul_rn(__dmul_rn(kTwoPi, f), c.ts - c.td[id]), c.lam[id]), -ph);
    }
  }
}

void launch_fullphaseamp(const double* d_params, const NetGeom& g, const QnmTable& q, const double* d_freq, int n,
                         PhdRec* d_rec, int* d_status, double* d_amp, double* d_phase, cudaStream_t s) {
  launch_setup(d_params, 1, g, q, d_rec, d_status, s);
  int blocks = (n + 255) / 256;
  if (blocks > 2368) blocks = 2368;
  if (blocks < 1) blocks = 1;
  k_fullphaseamp<<<blocks, 256, 0, s>>>(d_rec, g, d_freq, n, d_amp, d_phase);
}

// ---------------------------------------------------------------- heterodyne setup (FP64)
// Per bin j in [1, N/2): residual r = D - h, RC = 2 (r_re cos p + r_im sin p) A / S,
// RS = 2 (-r_re sin p + r_im cos p) A / S, AA = A^2 / S  (QuickCBC.c:5190-5203).
__global__ void k_het_bins(const double* __restrict__ h, const double* __restrict__ amp,
                           const double* __restrict__ phase, const double* __restrict__ D,
                           const double* __restrict__ S, int sn_stride, int N, int nifo, double* __restrict__ RC,
                           double* __restrict__ RS, double* __restrict__ AA) {
  const int half = N / 2;
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < nifo * half; idx += gridDim.x * blockDim.x) {
    int id = idx / half, j = idx - id * half;
    size_t o = (size_t)id * half + j;
    if (j == 0) { RC[o] = 0.0; RS[o] = 0.0; AA[o] = 0.0; continue; }
    const double* hr = h + (size_t)id * N;
    const double* dr = D + (size_t)id * N;
    double rre = dr[j] - hr[j], rim = dr[N - j] - hr[N - j];
    double a = amp[o], s = S[(size_t)id * sn_stride + j];
    double sp, cp;
    sincos(phase[o], &sp, &cp);
    double x = a / s;
    RC[o] = 2.0 * (rre * cp + rim * sp) * x;
    RS[o] = 2.0 * (-rre * sp + rim * cp) * x;
    AA[o] = a * a / s;
  }
}

void launch_het_bins(const double* d_h, const double* d_amp, const double* d_phase, const double* d_D,
                     const double* d_S, int sn_stride, int N, int nifo, double* d_RC, double* d_RS, double* d_AA,
                     cudaStream_t s) {
  int total = nifo * (N / 2);
  int blocks = (total + 255) / 256;
  if (blocks > 4736) blocks = 4736;
  k_het_bins<<<blocks, 256, 0, s>>>(d_h, d_amp, d_phase, d_D, d_S, sn_stride, N, nifo, d_RC, d_RS, d_AA);
}

// One block per (region, detector): sums over the region's U+1 bins of AA, RC, RS times the
// discrete Legendre polynomials P_a(n) (QuickCBC.c:5265-5281, recurrence of 5055-5094).
__global__ void k_het_region_sums(const double* __restrict__ RC, const double* __restrict__ RS,
                                  const double* __restrict__ AA, const int* __restrict__ fgrid, int M, int J,
                                  int nifo, int nh, double* __restrict__ SL, double* __restrict__ lc,
                                  double* __restrict__ ls) {
  __shared__ double red[32 * 12];
  int r = blockIdx.x / nifo, id = blockIdx.x - r * nifo;
  int J1 = J + 1;
  int k0 = fgrid[r * J], U = fgrid[(r + 1) * J] - k0;
  double acc[12];
#pragma unroll
  for (int a = 0; a < 12; a++) acc[a] = 0.0;
  for (int n = threadIdx.x; n <= U; n += blockDim.x) {
    double P[4];
    double c0 = 0.0, c1 = (double)(U - 2 * n), c2 = (double)U;
    double d0 = c2, d1 = c1 + c1, d2 = d0;
    P[0] = 1.0;
    if (J >= 1) P[1] = c1 / (double)U;
    for (int i = 1; i < J && i < 3; i++) {
      d0 += 2.0; d2 -= 2.0; c0 += d0; c1 += d1; c2 += d2;
      P[i + 1] = (c1 * P[i] - c0 * P[i - 1]) / c2;
    }
    size_t k = (size_t)id * nh + k0 + n;
    double aa = AA[k], rc = RC[k], rs = RS[k];
    for (int a = 0; a < J1 && a < 4; a++) {
      acc[3 * a] += aa * P[a];
      acc[3 * a + 1] += rc * P[a];
      acc[3 * a + 2] += rs * P[a];
    }
  }
  block_sum<12>(acc, red);
  if (threadIdx.x == 0) {
    for (int a = 0; a < J1 && a < 4; a++) {
      size_t o = ((size_t)r * nifo + id) * J1 + a;
      SL[o] = acc[3 * a];
      lc[o] = acc[3 * a + 1];
      ls[o] = acc[3 * a + 2];
    }
  }
}

void launch_het_region_sums(const double* d_RC, const double* d_RS, const double* d_AA, const int* d_fgrid, int M,
                            int J, int nifo, int nh, double* d_SL, double* d_lc, double* d_ls, cudaStream_t s) {
  int NR = (M - 1) / J;
  if (NR <= 0) return;
  k_het_region_sums<<<NR * nifo, 256, 0, s>>>(d_RC, d_RS, d_AA, d_fgrid, M, J, nifo, nh, d_SL, d_lc, d_ls);
}

// <h|h> and <D-h|h> over [imin, imax) per detector, one block per detector (Utilities.c:716-736)
__global__ void k_nwip_pairs(const double* __restrict__ h, const double* __restrict__ D, const double* __restrict__ S,
                             int sn_stride, int N, int imin, int imax, double* __restrict__ out) {
  __shared__ double red[32 * 2];
  int id = blockIdx.x;
  const double* hr = h + (size_t)id * N;
  const double* dr = D + (size_t)id * N;
  const double* sr = S + (size_t)id * sn_stride;
  double acc[2] = {0.0, 0.0};
  for (int i = imin + threadIdx.x; i < imax; i += blockDim.x) {
    int k = N - i;
    double s = sr[i];
    acc[0] += (hr[i] * hr[i] + hr[k] * hr[k]) / s;
    acc[1] += ((dr[i] - hr[i]) * hr[i] + (dr[k] - hr[k]) * hr[k]) / s;
  }
  block_sum<2>(acc, red);
  if (threadIdx.x == 0) { out[2 * id] = 4.0 * acc[0]; out[2 * id + 1] = 4.0 * acc[1]; }
}

void launch_nwip_pairs(const double* d_h, const double* d_D, const double* d_S, int sn_stride, int N, int nifo,
                       int imin, int imax, double* d_out, cudaStream_t s) {
  k_nwip_pairs<<<nifo, 1024, 0, s>>>(d_h, d_D, d_S, sn_stride, N, imin, imax, d_out);
}

__global__ void k_nwip(const double* __restrict__ a, const double* __restrict__ b, const double* __restrict__ S,
                       int imin, int imax, int N, double* __restrict__ out) {
  __shared__ double red[32];
  double acc[1] = {0.0};
  for (int i = imin + threadIdx.x; i < imax; i += blockDim.x) {
    int k = N - i;
    acc[0] += (a[i] * b[i] + a[k] * b[k]) / S[i];
  }
  block_sum<1>(acc, red);
  if (threadIdx.x == 0) out[0] = 4.0 * acc[0];
}

void launch_nwip(const double* d_a, const double* d_b, const double* d_S, int imin, int imax, int N, double* d_out,
                 cudaStream_t s) {
  k_nwip<<<1, 1024, 0, s>>>(d_a, d_b, d_S, imin, imax, N, d_out);
}

// Lets the kernels with large dynamic shared memory (rotation tables of long tiles, heterodyne
// grids) use up to the device's opt-in limit.  Set once per device at initialisation, outside
// any stream capture.
// ---------------------------------------------------------------- sky-ring proposal
// update's fourth move (QuickCBC.c:2299-2331): a new sky position on the ring of equal time delay
// between two detectors (Ring_all, Utilities.c:1445-1560), the distance, polarisation, phase and
// inclination that keep the signal in both detectors (skymap_all with uvwz_all, uvwz_sol and
// exsolve_all, QuickCBC.c:7085-7150, 7295-7405, 7526-7545), and the log of the Jacobian of that
// map by one-sided differences of step 1e-6 (skydensity_all, QuickCBC.c:7411-7500).

// F+, Fx of detector l at psi = 0 (F_ant with psi = 0), as set_projection evaluates them
__device__ void sky_ant(int l, double alpha, double sind, double GMST, double& fp, double& fx) {
  const double cd = sqrt(1.0 - sind * sind);
  double sa, ca;
  sincos(GMST - alpha, &sa, &ca);
  double mp[21], mx[18];
  antenna_basis(1.0, 0.0, cd, sind, ca, -sa, mp, mx);
  fp = 0.0;
  fx = 0.0;
  for (int k = 0; k < 21; k++) fp += c_antP[l][k] * mp[k];
  for (int k = 0; k < 18; k++) fx += c_antX[l][k] * mx[k];
}

// delay from the geocentre to detector l (Times)
__device__ double sky_delay(int l, double alpha, double sind, double GMST) {
  const double cd = sqrt(1.0 - sind * sind);
  double sa, ca;
  sincos(GMST - alpha, &sa, &ca);
  return -(c_detpos[l][0] * cd * ca + c_detpos[l][1] * cd * sa + c_detpos[l][2] * sind) / kClight;
}

// new sky position: the propagation direction turned by `rot` about the line between detectors
// l1 and l2, which keeps the time delay between them
__device__ void sky_ring_rotate(const double* x, double* y, int l1, int l2, double GMST, double rot) {
  double z[3], zm = 0.0;
  for (int i = 0; i < 3; i++) {
    z[i] = c_detpos[l1][i] - c_detpos[l2][i];
    zm += z[i] * z[i];
  }
  zm = sqrt(zm);
  for (int i = 0; i < 3; i++) z[i] /= zm;
  const double sind = x[8], cosd = sqrt(1.0 - sind * sind);
  double sa, ca;
  sincos(x[7] - GMST, &sa, &ca);
  const double k[3] = {cosd * ca, -cosd * sa, sind};
  double cmu = z[0] * k[0] + z[1] * k[1] + z[2] * k[2];
  cmu = fmin(fmax(cmu, -0.999999), 0.999999);
  const double smu = sqrt(1.0 - cmu * cmu);
  const double u[3] = {(k[0] - cmu * z[0]) / smu, (k[1] - cmu * z[1]) / smu, (k[2] - cmu * z[2]) / smu};
  const double v[3] = {(z[1] * k[2] - z[2] * k[1]) / smu, (z[2] * k[0] - z[0] * k[2]) / smu,
                       (z[0] * k[1] - z[1] * k[0]) / smu};
  double sr, cr;
  sincos(rot, &sr, &cr);
  double kr[3];
  for (int i = 0; i < 3; i++) kr[i] = cmu * z[i] + smu * (cr * u[i] + sr * v[i]);
  y[8] = kr[2];
  double a = GMST - atan2(kr[1], kr[0]);
  if (a < 0.0) a += kTwoPi;
  y[7] = a;
}

// antenna patterns (psi = 0) of the two detectors at x's and at y's sky positions, and detector
// l1's delay at both: all that sky_map needs of the geometry
struct SkyPair {
  double fp1x, fc1x, fp2x, fc2x, fp1y, fc1y, fp2y, fc2y, dt1x, dt1y;
};
__device__ SkyPair sky_pair(const double* x, const double* y, double GMST, int l1, int l2) {
  SkyPair a;
  sky_ant(l1, x[7], x[8], GMST, a.fp1x, a.fc1x);
  sky_ant(l2, x[7], x[8], GMST, a.fp2x, a.fc2x);
  sky_ant(l1, y[7], y[8], GMST, a.fp1y, a.fc1y);
  sky_ant(l2, y[7], y[8], GMST, a.fp2y, a.fc2y);
  a.dt1x = sky_delay(l1, x[7], x[8], GMST);
  a.dt1y = sky_delay(l1, y[7], y[8], GMST);
  return a;
}

// distance, polarisation, phase, inclination and geocentre time at y's sky position that keep the
// strain in detectors l1 and l2 what it is at x
__device__ void sky_map(const double* x, double* y, const SkyPair& ap) {
  const double fp1x = ap.fp1x, fc1x = ap.fc1x, fp2x = ap.fp2x, fc2x = ap.fc2x;
  const double fp1y = ap.fp1y, fc1y = ap.fc1y, fp2y = ap.fp2y, fc2y = ap.fc2y;
  // the two polarisation amplitudes of x as (u, v, w, z)
  const double ci = x[10], Ap = 0.5 * (1.0 + ci * ci), ecc = -ci / Ap, A = Ap / exp(x[6]);
  double sphi, cphi, s2p, c2p;
  sincos(x[4], &sphi, &cphi);
  sincos(2.0 * x[9], &s2p, &c2p);
  const double ux = A * (cphi * c2p + ecc * sphi * s2p), vx = A * (cphi * s2p - ecc * sphi * c2p);
  const double wx = A * (sphi * c2p - ecc * cphi * s2p), zx = A * (sphi * s2p + ecc * cphi * c2p);
  // the same detector responses from y's antenna patterns
  const double den = fc1y * fp2y - fc2y * fp1y;
  const double a1 = fc1y * fc2x - fc1x * fc2y, a2 = fc1y * fp2x - fc2y * fp1x;
  const double b1 = fc1x * fp2y - fc2x * fp1y, b2 = fp2y * fp1x - fp1y * fp2x;
  const double uy = (vx * a1 + ux * a2) / den, vy = (vx * b1 + ux * b2) / den;
  const double wy = (zx * a1 + wx * a2) / den, zy = (zx * b1 + wx * b2) / den;
  // back to phase, polarisation, inclination and distance
  const double cross = uy * wy + vy * zy, diffn = (uy * uy + vy * vy) - (wy * wy + zy * zy);
  const double q = 2.0 * cross / diffn, rad = sqrt(1.0 + q * q);
  double t = atan2(2.0 * cross, diffn);
  if (t < 0.0) t += kTwoPi;
  const double phiy = 0.5 * t;
  const bool f1 = cos(t) > 0.0, f2 = cos(0.5 * t) > 0.0, f3 = sin(0.5 * t) > 0.0;
  const double pp = ((rad + 1.0) * (uy * uy + vy * vy) + (rad - 1.0) * (wy * wy + zy * zy) + 2.0 * q * cross) /
                    (2.0 * rad);
  const double det = uy * zy - vy * wy;
  const double e = f1 ? det / pp : pp / det;
  const double ciy = -(1.0 - sqrt(1.0 - e * e)) / e;
  const double c1 = (1.0 + rad) * uy + q * wy, c2 = (1.0 + rad) * vy + q * zy;
  double s;
  if (f1 && f2) s = atan2(c2, c1);
  else if (f1) s = atan2(-c2, -c1);
  else if (f3) s = atan2(e * c1, -e * c2);
  else s = atan2(-e * c1, e * c2);
  if (s < 0.0) s += kTwoPi;
  const double Ay = f1 ? sqrt(pp) : sqrt(pp) / fabs(e);
  y[9] = 0.5 * s;
  y[10] = ciy;
  y[6] = log((1.0 + ciy * ciy) / (2.0 * Ay));
  y[4] = phiy;
  y[5] = x[5] + ap.dt1x - ap.dt1y;
}

// parameters of the Jacobian: ln D, psi, phi, cos iota
__device__ __forceinline__ int sky_jidx(int j) { return j == 0 ? 6 : (j == 1 ? 9 : (j == 2 ? 4 : 10)); }
constexpr double kSkyEp = 1.0e-6;           // its difference step (skydensity_all)

// row i of the Jacobian from the perturbed image yp, with the other branch of the (psi, phi)
// solution mapped back onto y's
__device__ void sky_jrow(double* yp, const double* y, double* row) {
  if (fabs(yp[9] + 0.5 * kPi - y[9]) < fabs(yp[9] - y[9])) yp[9] += 0.5 * kPi;
  if (fabs(yp[9] - 0.5 * kPi - y[9]) < fabs(yp[9] - y[9])) yp[9] -= 0.5 * kPi;
  if (fabs(yp[4] + kPi - y[4]) < fabs(yp[4] - y[4])) yp[4] += kPi;
  if (fabs(yp[4] - kPi - y[4]) < fabs(yp[4] - y[4])) yp[4] -= kPi;
  for (int j = 0; j < 4; j++) row[j] = (yp[sky_jidx(j)] - y[sky_jidx(j)]) / kSkyEp;
}

// log |det| of a 4 x 4 matrix by elimination with partial pivoting
__device__ double log_abs_det4(double (&J)[4][4]) {
  double d = 1.0;
  for (int c = 0; c < 4; c++) {
    int p = c;
    for (int r = c + 1; r < 4; r++)
      if (fabs(J[r][c]) > fabs(J[p][c])) p = r;
    if (J[p][c] == 0.0) return -HUGE_VAL;
    if (p != c) {
      for (int k = 0; k < 4; k++) { const double t = J[c][k]; J[c][k] = J[p][k]; J[p][k] = t; }
      d = -d;
    }
    d *= J[c][c];
    for (int r = c + 1; r < 4; r++) {
      const double f = J[r][c] / J[c][c];
      for (int k = c; k < 4; k++) J[r][k] -= f * J[c][k];
    }
  }
  return log(fabs(d));
}

// One sky-ring proposal by a group of kSkyLanes lanes: lane 0 maps x, lanes 1..4 map x perturbed
// along the Jacobian's parameters (independent: the sky positions are fixed), then lane 0 gathers
// the rows by shuffles and takes log |det| (skydensity_all).  Every lane of the group must call it
// (the shuffles), with the same l1, l2, rot; y and the return value are lane 0's.
constexpr int kSkyLanes = 8;
__device__ double sky_ring_group(const double* x, double* y, int l1, int l2, double GMST, double rot, int gl) {
  double ys[11];
  for (int j = 0; j < 11; j++) ys[j] = x[j];
  sky_ring_rotate(x, ys, l1, l2, GMST, rot);
  const SkyPair ap = sky_pair(x, ys, GMST, l1, l2);
  double xp[11], yp[11];
  for (int j = 0; j < 11; j++) { xp[j] = x[j]; yp[j] = ys[j]; }
  if (gl >= 1 && gl <= 4) xp[sky_jidx(gl - 1)] += kSkyEp;
  if (gl <= 4) sky_map(xp, yp, ap);
  // lane 0's image to every lane of the group
  double yb[11];
  for (int j = 0; j < 11; j++) yb[j] = __shfl_sync(0xffffffffu, yp[j], 0, kSkyLanes);
  double row[4] = {0.0, 0.0, 0.0, 0.0};
  if (gl >= 1 && gl <= 4) sky_jrow(yp, yb, row);
  double J[4][4];
  for (int i = 0; i < 4; i++)
    for (int k = 0; k < 4; k++) J[i][k] = __shfl_sync(0xffffffffu, row[k], i + 1, kSkyLanes);
  for (int j = 0; j < 11; j++) y[j] = yb[j];
  return log_abs_det4(J);
}

// sky-ring proposals of the step: kSkyLanes lanes per chain, all lanes reach every shuffle
__global__ void k_pt_skyring(PtRun* __restrict__ runs, PtChains c, int B) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = t / kSkyLanes, gl = t % kSkyLanes;
  const bool ring = b < B && c.kind[b] == kKindSkyRing;
  // the group's draws, by lane 0 from the chain's stream
  int l1 = 0, l2 = 1;
  double rot = 0.0, half = 0.0, GMST = 0.0;
  const double* x = nullptr;
  if (ring) {
    const PtRun& r = runs[c.run[b]];
    GMST = r.GMST;
    x = c.x + (size_t)b * 11;
    if (gl == 0) {
      Xoshiro g;
      g.load(c.rng + (size_t)b * 4);
      int id1 = 0, id2 = 1;
      if (r.nifo > 2) {              // a random pair of the network's detectors
        id1 = min((int)(r.nifo * g.uniform()), r.nifo - 1);
        id2 = id1;
        for (int k = 0; id2 == id1 && k < 64; k++) id2 = min((int)(r.nifo * g.uniform()), r.nifo - 1);
        if (id2 == id1) id2 = (id1 + 1) % r.nifo;
      }
      l1 = r.labels[id1];
      l2 = r.labels[id2];
      rot = kTwoPi * g.uniform();
      half = g.uniform();
      g.store(c.rng + (size_t)b * 4);
    }
  }
  l1 = __shfl_sync(0xffffffffu, l1, 0, kSkyLanes);
  l2 = __shfl_sync(0xffffffffu, l2, 0, kSkyLanes);
  rot = __shfl_sync(0xffffffffu, rot, 0, kSkyLanes);
  half = __shfl_sync(0xffffffffu, half, 0, kSkyLanes);
  double xl[11];
  for (int j = 0; j < 11; j++) xl[j] = ring ? x[j] : 0.5;   // lanes of other chains map a dummy point
  double y[11];
  const double lj = sky_ring_group(xl, y, l1, l2, GMST, rot, gl);
  if (!ring || gl != 0) return;
  const PtRun& r = runs[c.run[b]];
  if (half > 0.5) {                  // the other half of the (phi, psi) range
    y[4] += kPi;
    y[9] += 0.5 * kPi;
  }
  pt_wrap_angles(y);
  for (int j = 0; j < 11; j++) c.y[(size_t)b * 11 + j] = y[j];
  c.jack[b] = lj;
  c.eo[b] = (isfinite(lj) && pt_in_prior(r.pmin, r.pmax, y)) ? r.slot : -1;
}

void launch_pt_skyring(PtRun* d_runs, PtChains c, int B, cudaStream_t s) {
  if (B > 0) k_pt_skyring<<<(B * kSkyLanes + 127) / 128, 128, 0, s>>>(d_runs, c, B);
}

// one point: the first group of the one warp maps it, the other groups map a dummy point
__global__ void k_sky_ring_map(const double* __restrict__ x, double* __restrict__ y, double GMST, int l1, int l2,
                               double rot, double* __restrict__ lj) {
  const int gl = threadIdx.x % kSkyLanes;
  double xl[11], yl[11];
  for (int j = 0; j < 11; j++) xl[j] = threadIdx.x < kSkyLanes ? x[j] : 0.5;
  const double v = sky_ring_group(xl, yl, l1, l2, GMST, rot, gl);
  if (threadIdx.x == 0) {
    for (int j = 0; j < 11; j++) y[j] = yl[j];
    *lj = v;
  }
}

void launch_sky_ring_map(const double* d_x, double* d_y, double GMST, int l1, int l2, double rot, double* d_lj,
                         cudaStream_t s) {
  k_sky_ring_map<<<1, 32, 0, s>>>(d_x, d_y, GMST, l1, l2, rot, d_lj);
}

void allow_dynamic_smem() {
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  auto allow = [&](const void* f) {
    cudaFuncAttributes a;
    if (cudaFuncGetAttributes(&a, f) == cudaSuccess)
      cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
  };
  allow((const void*)k_lnl_full_mixed<1>);
  allow((const void*)k_lnl_full_mixed<2>);
  allow((const void*)k_lnl_full_mixed<3>);
  allow((const void*)k_lnl_multi<kFP64>);
  allow((const void*)k_lnl_multi<kMixed>);
  allow((const void*)k_lnl_het_multi<kFP64>);
  allow((const void*)k_lnl_het_multi<kMixed>);
  allow((const void*)k_lnl_het<kFP64>);
  allow((const void*)k_lnl_het<kMixed>);
  allow((const void*)k_lnl_het_wide<kFP64>);
  allow((const void*)k_lnl_het_wide<kMixed>);
}

}  // namespace qcbc
