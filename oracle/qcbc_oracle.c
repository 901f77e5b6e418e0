/*
 * CPU restatement (FP64) of the QuickCBC likelihood hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA kernels, never the
 * product.  Every routine below restates the reference algorithm at the
 * cited file:line; parity with the reference itself (oracle/_ref) is tested
 * in tests/test_oracle.py (against the golden fixtures the reference wrote and
 * against the reference library on fresh seeds).
 *
 * Structure (not the reference's): one coefficient record per parameter set
 * (struct phd) holds everything frequency independent; phd_eval() maps one
 * geometric frequency to (amplitude, phase).  The phenomenological fits of
 * arXiv:1508.07253 Table V are kept as an 11-number table per coefficient
 * and evaluated by one routine; the intermediate amplitude is kept in
 * Newton (Hermite) form rather than expanded monomials.
 */
#include "qcbc_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "_build/qnm_table.h"

/* ---- constants (IMRPhenomD_internals.h:106-136, Constants.h, ConstCBC.h:31) */
#define O_PI 3.141592653589793238462643383279502884
#define O_PI_4 0.785398163397448309615660845819875721
#define O_GAMMA 0.577215664901532860606512090082402431
#define O_MSUN 1.988546954961461467461011951140572744e30
#define O_MTSUN 4.925491025543575903411922162094833998e-6
#define O_MRSUN 1.476625061404649406193430731479084713e3
#define O_TSUN 4.92569043916e-6          /* Constants.h:1, used by fbegin */
#define O_TPI 6.2831853071795862319959269370884
#define O_CLIGHT 299792458.0
#define O_H22FAC 0.31539156525252
#define O_FREF 100.0
#define F_CUT 0.2
#define AMP_FJOIN 0.014
#define PHI_FJOIN 0.018

/* ---------------------------------------------------------------- QNM spline */
/* Natural cubic spline of fring/fdamp over final spin (IMRPhenomD_internals.c:479-513,
 * GSL cspline = natural end conditions). */
static int qnm_n = 0;
static double *qnm_x = NULL, *qnm_y[2] = {NULL, NULL}, *qnm_m2[2] = {NULL, NULL};

static void spline_second_derivs(const double *x, const double *y, int n, double *M) {
  double *diag = (double *)malloc(sizeof(double) * n), *rhs = (double *)malloc(sizeof(double) * n);
  for (int i = 0; i < n; i++) M[i] = 0.0;
  for (int i = 1; i < n - 1; i++) {
    double h0 = x[i] - x[i - 1], h1 = x[i + 1] - x[i];
    diag[i] = 2.0 * (h0 + h1);
    rhs[i] = 6.0 * ((y[i + 1] - y[i]) / h1 - (y[i] - y[i - 1]) / h0);
  }
  for (int i = 2; i < n - 1; i++) {       /* eliminate sub-diagonal h_{i-1} */
    double w = (x[i] - x[i - 1]) / diag[i - 1];
    diag[i] -= w * (x[i] - x[i - 1]);
    rhs[i] -= w * rhs[i - 1];
  }
  for (int i = n - 2; i >= 1; i--) M[i] = (rhs[i] - (x[i + 1] - x[i]) * M[i + 1]) / diag[i];
  free(diag); free(rhs);
}

int ora_set_qnm(const double *a, const double *fr, const double *fd, int n) {
  free(qnm_x); free(qnm_y[0]); free(qnm_y[1]); free(qnm_m2[0]); free(qnm_m2[1]);
  qnm_n = n;
  qnm_x = (double *)malloc(sizeof(double) * n);
  memcpy(qnm_x, a, sizeof(double) * n);
  for (int k = 0; k < 2; k++) {
    qnm_y[k] = (double *)malloc(sizeof(double) * n);
    qnm_m2[k] = (double *)malloc(sizeof(double) * n);
    memcpy(qnm_y[k], k == 0 ? fr : fd, sizeof(double) * n);
    spline_second_derivs(qnm_x, qnm_y[k], n, qnm_m2[k]);
  }
  return 0;
}

static void qnm_default(void) {
  if (qnm_n == 0) ora_set_qnm(ORA_QNM_A, ORA_QNM_FRING, ORA_QNM_FDAMP, ORA_QNM_N);
}

static double qnm_eval(int k, double s) {
  int lo = 0, hi = qnm_n - 1;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (qnm_x[mid] > s) hi = mid; else lo = mid;
  }
  double h = qnm_x[lo + 1] - qnm_x[lo], dx = s - qnm_x[lo];
  double Ml = qnm_m2[k][lo], Mr = qnm_m2[k][lo + 1];
  double b = (qnm_y[k][lo + 1] - qnm_y[k][lo]) / h - h * (2.0 * Ml + Mr) / 6.0;
  return qnm_y[k][lo] + dx * (b + dx * (0.5 * Ml + dx * (Mr - Ml) / (6.0 * h)));
}

/* ------------------------------------------------- Table V fits (1508.07253) */
/* lambda = l00 + l10 eta + (l01 + l11 eta + l21 eta^2) xi + (..) xi^2 + (..) xi^3,
 * xi = chiPN - 1 (IMRPhenomD_internals.c:537-1399, one function per coefficient). */
enum { F_RHO1, F_RHO2, F_RHO3, F_GAM1, F_GAM2, F_GAM3, F_V2, F_AL1, F_AL2, F_AL3, F_AL4, F_AL5,
       F_BE1, F_BE2, F_BE3, F_SI1, F_SI2, F_SI3, F_SI4, F_COUNT };
static const double FITS[F_COUNT][11] = {
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

static double fit(int k, double eta, double chi) {
  const double *c = FITS[k];
  double xi = -1 + chi, xi2 = xi * xi, xi3 = xi2 * xi, eta2 = eta * eta;
  return c[0] + c[1] * eta + (c[2] + c[3] * eta + c[4] * eta2) * xi + (c[5] + c[6] * eta + c[7] * eta2) * xi2 +
         (c[8] + c[9] * eta + c[10] * eta2) * xi3;
}

/* Powers of a positive number from one pow(x, 1/6) (IMRPhenomD_internals.c:515-533). */
typedef struct { double sixth, third, two_thirds, four_thirds, five_thirds, two, seven_thirds, eight_thirds; } pw_t;
static pw_t powers(double x) {
  pw_t p;
  if (x < 0.0) x = 1.0e-10;
  p.sixth = pow(x, 1 / 6.0);
  p.third = p.sixth * p.sixth;
  p.two_thirds = x / p.third;
  p.four_thirds = x * p.third;
  p.five_thirds = p.four_thirds * p.third;
  p.two = x * x;
  p.seven_thirds = p.third * p.two;
  p.eight_thirds = p.two_thirds * p.two;
  return p;
}

/* ------------------------------------------------------- coefficient record */
typedef struct {
  double eta, chi1, chi2, chi, fRD, fDM, fmax;   /* fmax = fmaxCalc */
  double pi_pw[3];                               /* pi^{1/3}, pi^{2/3}, pi^{5/3} ... see setup */
  pw_t pip;
  /* amplitude */
  double a0;                                     /* amp0Func(eta) */
  double ai[8];                                  /* inspiral prefactors: Mf^{2/3},Mf,4/3,5/3,2,7/3,8/3,3 */
  double g1, g2, g3;
  double hx1, hx2, hx3, hc[5];                   /* intermediate Hermite nodes + Newton coefficients */
  /* phase */
  double pv[8], pvl[8];                          /* TaylorF2 v[k], vlogv[k] (k<8) incl. pfaN */
  double pi_[13];                                /* PhiInsAnsatzInt prefactors */
  double s1, s2, s3, s4, b1, b2, b3, al1, al2, al3, al4, al5;
  double C1Int, C2Int, C1MRD, C2MRD, fMRDJoin;
  double t0, MfRef, phi_pre;
  /* dimensional */
  double Msec, fCut, amp_scale;
} phd;

/* Final spin, eq. 3.6 of arXiv:1508.07250 (IMRPhenomD_internals.c:402-434). */
static double final_spin(double eta, double chi1, double chi2) {
  double Seta = sqrt(1.0 - 4.0 * eta), m1 = 0.5 * (1.0 + Seta), m2 = 0.5 * (1.0 - Seta);
  double s = m1 * m1 * chi1 + m2 * m2 * chi2;
  double e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta, s2 = s * s, s3 = s2 * s, s4 = s3 * s;
  return 3.4641016151377544 * eta - 4.399247300629289 * e2 + 9.397292189321194 * e3 - 13.180949901606242 * e4 +
         (1 - 0.0850917821418767 * eta - 5.837029316602263 * e2) * s +
         (0.1014665242971878 * eta - 2.0967746996832157 * e2) * s2 +
         (-1.3546806617824356 * eta + 4.108962025369336 * e2) * s3 +
         (-0.8676969352555539 * eta + 2.064046835273906 * e2) * s4;
}

/* Radiated energy, eqs. 3.7-3.8 of arXiv:1508.07250 (IMRPhenomD_internals.c:440-474). */
static double erad(double eta, double chi1, double chi2) {
  double Seta = sqrt(1.0 - 4.0 * eta), m1 = 0.5 * (1.0 + Seta), m2 = 0.5 * (1.0 - Seta);
  double m1s = m1 * m1, m2s = m2 * m2, s = (m1s * chi1 + m2s * chi2) / (m1s + m2s);
  double e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta;
  return ((0.055974469826360077 * eta + 0.5809510763115132 * e2 - 0.9606726679372312 * e3 + 3.352411249771192 * e4) *
          (1. + (-0.0030302335878845507 - 2.0066110851351073 * eta + 7.7050567802399215 * e2) * s)) /
         (1. + (-0.6714403054720589 - 1.4756929437702908 * eta + 7.304676214885011 * e2) * s);
}

static double amp_mrd(const phd *c, double f) {          /* eq. 19, internals.c:715-726 */
  double fg = c->fDM * c->g3, df = f - c->fRD;
  return exp(-df * c->g2 / fg) * (fg * c->g1) / (df * df + fg * fg);
}
static double damp_mrd(const phd *c, double f) {         /* d/df of amp_mrd, internals.c:731-747 */
  double fg = c->fDM * c->g3, df = f - c->fRD, den = df * df + fg * fg;
  return amp_mrd(c, f) * (-c->g2 / fg - 2.0 * df / den);
}
static double amp_ins(const phd *c, double Mf, const pw_t *p) {   /* eqs. 29-30, internals.c:594-604 */
  return 1.0 + p->two_thirds * c->ai[0] + Mf * c->ai[1] + p->four_thirds * c->ai[2] + p->five_thirds * c->ai[3] +
         p->two * c->ai[4] + p->seven_thirds * c->ai[5] + p->eight_thirds * c->ai[6] + Mf * p->two * c->ai[7];
}
static double damp_ins(const phd *c, double Mf) {        /* d/dMf of amp_ins (internals.c:660-692) */
  pw_t p = powers(Mf);
  return (2.0 / 3.0) * c->ai[0] / p.third + c->ai[1] + (4.0 / 3.0) * c->ai[2] * p.third +
         (5.0 / 3.0) * c->ai[3] * p.two_thirds + 2.0 * c->ai[4] * Mf + (7.0 / 3.0) * c->ai[5] * p.four_thirds +
         (8.0 / 3.0) * c->ai[6] * p.five_thirds + 3.0 * c->ai[7] * p.two;
}

/* TaylorF2 phase coefficients with the 3.5PN spin-orbit, 3PN spin-orbit +
 * spin-spin, 2.5PN, 2PN, 1.5PN spin terms, all times pfaN = 3/(128 eta)
 * (IMRPhenomD_internals.c:244-365), then minus the 3PN spin-spin term that
 * PhenomD was not tuned with (IMRPhenomD.c:478, internals.c:1619-1629). */
static void taylorf2(phd *c, double m1, double m2) {
  double mt = m1 + m2, d = (m1 - m2) / mt, eta = m1 * m2 / mt / mt, m1M = m1 / mt, m2M = m2 / mt;
  double x1 = c->chi1, x2 = c->chi2;
  double SL = m1M * m1M * x1 + m2M * m2M * x2, dSigmaL = d * (m2M * x2 - m1M * x1);
  double pfaN = 3.0 / (128.0 * eta);
  double v[8] = {0}, vl[8] = {0};
  v[0] = 1.0;
  v[2] = 5.0 * (743.0 / 84.0 + 11.0 * eta) / 9.0;
  v[3] = -16.0 * O_PI;
  v[4] = 5.0 * (3058.673 / 7.056 + 5429.0 / 7.0 * eta + 617.0 * eta * eta) / 72.0;
  v[5] = 5.0 / 9.0 * (7729.0 / 84.0 - 13.0 * eta) * O_PI;
  vl[5] = 5.0 / 3.0 * (7729.0 / 84.0 - 13.0 * eta) * O_PI;
  v[6] = (11583.231236531 / 4.694215680 - 640.0 / 3.0 * O_PI * O_PI - 6848.0 / 21.0 * O_GAMMA) +
         eta * (-15737.765635 / 3.048192 + 2255. / 12. * O_PI * O_PI) + eta * eta * 76055.0 / 1728.0 -
         eta * eta * eta * 127825.0 / 1296.0;
  v[6] += (-6848.0 / 21.0) * log(4.);
  vl[6] = -6848.0 / 21.0;
  v[7] = O_PI * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta * eta);
  /* spin terms (quadrupole-monopole parameters = 1) */
  double sigma = eta * (721.0 / 48.0 * x1 * x2 - 247.0 / 48.0 * x1 * x2);
  sigma += (720.0 - 1.0) / 96.0 * m1M * m1M * x1 * x1;
  sigma += (720.0 - 1.0) / 96.0 * m2M * m2M * x2 * x2;
  sigma -= (240.0 - 7.0) / 96.0 * m1M * m1M * x1 * x1;
  sigma -= (240.0 - 7.0) / 96.0 * m2M * m2M * x2 * x2;
  double ss3 = (326.75 / 1.12 + 557.5 / 1.8 * eta) * eta * x1 * x2;
  ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m1M - 120.0 * m1M * m1M) +
          (-4108.25 / 6.72 - 108.5 / 1.2 * m1M + 125.5 / 3.6 * m1M * m1M)) * m1M * m1M * x1 * x1;
  ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m2M - 120.0 * m2M * m2M) +
          (-4108.25 / 6.72 - 108.5 / 1.2 * m2M + 125.5 / 3.6 * m2M * m2M)) * m2M * m2M * x2 * x2;
  double gam = (554345.0 / 1134.0 + 110.0 * eta / 9.0) * SL + (13915.0 / 84.0 - 10.0 * eta / 3.0) * dSigmaL;
  v[7] += (-8980424995.0 / 762048.0 + 6586595.0 * eta / 756.0 - 305.0 * eta * eta / 36.0) * SL -
          (170978035.0 / 48384.0 - 2876425.0 * eta / 672.0 - 4735.0 * eta * eta / 144.0) * dSigmaL;
  v[6] += O_PI * (3760.0 * SL + 1490.0 * dSigmaL) / 3.0 + ss3;
  v[5] += -1.0 * gam;
  vl[5] += -3.0 * gam;
  v[4] += -10.0 * sigma;
  v[3] += 188.0 * SL / 3.0 + 25.0 * dSigmaL;
  for (int k = 0; k < 8; k++) { c->pv[k] = v[k] * pfaN; c->pvl[k] = vl[k] * pfaN; }
  c->pv[6] -= ss3 * c->pv[0];
}

static double phi_ins(const phd *c, double Mf, const pw_t *p) {   /* eqs. 27-28, internals.c:1399-1425 */
  double v = p->third * c->pip.third, logv = log(v);
  const double *q = c->pi_;
  double ph = q[0];
  ph += q[1] * p->two_thirds;
  ph += q[2] * p->third;
  ph += q[3] * logv * p->third;
  ph += q[4] * logv;
  ph += q[5] / p->third;
  ph += q[6] / p->two_thirds;
  ph += q[7] / Mf;
  ph += q[8] / p->five_thirds;
  ph += (q[9] * Mf + q[10] * p->four_thirds + q[11] * p->five_thirds + q[12] * p->two) / c->eta;
  return ph;
}
static double dphi_ins(const phd *c, double Mf) {        /* internals.c:1455-1493 */
  double v = cbrt(O_PI * Mf), logv = log(v);
  double v2 = v * v, v3 = v * v2, v4 = v * v3, v5 = v * v4, v6 = v * v5, v7 = v * v6, v8 = v * v7;
  double D = 0.0;
  D += 2.0 * c->pv[7] * v7;
  D += (c->pv[6] + c->pvl[6] * (1.0 + logv)) * v6;
  D += c->pvl[5] * v5;
  D += -1.0 * c->pv[4] * v4;
  D += -2.0 * c->pv[3] * v3;
  D += -3.0 * c->pv[2] * v2;
  D += -4.0 * c->pv[1] * v;
  D += -5.0 * c->pv[0];
  D /= v8 * 3.0 / O_PI;
  D += (c->s1 + c->s2 * v / c->pip.third + c->s3 * v2 / c->pip.two_thirds + (c->s4 / O_PI) * v3) / c->eta;
  return D;
}
static double phi_int(const phd *c, double f) { return c->b1 * f - c->b3 / (3. * f * f * f) + c->b2 * log(f); }
static double dphi_int(const phd *c, double f) { return (c->b1 + c->b3 / (f * f * f * f) + c->b2 / f) / c->eta; }
static double phi_mrd(const phd *c, double f) {          /* eq. 14, internals.c:1222-1233 */
  double sq = sqrt(f), f34 = sqrt(f * sq);
  return -(c->al2 / f) + (4.0 / 3.0) * (c->al3 * f34) + c->al1 * f + c->al4 * atan((f - c->al5 * c->fRD) / c->fDM);
}
static double dphi_mrd(const phd *c, double f) {         /* internals.c:1238-1240 */
  double x = f - c->al5 * c->fRD;
  return (c->al1 + c->al2 / (f * f) + c->al3 / pow(f, 0.25) + c->al4 / (c->fDM * (1 + x * x / (c->fDM * c->fDM)))) / c->eta;
}

static double phase_geom(const phd *c, double Mf, const pw_t *p) {   /* internals.c:1590-1617 */
  if (Mf < PHI_FJOIN) return phi_ins(c, Mf, p);
  if (Mf >= c->fMRDJoin) return phi_mrd(c, Mf) / c->eta + c->C1MRD + c->C2MRD * Mf;
  return phi_int(c, Mf) / c->eta + c->C1Int + c->C2Int * Mf;
}
static double amp_geom(const phd *c, double Mf, const pw_t *p) {     /* internals.c:1107-1134 */
  double pre = c->a0 / (Mf * p->sixth);
  if (Mf < AMP_FJOIN) return pre * amp_ins(c, Mf, p);
  if (Mf >= c->fmax) return pre * amp_mrd(c, Mf);
  double x = Mf - c->hx1;
  double poly = c->hc[0] + x * (c->hc[1] + x * (c->hc[2] + (Mf - c->hx2) * (c->hc[3] + (Mf - c->hx3) * c->hc[4])));
  return pre * poly;
}

/* All frequency-independent work for one parameter set
 * (IMRPhenomD.c:413-503 + the coefficient routines it calls). */
static void phd_setup(phd *c, double phi0, double fRef, double m1_in, double m2_in, double chi1_in,
                      double chi2_in, double dist) {
  qnm_default();
  double m1 = m1_in, m2 = m2_in, chi1 = chi1_in, chi2 = chi2_in;
  if (!(m1_in > m2_in)) { m1 = m2_in; m2 = m1_in; chi1 = chi2_in; chi2 = chi1_in; }
  memset(c, 0, sizeof(*c));
  c->pip = powers(O_PI);
  double M = m1 + m2, eta = m1 * m2 / (M * M);
  c->eta = eta; c->chi1 = chi1; c->chi2 = chi2;
  c->Msec = M * O_MTSUN;
  c->amp_scale = M * O_MRSUN * M * O_MTSUN / dist;
  c->fCut = F_CUT / c->Msec;
  double Seta = sqrt(1.0 - 4.0 * eta);
  c->chi = (chi1 + chi2) / 2.0 * (1.0 - eta * 76.0 / 113.0) + Seta * ((chi1 - chi2) / 2.0);   /* internals.c:371-377 */
  double fs = final_spin(eta, chi1, chi2), er = erad(eta, chi1, chi2);
  c->fRD = qnm_eval(0, fs) / (1.0 - er);
  c->fDM = qnm_eval(1, fs) / (1.0 - er);
  double chi = c->chi;
  /* amplitude (internals.c:1072-1100) */
  c->g1 = fit(F_GAM1, eta, chi); c->g2 = fit(F_GAM2, eta, chi); c->g3 = fit(F_GAM3, eta, chi);
  if (c->g2 <= 1)
    c->fmax = fabs(c->fRD + (c->fDM * (-1 + sqrt(1 - c->g2 * c->g2)) * c->g3) / c->g2);
  else
    c->fmax = fabs(c->fRD + (c->fDM * (-1) * c->g3) / c->g2);
  c->a0 = (sqrt(2.0 / 3.0) * sqrt(eta)) / c->pip.sixth;
  /* inspiral amplitude prefactors, Appendix B of 1508.07253 (internals.c:612-654) */
  {
    double x1 = chi1, x2 = chi2, x1s = x1 * x1, x2s = x2 * x2, e2 = eta * eta, e3 = eta * e2, Pi = O_PI;
    double Pi2 = c->pip.two;
    c->ai[0] = ((-969 + 1804 * eta) * c->pip.two_thirds) / 672.;
    c->ai[1] = ((x1 * (81 * (1 + Seta) - 44 * eta) + x2 * (81 - 81 * Seta - 44 * eta)) * Pi) / 48.;
    c->ai[2] = ((-27312085.0 - 10287648 * x2s - 10287648 * x1s * (1 + Seta) + 10287648 * x2s * Seta +
                 24 * (-1975055 + 857304 * x1s - 994896 * x1 * x2 + 857304 * x2s) * eta + 35371056 * e2) *
                c->pip.four_thirds) / 8.128512e6;
    c->ai[3] = (c->pip.five_thirds * (x2 * (-285197 * (-1 + Seta) + 4 * (-91902 + 1579 * Seta) * eta - 35632 * e2) +
                                      x1 * (285197 * (1 + Seta) - 4 * (91902 + 1579 * Seta) * eta - 35632 * e2) +
                                      42840 * (-1.0 + 4 * eta) * Pi)) / 32256.;
    c->ai[4] = -(Pi2 * (-336 * (-3248849057.0 + 2943675504 * x1s - 3339284256 * x1 * x2 + 2943675504 * x2s) * e2 -
                        324322727232 * e3 -
                        7 * (-177520268561 + 107414046432 * x2s + 107414046432 * x1s * (1 + Seta) -
                             107414046432 * x2s * Seta + 11087290368 * (x1 + x2 + x1 * Seta - x2 * Seta) * Pi) +
                        12 * eta * (-545384828789 - 176491177632 * x1 * x2 + 202603761360 * x2s +
                                    77616 * x1s * (2610335 + 995766 * Seta) - 77287373856 * x2s * Seta +
                                    5841690624 * (x1 + x2) * Pi + 21384760320 * Pi2))) / 6.0085960704e10;
    c->ai[5] = fit(F_RHO1, eta, chi);
    c->ai[6] = fit(F_RHO2, eta, chi);
    c->ai[7] = fit(F_RHO3, eta, chi);
  }
  /* intermediate amplitude: quartic through (f1,v1,d1), (f2,v2), (f3,v3,d2)
   * -- eqs. 21-26 of 1508.07253 -- in Newton form on nodes f1,f1,f2,f3,f3
   * (the reference solves the same conditions in closed form, internals.c:1005-1067). */
  {
    double f1 = AMP_FJOIN, f3 = c->fmax, f2 = f1 + (f3 - f1) / 2.0;
    pw_t p1 = powers(f1);
    double v1 = amp_ins(c, f1, &p1), d1 = damp_ins(c, f1);
    double v3 = amp_mrd(c, f3), d2 = damp_mrd(c, f3);
    double v2 = fit(F_V2, eta, chi);
    double q01 = d1, q12 = (v2 - v1) / (f2 - f1), q23 = (v3 - v2) / (f3 - f2), q34 = d2;
    double q012 = (q12 - q01) / (f2 - f1), q123 = (q23 - q12) / (f3 - f1), q234 = (q34 - q23) / (f3 - f2);
    double q0123 = (q123 - q012) / (f3 - f1), q1234 = (q234 - q123) / (f3 - f1);
    double q01234 = (q1234 - q0123) / (f3 - f1);
    c->hx1 = f1; c->hx2 = f2; c->hx3 = f3;
    c->hc[0] = v1; c->hc[1] = q01; c->hc[2] = q012; c->hc[3] = q0123; c->hc[4] = q01234;
  }
  /* phase (internals.c:1509-1540, 1547-1584) */
  c->s1 = fit(F_SI1, eta, chi); c->s2 = fit(F_SI2, eta, chi); c->s3 = fit(F_SI3, eta, chi); c->s4 = fit(F_SI4, eta, chi);
  c->b1 = fit(F_BE1, eta, chi); c->b2 = fit(F_BE2, eta, chi); c->b3 = fit(F_BE3, eta, chi);
  c->al1 = fit(F_AL1, eta, chi); c->al2 = fit(F_AL2, eta, chi); c->al3 = fit(F_AL3, eta, chi);
  c->al4 = fit(F_AL4, eta, chi); c->al5 = fit(F_AL5, eta, chi);
  taylorf2(c, m1, m2);
  {
    double *q = c->pi_;
    q[0] = c->pv[5] - O_PI_4;
    q[1] = c->pv[7] * c->pip.two_thirds;
    q[2] = c->pv[6] * c->pip.third;
    q[3] = c->pvl[6] * c->pip.third;
    q[4] = c->pvl[5];
    q[5] = c->pv[4] / c->pip.third;
    q[6] = c->pv[3] / c->pip.two_thirds;
    q[7] = c->pv[2] / O_PI;
    q[8] = c->pv[0] / c->pip.five_thirds;
    q[9] = c->s1;
    q[10] = c->s2 * 3.0 / 4.0;
    q[11] = c->s3 * 3.0 / 5.0;
    q[12] = c->s4 / 2.0;
  }
  {
    double fj = PHI_FJOIN;
    c->C2Int = dphi_ins(c, fj) - dphi_int(c, fj);
    pw_t pj = powers(fj);
    c->C1Int = phi_ins(c, fj, &pj) - 1.0 / eta * phi_int(c, fj) - c->C2Int * fj;
    c->fMRDJoin = 0.5 * c->fRD;
    double fm = c->fMRDJoin;
    double phiT = 1.0 / eta * phi_int(c, fm) + c->C1Int + c->C2Int * fm;
    double dphiT = c->C2Int + dphi_int(c, fm);
    c->C2MRD = dphiT - dphi_mrd(c, fm);
    c->C1MRD = phiT - 1.0 / eta * phi_mrd(c, fm) - c->C2MRD * fm;
  }
  c->t0 = dphi_mrd(c, c->fmax);
  c->MfRef = c->Msec * fRef;
  pw_t pr = powers(c->MfRef);
  c->phi_pre = 2. * phi0 + phase_geom(c, c->MfRef, &pr);
}

/* amplitude and phase at one frequency in Hz (IMRPhenomD.c:527-556) */
static void phd_eval(const phd *c, double f, double *amp, double *phase) {
  if (f > c->fCut) { *amp = 0.0; *phase = 0.0; return; }
  double Mf = c->Msec * f;
  pw_t p = powers(Mf);
  double a = amp_geom(c, Mf, &p);
  double ph = phase_geom(c, Mf, &p);
  ph -= c->t0 * (Mf - c->MfRef) + c->phi_pre;
  *amp = c->amp_scale * a;
  *phase = ph;
}

int ora_amp_phase(const double *freq, int n, double phi0, double fRef, double m1_SI, double m2_SI,
                  double chi1, double chi2, double dist, double *amp, double *phase) {
  phd c;
  phd_setup(&c, phi0, fRef, m1_SI / O_MSUN, m2_SI / O_MSUN, chi1, chi2, dist);
  for (int i = 0; i < n; i++) phd_eval(&c, freq[i], &amp[i], &phase[i]);
  return 0;
}

/* ------------------------------------------------- start frequency (3PN) */
/* Frequency at time tc before merger, 3PN t(f) inversion (Utilities.c:587-629). */
double ora_fbegin(const double *p) {
  const double gE = 0.5772156649, PI = O_PI;
  double Mc = exp(p[0]) / O_MSUN * O_TSUN, M = exp(p[1]) / O_MSUN * O_TSUN;
  double eta = pow(Mc / M, 5.0 / 3.0);
  if (eta > 0.25) eta = 0.25;
  double dm = sqrt(1.0 - 4.0 * eta), m1 = M * (1.0 + dm) / 2.0, m2 = M * (1.0 - dm) / 2.0;
  double c1 = p[2], c2 = p[3], chi = (m1 * c1 + m2 * c2) / M, tc = p[5];
  double th = pow(eta * tc / (5.0 * M), -1.0 / 8.0);
  double t2 = th * th, t3 = t2 * th, t4 = t2 * t2, t5 = t2 * t3, t6 = t3 * t3;
  double PN1 = (11.0 / 32.0 * eta + 743.0 / 2688.0) * t2;
  double PN15 = -3.0 * PI / 10.0 * t3 + (1.0 / 160.0) * (113.0 * chi - 38.0 * eta * (c1 + c2)) * t3;
  double PN2 = (1855099.0 / 14450688.0 + 56975.0 / 258048.0 * eta + 371.0 / 2048.0 * eta * eta) * t4 +
               (1.0 / 14450688.0) * (-3386880.0 * chi * chi + 1512.0 * c1 * c2) * t4;
  double PN25 = -(7729.0 / 21504.0 - 13.0 / 256.0 * eta) * PI * t5;
  double PN3 = (-720817631400877.0 / 288412611379200.0 + 53.0 / 200.0 * PI * PI + 107.0 / 280.0 * gE +
                (25302017977.0 / 4161798144.0 - 451.0 / 2048.0 * PI * PI) * eta - 30913.0 / 1835008.0 * eta * eta +
                235925.0 / 1769472.0 * eta * eta * eta + 107.0 / 280.0 * log(2.0 * th)) * t6;
  return t3 / (8.0 * M * PI) * (1.0 + PN1 + PN15 + PN2 + PN25 + PN3);
}

/* ------------------------------------------------- antenna patterns, delays */
/* F+ and Fx for H1, L1, V1 as polynomials in cos/sin of psi, delta and
 * (alpha - GMST) with the reference's rounded coefficients
 * (Utilities.c:1004-1076).  exps: cpsi, spsi, cdelta, sdelta, calpha, salpha. */
typedef struct { double c; unsigned char e[6]; } mono;
static const mono ANT_P[3][21] = {
  {{0.3104536562,{2,0,0,0,1,1}},{0.494778091,{0,0,1,1,1,0}},{1.424276331,{2,0,0,2,2,0}},{-0.4559956644,{0,0,1,1,0,1}},
   {-0.1552268274,{0,0,0,2,1,1}},{0.3104536562,{1,1,0,1,0,0}},{-0.1552268276,{0,0,0,0,1,1}},{-0.4928680677,{2,0,0,2,0,0}},
   {1.424276334,{2,0,0,0,2,0}},{0.3104536558,{2,0,0,2,1,1}},{-0.9119913289,{1,1,1,0,1,0}},{-0.9314082637,{2,0,0,0,0,0}},
   {-0.712138166,{0,0,0,0,2,0}},{0.9119913288,{2,0,1,1,0,1}},{-0.6209073089,{1,1,0,1,2,0}},{2.848552667,{1,1,0,1,1,1}},
   {-0.9895561804,{2,0,1,1,1,0}},{0.2464340337,{0,0,0,2,0,0}},{-0.9895561811,{1,1,1,0,0,1}},{-0.7121381653,{0,0,0,2,2,0}},
   {0.4657041323,{0,0,0,0,0,0}}},
  {{-0.5608410611,{2,0,0,0,1,1}},{-0.4945891833,{0,0,1,1,1,0}},{-1.040573095,{2,0,0,2,2,0}},{0.363231261,{0,0,1,1,0,1}},
   {0.2804205304,{0,0,0,2,1,1}},{-0.5608410611,{1,1,0,1,0,0}},{0.2804205305,{0,0,0,0,1,1}},{-0.3865389475,{2,0,0,2,0,0}},
   {-1.040573095,{2,0,0,0,2,0}},{-0.5608410611,{2,0,0,2,1,1}},{0.7264625218,{1,1,1,0,1,0}},{-0.7135560209,{0,0,0,0,0,0}},
   {1.427112041,{2,0,0,0,0,0}},{0.5202865467,{0,0,0,0,2,0}},{-0.7264625224,{2,0,1,1,0,1}},{1.121682123,{1,1,0,1,2,0}},
   {-2.081146187,{1,1,0,1,1,1}},{0.9891783667,{2,0,1,1,1,0}},{0.1932694762,{0,0,0,2,0,0}},{0.9891783666,{1,1,1,0,0,1}},
   {0.5202865474,{0,0,0,2,2,0}}},
  {{0.3963351156,{2,0,0,0,1,1}},{0.465152434,{0,0,1,1,1,0}},{-1.383399753,{2,0,0,2,2,0}},{-0.3756662059,{0,0,1,1,0,1}},
   {-0.1981675579,{0,0,0,2,1,1}},{0.3963351153,{1,1,0,1,0,0}},{-0.1981675578,{0,0,0,0,1,1}},{1.303555289,{2,0,0,2,0,0}},
   {-1.383399752,{2,0,0,0,2,0}},{-0.039922232,{0,0,0,0,0,0}},{0.3963351158,{2,0,0,2,1,1}},{-0.7513324118,{1,1,1,0,1,0}},
   {0.0798444642,{2,0,0,0,0,0}},{0.6916998761,{0,0,0,0,2,0}},{0.7513324118,{2,0,1,1,0,1}},{-0.792670233,{1,1,0,1,2,0}},
   {-2.766799504,{1,1,0,1,1,1}},{-0.9303048681,{2,0,1,1,1,0}},{-0.6517776444,{0,0,0,2,0,0}},{-0.9303048681,{1,1,1,0,0,1}},
   {0.6916998765,{0,0,0,2,2,0}}},
};
static const mono ANT_X[3][18] = {
  {{-1.424276332,{1,1,0,2,2,0}},{-0.3104536551,{1,1,0,0,1,1}},{-0.6209073087,{2,0,0,1,2,0}},{-0.989556182,{2,0,1,0,0,1}},
   {0.3104536561,{0,0,0,1,2,0}},{0.9895561812,{1,1,1,1,1,0}},{-1.424276332,{0,0,0,1,1,1}},{-0.9119913298,{2,0,1,0,1,0}},
   {2.848552668,{2,0,0,1,1,1}},{-0.911991329,{1,1,1,1,0,1}},{0.9314082638,{1,1,0,0,0,0}},{-1.424276333,{1,1,0,0,2,0}},
   {-0.1552268276,{0,0,0,1,0,0}},{0.3104536564,{2,0,0,1,0,0}},{0.4947780906,{0,0,1,0,0,1}},{-0.3104536556,{1,1,0,2,1,1}},
   {0.4928680679,{1,1,0,2,0,0}},{0.4559956636,{0,0,1,0,1,0}}},
  {{1.040573095,{1,1,0,2,2,0}},{0.5608410611,{1,1,0,0,1,1}},{1.121682122,{2,0,0,1,2,0}},{0.9891783668,{2,0,1,0,0,1}},
   {-0.5608410611,{0,0,0,1,2,0}},{-0.9891783668,{1,1,1,1,1,0}},{1.040573095,{0,0,0,1,1,1}},{0.7264625222,{2,0,1,0,1,0}},
   {-2.081146187,{2,0,0,1,1,1}},{0.7264625218,{1,1,1,1,0,1}},{-1.427112042,{1,1,0,0,0,0}},{1.040573094,{1,1,0,0,2,0}},
   {0.2804205304,{0,0,0,1,0,0}},{-0.560841061,{2,0,0,1,0,0}},{-0.4945891833,{0,0,1,0,0,1}},{0.5608410611,{1,1,0,2,1,1}},
   {0.3865389466,{1,1,0,2,0,0}},{-0.3632312614,{0,0,1,0,1,0}}},
  {{1.383399753,{1,1,0,2,2,0}},{-0.396335116,{1,1,0,0,1,1}},{-0.7926702326,{2,0,0,1,2,0}},{-0.9303048681,{2,0,1,0,0,1}},
   {0.3963351158,{0,0,0,1,2,0}},{0.9303048686,{1,1,1,1,1,0}},{1.383399752,{0,0,0,1,1,1}},{-0.7513324118,{2,0,1,0,1,0}},
   {-2.766799505,{2,0,0,1,1,1}},{-0.7513324118,{1,1,1,1,0,1}},{-0.0798444646,{1,1,0,0,0,0}},{1.383399752,{1,1,0,0,2,0}},
   {-0.1981675579,{0,0,0,1,0,0}},{0.3963351158,{2,0,0,1,0,0}},{0.465152434,{0,0,1,0,0,1}},{-0.3963351158,{1,1,0,2,1,1}},
   {-1.303555288,{1,1,0,2,0,0}},{0.3756662059,{0,0,1,0,1,0}}},
};

static double mono_sum(const mono *t, int n, const double *v) {
  double s = 0.0;
  for (int k = 0; k < n; k++) {
    double term = t[k].c;
    for (int j = 0; j < 6; j++)
      for (int e = 0; e < t[k].e[j]; e++) term *= v[j];
    s += term;
  }
  return s;
}

void ora_antenna(double psi, double alpha, double sindelta, double GMST, int ifo, double *fpfc) {
  double v[6] = {cos(psi), sin(psi), sqrt(1.0 - sindelta * sindelta), sindelta, cos(alpha - GMST), sin(alpha - GMST)};
  if (ifo < 0 || ifo > 2) { fpfc[0] = fpfc[1] = 0.0; return; }
  fpfc[0] = mono_sum(ANT_P[ifo], 21, v);
  fpfc[1] = mono_sum(ANT_X[ifo], 18, v);
}

/* Earth-fixed detector vertex positions in metres (Utilities.c:1078-1109). */
static const double DET_R[3][3] = {
  {-2.161414928e6, 3.834695183e6, 4.600350224e6},
  {-74276.04192, 5.496283721e6, 3.224257016e6},
  {4546374.098, -842989.6972, 4378576.963},
};
void ora_delays(double alpha, double sindelta, double GMST, double *dt3) {
  double cd = sqrt(1.0 - sindelta * sindelta), ca = cos(GMST - alpha), sa = sin(GMST - alpha);
  for (int k = 0; k < 3; k++) {
    double r = DET_R[k][0] * cd * ca + DET_R[k][1] * cd * sa + DET_R[k][2] * sindelta;
    dt3[k] = -r / O_CLIGHT;
  }
}

/* ------------------------------------------------------ projection */
typedef struct { double m1, m2, chi1, chi2, phi0, ts, dist, fs; double Fs[3], lam[3], td[3]; } proj_t;

/* Parameter mapping + per-detector response (QuickCBC.c:3698-3755). */
static void project_setup(proj_t *q, const int *labels, int nifo, double GMST, double Tobs, const double *p) {
  q->fs = ora_fbegin(p);
  double mc = exp(p[0]), mt = exp(p[1]);
  double eta = pow((mc / mt), (5.0 / 3.0));
  double dm = eta > 0.25 ? 0.0 : sqrt(1.0 - 4.0 * eta);
  q->m1 = mt * (1.0 + dm) / 2.0;
  q->m2 = mt * (1.0 - dm) / 2.0;
  q->chi1 = p[2]; q->chi2 = p[3];
  q->phi0 = 0.5 * p[4];
  q->ts = Tobs - p[5];
  q->dist = exp(p[6]);
  double Ap = (1.0 + p[10] * p[10]) / 2.0, Ac = -p[10];
  double dt[3];
  ora_delays(p[7], p[8], GMST, dt);
  for (int id = 0; id < nifo; id++) {
    double fpfc[2];
    ora_antenna(p[9], p[7], p[8], GMST, labels[id], fpfc);
    q->Fs[id] = sqrt(Ap * Ap * fpfc[0] * fpfc[0] + Ac * Ac * fpfc[1] * fpfc[1]);
    double lam = atan2(Ac * fpfc[1], Ap * fpfc[0]);
    if (lam < 0.0) lam += O_TPI;
    q->lam[id] = lam;
    q->td[id] = dt[labels[id]];
  }
}

/* h[id][i] = A cos x, h[id][N-i] = A sin x, zero for f <= fbegin
 * (QuickCBC.c:3683-3777; Tobs taken as 1/freq[1] there). */
void ora_fulltemplates(const int *labels, int nifo, double GMST, const double *freq, const double *params,
                       int N, double *h) {
  double Tobs = 1.0 / freq[1], sqT = sqrt(Tobs);
  proj_t q;
  project_setup(&q, labels, nifo, GMST, Tobs, params);
  phd c;
  phd_setup(&c, q.phi0, O_FREF, q.m1 / O_MSUN, q.m2 / O_MSUN, q.chi1, q.chi2, q.dist);
  for (int id = 0; id < nifo; id++) {
    double *row = h + (size_t)id * N;
    row[0] = 0.0; row[N / 2] = 0.0;
  }
  for (int i = 1; i < N / 2; i++) {
    double f = freq[i], a, ph;
    if (!(f > q.fs)) {
      for (int id = 0; id < nifo; id++) { h[(size_t)id * N + i] = 0.0; h[(size_t)id * N + N - i] = 0.0; }
      continue;
    }
    phd_eval(&c, f, &a, &ph);
    for (int id = 0; id < nifo; id++) {
      double A = q.Fs[id] * O_H22FAC * a / sqT;
      double x = O_TPI * f * (q.ts - q.td[id]) + q.lam[id] - ph;
      h[(size_t)id * N + i] = A * cos(x);
      h[(size_t)id * N + N - i] = A * sin(x);
    }
  }
}

/* amp[id][i] = A * taper, phase[id][i] = x on the first N/2 entries of freq
 * (QuickCBC.c:3780-3869; taper exp(10(f-fs)/fs) below fbegin). */
void ora_fullphaseamp(const int *labels, int nifo, double GMST, double Tobs, const double *freq,
                      const double *params, int N, double *amp, double *phase) {
  double sqT = sqrt(Tobs);
  int n = N / 2;
  proj_t q;
  project_setup(&q, labels, nifo, GMST, Tobs, params);
  phd c;
  phd_setup(&c, q.phi0, O_FREF, q.m1 / O_MSUN, q.m2 / O_MSUN, q.chi1, q.chi2, q.dist);
  for (int i = 0; i < n; i++) {
    double f = freq[i], a, ph;
    phd_eval(&c, f, &a, &ph);
    double y = 1.0;
    if (f < q.fs) y = exp(10.0 * (f - q.fs) / q.fs);
    for (int id = 0; id < nifo; id++) {
      double A = q.Fs[id] * O_H22FAC * a / sqT;
      amp[(size_t)id * n + i] = A * y;
      phase[(size_t)id * n + i] = O_TPI * f * (q.ts - q.td[id]) + q.lam[id] - ph;
    }
  }
}

double ora_fourier_nwip(const double *a, const double *b, const double *S, int imin, int imax, int N) {
  double s = 0.0;                                   /* Utilities.c:716-736 */
  for (int i = imin; i < imax; i++) s += (a[i] * b[i] + a[N - i] * b[N - i]) / S[i];
  return 4.0 * s;
}

/* sum_id <d|h> - <h|h>/2 over [Tobs fmin, min(Tobs fmax, N/2)) (QuickCBC.c:4236-4273) */
double ora_lnl_full(const int *labels, int nifo, double GMST, const double *D, const double *SN, int sn_stride,
                    const double *freq, const double *params, int N, double Tobs, double fmin, double fmax,
                    double *rho) {
  int imin = (int)(Tobs * fmin), imax = (int)(Tobs * fmax);
  if (imax > N / 2) imax = N / 2;
  double *h = (double *)malloc(sizeof(double) * (size_t)nifo * N);
  ora_fulltemplates(labels, nifo, GMST, freq, params, N, h);
  double L = 0.0;
  for (int id = 0; id < nifo; id++) {
    const double *hr = h + (size_t)id * N, *dr = D + (size_t)id * N, *sr = SN + (size_t)id * sn_stride;
    double HH = ora_fourier_nwip(hr, hr, sr, imin, imax, N);
    double HD = ora_fourier_nwip(dr, hr, sr, imin, imax, N);
    if (rho) rho[id] = HD / sqrt(HH);
    L += HD - 0.5 * HH;
  }
  free(h);
  return L;
}

double ora_lnl_full_batch(const int *labels, int nifo, double GMST, const double *D, const double *SN,
                          int sn_stride, const double *freq, const double *params, int B, int N, double Tobs,
                          double fmin, double fmax, double *lnl, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int b = 0; b < B; b++)
    lnl[b] = ora_lnl_full(labels, nifo, GMST, D, SN, sn_stride, freq, params + (size_t)b * 11, N, Tobs, fmin,
                          fmax, NULL);
#ifdef _OPENMP
  return omp_get_wtime() - t0;
#else
  return 0.0;
#endif
}

/* ------------------------------------------------------ heterodyne */
/* Discrete Legendre (Gram) polynomials on U+1 points by the three-term
 * recurrence of QuickCBC.c:5055-5094. P is (J+1) x (U+1). */
static void gram_poly(int J, int U, double *P) {
  for (int k = 0; k <= U; k++) {
    double c0 = 0.0, c1 = (double)(U - 2 * k), c2 = (double)U;
    double d0 = c2, d1 = c1 + c1, d2 = d0;
    P[0 * (U + 1) + k] = 1.0;
    if (J >= 1) P[1 * (U + 1) + k] = c1 / (double)U;
    for (int i = 1; i < J; i++) {
      d0 += 2.0; d2 -= 2.0; c0 += d0; c1 += d1; c2 += d2;
      P[(i + 1) * (U + 1) + k] = (c1 * P[i * (U + 1) + k] - c0 * P[(i - 1) * (U + 1) + k]) / c2;
    }
  }
}

/* Inverse of an n x n matrix by Gauss-Jordan elimination with partial pivoting. */
static void invert(const double *A, double *Ainv, int n) {
  double W[8][16];
  for (int i = 0; i < n; i++)
    for (int j = 0; j < 2 * n; j++) W[i][j] = j < n ? A[i * n + j] : (j - n == i ? 1.0 : 0.0);
  for (int col = 0; col < n; col++) {
    int piv = col;
    for (int i = col + 1; i < n; i++) if (fabs(W[i][col]) > fabs(W[piv][col])) piv = i;
    if (piv != col) for (int j = 0; j < 2 * n; j++) { double t = W[col][j]; W[col][j] = W[piv][j]; W[piv][j] = t; }
    double d = W[col][col];
    for (int j = 0; j < 2 * n; j++) W[col][j] /= d;
    for (int i = 0; i < n; i++) {
      if (i == col) continue;
      double f = W[i][col];
      for (int j = 0; j < 2 * n; j++) W[i][j] -= f * W[col][j];
    }
  }
  for (int i = 0; i < n; i++) for (int j = 0; j < n; j++) Ainv[i * n + j] = W[i][n + j];
}

/* Summary tables of the heterodyned likelihood for a given grid (QuickCBC.c:5112-5299).
 * Layouts: amp/phase [nifo][M], IP [NR][J+1][J+1] (transpose of the inverse of the
 * sampled basis, as stored by the reference), SL/lc/ls [NR][nifo][J+1], aa/rc/rs [nifo][NR]. */
int ora_heterodyne(const int *labels, int nifo, double GMST, const double *D, const double *SN, int sn_stride,
                   const double *freq, const double *params, int N, double Tobs, const int *fgrid, int M, int MN,
                   int MM, int J, double *amp, double *phase, double *IP, double *SL, double *lc, double *ls,
                   double *aa, double *rc, double *rs, double *logLb) {
  int NR = (M - 1) / J, half = N / 2, J1 = J + 1;
  double *hb = (double *)malloc(sizeof(double) * (size_t)nifo * N);
  double *ab = (double *)malloc(sizeof(double) * (size_t)nifo * half);
  double *pb = (double *)malloc(sizeof(double) * (size_t)nifo * half);
  double *RC = (double *)calloc((size_t)nifo * half, sizeof(double));
  double *RS = (double *)calloc((size_t)nifo * half, sizeof(double));
  double *AA = (double *)calloc((size_t)nifo * half, sizeof(double));
  ora_fulltemplates(labels, nifo, GMST, freq, params, N, hb);
  ora_fullphaseamp(labels, nifo, GMST, Tobs, freq, params, N, ab, pb);
  for (int id = 0; id < nifo; id++)
    for (int j = 0; j < M; j++) {
      amp[id * M + j] = ab[(size_t)id * half + fgrid[j]];
      phase[id * M + j] = pb[(size_t)id * half + fgrid[j]];
    }
  double L = 0.0;
  double *rb = (double *)malloc(sizeof(double) * N);
  for (int id = 0; id < nifo; id++) {
    const double *h = hb + (size_t)id * N, *d = D + (size_t)id * N, *s = SN + (size_t)id * sn_stride;
    for (int j = 0; j < N; j++) rb[j] = d[j] - h[j];
    double HH = ora_fourier_nwip(h, h, s, MN, MM, N);
    double HR = ora_fourier_nwip(rb, h, s, MN, MM, N);
    L += HR + 0.5 * HH;
    for (int j = 1; j < half; j++) {
      double a = ab[(size_t)id * half + j], ph = pb[(size_t)id * half + j];
      double cp = cos(ph), sp = sin(ph), x = a / s[j];
      RC[(size_t)id * half + j] = 2.0 * (rb[j] * cp + rb[N - j] * sp) * x;
      RS[(size_t)id * half + j] = 2.0 * (-rb[j] * sp + rb[N - j] * cp) * x;
      AA[(size_t)id * half + j] = a * a / s[j];
    }
  }
  *logLb = L;
  for (int id = 0; id < nifo; id++)
    for (int i = 0; i < NR; i++) {
      int k = fgrid[i * J];
      rc[id * NR + i] = RC[(size_t)id * half + k];
      rs[id * NR + i] = RS[(size_t)id * half + k];
      aa[id * NR + i] = AA[(size_t)id * half + k];
    }
  for (int i = 0; i < NR; i++) {
    int U = fgrid[(i + 1) * J] - fgrid[i * J];
    double *P = (double *)malloc(sizeof(double) * J1 * (U + 1));
    gram_poly(J, U, P);
    double PP[64], inv[64];
    for (int a = 0; a <= J; a++)
      for (int b = 0; b <= J; b++) PP[a * J1 + b] = P[a * (U + 1) + fgrid[i * J + b] - fgrid[i * J]];
    invert(PP, inv, J1);
    for (int a = 0; a <= J; a++)
      for (int b = 0; b <= J; b++) IP[((size_t)i * J1 + a) * J1 + b] = inv[b * J1 + a];
    for (int id = 0; id < nifo; id++) {
      for (int a = 0; a <= J; a++) {
        double s1 = 0.0, s2 = 0.0, s3 = 0.0;
        for (int n = 0; n <= U; n++) {
          size_t k = (size_t)id * half + fgrid[i * J] + n;
          double pv = P[a * (U + 1) + n];
          s1 += AA[k] * pv; s2 += RC[k] * pv; s3 += RS[k] * pv;
        }
        size_t o = ((size_t)i * nifo + id) * J1 + a;
        SL[o] = s1; lc[o] = s2; ls[o] = s3;
      }
    }
    free(P);
  }
  free(rb); free(hb); free(ab); free(pb); free(RC); free(RS); free(AA);
  return NR;
}

/* logLb - sum_id (HR + HH/2) from the grid-point waveform (QuickCBC.c:5303-5444). */
double ora_lnl_het(const int *labels, int nifo, double GMST, double Tobs, const double *hfreq, int M, int J,
                   const double *amp, const double *phase, const double *IP, const double *SL, const double *lc,
                   const double *ls, const double *aa, const double *rc, const double *rs, double logLb,
                   const double *params) {
  int NR = (M - 1) / J, J1 = J + 1;
  double *A = (double *)malloc(sizeof(double) * (size_t)nifo * M), *P = (double *)malloc(sizeof(double) * (size_t)nifo * M);
  ora_fullphaseamp(labels, nifo, GMST, Tobs, hfreq, params, 2 * M, A, P);
  double *hc = (double *)malloc(sizeof(double) * M), *hs = (double *)malloc(sizeof(double) * M),
         *cc = (double *)malloc(sizeof(double) * M);
  double L = logLb;
  for (int id = 0; id < nifo; id++) {
    for (int j = 0; j < M; j++) {
      double ar = amp[id * M + j], d = phase[id * M + j] - P[(size_t)id * M + j], a = A[(size_t)id * M + j];
      double c = 2.0 * (ar - a * cos(d)), s = 2.0 * a * sin(d);
      hc[j] = c / ar; hs[j] = s / ar;
      cc[j] = hc[j] * hc[j] + hs[j] * hs[j];
    }
    double HH = 0.0, HR = 0.0, x = 0.0, y = 0.0;
    for (int i = 0; i < NR; i++) {
      const double *ip = IP + (size_t)i * J1 * J1;
      const double *sl = SL + ((size_t)i * nifo + id) * J1, *lcv = lc + ((size_t)i * nifo + id) * J1,
                   *lsv = ls + ((size_t)i * nifo + id) * J1;
      /* same accumulation order as the reference: cc, then hc, then hs */
      const double *vecs[3] = {cc + i * J, hc + i * J, hs + i * J};
      const double *proj[3] = {sl, lcv, lsv};
      for (int t = 0; t < 3; t++) {
        double u[8];
        for (int a = 0; a <= J; a++) {
          u[a] = 0.0;
          for (int b = 0; b <= J; b++) u[a] += ip[a * J1 + b] * vecs[t][b];
        }
        for (int a = 0; a <= J; a++) {
          if (t == 0) HH += u[a] * proj[t][a]; else HR += u[a] * proj[t][a];
        }
        if (i < NR - 2) {
          if (t == 0) x += aa[id * NR + i + 1] * vecs[t][J];
          else if (t == 1) y += rc[id * NR + i + 1] * vecs[t][J];
          else y += rs[id * NR + i + 1] * vecs[t][J];
        }
      }
    }
    HH -= x;
    HR -= y;
    L -= (HR + 0.5 * HH);
  }
  free(A); free(P); free(hc); free(hs); free(cc);
  return L;
}

double ora_lnl_het_batch(const int *labels, int nifo, double GMST, double Tobs, const double *hfreq, int M, int J,
                         const double *amp, const double *phase, const double *IP, const double *SL,
                         const double *lc, const double *ls, const double *aa, const double *rc, const double *rs,
                         double logLb, const double *params, int B, double *lnl, int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  double t0 = omp_get_wtime();
#pragma omp parallel for schedule(dynamic, 4)
#endif
  for (int b = 0; b < B; b++)
    lnl[b] = ora_lnl_het(labels, nifo, GMST, Tobs, hfreq, M, J, amp, phase, IP, SL, lc, ls, aa, rc, rs, logLb,
                         params + (size_t)b * 11);
#ifdef _OPENMP
  return omp_get_wtime() - t0;
#else
  return 0.0;
#endif
}
