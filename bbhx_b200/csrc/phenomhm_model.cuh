// PhenomHM / PhenomD amplitude, phase and t(f) model (device side).
//
// The model follows the reference's PhenomHM implementation (src/bbhx/cutils/
// PhenomHMWaveform.cu), which is the LAL IMRPhenomD (arXiv:1508.07250, 1508.07253) +
// IMRPhenomHM (arXiv:1708.00404) model.  The phenomenological fit tables (Table 5 of
// 1508.07253, the final-spin / radiated-energy fits of 1508.07250, the QNM fits of
// arXiv:1810.03550 and the PN amplitude ratios of the HM paper) are published data and
// are reproduced with the same numbers.
//
// Organisation (B200-first, unlike the reference's block-per-binary kernel that redoes
// the setup in every thread, PhenomHMWaveform.cu:2811-2842):
//   * phm_setup_mode() builds everything that depends only on (binary, mode) once into a
//     ModeCoeffs record (one thread per (binary, mode)),
//   * phm_eval_point() evaluates amplitude, phase and t(f) at one frequency from that
//     record (one thread per (binary, mode, frequency)).
// The intermediate-region amplitude (reference: closed-form Mathematica monomial
// coefficients delta0..4, PhenomHMWaveform.cu:650-833) is the same unique quartic
// fixed by p(f1)=v1, p'(f1)=d1, p(f2)=v2, p(f3)=v3, p'(f3)=d2, but built here as a
// confluent Hermite interpolant in Newton divided-difference form, which is better
// conditioned and cheaper to evaluate.
#pragma once

#include "bbhx_common.cuh"
#include "dual.cuh"

namespace bbhx {

constexpr double AMP_FJOIN_INS = 0.014;  // PhenomHMWaveform.hh:62
constexpr double PHI_FJOIN_INS = 0.018;  // PhenomHMWaveform.hh:68
constexpr int MAX_MODES = 6;

// ---------------------------------------------------------------------------------
// Fits that depend on (eta, chi_PN): each is c00 + c01 eta + sum_k xi^k (ck0 + ck1 eta +
// ck2 eta^2), xi = chi - 1 (PhenomHMWaveform.cu:394-457, 498-540, 603-620, 895-963,
// 1005-1047, 1109-1163).
// ---------------------------------------------------------------------------------
struct Fit11 {
  double c00, c01, c10, c11, c12, c20, c21, c22, c30, c31, c32;
};

template <typename T>
__device__ __forceinline__ T eval_fit(const Fit11& c, const T& eta, const T& chi) {
  T xi = chi - 1.0;
  T e2 = eta * eta;
  T t1 = c.c10 + c.c11 * eta + c.c12 * e2;
  T t2 = c.c20 + c.c21 * eta + c.c22 * e2;
  T t3 = c.c30 + c.c31 * eta + c.c32 * e2;
  return c.c00 + c.c01 * eta + xi * (t1 + xi * (t2 + xi * t3));
}

// rho1..3 (inspiral amplitude), gamma1..3 (merger-ringdown amplitude), v2 (intermediate
// collocation value), sigma1..4 (inspiral phase), beta1..3 (intermediate phase),
// alpha1..5 (merger-ringdown phase).
__constant__ Fit11 kFitRho[3] = {
    {3931.8979897196696, -17395.758706812805, 3132.375545898835, 343965.86092361377,
     -1.2162565819981997e6, -70698.00600428853, 1.383907177859705e6, -3.9662761890979446e6,
     -60017.52423652596, 803515.1181825735, -2.091710365941658e6},
    {-40105.47653771657, 112253.0169706701, 23561.696065836168, -3.476180699403351e6,
     1.137593670849482e7, 754313.1127166454, -1.308476044625268e7, 3.6444584853928134e7,
     596226.612472288, -7.4277901143564405e6, 1.8928977514040343e7},
    {83208.35471266537, -191237.7264145924, -210916.2454782992, 8.71797508352568e6,
     -2.6914942420669552e7, -1.9889806527362722e6, 3.0888029960154563e7, -8.390870279256162e7,
     -1.4535031953446497e6, 1.7063528990822166e7, -4.2748659731120914e7}};
__constant__ Fit11 kFitGamma[3] = {
    {0.006927402739328343, 0.03020474290328911, 0.006308024337706171, -0.12074130661131138,
     0.26271598905781324, 0.0034151773647198794, -0.10779338611188374, 0.27098966966891747,
     0.0007374185938559283, -0.02749621038376281, 0.0733150789135702},
    {1.010344404799477, 0.0008993122007234548, 0.283949116804459, -4.049752962958005,
     13.207828172665366, 0.10396278486805426, -7.025059158961947, 24.784892370130475,
     0.03093202475605892, -2.6924023896851663, 9.609374464684983},
    {1.3081615607036106, -0.005537729694807678, -0.06782917938621007, -0.6689834970767117,
     3.403147966134083, -0.05296577374411866, -0.9923793203111362, 4.820681208409587,
     -0.006134139870393713, -0.38429253308696365, 1.7561754421985984}};
__constant__ Fit11 kFitV2 = {0.8149838730507785, 2.5747553517454658, 1.1610198035496786,
                             -2.3627771785551537, 6.771038707057573, 0.7570782938606834,
                             -2.7256896890432474, 7.1140380397149965, 0.1766934149293479,
                             -0.7978690983168183, 2.1162391502005153};
__constant__ Fit11 kFitSigma[4] = {
    {2096.551999295543, 1463.7493168261553, 1312.5493286098522, 18307.330017082117,
     -43534.1440746107, -833.2889543511114, 32047.31997183187, -108609.45037520859,
     452.25136398112204, 8353.439546391714, -44531.3250037322},
    {-10114.056472621156, -44631.01109458185, -6541.308761668722, -266959.23419307504,
     686328.3229317984, 3405.6372187679685, -437507.7208209015, 1.6318171307344697e6,
     -7462.648563007646, -114585.25177153319, 674402.4689098676},
    {22933.658273436497, 230960.00814979506, 14961.083974183695, 1.1940181342318142e6,
     -3.1042239693052764e6, -3038.166617199259, 1.8720322849093592e6, -7.309145012085539e6,
     42738.22871475411, 467502.018616601, -3.064853498512499e6},
    {-14621.71522218357, -377812.8579387104, -9608.682631509726, -1.7108925257214056e6,
     4.332924601416521e6, -22366.683262266528, -2.5019716386377467e6, 1.0274495902259542e7,
     -85360.30079034246, -570025.3441737515, 4.396844346849777e6}};
__constant__ Fit11 kFitBeta[3] = {
    {97.89747327985583, -42.659730877489224, 153.48421037904913, -1417.0620760768954,
     2752.8614143665027, 138.7406469558649, -1433.6585075135881, 2857.7418952430758,
     41.025109467376126, -423.680737974639, 850.3594335657173},
    {-3.282701958759534, -9.051384468245866, -12.415449742258042, 55.4716447709787,
     -106.05109938966335, -11.953044553690658, 76.80704618365418, -155.33172948098394,
     -3.4129261592393263, 25.572377569952536, -54.408036707740465},
    {-0.000025156429818799565, 0.000019750256942201327, -0.000018370671469295915,
     0.000021886317041311973, 0.00008250240316860033, 7.157371250566708e-6,
     -0.000055780000112270685, 0.00019142082884072178, 5.447166261464217e-6,
     -0.00003220610095021982, 0.00007974016714984341}};
__constant__ Fit11 kFitAlpha[5] = {
    {43.31514709695348, 638.6332679188081, -32.85768747216059, 2415.8938269370315,
     -5766.875169379177, -61.85459307173841, 2953.967762459948, -8986.29057591497,
     -21.571435779762044, 981.2158224673428, -3239.5664895930286},
    {-0.07020209449091723, -0.16269798450687084, -0.1872514685185499, 1.138313650449945,
     -2.8334196304430046, -0.17137955686840617, 1.7197549338119527, -4.539717148261272,
     -0.049983437357548705, 0.6062072055948309, -1.682769616644546},
    {9.5988072383479, -397.05438595557433, 16.202126189517813, -1574.8286986717037,
     3600.3410843831093, 27.092429659075467, -1786.482357315139, 5152.919378666511,
     11.175710130033895, -577.7999423177481, 1808.730762932043},
    {-0.02989487384493607, 1.4022106448583738, -0.07356049468633846, 0.8337006542278661,
     0.2240008282397391, -0.055202870001177226, 0.5667186343606578, 0.7186931973380503,
     -0.015507437354325743, 0.15750322779277187, 0.21076815715176228},
    {0.9974408278363099, -0.007884449714907203, -0.059046901195591035, 1.3958712396764088,
     -4.516631601676276, -0.05585343136869692, 1.7516580039343603, -5.990208965347804,
     -0.017945336522161195, 0.5965097794825992, -2.0608879367971804}};

// ---------------------------------------------------------------------------------
// QNM frequencies of the remnant (London & Fauchon-Jones fits, PhenomHMWaveform.cu:55-211)
// ans = base + kappa^s * sum_k A_k exp(i phi_k) kappa^k with base = m/2, s = 1 for the
// zero-damped modes, base = 0, s = 0 for (2,1) and (3,2).
// ---------------------------------------------------------------------------------
struct QnmFit {
  int ell, mm, nterms, shift;
  double base;
  double A[7];
  double ph[7];
};
__constant__ QnmFit kQnm[6] = {
    {2, 2, 5, 1, 1.0, {1.557847, 1.95097051, 2.09971716, 1.41094660, 0.41063923},
     {2.903124, 5.920970, 2.760585, 5.914340, 2.795235}},
    {3, 3, 5, 1, 1.5, {2.095657, 2.46964352, 2.66552551, 1.75836443, 0.49905688},
     {2.964973, 5.996734, 2.817591, 5.932693, 2.781658}},
    {4, 4, 5, 1, 2.0, {2.658908, 2.97825567, 3.21842350, 2.12764967, 0.60338186},
     {3.002787, 6.050955, 2.877514, 5.989669, 2.830031}},
    {2, 1, 7, 0, 0.0,
     {0.589113, 0.18896353, 1.15012965, 6.04585476, 11.12627777, 9.34711461, 3.03838318},
     {0.043525, 2.289868, 5.810057, 2.741967, 5.844130, 2.669372, 5.791518}},
    {3, 2, 7, 0, 0.0,
     {1.022464, 0.24731213, 1.70468239, 0.94604882, 1.53189884, 2.28052668, 0.92150314},
     {0.004870, 0.665292, 3.138283, 0.163247, 5.703573, 2.685231, 5.841704}},
    {4, 3, 5, 1, 1.5, {0.205046, 3.10333396, 4.23612166, 3.02890198, 0.90843949},
     {0.595328, 3.016200, 6.038842, 2.826239, 5.915164}}};

// Complex dimensionless QNM frequency M*omega for mode (l, m, n=0); zero if unsupported.
template <typename T>
__device__ inline cplxT<T> qnm_cw(T jf, int ell, int mm) {
  int idx = -1;
  for (int k = 0; k < 6; ++k)
    if (kQnm[k].ell == ell && kQnm[k].mm == mm) idx = k;
  if (idx < 0) return cmk(T(0.0), T(0.0));
  const QnmFit& q = kQnm[idx];
  T kappa = pow(log(2.0 - jf) / log(3.0), 1.0 / (2.0 + ell - abs(mm)));
  cplxT<T> sum = cmk(T(0.0), T(0.0));
  T kp = 1.0;
  for (int k = 0; k < q.nterms; ++k) {
    double s, c;
    sincos(q.ph[k], &s, &c);
    sum = sum + cmk(T(q.A[k] * c * kp), T(q.A[k] * s * kp));
    kp *= kappa;
  }
  if (q.shift) sum = kappa * sum;
  return cmk(T(q.base + sum.re), sum.im);
}

// Final spin (1508.07250 eq. 3.6) and radiated energy (eqs. 3.7-3.8); masses in any units
// with m1 >= m2 enforced inside (PhenomHMWaveform.cu:1679-1814).
template <typename T>
__device__ inline void final_mass_spin(T m1, T m2, T chi1, T chi2,
                                       T* finmass, T* finspin) {
  if (!(m1 > m2)) {  // the reference swaps unless m1 > m2 strictly
    T t = m1; m1 = m2; m2 = t;
    t = chi1; chi1 = chi2; chi2 = t;
  }
  T M = m1 + m2;
  T eta = m1 * m2 / (M * M);
  T Seta = sqrt(1.0 - 4.0 * eta);
  T q1 = 0.5 * (1.0 + Seta), q2 = 0.5 * (1.0 - Seta);
  T q1s = q1 * q1, q2s = q2 * q2;
  T e2 = eta * eta, e3 = e2 * eta, e4 = e3 * eta;
  // final spin
  T s = q1s * chi1 + q2s * chi2;
  T s2 = s * s, s3 = s2 * s, s4 = s3 * s;
  *finspin = 3.4641016151377544 * eta - 4.399247300629289 * e2 + 9.397292189321194 * e3 -
             13.180949901606242 * e4 + (1 - 0.0850917821418767 * eta - 5.837029316602263 * e2) * s +
             (0.1014665242971878 * eta - 2.0967746996832157 * e2) * s2 +
             (-1.3546806617824356 * eta + 4.108962025369336 * e2) * s3 +
             (-0.8676969352555539 * eta + 2.064046835273906 * e2) * s4;
  // radiated energy
  T sr = (q1s * chi1 + q2s * chi2) / (q1s + q2s);
  T erad = ((0.055974469826360077 * eta + 0.5809510763115132 * e2 - 0.9606726679372312 * e3 +
                  3.352411249771192 * e4) *
                 (1. + (-0.0030302335878845507 - 2.0066110851351073 * eta + 7.7050567802399215 * e2) * sr)) /
                (1. + (-0.6714403054720589 - 1.4756929437702908 * eta + 7.304676214885011 * e2) * sr);
  *finmass = 1.0 - erad;
}

// ---------------------------------------------------------------------------------
// PhenomD coefficients for one (binary, fRD, fDM, Rholm, Taulm)
// ---------------------------------------------------------------------------------
template <typename T>
struct PhenomDT {
  T eta, etaInv, chi;
  T fRD, fDM;
  // amplitude
  T amp0;        // sqrt(2/3) sqrt(eta) / pi^(1/6)
  T ains[8];     // Mf^{2/3,1,4/3,5/3,2,7/3,8/3,3} coefficients of the inspiral ansatz
  T g1, g2, g3;  // gamma_1..3
  T fpeak;       // fmaxCalc (1508.07253 eq. 20)
  T hf1, hf2, hf3, hc0, hc1, hc2, hc3, hc4;  // Hermite nodes and Newton coefficients
  // phase
  T pn_v[8], pn_vlogv5, pn_vlogv6;
  T sig1, sig2, sig3, sig4, bet1, bet2, bet3, alp1, alp2, alp3, alp4, alp5;
  T pins_init, pins_23, pins_13, pins_13log, pins_log, pins_m13, pins_m23, pins_m1,
      pins_m53, pins_1, pins_43, pins_53, pins_2;
  T C1Int, C2Int, C1MRD, C2MRD, fMRDJoin;
  T Rholm, Taulm;
  T inv_atan_scale;  // 1 / (Rholm fDM Taulm)
};
using PhenomD = PhenomDT<double>;

template <typename T>
struct PowersT {  // PhenomHMWaveform.cu:348-362 (same derivation of the fractional powers)
  T sixth, third, two_thirds, four_thirds, five_thirds, two, seven_thirds, eight_thirds;
};
using Powers = PowersT<double>;

template <typename T>
__device__ __forceinline__ PowersT<T> make_powers(T x) {
  PowersT<T> p;
  p.third = cbrt(x);
  p.sixth = sqrt(p.third);
  p.two_thirds = p.third * p.third;
  p.four_thirds = x * p.third;
  p.five_thirds = p.four_thirds * p.third;
  p.two = x * x;
  p.seven_thirds = p.third * p.two;
  p.eight_thirds = p.two_thirds * p.two;
  return p;
}

template <typename T>
__device__ __forceinline__ T amp_ins_ansatz(const PhenomDT<T>& d, T Mf, const PowersT<T>& p) {
  return 1.0 + p.two_thirds * d.ains[0] + Mf * d.ains[1] + p.four_thirds * d.ains[2] +
         p.five_thirds * d.ains[3] + p.two * d.ains[4] + p.seven_thirds * d.ains[5] +
         p.eight_thirds * d.ains[6] + Mf * p.two * d.ains[7];
}

// derivative of amp_ins_ansatz: sum_k (k/3) c_k Mf^{k/3-1}
template <typename T>
__device__ __forceinline__ T amp_ins_ansatz_deriv(const PhenomDT<T>& d, T Mf) {
  T t = cbrt(Mf);
  T t2 = t * t;
  return (2.0 / 3.0) * d.ains[0] / t + d.ains[1] + (4.0 / 3.0) * d.ains[2] * t +
         (5.0 / 3.0) * d.ains[3] * t2 + 2.0 * d.ains[4] * Mf + (7.0 / 3.0) * d.ains[5] * Mf * t +
         (8.0 / 3.0) * d.ains[6] * Mf * t2 + 3.0 * d.ains[7] * Mf * Mf;
}

template <typename T>
__device__ __forceinline__ T amp_mrd_ansatz(const PhenomDT<T>& d, T f) {
  T s = d.fDM * d.g3;
  T x = f - d.fRD;
  return exp(-x * d.g2 / s) * (s * d.g1) / (x * x + s * s);
}

template <typename T>
__device__ __forceinline__ T amp_mrd_ansatz_deriv(const PhenomDT<T>& d, T f) {
  T s = d.fDM * d.g3;
  T x = f - d.fRD;
  T den = x * x + s * s;
  return amp_mrd_ansatz(d, f) * (-d.g2 / s - 2.0 * x / den);
}

template <typename T>
__device__ __forceinline__ T amp_int_ansatz(const PhenomDT<T>& d, T f) {
  T u = f - d.hf1;
  return d.hc0 + u * (d.hc1 + u * (d.hc2 + (f - d.hf2) * (d.hc3 + (f - d.hf3) * d.hc4)));
}

// Full PhenomD amplitude (without the distance/mass scale), PhenomHMWaveform.cu:1508-1537
template <typename T>
__device__ __forceinline__ T phenomd_amp(const PhenomDT<T>& d, T Mf) {
  PowersT<T> p = make_powers(Mf);
  T pre = d.amp0 / (Mf * p.sixth);
  if (Mf < AMP_FJOIN_INS) return pre * amp_ins_ansatz(d, Mf, p);
  if (Mf >= d.fpeak) return pre * amp_mrd_ansatz(d, Mf);
  return pre * amp_int_ansatz(d, Mf);
}

// inspiral phase, PhenomHMWaveform.cu:1077-1117
template <typename T>
__device__ __forceinline__ T phi_ins(const PhenomDT<T>& d, T Mf, const PowersT<T>& p) {
  const double PI_THIRD = 1.4645918875615231;  // pi^(1/3)
  T v = p.third * PI_THIRD;
  T logv = log(v);
  T ph = d.pins_init;
  ph += d.pins_23 * p.two_thirds;
  ph += d.pins_13 * p.third;
  ph += d.pins_13log * logv * p.third;
  ph += d.pins_log * logv;
  ph += d.pins_m13 / p.third;
  ph += d.pins_m23 / p.two_thirds;
  ph += d.pins_m1 / Mf;
  ph += d.pins_m53 / p.five_thirds;
  ph += (d.pins_1 * Mf + d.pins_43 * p.four_thirds + d.pins_53 * p.five_thirds + d.pins_2 * p.two) *
        d.etaInv;
  return ph;
}

// d(phi_ins)/dMf, PhenomHMWaveform.cu:1214-1250
template <typename T>
__device__ __forceinline__ T dphi_ins(const PhenomDT<T>& d, T Mf) {
  const double PI_THIRD = 1.4645918875615231;
  const double PI_TWOTHIRDS = 2.1450293971110255;
  T v = cbrt(PI * Mf);
  T logv = log(v);
  T v2 = v * v, v3 = v2 * v, v4 = v3 * v, v5 = v4 * v, v6 = v5 * v, v7 = v6 * v, v8 = v7 * v;
  T s = 2.0 * d.pn_v[7] * v7;
  s += (d.pn_v[6] + d.pn_vlogv6 * (1.0 + logv)) * v6;
  s += d.pn_vlogv5 * v5;
  s -= d.pn_v[4] * v4;
  s -= 2.0 * d.pn_v[3] * v3;
  s -= 3.0 * d.pn_v[2] * v2;
  s -= 4.0 * d.pn_v[1] * v;
  s -= 5.0 * d.pn_v[0];
  s /= v8 * 3.0 / PI;
  s += (d.sig1 + d.sig2 * v / PI_THIRD + d.sig3 * v2 / PI_TWOTHIRDS + (d.sig4 / PI) * v3) / d.eta;
  return s;
}

template <typename T>
__device__ __forceinline__ T phi_int(const PhenomDT<T>& d, T Mf) {
  return d.bet1 * Mf - d.bet3 / (3.0 * Mf * Mf * Mf) + d.bet2 * log(Mf);
}
template <typename T>
__device__ __forceinline__ T dphi_int(const PhenomDT<T>& d, T Mf) {
  T Mf2 = Mf * Mf;
  return (d.bet1 + d.bet3 / (Mf2 * Mf2) + d.bet2 / Mf) / d.eta;
}
template <typename T>
__device__ __forceinline__ T phi_mrd(const PhenomDT<T>& d, T f, T Rho, T Tau) {
  T sq = sqrt(f);
  T f075 = sqrt(f * sq);
  return -(d.alp2 / f) + (4.0 / 3.0) * (d.alp3 * f075) + d.alp1 * f +
         d.alp4 * Rho * atan((f - d.alp5 * d.fRD) / (Rho * d.fDM * Tau));
}
template <typename T>
__device__ __forceinline__ T dphi_mrd(const PhenomDT<T>& d, T f, T Rho, T Tau) {
  T x = f - d.alp5 * d.fRD;
  T w = d.fDM * Tau * Rho;
  return (d.alp1 + d.alp2 / (f * f) + d.alp3 / pow(f, 0.25) +
          d.alp4 / (d.fDM * Tau * (1.0 + x * x / (w * w)))) *
         d.etaInv;
}

// Full PhenomD phase with the mode's connection constants (PhenomHMWaveform.cu:1360-1381)
template <typename T>
__device__ __forceinline__ T phenomd_phase(const PhenomDT<T>& d, T Mf) {
  if (Mf < PHI_FJOIN_INS) {
    PowersT<T> p = make_powers(Mf);
    return phi_ins(d, Mf, p);
  }
  if (Mf >= d.fMRDJoin) return d.etaInv * phi_mrd(d, Mf, d.Rholm, d.Taulm) + d.C1MRD + d.C2MRD * Mf;
  return d.etaInv * phi_int(d, Mf) + d.C1Int + d.C2Int * Mf;
}
template <typename T>
__device__ __forceinline__ T phenomd_dphase(const PhenomDT<T>& d, T Mf) {
  if (Mf < PHI_FJOIN_INS) return dphi_ins(d, Mf);
  if (Mf >= d.fMRDJoin) return dphi_mrd(d, Mf, d.Rholm, d.Taulm) + d.C2MRD;
  return dphi_int(d, Mf) + d.C2Int;
}

// Phase and d(phase)/dMf at one frequency together (the two branches of phenomd_phase and
// phenomd_dphase), sharing the fractional powers, the logarithm and the reciprocals.
template <typename T>
__device__ __forceinline__ void phenomd_phase_dphase(const PhenomDT<T>& d, T Mf, T* ph,
                                                     T* dph) {
  const double PI_THIRD = 1.4645918875615231;  // pi^(1/3)
  if (Mf < PHI_FJOIN_INS) {
    const T t = cbrt(Mf);  // Mf^(1/3)
    const T it = 1.0 / t;
    const T t2 = t * t, it2 = it * it;
    const T v = t * PI_THIRD;
    const T logv = log(v);
    T p = d.pins_init;
    p += d.pins_23 * t2;
    p += d.pins_13 * t;
    p += d.pins_13log * logv * t;
    p += d.pins_log * logv;
    p += d.pins_m13 * it;
    p += d.pins_m23 * it2;
    p += d.pins_m1 * (it2 * it);
    p += d.pins_m53 * (it2 * it2 * it);
    p += (d.pins_1 * Mf + d.pins_43 * (Mf * t) + d.pins_53 * (Mf * t2) + d.pins_2 * (Mf * Mf)) *
         d.etaInv;
    *ph = p;
    const T v2 = v * v, v3 = v2 * v, v4 = v3 * v, v5 = v4 * v, v6 = v5 * v, v7 = v6 * v;
    T s = 2.0 * d.pn_v[7] * v7;
    s += (d.pn_v[6] + d.pn_vlogv6 * (1.0 + logv)) * v6;
    s += d.pn_vlogv5 * v5;
    s -= d.pn_v[4] * v4;
    s -= 2.0 * d.pn_v[3] * v3;
    s -= 3.0 * d.pn_v[2] * v2;
    s -= 4.0 * d.pn_v[1] * v;
    s -= 5.0 * d.pn_v[0];
    const T iv = it * (1.0 / PI_THIRD);
    const T iv2 = iv * iv, iv4 = iv2 * iv2;
    s *= (PI / 3.0) * (iv4 * iv4);
    s += (d.sig1 + d.sig2 * t + d.sig3 * t2 + d.sig4 * Mf) * d.etaInv;
    *dph = s;
    return;
  }
  if (Mf >= d.fMRDJoin) {
    const T sq = sqrt(Mf);
    const T q = sqrt(sq);  // Mf^(1/4)
    const T f075 = sq * q;
    const T iF = 1.0 / Mf;
    const T x = Mf - d.alp5 * d.fRD;
    const T y = x * d.inv_atan_scale;
    *ph = d.etaInv * (-(d.alp2 * iF) + (4.0 / 3.0) * (d.alp3 * f075) + d.alp1 * Mf +
                      d.alp4 * d.Rholm * atan(y)) +
          d.C1MRD + d.C2MRD * Mf;
    *dph = (d.alp1 + d.alp2 * (iF * iF) + d.alp3 * (f075 * iF) +
            d.alp4 / (d.fDM * d.Taulm * (1.0 + y * y))) *
               d.etaInv +
           d.C2MRD;
    return;
  }
  const T iF = 1.0 / Mf;
  const T iF2 = iF * iF;
  *ph = d.etaInv * (d.bet1 * Mf - d.bet3 * (1.0 / 3.0) * (iF2 * iF) + d.bet2 * log(Mf)) + d.C1Int +
        d.C2Int * Mf;
  *dph = (d.bet1 + d.bet3 * (iF2 * iF2) + d.bet2 * iF) * d.etaInv + d.C2Int;
}

// Build the PhenomD coefficient set.  m1, m2 in solar masses with m1 >= m2 already
// enforced; fring/fdamp dimensionless; Rholm/Taulm mode ratios (1, 1 for PhenomD).
template <typename T>
__device__ inline void phenomd_setup(PhenomDT<T>& d, T m1, T m2, T chi1, T chi2,
                                     T fring, T fdamp, T Rholm, T Taulm) {
  const T M = m1 + m2;
  const T eta = m1 * m2 / (M * M);
  d.eta = eta;
  d.etaInv = 1.0 / eta;
  const T Seta = sqrt(1.0 - 4.0 * eta);
  // reduced spin chi_PN (1107.1267 eq. 5.9)
  d.chi = 0.5 * (chi1 + chi2) * (1.0 - eta * 76.0 / 113.0) + Seta * 0.5 * (chi1 - chi2);
  const T chi = d.chi;
  d.fRD = fring;
  d.fDM = fdamp;
  d.Rholm = Rholm;
  d.Taulm = Taulm;
  d.inv_atan_scale = 1.0 / (Rholm * fdamp * Taulm);

  // ---------------- amplitude ----------------
  const double pi16 = pow(PI, 1.0 / 6.0);
  d.amp0 = sqrt(2.0 / 3.0) * sqrt(eta) / pi16;
  const PowersT<double> pp = make_powers(PI);
  const double Pi = PI, Pi2 = pp.two;
  const T c12 = chi1 * chi1, c22 = chi2 * chi2, e2 = eta * eta, e3 = e2 * eta;
  T rho1 = eval_fit(kFitRho[0], eta, chi);
  T rho2 = eval_fit(kFitRho[1], eta, chi);
  T rho3 = eval_fit(kFitRho[2], eta, chi);
  // TaylorF2-amplitude re-expansion coefficients (1508.07253 eqs. 29-30, appendix B)
  d.ains[0] = ((-969 + 1804 * eta) * pp.two_thirds) / 672.;
  d.ains[1] = ((chi1 * (81 * (1 + Seta) - 44 * eta) + chi2 * (81 - 81 * Seta - 44 * eta)) * Pi) / 48.;
  d.ains[2] = ((-27312085.0 - 10287648 * c22 - 10287648 * c12 * (1 + Seta) + 10287648 * c22 * Seta +
                24 * (-1975055 + 857304 * c12 - 994896 * chi1 * chi2 + 857304 * c22) * eta +
                35371056 * e2) *
               pp.four_thirds) /
              8.128512e6;
  d.ains[3] = (pp.five_thirds *
               (chi2 * (-285197 * (-1 + Seta) + 4 * (-91902 + 1579 * Seta) * eta - 35632 * e2) +
                chi1 * (285197 * (1 + Seta) - 4 * (91902 + 1579 * Seta) * eta - 35632 * e2) +
                42840 * (-1.0 + 4 * eta) * Pi)) /
              32256.;
  d.ains[4] = -(Pi2 * (-336 * (-3248849057.0 + 2943675504 * c12 - 3339284256 * chi1 * chi2 +
                               2943675504 * c22) *
                           e2 -
                       324322727232 * e3 -
                       7 * (-177520268561 + 107414046432 * c22 + 107414046432 * c12 * (1 + Seta) -
                            107414046432 * c22 * Seta +
                            11087290368 * (chi1 + chi2 + chi1 * Seta - chi2 * Seta) * Pi) +
                       12 * eta *
                           (-545384828789 - 176491177632 * chi1 * chi2 + 202603761360 * c22 +
                            77616 * c12 * (2610335 + 995766 * Seta) - 77287373856 * c22 * Seta +
                            5841690624 * (chi1 + chi2) * Pi + 21384760320 * Pi2))) /
              6.0085960704e10;
  d.ains[5] = rho1;
  d.ains[6] = rho2;
  d.ains[7] = rho3;
  d.g1 = eval_fit(kFitGamma[0], eta, chi);
  d.g2 = eval_fit(kFitGamma[1], eta, chi);
  d.g3 = eval_fit(kFitGamma[2], eta, chi);
  if (d.g2 <= 1.0)
    d.fpeak = fabs(fring + (fdamp * (-1 + sqrt(1 - d.g2 * d.g2)) * d.g3) / d.g2);
  else
    d.fpeak = fabs(fring + (fdamp * (-1) * d.g3) / d.g2);
  // intermediate amplitude: Hermite data at f1 (value+slope), f2 (value), f3 (value+slope)
  {
    const T f1 = AMP_FJOIN_INS, f3 = d.fpeak;
    const T f2 = f1 + (f3 - f1) / 2.0;
    PowersT<T> p1 = make_powers(f1);
    const T v1 = amp_ins_ansatz(d, f1, p1);
    const T d1 = amp_ins_ansatz_deriv(d, f1);
    const T v3 = amp_mrd_ansatz(d, f3);
    const T d2 = amp_mrd_ansatz_deriv(d, f3);
    const T v2 = eval_fit(kFitV2, eta, chi);
    // divided differences on nodes (f1, f1, f2, f3, f3)
    const T z01 = d1;
    const T z12 = (v2 - v1) / (f2 - f1);
    const T z23 = (v3 - v2) / (f3 - f2);
    const T z34 = d2;
    const T z012 = (z12 - z01) / (f2 - f1);
    const T z123 = (z23 - z12) / (f3 - f1);
    const T z234 = (z34 - z23) / (f3 - f2);
    const T z0123 = (z123 - z012) / (f3 - f1);
    const T z1234 = (z234 - z123) / (f3 - f1);
    const T z01234 = (z1234 - z0123) / (f3 - f1);
    d.hf1 = f1;
    d.hf2 = f2;
    d.hf3 = f3;
    d.hc0 = v1;
    d.hc1 = z01;
    d.hc2 = z012;
    d.hc3 = z0123;
    d.hc4 = z01234;
  }

  // ---------------- phase ----------------
  d.sig1 = eval_fit(kFitSigma[0], eta, chi);
  d.sig2 = eval_fit(kFitSigma[1], eta, chi);
  d.sig3 = eval_fit(kFitSigma[2], eta, chi);
  d.sig4 = eval_fit(kFitSigma[3], eta, chi);
  d.bet1 = eval_fit(kFitBeta[0], eta, chi);
  d.bet2 = eval_fit(kFitBeta[1], eta, chi);
  d.bet3 = eval_fit(kFitBeta[2], eta, chi);
  d.alp1 = eval_fit(kFitAlpha[0], eta, chi);
  d.alp2 = eval_fit(kFitAlpha[1], eta, chi);
  d.alp3 = eval_fit(kFitAlpha[2], eta, chi);
  d.alp4 = eval_fit(kFitAlpha[3], eta, chi);
  d.alp5 = eval_fit(kFitAlpha[4], eta, chi);

  // TaylorF2 aligned-spin phasing (LAL PNPhasing_F2, PhenomHMWaveform.cu:253-335)
  {
    const T m1M = m1 / M, m2M = m2 / M;
    const T dm = (m1 - m2) / M;
    const T SL = m1M * m1M * chi1 + m2M * m2M * chi2;
    const T dSigmaL = dm * (m2M * chi2 - m1M * chi1);
    const T pfaN = 3.0 / (128.0 * eta);
    T v0 = pfaN;
    T v1 = 0.0;
    T v2 = pfaN * (5.0 * (743.0 / 84.0 + 11.0 * eta) / 9.0);
    T v3 = pfaN * (-16.0 * PI);
    T v4 = pfaN * (5.0 * (3058.673 / 7.056 + 5429.0 / 7.0 * eta + 617.0 * eta * eta) / 72.0);
    T v5 = pfaN * (5.0 / 9.0 * (7729.0 / 84.0 - 13.0 * eta) * PI);
    T vlogv5 = pfaN * (5.0 / 3.0 * (7729.0 / 84.0 - 13.0 * eta) * PI);
    T v6 = pfaN * ((11583.231236531 / 4.694215680 - 640.0 / 3.0 * PI * PI - 6848.0 / 21.0 * GAMMA_E) +
                        eta * (-15737.765635 / 3.048192 + 2255. / 12. * PI * PI) +
                        eta * eta * 76055.0 / 1728.0 - eta * eta * eta * 127825.0 / 1296.0);
    v6 += pfaN * (-6848.0 / 21.0) * log(4.);
    T vlogv6 = pfaN * (-6848.0 / 21.0);
    T v7 = pfaN * (PI * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta * eta));
    // spin-spin (2PN) and self-spin terms with qm_def = 1
    T pn_sigma = eta * (721.0 / 48.0 * chi1 * chi2 - 247.0 / 48.0 * chi1 * chi2);
    pn_sigma += (720.0 - 1.0) / 96.0 * m1M * m1M * chi1 * chi1;
    pn_sigma += (720.0 - 1.0) / 96.0 * m2M * m2M * chi2 * chi2;
    pn_sigma -= (240.0 - 7.0) / 96.0 * m1M * m1M * chi1 * chi1;
    pn_sigma -= (240.0 - 7.0) / 96.0 * m2M * m2M * chi2 * chi2;
    T pn_ss3 = (326.75 / 1.12 + 557.5 / 1.8 * eta) * eta * chi1 * chi2;
    pn_ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m1M - 120.0 * m1M * m1M) +
               (-4108.25 / 6.72 - 108.5 / 1.2 * m1M + 125.5 / 3.6 * m1M * m1M)) *
              m1M * m1M * chi1 * chi1;
    pn_ss3 += ((4703.5 / 8.4 + 2935.0 / 6.0 * m2M - 120.0 * m2M * m2M) +
               (-4108.25 / 6.72 - 108.5 / 1.2 * m2M + 125.5 / 3.6 * m2M * m2M)) *
              m2M * m2M * chi2 * chi2;
    const T pn_gamma = (554345.0 / 1134.0 + 110.0 * eta / 9.0) * SL + (13915.0 / 84.0 - 10.0 * eta / 3.0) * dSigmaL;
    v7 += pfaN * ((-8980424995.0 / 762048.0 + 6586595.0 * eta / 756.0 - 305.0 * eta * eta / 36.0) * SL -
                  (170978035.0 / 48384.0 - 2876425.0 * eta / 672.0 - 4735.0 * eta * eta / 144.0) * dSigmaL);
    v6 += pfaN * (PI * (3760.0 * SL + 1490.0 * dSigmaL) / 3.0 + pn_ss3);
    v5 += pfaN * (-1.0 * pn_gamma);
    vlogv5 += pfaN * (-3.0 * pn_gamma);
    v4 += pfaN * (-10.0 * pn_sigma);
    v3 += pfaN * (188.0 * SL / 3.0 + 25.0 * dSigmaL);
    // PhenomD was tuned without the 3PN spin-spin term: remove it (PhenomHMWaveform.cu:1406-1424)
    v6 -= pn_ss3 * v0;
    d.pn_v[0] = v0; d.pn_v[1] = v1; d.pn_v[2] = v2; d.pn_v[3] = v3;
    d.pn_v[4] = v4; d.pn_v[5] = v5; d.pn_v[6] = v6; d.pn_v[7] = v7;
    d.pn_vlogv5 = vlogv5;
    d.pn_vlogv6 = vlogv6;
  }
  // inspiral phase prefactors (PhenomHMWaveform.cu:1180-1207)
  d.pins_init = d.pn_v[5] - PI_4;
  d.pins_23 = d.pn_v[7] * pp.two_thirds;
  d.pins_13 = d.pn_v[6] * pp.third;
  d.pins_13log = d.pn_vlogv6 * pp.third;
  d.pins_log = d.pn_vlogv5;
  d.pins_m13 = d.pn_v[4] / pp.third;
  d.pins_m23 = d.pn_v[3] / pp.two_thirds;
  d.pins_m1 = d.pn_v[2] / Pi;
  d.pins_m53 = d.pn_v[0] / pp.five_thirds;
  d.pins_1 = d.sig1;
  d.pins_43 = d.sig2 * 3.0 / 4.0;
  d.pins_53 = d.sig3 * 3.0 / 5.0;
  d.pins_2 = d.sig4 / 2.0;

  // C1 joins (PhenomHMWaveform.cu:1263-1303)
  {
    const T fj = PHI_FJOIN_INS;
    d.C2Int = dphi_ins(d, fj) - dphi_int(d, fj);
    PowersT<T> pj = make_powers(fj);
    d.C1Int = phi_ins(d, fj, pj) - d.etaInv * phi_int(d, fj) - d.C2Int * fj;
    d.fMRDJoin = 0.5 * fring;
    const T fm = d.fMRDJoin;
    const T phi_int_val = d.etaInv * phi_int(d, fm) + d.C1Int + d.C2Int * fm;
    const T dphi_int_val = d.C2Int + dphi_int(d, fm);
    d.C2MRD = dphi_int_val - dphi_mrd(d, fm, Rholm, Taulm);
    d.C1MRD = phi_int_val - d.etaInv * phi_mrd(d, fm, Rholm, Taulm) - d.C2MRD * fm;
  }
}

// ---------------------------------------------------------------------------------
// PhenomHM per-(binary, mode) record
// ---------------------------------------------------------------------------------
template <typename T>
struct ModeCoeffsT {
  PhenomDT<T> d;
  int ell, mm, phenomd_only, pad;
  // phase frequency map Mf22 = a Mf + b by region (PhenomHMWaveform.cu:2130-2369)
  T ph_fi, ph_fr, ph_ai, ph_am, ph_bm, ph_ar, ph_constB, ph_constC;
  // amplitude frequency map
  T am_fi, am_fr, am_ai, am_am, am_bm, am_br;
  // PN amplitude ratio inputs (PhenomHMWaveform.cu:2375-2455)
  T pn_m1, pn_m2, pn_chi1, pn_chi2;
  // |H_lm(v)| constants: leading factor, eta, delta, chi_s, chi_a; case 0 = 22 / PhenomD,
  // 1..5 = 21, 33, 32, 44, 43, 6 = no PN amplitude
  T pn_k, pn_eta, pn_delta, pn_Xs, pn_Xa, pn_2pi_m, pn_4pi_m2;
  int pn_case, pad2;
  T ph_inv_ai, ph_inv_am, ph_inv_ar;
  // overall shifts / scales
  T t0, phi0, Mf_ref, amp_scale, M_sec, cshift;
};
using ModeCoeffs = ModeCoeffsT<double>;

__device__ __forceinline__ double cshift_of(int mm) {
  // Blanchet arXiv:1310.1528 sec. 9.5 leading-order complex-amplitude phase shifts by m
  switch (mm) {
    case 1: return PI_2;
    case 3: return -PI_2;
    case 4: return PI;
    case 5: return PI_2;
    default: return 0.0;
  }
}

// Set up one (binary, mode) record.  Inputs as the reference's IMRPhenomHM kernel:
// SI masses (kg), distance (m), the mode's QNM ringdown / damping frequencies and the
// PhenomD spline values appended after the modes (phenomhm.py:424-463).
template <typename T>
__device__ inline void phm_setup_mode(ModeCoeffsT<T>& c, T m1_SI, T m2_SI, T chi1,
                                      T chi2, T distance, int ell, int mm,
                                      T Mf_RD_lm, T Mf_DM_lm, T Mf_RD_22_in,
                                      T Mf_DM_22_in, int run_phenomd) {
  T m1 = m1_SI / MSUN_SI, m2 = m2_SI / MSUN_SI;
  if (!(m1 > m2)) {
    T t = m1; m1 = m2; m2 = t;
    t = chi1; chi1 = chi2; chi2 = t;
  }
  const T Mtot = m1 + m2;
  T finmass, finspin;
  final_mass_spin(m1, m2, chi1, chi2, &finmass, &finspin);
  T Mf_RD_22, Mf_DM_22;
  if (!run_phenomd) {
    cplxT<T> z = qnm_cw(finspin, 2, 2);
    Mf_RD_22 = (0.5 / PI) * z.re / finmass;
    Mf_DM_22 = (0.5 / PI) * z.im / finmass;
  } else {
    Mf_RD_22 = Mf_RD_lm;
    Mf_DM_22 = Mf_DM_lm;
  }
  // 22-mode PhenomD: reference frequency = amplitude peak, t0 and phi0 from there
  PhenomDT<T> d22;
  phenomd_setup(d22, m1, m2, chi1, chi2, Mf_RD_22_in, Mf_DM_22_in, T(1.0), T(1.0));
  const T Mf_ref = d22.fpeak;
  const T phi22_ref = phenomd_phase(d22, Mf_ref);
  c.phi0 = 0.5 * phi22_ref;
  c.t0 = phenomd_dphase(d22, Mf_ref);
  c.Mf_ref = Mf_ref;
  c.amp_scale = ((m1_SI + m2_SI) / MSUN_SI) * MRSUN_SI * ((m1_SI + m2_SI) / MSUN_SI) * MTSUN_SI / distance;
  c.M_sec = Mtot * MTSUN_SI;
  c.ell = ell;
  c.mm = mm;
  c.phenomd_only = run_phenomd;
  c.pn_m1 = m1;
  c.pn_m2 = m2;
  c.pn_chi1 = chi1;
  c.pn_chi2 = chi2;
  {
    const T M1 = m1 / (m1 + m2), M2 = m2 / (m1 + m2);
    const T eta = M1 * M2 / ((M1 + M2) * (M1 + M2));
    c.pn_eta = eta;
    c.pn_delta = sqrt(1.0 - 4 * eta);
    c.pn_Xs = 0.5 * (chi1 + chi2);
    c.pn_Xa = 0.5 * (chi1 - chi2);
    c.pn_2pi_m = 2.0 * PI / mm;
    c.pn_4pi_m2 = 4.0 * PI / ((T)mm * mm);
    if (run_phenomd || (ell == 2 && mm == 2)) { c.pn_case = 0; c.pn_k = 1.0; }
    else if (ell == 2 && mm == 1) { c.pn_case = 1; c.pn_k = sqrt(2.0) / 3.0; }
    else if (ell == 3 && mm == 3) { c.pn_case = 2; c.pn_k = 0.75 * sqrt(5.0 / 7.0); }
    else if (ell == 3 && mm == 2) { c.pn_case = 3; c.pn_k = (1.0 / 3.0) * sqrt(5.0 / 7.0); }
    else if (ell == 4 && mm == 4) { c.pn_case = 4; c.pn_k = (4.0 / 9.0) * sqrt(10.0 / 7.0); }
    else if (ell == 4 && mm == 3) { c.pn_case = 5; c.pn_k = 0.75 * sqrt(3.0 / 35.0); }
    else { c.pn_case = 6; c.pn_k = 0.0; }
    c.pad2 = 0;
  }
  if (run_phenomd) {
    c.d = d22;
    c.cshift = cshift_of(2);
    return;
  }
  c.cshift = cshift_of(mm);
  const T Rholm = Mf_RD_22 / Mf_RD_lm;
  const T Taulm = Mf_DM_lm / Mf_DM_22;
  phenomd_setup(c.d, m1, m2, chi1, chi2, Mf_RD_22_in, Mf_DM_22_in, Rholm, Taulm);
  // phase map: inspiral Mf22 = (2/m) Mf; ringdown Mf22 = Rholm Mf; linear in between
  {
    const T fi = PHI_FJOIN_INS / Rholm;
    const T fr = Mf_RD_lm;
    const T ai = 2.0 / mm;
    const T Trd = Rholm * fr;
    const T Ti = 2.0 * fi / mm;
    const T am = (Trd - Ti) / (fr - fi);
    const T bm = Ti - fi * am;
    const T ar = Rholm;
    c.ph_fi = fi;
    c.ph_fr = fr;
    c.ph_ai = ai;
    c.ph_am = am;
    c.ph_bm = bm;
    c.ph_ar = ar;
    c.ph_inv_ai = 1.0 / ai;
    c.ph_inv_am = 1.0 / am;
    c.ph_inv_ar = 1.0 / ar;
    const T PhDBconst = phenomd_phase(c.d, am * fi + bm) / am;
    const T PhDCconst = phenomd_phase(c.d, ar * fr) / ar;
    const T PhDBAterm = phenomd_phase(c.d, ai * fi) / ai;
    const T tmpC = phenomd_phase(c.d, am * fr + bm) / am - PhDBconst + PhDBAterm;
    c.ph_constB = -PhDBconst + PhDBAterm;
    c.ph_constC = -PhDCconst + tmpC;
  }
  // amplitude map: inspiral (2/m) Mf; ringdown Mf - Mf_RD_lm + Mf_RD_22
  {
    const T fi = AMP_FJOIN_INS / Rholm;
    const T fr = Mf_RD_lm;
    const T Trd = fr - Mf_RD_lm + Mf_RD_22;
    const T Ti = 2.0 * fi / mm;
    const T am = (Trd - Ti) / (fr - fi);
    c.am_fi = fi;
    c.am_fr = fr;
    c.am_ai = 2.0 / mm;
    c.am_am = am;
    c.am_bm = Ti - fi * am;
    c.am_br = -Mf_RD_lm + Mf_RD_22;
  }
}

// |H_lm(v)| of the 1.5PN spinning amplitude (IMRPhenomHMOnePointFiveSpinPN,
// PhenomHMWaveform.cu:2375-2455) for the non-22 cases.
template <typename T>
__device__ __forceinline__ T pn_habs(const ModeCoeffsT<T>& c, T v) {
  const T v2 = v * v, v3 = v2 * v;
  switch (c.pn_case) {
    case 1: {
      const T v4 = v3 * v;
      const T re = c.pn_k * (v * c.pn_delta - v2 * 1.5 * (c.pn_Xa + c.pn_delta * c.pn_Xs) +
                                  v3 * c.pn_delta * ((335.0 / 672.0) + (c.pn_eta * 117.0 / 56.0)) +
                                  v4 * (c.pn_Xa * (3427.0 / 1344 - c.pn_eta * 2101.0 / 336) +
                                        c.pn_delta * c.pn_Xs * (3427.0 / 1344 - c.pn_eta * 965 / 336) +
                                        c.pn_delta * (-PI)));
      const T im = c.pn_k * v4 * c.pn_delta * (-0.5 - 2.0 * 0.69314718056);
      return hypot(re, im);
    }
    case 2: return fabs(c.pn_k * (v * c.pn_delta));
    case 3: return fabs(c.pn_k * (v2 * (1.0 - 3.0 * c.pn_eta)));
    case 4: return fabs(c.pn_k * v2 * (1.0 - 3.0 * c.pn_eta));
    case 5: return fabs(c.pn_k * v3 * c.pn_delta * (1.0 - 2.0 * c.pn_eta));
    default: return 0.0;
  }
}

// HM amplitude factor of get_amp (PhenomHMWaveform.cu:2461-2514): beta * HMamp1 / HMamp2 =
// [P(Mf) / P(2Mf/m)] * [P_lm(Mfa) / P_22(Mfa)] with P = v^-3.5 |H(v)|, v = (2 pi x / m)^(1/3).
// The v^-3.5 factors cancel exactly (v(2Mf/m) / v(Mf) = (2/m)^(1/3), v_22(Mfa) / v_lm(Mfa)
// = (m/2)^(1/3)), leaving |H(v(Mf))| |H(v(Mfa))| / |H(v(2Mf/m))|; zero where |H(v(Mf))| = 0
// (the reference's equal-mass guard).
template <typename T>
__device__ __forceinline__ T hm_amp_factor(const ModeCoeffsT<T>& c, T Mf, T Mfa) {
  if (c.pn_case == 0) return 1.0;
  const T t1 = pn_habs(c, cbrt(c.pn_2pi_m * Mf));
  if (t1 == 0.0) return 0.0;
  const T t2 = pn_habs(c, cbrt(c.pn_4pi_m2 * Mf));
  const T h1 = pn_habs(c, cbrt(c.pn_2pi_m * Mfa));
  return (t1 / t2) * h1;
}

// Mapped PhenomD frequency and phase constants of the HM phase map (get_phase,
// PhenomHMWaveform.cu:2517-2565): ph = phase(Mfp) * inv + add.
template <typename T>
__device__ __forceinline__ void hm_phase_map(const ModeCoeffsT<T>& c, T Mf, T* Mfp,
                                             T* inv, T* add) {
  if (!(Mf > c.ph_fi)) {
    *Mfp = c.ph_ai * Mf;
    *inv = c.ph_inv_ai;
    *add = 0.0;
  } else if (!(Mf > c.ph_fr)) {
    *Mfp = c.ph_am * Mf + c.ph_bm;
    *inv = c.ph_inv_am;
    *add = c.ph_constB;
  } else {
    *Mfp = c.ph_ar * Mf;
    *inv = c.ph_inv_ar;
    *add = c.ph_constC;
  }
}

// Phase and t(f) of one mode at Mf (no t_ref shift).
template <typename T>
__device__ __forceinline__ void mode_phase_tf(const ModeCoeffsT<T>& c, T Mf, T* phase,
                                              T* tf) {
  T ph, dph;
  if (c.phenomd_only) {
    phenomd_phase_dphase(c.d, Mf, &ph, &dph);
    *phase = -c.t0 * (Mf - c.Mf_ref) + ((c.cshift + ph) - 2 * c.phi0);
  } else {
    T Mfp, inv, add;
    hm_phase_map(c, Mf, &Mfp, &inv, &add);
    phenomd_phase_dphase(c.d, Mfp, &ph, &dph);
    *phase = -c.t0 * (Mf - c.Mf_ref) + ((c.cshift + (ph * inv + add)) - c.mm * c.phi0);
  }
  const double INV_2PI = 0.15915494309189533577;  // 1 / (2 pi)
  *tf = c.M_sec * (dph * INV_2PI) - (c.t0 * INV_2PI * c.M_sec);
}

// Mapped amplitude frequency (IMRPhenomHMFreqDomainMap with AmpFlag, :2295-2315).
template <typename T>
__device__ __forceinline__ T hm_amp_map(const ModeCoeffsT<T>& c, T Mf) {
  if (Mf > c.am_fi) return (Mf > c.am_fr) ? Mf + c.am_br : c.am_am * Mf + c.am_bm;
  return c.am_ai * Mf;
}

template <typename T>
struct PointOutT {
  T amp, phase, tf;
};
using PointOut = PointOutT<double>;

// Amplitude, phase and t(f) of one mode at frequency f (Hz).  t(f) and phase do not yet
// include the t_ref shift (added by the caller, phenomhm.py:485-507).
template <typename T>
__device__ inline PointOutT<T> phm_eval_point(const ModeCoeffsT<T>& c, T f) {
  PointOutT<T> o;
  const T Mf = f * c.M_sec;
  if (c.phenomd_only) {
    o.amp = phenomd_amp(c.d, Mf) * c.amp_scale;
  } else {
    const T Mfa = hm_amp_map(c, Mf);
    o.amp = phenomd_amp(c.d, Mfa) * hm_amp_factor(c, Mf, Mfa) * c.amp_scale;
  }
  mode_phase_tf(c, Mf, &o.phase, &o.tf);
  return o;
}

}  // namespace bbhx
