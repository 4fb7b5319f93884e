// cp_opcount.cc -- the algorithmic operation count of the hadronic integrand, per point.
//
// TEST INFRASTRUCTURE ONLY (like the rest of oracle/): it pins the per-point work that the
// integrand kernels' roofline is quoted on.  Nothing in the product calls it.
//
// The integrand of cp_oracle_body.h (Pythia's formulas: PartonDistributions.cc:922-1062 CTEQ5L,
// StandardModel.cc:42-64,189-215 first-order alpha_s, SigmaQCD.cc:115-325 matrix elements,
// SigmaProcess.cc:423-480 sigmaPDF, PhaseSpace.cc:1149-1250 the tau/y/z region and weights)
// restated once more over a scalar type T, in the form with the least arithmetic that computes
// the same function -- the algorithm's own work, without the precision bookkeeping of an FP32
// implementation (compensated sums, (hi, lo) logarithms) and without redundant evaluation:
//   * the CTEQ5L terms that depend on Q alone (ln Q, ln ln(Q / alpha_i), the 9 scale polynomials
//     of each of the 8 parametrisations) once per point, not once per beam;
//   * pow(y, p) as exp(p ln y) with ln y once per beam; ln x of each beam from the phase-space
//     map (ln x = ln tau / 2 +- y) rather than a logarithm;
//   * polynomials whose three CTEQ5L coefficients are all zero skipped;
//   * the channel sums of sigmaPDF factorised: gg once, qg from the quark sums of the two beams,
//     qq from the quark sums and the same-flavour and opposite-flavour products, qqbar from the
//     opposite-flavour products; one reciprocal each of tHat/sHat and uHat/sHat shared by the
//     five matrix elements;
//   * the VEGAS map per dimension (x = low edge + fraction x width, Jacobian nb x width); the
//     bin and fraction themselves are integer work (Philox words), as is the Philox draw.
// With T = double it must equal cpo_had_weight_x (the literal restatement) to rounding
// (tests/test_opcount.py: 1e-12 relative); with T = a counting scalar every +, -, x, / and every
// exp, log, sqrt of one point is tallied (a negation and constants are free).
#include <cmath>
#include <cstdint>
#include <cstring>

#include "cp_oracle.h"

namespace {

struct Tally {
  double add, mul, div, exp, log, sqrt;
};
Tally* g_tally = nullptr;

struct CR {
  double v;
  CR() : v(0.0) {}
  CR(double x) : v(x) {}
};
inline CR operator+(CR a, CR b) { g_tally->add += 1; return CR(a.v + b.v); }
inline CR operator-(CR a, CR b) { g_tally->add += 1; return CR(a.v - b.v); }
inline CR operator*(CR a, CR b) { g_tally->mul += 1; return CR(a.v * b.v); }
inline CR operator/(CR a, CR b) { g_tally->div += 1; return CR(a.v / b.v); }
inline CR operator-(CR a) { return CR(-a.v); }
inline CR exp(CR a) { g_tally->exp += 1; return CR(std::exp(a.v)); }
inline CR log(CR a) { g_tally->log += 1; return CR(std::log(a.v)); }
inline CR sqrt(CR a) { g_tally->sqrt += 1; return CR(std::sqrt(a.v)); }
inline double val(CR a) { return a.v; }
inline double val(double a) { return a; }
using std::exp;
using std::log;
using std::sqrt;

// Per-configuration constants (formed once, outside the per-point count).
struct Consts {
  double s, lnTauMin, pT2min4, kR, kF, conv, nQuarkNew, K0;
  double lnL2[4], thr2[3], scale2Min, aCoef[4];   // alpha_s: 12 pi / (33 - 2 nf) per nf = 3..6
  const double* am;                                // CTEQ5L [8][9][3]
  double lnAlpha[8], qlim[8], qmin[8], ut1[8], eut2[8];
  bool useX1L[8], nz[8][9];
  double ln1em5;
};

void make_consts(const cpo_had_cfg* c, Consts& K)
{
  K.s = c->sqrtS * c->sqrtS;
  double tauMin = 4.0 * c->pTmin * c->pTmin / K.s;
  if (tauMin < 16.0 / K.s) tauMin = 16.0 / K.s;
  K.lnTauMin = std::log(tauMin);
  K.pT2min4 = 4.0 * c->pTmin * c->pTmin;
  K.kR = c->kR;
  K.kF = c->kF;
  K.conv = c->convert2mb;
  K.nQuarkNew = c->nQuarkNew;
  // w = sigmaPDF (mHat pAbs / tau) jTau jY jZ with sigmaPDF = conv pi alpha_s^2 / sH^2 x (bracket
  // sum): (0.5 sH / tau)(-lnTauMin tau)(2 yMax)(2 zMax) conv pi alpha_s^2 / sH^2
  //     = K0 alpha_s^2 yMax zMax / sH x (bracket sum), K0 = -2 pi conv lnTauMin
  K.K0 = -2.0 * M_PI * K.conv * K.lnTauMin;
  const double MZ = 91.188, mc = 1.5, mb = 4.8, mt = 171.0;
  const double L5 = MZ * std::exp(-6.0 * M_PI / (23.0 * c->aSmZ));
  const double L6 = L5 * std::pow(L5 / mt, 2.0 / 21.0);
  const double L4 = L5 * std::pow(mb / L5, 2.0 / 25.0);
  const double L3 = L4 * std::pow(mc / L4, 2.0 / 27.0);
  K.lnL2[0] = std::log(L3 * L3); K.lnL2[1] = std::log(L4 * L4);
  K.lnL2[2] = std::log(L5 * L5); K.lnL2[3] = std::log(L6 * L6);
  K.thr2[0] = mc * mc; K.thr2[1] = mb * mb; K.thr2[2] = mt * mt;
  K.scale2Min = (1.07 * L3) * (1.07 * L3);
  for (int k = 0; k < 4; ++k) K.aCoef[k] = 12.0 * M_PI / (27.0 - 2.0 * k);
  const double *qmin, *alpha, *ut1, *ut2;
  cpo_cteq5l_table(&K.am, &qmin, &alpha, &ut1, &ut2);
  for (int i = 0; i < 8; ++i) {
    K.lnAlpha[i] = std::log(alpha[i]);
    K.qmin[i] = qmin[i];
    K.qlim[i] = qmin[i] > alpha[i] ? qmin[i] : alpha[i];
    K.ut1[i] = ut1[i];
    K.useX1L[i] = ut2[i] < -100.0;
    K.eut2[i] = K.useX1L[i] ? 0.0 : std::exp(ut2[i]);
    for (int j = 0; j < 9; ++j) {
      const double* a = K.am + (i * 9 + j) * 3;
      K.nz[i][j] = a[0] != 0.0 || a[1] != 0.0 || a[2] != 0.0;
    }
  }
  K.ln1em5 = std::log(1e-5);
}

// first-order alpha_s (StandardModel.cc:189-215)
template <class T>
T alphas(const Consts& K, T Q2)
{
  if (val(Q2) < K.scale2Min) Q2 = T(K.scale2Min);
  const T lq = log(Q2);
  int k = 0;
  if (val(Q2) > K.thr2[2]) k = 3;
  else if (val(Q2) > K.thr2[1]) k = 2;
  else if (val(Q2) > K.thr2[0]) k = 1;
  return T(K.aCoef[k]) / (lq - K.lnL2[k]);
}

// The Q-dependent part of CTEQ5L, shared by the two beams.
template <class T>
struct CteqQ {
  bool on[8];
  T af[8][9], p[8], qfac[8];
};

template <class T>
void cteq_q(const Consts& K, T Q2, CteqQ<T>& C)
{
  if (val(Q2) > 1e8) Q2 = T(1e8);
  if (val(Q2) < 1.0) Q2 = T(1.0);
  const T lnQ = 0.5 * log(Q2);
  T Q = T(0.0);
  bool needQ = false;
  for (int i = 0; i < 8; ++i) needQ = needQ || K.qmin[i] > 0.0;
  if (needQ) Q = sqrt(Q2);
  for (int i = 0; i < 8; ++i) {
    C.on[i] = std::exp(val(lnQ)) > K.qlim[i];
    if (!C.on[i]) continue;
    const T tmp = lnQ - K.lnAlpha[i];
    const T sb1 = log(tmp) - 1.2;
    const T sb2 = sb1 * sb1;
    for (int j = 0; j < 9; ++j) {
      const double* a = K.am + (i * 9 + j) * 3;
      C.af[i][j] = K.nz[i][j] ? T(a[0]) + sb1 * a[1] + sb2 * a[2] : T(0.0);
    }
    C.p[i] = 1.0 + 0.01 * C.af[i][4];
    C.qfac[i] = K.qmin[i] > 0.0 ? 1.0 - K.qmin[i] / Q : T(1.0);
  }
}

// The x-dependent part of one beam: xf = {d, u, g, ubar, dbar, s, c, b}
template <class T>
void cteq_x(const Consts& K, const CteqQ<T>& C, T lnx, T x, T xf[8])
{
  const T y = -lnx;
  const T lny = log(y);
  const T u = lnx - K.ln1em5;
  const T x1 = 1.0 - x;
  const T x1L = log(x1);
  const T xx1 = x * x1;
  T ans[8];
  for (int i = 0; i < 8; ++i) {
    if (!C.on[i]) { ans[i] = T(0.0); continue; }
    const T* af = C.af[i];
    T part1 = af[1] * exp(C.p[i] * lny);
    if (K.nz[i][8]) part1 = part1 * (1.0 + af[8] * u);
    const T part2 = af[0] * x1 + af[3] * x;
    T in3 = af[5] + af[6] * x1;
    if (K.nz[i][7]) in3 = in3 + af[7] * xx1;
    const T part3 = xx1 * in3;
    const T L = K.useX1L[i] ? x1L : log(x1 + K.eut2[i]);
    const T part4 = K.ut1[i] * x1L + af[2] * L;
    T a = x * exp(part1 + part2 + part3 + part4);
    if (K.qmin[i] > 0.0) a = a * C.qfac[i];
    ans[i] = a;
  }
  xf[0] = x * ans[0];
  xf[1] = x * ans[1];
  xf[2] = x * ans[2];
  // ubar + dbar and dbar/ubar (PartonDistributions.cc:1052-1054)
  const T S = x * ans[3];
  const T ubar = S / (1.0 + ans[4]);
  xf[3] = ubar;
  xf[4] = S - ubar;
  xf[5] = x * ans[5];
  xf[6] = x * ans[6];
  xf[7] = x * ans[7];
  for (int k = 0; k < 8; ++k)
    if (val(xf[k]) < 0.0) xf[k] = T(0.0);   // max(0, .) of PDF::xf
}

// The weight of the base-map point x in [0,1]^3 (cpo_had_weight_x), all five processes.
template <class T>
T weight_x(const Consts& K, const T x[3])
{
  const T lnTau = (1.0 - x[0]) * K.lnTauMin;
  const T tau = exp(lnTau);
  const T yMax = -0.5 * lnTau;
  const T y = yMax * (2.0 * x[1] - 1.0);
  const T sH = tau * K.s;
  T zArg = 1.0 - K.pT2min4 / sH;
  if (val(zArg) <= 0.0) return T(0.0);
  const T zMax = sqrt(zArg);
  const T z = zMax * (2.0 * x[2] - 1.0);
  // tHat / sHat = -(1 - z) / 2, uHat / sHat = -(1 + z) / 2, pT^2 = sH (1 - z)(1 + z) / 4
  const T omz = 1.0 - z, opz = 1.0 + z;
  const T tp = -0.5 * omz, up = -0.5 * opz;
  const T pT2 = 0.25 * (sH * (omz * opz));
  const T alpS = alphas(K, K.kR == 1.0 ? pT2 : pT2 * K.kR);
  // incoming momentum fractions: ln x1,2 = ln tau / 2 +- y
  const T hl = 0.5 * lnTau;
  const T lnx1 = hl + y, lnx2 = hl - y;
  T x1 = exp(lnx1), x2 = exp(lnx2);
  if (val(x1) > 1.0 - 1e-10) x1 = T(1.0 - 1e-10);
  if (val(x2) > 1.0 - 1e-10) x2 = T(1.0 - 1e-10);
  CteqQ<T> C;
  cteq_q(K, K.kF == 1.0 ? pT2 : pT2 * K.kF, C);
  T fa[8], fb[8];
  cteq_x(K, C, lnx1, x1, fa);
  cteq_x(K, C, lnx2, x2, fb);
  // matrix elements per (pi / sH^2) alpha_s^2 (SigmaQCD.cc), one reciprocal each of tp and up
  const T rt = 1.0 / tp, ru = 1.0 / up;
  const T tr = tp * ru, ur = up * rt;
  const T tp2 = tp * tp, up2 = up * up, rt2 = rt * rt, ru2 = ru * ru, tr2 = tr * tr, ur2 = ur * ur;
  const T gg2gg = (9.0 / 8.0) * ((tp2 + up2 + rt2 + ru2 + tr2 + ur2) + 2.0 * (tp + up + rt + ru + tr + ur) + 9.0);
  const T gg2qq = K.nQuarkNew * ((1.0 / 6.0) * (ur + tr) - (3.0 / 8.0) * (up2 + tp2));
  const T qg2qg = ur2 + rt2 - (4.0 / 9.0) * (up + ru);
  const T qqT = (4.0 / 9.0) * ((1.0 + up2) * rt2);
  const T qqU = (4.0 / 9.0) * ((1.0 + tp2) * ru2);
  const T qqTU = (-8.0 / 27.0) * (rt * ru);
  const T qqST = (-8.0 / 27.0) * (up2 * rt);
  const T qqbar2gg = (16.0 / 27.0) * (ur + tr) - (4.0 / 3.0) * (up2 + tp2);
  // factorised channel sums (SigmaProcess.cc:423-480 over the initFlux lists, nQuarkIn = 5)
  const T heavyA = fa[5] + fa[6] + fa[7], heavyB = fb[5] + fb[6] + fb[7];
  const T QA = (fa[0] + fa[1]) + (fa[3] + fa[4]) + 2.0 * heavyA;
  const T QB = (fb[0] + fb[1]) + (fb[3] + fb[4]) + 2.0 * heavyB;
  const T HH = 2.0 * (fa[5] * fb[5] + fa[6] * fb[6] + fa[7] * fb[7]);
  const T Dsame = fa[0] * fb[0] + fa[1] * fb[1] + fa[3] * fb[3] + fa[4] * fb[4] + HH;
  const T Dopp = fa[0] * fb[4] + fa[4] * fb[0] + fa[1] * fb[3] + fa[3] * fb[1] + HH;
  const T G = fa[2] * fb[2];
  const T sum = G * (gg2gg + gg2qq) + qg2qg * (QA * fb[2] + fa[2] * QB) +
                (qqT * (QA * QB) + Dsame * (0.5 * (qqU + qqTU - qqT)) + Dopp * qqST) + Dopp * qqbar2gg;
  return K.K0 * ((alpS * alpS) * (yMax * zMax)) / sH * sum;
}

}  // namespace

extern "C" {

// The weight of cpo_had_weight_x in the counted form (T = double).
double cpo_opcount_weight(const cpo_had_cfg* c, const double x[3])
{
  Consts K;
  make_consts(c, K);
  const double xx[3] = {x[0], x[1], x[2]};
  return weight_x<double>(K, xx);
}

// Mean operation counts per point over the n base-map points x (3n doubles), in the order
// add, mul, div, exp, log, sqrt (out[6]); out[6] = the largest relative difference of the
// counted evaluation from cpo_had_weight_x over the points.  The VEGAS map is added per point:
// per dimension x = low + fraction * width (1 mul, 1 add) and the Jacobian factor nb * width
// (1 mul) times the running product (1 mul), then the weight times the product (1 mul).
void cpo_opcount_counts(const cpo_had_cfg* c, const double* x, int64_t n, double out[7])
{
  Consts K;
  make_consts(c, K);
  Tally t{};
  g_tally = &t;
  double worst = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    const CR xx[3] = {CR(x[3 * i]), CR(x[3 * i + 1]), CR(x[3 * i + 2])};
    const CR w = weight_x<CR>(K, xx);
    const double ref = cpo_had_weight_x(c, x + 3 * i, nullptr);
    if (ref != 0.0) {
      const double r = std::fabs(w.v - ref) / std::fabs(ref);
      if (r > worst) worst = r;
    }
  }
  g_tally = nullptr;
  const double vegas_add = 3.0, vegas_mul = 3.0 * 3.0 + 1.0;
  const double dn = n > 0 ? (double)n : 1.0;
  out[0] = t.add / dn + vegas_add;
  out[1] = t.mul / dn + vegas_mul;
  out[2] = t.div / dn;
  out[3] = t.exp / dn;
  out[4] = t.log / dn;
  out[5] = t.sqrt / dn;
  out[6] = worst;
}

}  // extern "C"
