/*
 * cp_oracle.c -- CPU FP64 restatement of the QCD 2->2 integrator path (test infrastructure;
 * see cp_oracle.h for the rules on who may call it).
 */
#define _GNU_SOURCE
#include "cp_oracle.h"
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ======================= counter RNGs ======================= */

/* SplitMix64, cuPythia/common/rng.cuh:47-52 */
uint64_t cpo_splitmix64(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}
/* top 53 bits -> [0,1), cuPythia/common/rng.cuh:55-57 */
double cpo_u01(uint64_t u) { return (double)(u >> 11) * (1.0 / 9007199254740992.0); }
/* per-thread stream start, cuPythia/03_fused_resident_me/fused_gg2gg.cu:43 */
uint64_t cpo_thread_counter(uint64_t seed, uint64_t tid) { return seed + tid * 0x100000001B3ULL; }
/* per-event key, cuPythia/05_reproducible_events/repro_events.cu:43 and
 * cuPythia/pipeline/generate.cu:33 */
uint64_t cpo_event_key(uint64_t base, uint64_t e)
{
  return cpo_splitmix64(base ^ (e * 0x9E3779B97F4A7C15ULL));
}

/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of
 * (L0,R0,L1,R1) -> (hi(M1 R1) ^ L0' ^ k0, lo(M1 R1), hi(M0 R0) ^ L1' ^ k1, lo(M0 R0)),
 * round keys bumped by the Weyl constants between rounds. */
void cpo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
  uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
  uint32_t k0 = key[0], k1 = key[1];
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void cpo_point_words(uint64_t seed, uint64_t point, uint32_t iter, uint32_t stream, uint32_t out[4])
{
  uint32_t ctr[4] = {(uint32_t)point, (uint32_t)(point >> 32), iter, stream};
  uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
  cpo_philox4x32_10(ctr, key, out);
}
double cpo_u24(uint32_t w) { return (double)(w >> 8) * (1.0 / 16777216.0); }
double cpo_u53(uint32_t lo, uint32_t hi)
{
  uint64_t v = ((uint64_t)hi << 32) | lo;
  return (double)(v >> 11) * (1.0 / 9007199254740992.0);
}

/* ======================= CTEQ5L coefficients ======================= */
/* pythia8317/src/PartonDistributions.cc:936-1023 (published CTEQ5L fit parameters) */
static const double CTEQ5L_QMIN[8] = {0., 0., 0., 0., 0., 0., 1.3, 4.5};
static const double CTEQ5L_ALPHA[8] = {0.2987216, 0.3407552, 0.4491863, 0.2457668,
                                       0.5293999, 0.3713141, 0.03712017, 0.004952010};
static const double CTEQ5L_UT1[8] = {4.971265, 2.612618, -0.4656819, 3.862583,
                                     0.1895615, 3.753257, 4.400772, 5.562568};
static const double CTEQ5L_UT2[8] = {-1.105128, -1.258304e5, -274.2390, -1.265969,
                                     -3.069097, -1.113085, -1.356116, -1.801317};
static const double CTEQ5L_AM[8][9][3] = {
  /* d */
  {{0.5292616E+01, -0.2751910E+01, -0.2488990E+01}, {0.9714424E+00, 0.1011827E-01, -0.1023660E-01},
   {-0.1651006E+02, 0.7959721E+01, 0.8810563E+01}, {-0.1643394E+02, 0.5892854E+01, 0.9348874E+01},
   {0.3067422E+02, 0.4235796E+01, -0.5112136E+00}, {0.2352526E+02, -0.5305168E+01, -0.1169174E+02},
   {-0.1095451E+02, 0.3006577E+01, 0.5638136E+01}, {-0.1172251E+02, -0.2183624E+01, 0.4955794E+01},
   {0.1662533E-01, 0.7622870E-02, -0.4895887E-03}},
  /* u */
  {{0.9905300E+00, -0.4502235E+00, 0.1624441E+00}, {0.8867534E+00, 0.1630829E-01, -0.4049085E-01},
   {0.8547974E+00, 0.3336301E+00, 0.1371388E+00}, {0.2941113E+00, -0.1527905E+01, 0.2331879E+00},
   {0.3384235E+02, 0.3715315E+01, 0.8276930E+00}, {0.6230115E+01, 0.3134639E+01, -0.1729099E+01},
   {-0.1186928E+01, -0.3282460E+00, 0.1052020E+00}, {-0.8545702E+01, -0.6247947E+01, 0.3692561E+01},
   {0.1724598E-01, 0.7120465E-02, 0.4003646E-04}},
  /* g */
  {{0.1193572E+03, -0.3886845E+01, -0.1133965E+01}, {-0.9421449E+02, 0.3995885E+01, 0.1607363E+01},
   {0.4206383E+01, 0.2485954E+00, 0.2497468E+00}, {0.1210557E+03, -0.3015765E+01, -0.1423651E+01},
   {-0.1013897E+03, -0.7113478E+00, 0.2621865E+00}, {-0.1312404E+01, -0.9297691E+00, -0.1562531E+00},
   {0.1627137E+01, 0.4954111E+00, -0.6387009E+00}, {0.1537698E+00, -0.2487878E+00, 0.8305947E+00},
   {0.2496448E-01, 0.2457823E-02, 0.8234276E-03}},
  /* ubar + dbar */
  {{0.2647441E+02, 0.1059277E+02, -0.9176654E+00}, {0.1990636E+01, 0.8558918E-01, 0.4248667E-01},
   {-0.1476095E+02, -0.3276255E+02, 0.1558110E+01}, {-0.2966889E+01, -0.3649037E+02, 0.1195914E+01},
   {-0.1000519E+03, -0.2464635E+01, 0.1964849E+00}, {0.3718331E+02, 0.4700389E+02, -0.2772142E+01},
   {-0.1872722E+02, -0.2291189E+02, 0.1089052E+01}, {-0.1628146E+02, -0.1823993E+02, 0.2537369E+01},
   {-0.1156300E+01, -0.1280495E+00, 0.5153245E-01}},
  /* dbar / ubar */
  {{-0.6556775E+00, 0.2490190E+00, 0.3966485E-01}, {0.1305102E+01, -0.1188925E+00, -0.4600870E-02},
   {-0.2371436E+01, 0.3566814E+00, -0.2834683E+00}, {-0.6152826E+01, 0.8339877E+00, -0.7233230E+00},
   {-0.8346558E+01, 0.2892168E+01, 0.2137099E+00}, {0.1279530E+02, 0.1021114E+00, 0.5787439E+00},
   {0.5858816E+00, -0.1940375E+01, -0.4029269E+00}, {-0.2795725E+02, -0.5263392E+00, 0.1290229E+01},
   {0.0, 0.0, 0.0}},
  /* sbar */
  {{0.1580931E+01, -0.2273826E+01, -0.1822245E+01}, {0.2702644E+01, 0.6763243E+00, 0.7231586E-02},
   {-0.1857924E+02, 0.3907500E+01, 0.5850109E+01}, {-0.3044793E+02, 0.2639332E+01, 0.5566644E+01},
   {-0.4258011E+01, -0.5429244E+01, 0.4418946E+00}, {0.3465259E+02, -0.5532604E+01, -0.4904153E+01},
   {-0.1658858E+02, 0.2923275E+01, 0.2266286E+01}, {-0.1149263E+02, 0.2877475E+01, -0.7999105E+00},
   {0.0, 0.0, 0.0}},
  /* cbar */
  {{-0.8293661E+00, -0.3982375E+01, -0.6494283E-01}, {0.2754618E+01, 0.8338636E+00, -0.6885160E-01},
   {-0.1657987E+02, 0.1439143E+02, -0.6887240E+00}, {-0.2800703E+02, 0.1535966E+02, -0.7377693E+00},
   {-0.6460216E+01, -0.4783019E+01, 0.4913297E+00}, {0.3141830E+02, -0.3178031E+02, 0.7136013E+01},
   {-0.1802509E+02, 0.1862163E+02, -0.4632843E+01}, {-0.1240412E+02, 0.2565386E+02, -0.1066570E+02},
   {0.0, 0.0, 0.0}},
  /* bbar */
  {{-0.6031237E+01, 0.1992727E+01, -0.1076331E+01}, {0.2933912E+01, 0.5839674E+00, 0.7509435E-01},
   {-0.8284919E+01, 0.1488593E+01, -0.8251678E+00}, {-0.1925986E+02, 0.2805753E+01, -0.3015446E+01},
   {-0.9480483E+01, -0.9767837E+00, -0.1165544E+01}, {0.2193195E+02, -0.1788518E+02, 0.9460908E+01},
   {-0.1327377E+02, 0.1201754E+02, -0.6277844E+01}, {0.0, 0.0, 0.0},
   {0.0, 0.0, 0.0}}};

/* read-only view of the tables above (the operation-count restatement, cp_opcount.cc) */
void cpo_cteq5l_table(const double** am, const double** qmin, const double** alpha, const double** ut1,
                      const double** ut2)
{
  *am = &CTEQ5L_AM[0][0][0];
  *qmin = CTEQ5L_QMIN;
  *alpha = CTEQ5L_ALPHA;
  *ut1 = CTEQ5L_UT1;
  *ut2 = CTEQ5L_UT2;
}

/* ======================= the integrand, twice ======================= */
#define REAL double
#define FN(n) n##_r
#define RE(x) (x)
#define R_EXP exp
#define R_LOG log
#define R_SQRT sqrt
#define R_POW pow
#include "cp_oracle_body.h"
#undef REAL
#undef FN
#undef RE
#undef R_EXP
#undef R_LOG
#undef R_SQRT
#undef R_POW

static double complex cpow_pos(double complex a, double complex b) { return cexp(b * clog(a)); }
#define REAL double complex
#define FN(n) n##_c
#define RE(x) creal(x)
#define R_EXP cexp
#define R_LOG clog
#define R_SQRT csqrt
#define R_POW cpow_pos
#include "cp_oracle_body.h"
#undef REAL
#undef FN
#undef RE
#undef R_EXP
#undef R_LOG
#undef R_SQRT
#undef R_POW

/* ======================= public wrappers ======================= */
double cpo_sigma_gg2gg(double sH, double tH, double uH, double a) { return me_gg2gg_r(sH, tH, uH, a); }
double cpo_sigma_gg2qqbar(double sH, double tH, double uH, double a, int nq)
{
  return me_gg2qqbar_r(sH, tH, uH, a, nq);
}
double cpo_sigma_qg2qg(double sH, double tH, double uH, double a) { return me_qg2qg_r(sH, tH, uH, a); }
double cpo_sigma_qq2qq(double sH, double tH, double uH, double a, int i1, int i2)
{
  return me_qq2qq_r(sH, tH, uH, a, i1, i2);
}
double cpo_sigma_qqbar2gg(double sH, double tH, double uH, double a)
{
  return me_qqbar2gg_r(sH, tH, uH, a);
}
/* cuPythia/pipeline/physics.cuh:9-16 (reciprocal-precompute form of the same bracket) */
double cpo_gg2gg_recip(double sH, double tH, double uH, double aS)
{
  double is = 1.0 / sH, it = 1.0 / tH, iu = 1.0 / uH;
  double rts = tH * is, rst = sH * it, rus = uH * is, rsu = sH * iu, rtu = tH * iu, rut = uH * it;
  double a = (9. / 4.) * (rts * rts + 2. * rts + 3. + 2. * rst + rst * rst);
  double b = (9. / 4.) * (rus * rus + 2. * rus + 3. + 2. * rsu + rsu * rsu);
  double c = (9. / 4.) * (rtu * rtu + 2. * rtu + 3. + 2. * rut + rut * rut);
  return (M_PI * is * is) * (aS * aS) * 0.5 * (a + b + c);
}

void cpo_cteq5l_raw(double x, double Q2, double out[8]) { cteq5l_r(x, Q2, out); }
double cpo_pdf_xf(int id, double x, double Q2)
{
  double raw[8];
  cteq5l_r(x, Q2, raw);
  return xf_of_r(raw, id);
}

void cpo_alphas_init(cpo_alphas* a, double aSmZ)
{
  const double MZ = 91.188, mc = 1.5, mb = 4.8, mt = 171.0;
  double L5 = MZ * exp(-6. * M_PI / (23. * aSmZ));
  double L6 = L5 * pow(L5 / mt, 2. / 21.);
  double L4 = L5 * pow(mb / L5, 2. / 25.);
  double L3 = L4 * pow(mc / L4, 2. / 27.);
  a->aSmZ = aSmZ;
  a->L3_2 = L3 * L3; a->L4_2 = L4 * L4; a->L5_2 = L5 * L5; a->L6_2 = L6 * L6;
  a->mc2 = mc * mc; a->mb2 = mb * mb; a->mt2 = mt * mt;
  a->scale2Min = (1.07 * L3) * (1.07 * L3);
  a->nfmax = 6;
}
double cpo_alphas_eval(const cpo_alphas* a, double Q2) { return alphas_r(a->aSmZ, Q2); }

void cpo_had_default(cpo_had_cfg* c)
{
  c->sqrtS = 13000.0;
  c->pTmin = 20.0;
  c->aSmZ = 0.13;
  c->kR = 1.0;
  c->kF = 1.0;
  c->convert2mb = 0.389380; /* SigmaProcess::CONVERT2MB, SigmaProcess.cc:24 */
  c->nQuarkIn = 5;          /* PDFinProcess:nQuarkIn default */
  c->nQuarkNew = 3;         /* HardQCD:nQuarkNew default     */
  c->procMask = CPO_ALLQCD;
}

void cpo_had_sigma_pdf(const cpo_had_cfg* c, double x1, double x2, double sH, double tH,
                       int procMask, double out[6])
{
  sigma_pdf_r(c, c->aSmZ, c->kR, c->kF, x1, x2, sH, tH, procMask, out);
}

double cpo_had_density(const cpo_had_cfg* c, double tau, double y, double z)
{
  const double s = c->sqrtS * c->sqrtS;
  double tauMin = 4.0 * c->pTmin * c->pTmin / s;
  if (tauMin < 16.0 / s) tauMin = 16.0 / s;
  if (tau < tauMin || tau > 1.0) return 0.0;
  double yMax = -0.5 * log(tau);
  if (fabs(y) > yMax) return 0.0;
  double sH = tau * s;
  double zA = 1.0 - c->pTmin * c->pTmin / (0.25 * sH);
  double zMax = zA > 0 ? sqrt(zA) : 0.0;
  if (fabs(z) > zMax) return 0.0;
  double tH = -0.5 * sH * (1.0 - z);
  double x1 = sqrt(tau) * exp(y), x2 = sqrt(tau) * exp(-y);
  double sig = sigma_pdf_r(c, c->aSmZ, c->kR, c->kF, x1, x2, sH, tH, c->procMask, NULL);
  return sig * 0.5 * sH / tau;
}

double cpo_had_weight_x(const cpo_had_cfg* c, const double x[3], double tyz[3])
{
  return weight_x_r(c, c->aSmZ, c->kR, c->pTmin, x, tyz);
}

/* ---------------------------------------------------------------------------------------
 * Record picks of one accepted point at x (FP64), the rules of the device record builder:
 *  process      k in proportion to the sum of its pair terms at the point (r0; the device's own
 *               rule: Pythia instead picks a process container by its sigmaMax first),
 *  pair         SigmaProcess::pickInState (pythia8317/src/SigmaProcess.cc:486-508): the first
 *               pair of the initFlux list (:124-193) at which the running sum of pair terms
 *               reaches r1 x the process total (the last pair if rounding leaves none),
 *  new flavour  Sigma2gg2qqbar::sigmaKin (pythia8317/src/SigmaQCD.cc:173): 1 + int(nQuarkNew r3),
 *  colour       the process's setIdColAcol (SigmaQCD.cc: gg2gg :135-148, gg2qqbar :195-205,
 *               qg2qg :232-244, qq2qq :292-304, qqbar2gg :331-342): topology with rc in
 *               proportion to its kinematic term, gg -> gg orientation swapped when rs > 0.5.
 * Returns the process code (0 if the point has no weight); id[4] and the colour code in the
 * record's encoding (bits 0-1 topology, bit 2 swapColAcol, bit 3 swapCol1234).
 * ------------------------------------------------------------------------------------- */
/* Pair lists of every process at one phase-space point, in initFlux order (SigmaProcess.cc:124-193),
 * each pair term sigmaHat(id1, id2) * xfA * xfB (the common factors dropped). */
typedef struct {
  int pa[5][128], pb[5][128], np[5];
  double ps[5][128], tot[5];
  double sH, tH, uH;
} cpo_pairs;

static void pick_lists(const cpo_had_cfg* c, double x1, double x2, double sH, double tH, cpo_pairs* L)
{
  const double uH = -sH - tH;
  const double pT2 = tH * uH / sH;
  const double alpS = alphas_r(c->aSmZ, pT2 * c->kR);
  double A[8], B[8];
  cteq5l_r(x1, pT2 * c->kF, A);
  cteq5l_r(x2, pT2 * c->kF, B);
  const int nQ = c->nQuarkIn;
  int (*pa)[128] = L->pa, (*pb)[128] = L->pb;
  int* np = L->np;
  double (*ps)[128] = L->ps;
  double* tot = L->tot;
  for (int k = 0; k < 5; ++k) { np[k] = 0; tot[k] = 0.0; }
  L->sH = sH; L->tH = tH; L->uH = uH;
  const int bit[5] = {CPO_GG2GG, CPO_GG2QQBAR, CPO_QG2QG, CPO_QQ2QQ, CPO_QQBAR2GG};
#define CPO_ADD(k, a, b, me)                                                       \
  do {                                                                             \
    const double v_ = (me) * xf_of_r(A, a) * xf_of_r(B, b);                        \
    pa[k][np[k]] = a; pb[k][np[k]] = b; ps[k][np[k]] = v_; ++np[k]; tot[k] += v_;  \
  } while (0)
  if (c->procMask & bit[0]) CPO_ADD(0, 21, 21, me_gg2gg_r(sH, tH, uH, alpS));
  if (c->procMask & bit[1]) CPO_ADD(1, 21, 21, me_gg2qqbar_r(sH, tH, uH, alpS, c->nQuarkNew));
  if (c->procMask & bit[2]) {
    const double me = me_qg2qg_r(sH, tH, uH, alpS);
    for (int q = -nQ; q <= nQ; ++q)
      if (q) { CPO_ADD(2, q, 21, me); CPO_ADD(2, 21, q, me); }
  }
  if (c->procMask & bit[3])
    for (int q1 = -nQ; q1 <= nQ; ++q1)
      for (int q2 = -nQ; q2 <= nQ; ++q2)
        if (q1 && q2) CPO_ADD(3, q1, q2, me_qq2qq_r(sH, tH, uH, alpS, q1, q2));
  if (c->procMask & bit[4]) {
    const double me = me_qqbar2gg_r(sH, tH, uH, alpS);
    for (int q = -nQ; q <= nQ; ++q)
      if (q) CPO_ADD(4, q, -q, me);
  }
#undef CPO_ADD
}

/* pickInState of process k with r1 (the first pair whose running sum of pair terms reaches
 * r1 x the process total; the last pair if rounding leaves none), the new flavour of
 * Sigma2gg2qqbar::sigmaKin (SigmaQCD.cc:173) from r3, and setIdColAcol's colour flow from rc, rs. */
/* The smallest distance of a draw from a selection boundary of this pick, relative to the
 * quantity it selects from (the process or pair total, the topology sum, the flavour count):
 * a pick whose margin is above the FP32 rounding of those sums is decided the same way in FP32. */
static void margin_upd(double* m, double v)
{
  if (m && v < *m) *m = v;
}

static int pick_finish(const cpo_had_cfg* c, int k, const cpo_pairs* L, double r1, double r3, double rc,
                       double rs, int id[4], int* colour, double* margin)
{
  const int (*pa)[128] = (const int (*)[128])L->pa, (*pb)[128] = (const int (*)[128])L->pb;
  const int* np = L->np;
  const double (*ps)[128] = (const double (*)[128])L->ps;
  const double* tot = L->tot;
  const double sH = L->sH, tH = L->tH, uH = L->uH;
  if (np[k] == 0) return 0;
  double u = r1 * tot[k];
  int i = 0;
  for (; i < np[k] - 1; ++i) {
    u -= ps[k][i];
    if (u <= 0.0) break;
  }
  if (margin) {
    double cum = 0.0;
    for (int j = 0; j < np[k] - 1; ++j) {
      cum += ps[k][j];
      margin_upd(margin, fabs(r1 * tot[k] - cum) / tot[k]);
    }
  }
  const int a = pa[k][i], b = pb[k][i];
  id[0] = a; id[1] = b;
  if (k == 0 || k == 4) { id[2] = 21; id[3] = 21; }
  else if (k == 1) {
    int qn = 1 + (int)(c->nQuarkNew * r3);
    if (qn > c->nQuarkNew) qn = c->nQuarkNew;
    id[2] = qn; id[3] = -qn;
    const double v = c->nQuarkNew * r3;
    for (int j = 1; j < c->nQuarkNew; ++j) margin_upd(margin, fabs(v - j) / c->nQuarkNew);
  } else { id[2] = a; id[3] = b; }
  /* colour flow */
  const double sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  int topo = 0, swapCA = 0, swap12 = 0;
  if (k == 0) {
    const double sTS = (9. / 4.) * (tH2 / sH2 + 2. * tH / sH + 3. + 2. * sH / tH + sH2 / tH2);
    const double sUS = (9. / 4.) * (uH2 / sH2 + 2. * uH / sH + 3. + 2. * sH / uH + sH2 / uH2);
    const double sTU = (9. / 4.) * (tH2 / uH2 + 2. * tH / uH + 3. + 2. * uH / tH + uH2 / tH2);
    const double r = (sTS + sUS + sTU) * rc;
    topo = r < sTS ? 0 : (r < sTS + sUS ? 1 : 2);
    swapCA = rs > 0.5;
    margin_upd(margin, fabs(r - sTS) / (sTS + sUS + sTU));
    margin_upd(margin, fabs(r - sTS - sUS) / (sTS + sUS + sTU));
    margin_upd(margin, fabs(rs - 0.5));
  } else if (k == 1) {
    const double sTS = (1. / 6.) * uH / tH - (3. / 8.) * uH2 / sH2;
    const double sUS = (1. / 6.) * tH / uH - (3. / 8.) * tH2 / sH2;
    topo = (sTS + sUS) * rc < sTS ? 0 : 1;
    margin_upd(margin, fabs((sTS + sUS) * rc - sTS) / fabs(sTS + sUS));
  } else if (k == 2) {
    const double sTS = uH2 / tH2 - (4. / 9.) * uH / sH;
    const double sTU = sH2 / tH2 - (4. / 9.) * sH / uH;
    topo = (sTS + sTU) * rc < sTS ? 0 : 1;
    margin_upd(margin, fabs((sTS + sTU) * rc - sTS) / fabs(sTS + sTU));
    swap12 = id[0] == 21;
    swapCA = id[0] < 0 || id[1] < 0;
  } else if (k == 3) {
    const double sT = (4. / 9.) * (sH2 + uH2) / tH2, sU = (4. / 9.) * (sH2 + tH2) / uH2;
    topo = id[0] * id[1] > 0 ? 0 : 1;
    if (id[1] == id[0] && (sT + sU) * rc > sT) topo = 2;
    if (id[1] == id[0]) margin_upd(margin, fabs((sT + sU) * rc - sT) / (sT + sU));
    swapCA = id[0] < 0;
  } else {
    const double sTS = (32. / 27.) * uH / tH - (8. / 3.) * uH2 / sH2;
    const double sUS = (32. / 27.) * tH / uH - (8. / 3.) * tH2 / sH2;
    topo = (sTS + sUS) * rc < sTS ? 0 : 1;
    margin_upd(margin, fabs((sTS + sUS) * rc - sTS) / fabs(sTS + sUS));
    swapCA = id[0] < 0;
  }
  *colour = topo | (swapCA << 2) | (swap12 << 3);
  return 111 + k;
}

int cpo_pick_state_margin(const cpo_had_cfg* c, int code, double x1, double x2, double sH, double tH, double r1,
                          double r3, double rc, double rs, int id[4], int* colour, double* margin)
{
  if (margin) *margin = 1.0;
  if (code < 111 || code > 115) return 0;
  cpo_pairs L;
  pick_lists(c, x1, x2, sH, tH, &L);
  return pick_finish(c, code - 111, &L, r1, r3, rc, rs, id, colour, margin);
}

int cpo_pick_state(const cpo_had_cfg* c, int code, double x1, double x2, double sH, double tH, double r1,
                   double r3, double rc, double rs, int id[4], int* colour)
{
  return cpo_pick_state_margin(c, code, x1, x2, sH, tH, r1, r3, rc, rs, id, colour, NULL);
}

int cpo_pick_record_margin(const cpo_had_cfg* c, const double x[3], double r0, double r1, double r3, double rc,
                           double rs, int id[4], int* colour, double* margin)
{
  if (margin) *margin = 1.0;
  double tyz[3];
  if (!(weight_x_r(c, c->aSmZ, c->kR, c->pTmin, x, tyz) > 0.0)) return 0;
  const double s = c->sqrtS * c->sqrtS;
  const double tau = tyz[0], y = tyz[1], z = tyz[2];
  const double sH = tau * s, tH = -0.5 * sH * (1.0 - z);
  const double x1 = sqrt(tau) * exp(y), x2 = sqrt(tau) * exp(-y);
  cpo_pairs L;
  pick_lists(c, x1, x2, sH, tH, &L);
  const double* tot = L.tot;
  double all = 0.0;
  for (int k = 0; k < 5; ++k) all += tot[k];
  double t = r0 * all;
  int k = 0;
  while (k < 4 && (t >= tot[k] || tot[k] <= 0.0)) { t -= tot[k]; ++k; }
  if (tot[k] <= 0.0) { k = 0; while (k < 4 && !(tot[k] > 0.0)) ++k; }
  if (margin) {
    double cum = 0.0;
    for (int j = 0; j < 4; ++j) {
      cum += tot[j];
      margin_upd(margin, fabs(r0 * all - cum) / all);
    }
  }
  return pick_finish(c, k, &L, r1, r3, rc, rs, id, colour, margin);
}

int cpo_pick_record(const cpo_had_cfg* c, const double x[3], double r0, double r1, double r3, double rc,
                    double rs, int id[4], int* colour)
{
  return cpo_pick_record_margin(c, x, r0, r1, r3, rc, rs, id, colour, NULL);
}

double cpo_vegas_map(const double* edges, int nb, const uint32_t w[3], double x[3], int bins[3])
{
  double jac = 1.0;
  for (int d = 0; d < 3; ++d) {
    uint64_t m = (uint64_t)(w[d] >> 8) * (uint64_t)nb;
    int b = (int)(m >> 24);
    double frac = (double)(m & 0xFFFFFFu) * (1.0 / 16777216.0);
    const double* e = edges + d * (nb + 1);
    double lo = e[b], wd = e[b + 1] - e[b];
    x[d] = lo + frac * wd;
    jac *= (double)nb * wd;
    if (bins) bins[d] = b;
  }
  return jac;
}

double cpo_had_point_weight(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                            uint32_t iter, uint64_t point, int bins[3], double x[3])
{
  uint32_t w[4];
  double xx[3];
  int bb[3];
  cpo_point_words(seed, point, iter, 0, w);
  double jv = cpo_vegas_map(edges, nb, w, xx, bb);
  double f = weight_x_r(c, c->aSmZ, c->kR, c->pTmin, xx, NULL);
  if (bins) memcpy(bins, bb, sizeof bb);
  if (x) memcpy(x, xx, sizeof xx);
  return f * jv;
}

/* ---------------- threaded accumulation (disjoint point ranges, fixed-order combine) ---- */
typedef struct {
  const cpo_had_cfg* c;
  const double* edges;
  int nb;
  uint64_t seed;
  uint32_t iter, stream;
  uint64_t p0, n;
  double sums[2];
  double* hist;
  double* g; /* adjoint sums */
  int mode;  /* 0 accumulate, 1 adjoint */
} had_job;

static void had_accumulate_range(had_job* j)
{
  double s1 = 0, s2 = 0;
  for (uint64_t i = 0; i < j->n; ++i) {
    int b[3];
    double w = cpo_had_point_weight(j->c, j->edges, j->nb, j->seed, j->iter, j->p0 + i, b, NULL);
    s1 += w;
    s2 += w * w;
    if (j->hist)
      for (int d = 0; d < 3; ++d) j->hist[d * j->nb + b[d]] += w * w;
  }
  j->sums[0] = s1;
  j->sums[1] = s2;
}

static void had_adjoint_range(had_job* j);

static void* had_thread(void* arg)
{
  had_job* j = (had_job*)arg;
  if (j->mode == 0) had_accumulate_range(j);
  else had_adjoint_range(j);
  return NULL;
}

static int clamp_threads(int nthreads, uint64_t n)
{
  if (nthreads < 1) nthreads = 1;
  if (nthreads > 256) nthreads = 256;
  if ((uint64_t)nthreads > n && n > 0) nthreads = (int)n;
  return nthreads;
}

void cpo_had_accumulate(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                        uint32_t iter, uint64_t p0, uint64_t n, double sums[2], double* hist,
                        int nthreads)
{
  nthreads = clamp_threads(nthreads, n);
  had_job* jobs = (had_job*)calloc((size_t)nthreads, sizeof(had_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  uint64_t per = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads, off = p0;
  for (int t = 0; t < nthreads; ++t) {
    had_job* j = &jobs[t];
    j->c = c; j->edges = edges; j->nb = nb; j->seed = seed; j->iter = iter; j->stream = 0;
    j->p0 = off; j->n = per + ((uint64_t)t < rem ? 1 : 0); off += j->n;
    j->hist = hist ? (double*)calloc((size_t)(3 * nb), sizeof(double)) : NULL;
    j->mode = 0;
    if (nthreads > 1) pthread_create(&th[t], NULL, had_thread, j);
    else had_thread(j);
  }
  sums[0] = sums[1] = 0;
  for (int t = 0; t < nthreads; ++t) {
    if (nthreads > 1) pthread_join(th[t], NULL);
    sums[0] += jobs[t].sums[0];
    sums[1] += jobs[t].sums[1];
    if (hist) {
      for (int k = 0; k < 3 * nb; ++k) hist[k] += jobs[t].hist[k];
      free(jobs[t].hist);
    }
  }
  free(jobs);
  free(th);
}

/* ---------------- VEGAS refinement ---------------- */
void cpo_vegas_uniform(double* edges, int ndim, int nb)
{
  for (int d = 0; d < ndim; ++d)
    for (int k = 0; k <= nb; ++k) edges[d * (nb + 1) + k] = (double)k / (double)nb;
}

/* Lepage's refinement (G.P. Lepage, J. Comput. Phys. 27 (1978) 192): per dimension take the
 * per-bin second moments d_i, smooth them with the (1,1)/(1,1,1)/(1,1) neighbour average,
 * normalise, compress with r_i = ((d_i - 1)/ln d_i)^alpha, and place the new edges so that
 * every new bin holds an equal share of sum r_i, interpolating linearly inside old bins.
 * (The reference's 1-D rule, cuPythia/11_vegas_importance/vegas.cu:69-85, is the same
 * equal-share rebin on a different per-bin importance.) */
void cpo_vegas_refine(double* edges, const double* hist, int ndim, int nb, double alpha)
{
  double* d = (double*)malloc(sizeof(double) * (size_t)nb);
  double* r = (double*)malloc(sizeof(double) * (size_t)nb);
  double* ne = (double*)malloc(sizeof(double) * (size_t)(nb + 1));
  for (int dim = 0; dim < ndim; ++dim) {
    const double* h = hist + dim * nb;
    double* e = edges + dim * (nb + 1);
    double tot = 0.0;
    for (int i = 0; i < nb; ++i) {
      double s;
      if (i == 0) s = (h[0] + h[1]) / 2.0;
      else if (i == nb - 1) s = (h[nb - 2] + h[nb - 1]) / 2.0;
      else s = (h[i - 1] + h[i] + h[i + 1]) / 3.0;
      d[i] = s;
      tot += s;
    }
    if (!(tot > 0.0)) continue; /* no information: keep the grid */
    double rsum = 0.0;
    for (int i = 0; i < nb; ++i) {
      double di = d[i] / tot;
      double ri = 0.0;
      if (di >= 1.0) ri = 1.0;
      else if (di > 0.0) ri = pow((di - 1.0) / log(di), alpha);
      r[i] = ri;
      rsum += ri;
    }
    double step = rsum / (double)nb;
    ne[0] = e[0];
    ne[nb] = e[nb];
    double acc = 0.0;
    int j = 0;
    for (int k = 1; k < nb; ++k) {
      double need = step * (double)k;
      while (j < nb - 1 && acc + r[j] < need) { acc += r[j]; ++j; }
      double frac = r[j] > 0.0 ? (need - acc) / r[j] : 0.0;
      if (frac < 0.0) frac = 0.0;
      if (frac > 1.0) frac = 1.0;
      ne[k] = e[j] + frac * (e[j + 1] - e[j]);
    }
    memcpy(e, ne, sizeof(double) * (size_t)(nb + 1));
  }
  free(d); free(r); free(ne);
}

/* ======================= partonic gg -> gg ======================= */
/* one point: cuPythia/03_fused_resident_me/fused_gg2gg.cu:45-48 and :60-61 */
double cpo_partonic_weight(double sqrtShat, double alpS, double cMax, double conv, double u)
{
  double s = sqrtShat * sqrtShat;
  double c = (2.0 * u - 1.0) * cMax;
  double t = -0.5 * s * (1.0 - c);
  return cpo_gg2gg_recip(s, t, -s - t, alpS) * (2.0 * cMax) * (s / 2.0) * conv;
}

typedef struct {
  double sq, aS, cMax, conv;
  uint64_t seed, p0, n, kPer;
  int mode; /* 0 philox, 1 splitmix threads [p0, p0+n) */
  double sums[2];
} part_job;

static void* part_thread(void* arg)
{
  part_job* j = (part_job*)arg;
  double s1 = 0, s2 = 0;
  if (j->mode == 0) {
    for (uint64_t i = 0; i < j->n; ++i) {
      uint32_t w[4];
      cpo_point_words(j->seed, j->p0 + i, 0, 0, w);
      double v = cpo_partonic_weight(j->sq, j->aS, j->cMax, j->conv, cpo_u53(w[0], w[1]));
      s1 += v; s2 += v * v;
    }
  } else {
    for (uint64_t t = j->p0; t < j->p0 + j->n; ++t) {
      uint64_t ctr = cpo_thread_counter(j->seed, t);
      for (uint64_t i = 0; i < j->kPer; ++i) {
        double v = cpo_partonic_weight(j->sq, j->aS, j->cMax, j->conv, cpo_u01(cpo_splitmix64(ctr++)));
        s1 += v; s2 += v * v;
      }
    }
  }
  j->sums[0] = s1; j->sums[1] = s2;
  return NULL;
}

static void partonic_run(part_job proto, uint64_t p0, uint64_t n, double sums[2], int nthreads)
{
  nthreads = clamp_threads(nthreads, n);
  part_job* jobs = (part_job*)calloc((size_t)nthreads, sizeof(part_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  uint64_t per = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads, off = p0;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t] = proto;
    jobs[t].p0 = off; jobs[t].n = per + ((uint64_t)t < rem ? 1 : 0); off += jobs[t].n;
    if (nthreads > 1) pthread_create(&th[t], NULL, part_thread, &jobs[t]);
    else part_thread(&jobs[t]);
  }
  sums[0] = sums[1] = 0;
  for (int t = 0; t < nthreads; ++t) {
    if (nthreads > 1) pthread_join(th[t], NULL);
    sums[0] += jobs[t].sums[0];
    sums[1] += jobs[t].sums[1];
  }
  free(jobs);
  free(th);
}

void cpo_partonic_philox(double sqrtShat, double alpS, double cMax, double conv, uint64_t seed,
                         uint64_t p0, uint64_t n, double sums[2], int nthreads)
{
  part_job p = {sqrtShat, alpS, cMax, conv, seed, 0, 0, 0, 0, {0, 0}};
  partonic_run(p, p0, n, sums, nthreads);
}

void cpo_partonic_splitmix(double sqrtShat, double alpS, double cMax, double conv, uint64_t seed,
                           uint64_t nThreads, uint64_t kPer, double sums[2], int nthreads)
{
  part_job p = {sqrtShat, alpS, cMax, conv, seed, 0, 0, kPer, 1, {0, 0}};
  partonic_run(p, 0, nThreads, sums, nthreads);
}

/* Simpson quadrature, cuPythia/03_fused_resident_me/fused_gg2gg.cu:65-74, times conv */
double cpo_simpson_gg2gg(int N, double sqrtShat, double alpS, double cMax, double conv)
{
  double s = sqrtShat * sqrtShat;
  double a = -cMax, b = cMax, h = (b - a) / N, sum = 0.0;
  for (int i = 0; i <= N; ++i) {
    double c = a + i * h, t = -0.5 * s * (1.0 - c);
    double f = cpo_gg2gg_recip(s, t, -s - t, alpS);
    double w = (i == 0 || i == N) ? 1.0 : (i % 2 ? 4.0 : 2.0);
    sum += w * f;
  }
  return (sum * h / 3.0) * (s / 2.0) * conv;
}

/* ======================= derivatives by complex step ======================= */
#define CS_H 1e-30

void cpo_had_weight_grad(const cpo_had_cfg* c, const double x[3], double out[7])
{
  double complex xc[3] = {x[0], x[1], x[2]};
  out[0] = weight_x_r(c, c->aSmZ, c->kR, c->pTmin, x, NULL);
  for (int d = 0; d < 3; ++d) {
    double complex xp[3] = {xc[0], xc[1], xc[2]};
    xp[d] += I * CS_H;
    out[1 + d] = cimag(weight_x_c(c, c->aSmZ, c->kR, c->pTmin, xp, NULL)) / CS_H;
  }
  out[4] = cimag(weight_x_c(c, c->aSmZ + I * CS_H, c->kR, c->pTmin, xc, NULL)) / CS_H;
  out[5] = cimag(weight_x_c(c, c->aSmZ, c->kR + I * CS_H, c->pTmin, xc, NULL)) / CS_H;
  out[6] = cimag(weight_x_c(c, c->aSmZ, c->kR, c->pTmin + I * CS_H, xc, NULL)) / CS_H;
}

static void had_adjoint_range(had_job* j)
{
  const int nb = j->nb, E = 3 * (nb + 1);
  double* g = j->g;
  for (uint64_t i = 0; i < j->n; ++i) {
    uint32_t wd[4];
    double x[3];
    int b[3];
    cpo_point_words(j->seed, j->p0 + i, j->iter, j->stream, wd);
    double jv = cpo_vegas_map(j->edges, nb, wd, x, b);
    double gr[7];
    cpo_had_weight_grad(j->c, x, gr);
    double w = gr[0] * jv;
    g[0] += w;
    g[1] += w * w;
    for (int k = 0; k < 3; ++k) {
      double dw = gr[4 + k] * jv;
      g[2 + k] += dw;
      g[5 + k] += w * dw;
    }
    for (int d = 0; d < 3; ++d) {
      uint64_t m = (uint64_t)(wd[d] >> 8) * (uint64_t)nb;
      double frac = (double)(m & 0xFFFFFFu) * (1.0 / 16777216.0);
      const double* e = j->edges + d * (nb + 1);
      double wdth = e[b[d] + 1] - e[b[d]];
      double dxw = gr[1 + d] * jv; /* dw/dx_d at fixed Jacobian */
      double dlo = -w / wdth + dxw * (1.0 - frac);
      double dhi = w / wdth + dxw * frac;
      int klo = d * (nb + 1) + b[d], khi = klo + 1;
      g[8 + klo] += dlo;
      g[8 + khi] += dhi;
      g[8 + E + klo] += w * dlo;
      g[8 + E + khi] += w * dhi;
    }
  }
}

void cpo_had_adjoint_sums(const cpo_had_cfg* c, const double* edges, int nb, uint64_t seed,
                          uint32_t iter, uint32_t stream, uint64_t p0, uint64_t n, double* g,
                          int nthreads)
{
  const int G = 8 + 2 * 3 * (nb + 1);
  nthreads = clamp_threads(nthreads, n);
  had_job* jobs = (had_job*)calloc((size_t)nthreads, sizeof(had_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  uint64_t per = n / (uint64_t)nthreads, rem = n % (uint64_t)nthreads, off = p0;
  for (int t = 0; t < nthreads; ++t) {
    had_job* j = &jobs[t];
    j->c = c; j->edges = edges; j->nb = nb; j->seed = seed; j->iter = iter; j->stream = stream;
    j->p0 = off; j->n = per + ((uint64_t)t < rem ? 1 : 0); off += j->n;
    j->g = (double*)calloc((size_t)G, sizeof(double));
    j->mode = 1;
    if (nthreads > 1) pthread_create(&th[t], NULL, had_thread, j);
    else had_thread(j);
  }
  memset(g, 0, sizeof(double) * (size_t)G);
  for (int t = 0; t < nthreads; ++t) {
    if (nthreads > 1) pthread_join(th[t], NULL);
    for (int k = 0; k < G; ++k) g[k] += jobs[t].g[k];
    free(jobs[t].g);
  }
  free(jobs);
  free(th);
}

/* ======================= unweighting ======================= */
/* von Neumann accept, cuPythia/07_unweighting_lhe/unweight_lhe.cu:54: accept if u wMax < w */
int cpo_accept(double w, double wmax, uint32_t w3) { return cpo_u24(w3) * wmax < w; }

/* ======================= batch helpers for the parity tests ======================= */
typedef struct {
  const cpo_had_cfg* c;
  const float* x;
  double* out;
  int64_t i0, i1;
} wx_job;

static void* wx_thread(void* arg)
{
  wx_job* j = (wx_job*)arg;
  for (int64_t i = j->i0; i < j->i1; ++i) {
    double x[3] = {j->x[3 * i], j->x[3 * i + 1], j->x[3 * i + 2]};
    j->out[i] = cpo_had_weight_x(j->c, x, NULL);
  }
  return NULL;
}

void cpo_had_weight_x_batch(const cpo_had_cfg* c, const float* x, int64_t n, double* out, int nthreads)
{
  nthreads = clamp_threads(nthreads, (uint64_t)n);
  wx_job* jobs = (wx_job*)calloc((size_t)nthreads, sizeof(wx_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  int64_t per = n / nthreads, rem = n % nthreads, off = 0;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].c = c; jobs[t].x = x; jobs[t].out = out;
    jobs[t].i0 = off; off += per + (t < rem ? 1 : 0); jobs[t].i1 = off;
    if (nthreads > 1) pthread_create(&th[t], NULL, wx_thread, &jobs[t]);
    else wx_thread(&jobs[t]);
  }
  if (nthreads > 1)
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(jobs);
  free(th);
}

/* ======================= the learned proposal (flow), FP64 ======================= */
/* Same architecture and parameter layout as the CUDA flow: 4 affine couplings on logit space,
 * MLP in -> 64 -> 64 -> out (ReLU), s = 4 tanh(s_raw / 4).  The forward reproduces the kernels'
 * BF16 rounding points (weights, MLP inputs, post-ReLU activations); arithmetic is FP64.
 * The backward is plain reverse-mode differentiation of that forward (rounding treated as the
 * identity), the reference for the GPU's tensor-core training gradients. */
#define FL_NC 4
#define FL_PER 5768
#define FL_W1 0
#define FL_B1 1024
#define FL_W2 1088
#define FL_B2 5184
#define FL_W3 5248
#define FL_B3 5760
#define FL_S 4.0

static int fl_round = 1;
void cpo_flow_set_rounding(int on) { fl_round = on; }

static double bf16r(double x)
{
  if (!fl_round) return x;
  float f = (float)x;
  uint32_t b;
  memcpy(&b, &f, 4);
  b = (b + 0x7FFFu + ((b >> 16) & 1u)) & 0xFFFF0000u;
  memcpy(&f, &b, 4);
  return (double)f;
}

static void fl_coupling(int c, int* nin, int cin[2], int* nt, int tr[2])
{
  static const int NIN[4] = {1, 2, 1, 2}, NT[4] = {2, 1, 2, 1};
  static const int CIN[4][2] = {{0, 0}, {1, 2}, {1, 1}, {0, 2}}, TR[4][2] = {{1, 2}, {0, 0}, {0, 2}, {1, 1}};
  *nin = NIN[c]; *nt = NT[c];
  cin[0] = CIN[c][0]; cin[1] = CIN[c][1]; tr[0] = TR[c][0]; tr[1] = TR[c][1];
}

typedef struct {
  double x[2], h1[64], h2[64], o[4], zin[3];
} fl_tape;

static void fl_mlp(const float* P, int c, int nin, const double in[2], fl_tape* t)
{
  const float* W1 = P + c * FL_PER + FL_W1;
  const float* W2 = P + c * FL_PER + FL_W2;
  const float* W3 = P + c * FL_PER + FL_W3;
  const float* B = P + c * FL_PER;
  for (int k = 0; k < 2; ++k) t->x[k] = k < nin ? bf16r(in[k]) : 0.0;
  for (int j = 0; j < 64; ++j) {
    double a = B[FL_B1 + j];
    for (int k = 0; k < nin; ++k) a += t->x[k] * bf16r(W1[k * 64 + j]);
    t->h1[j] = bf16r(a > 0 ? a : 0.0);
  }
  for (int j = 0; j < 64; ++j) {
    double a = B[FL_B2 + j];
    for (int k = 0; k < 64; ++k) a += t->h1[k] * bf16r(W2[k * 64 + j]);
    t->h2[j] = bf16r(a > 0 ? a : 0.0);
  }
  for (int j = 0; j < 4; ++j) {
    double a = B[FL_B3 + j];
    for (int k = 0; k < 64; ++k) a += t->h2[k] * bf16r(W3[k * 8 + j]);
    t->o[j] = a;
  }
}

void cpo_flow_forward(const float* P, const double u[3], double v[3], double* logJ)
{
  double z[3], ld = 0.0;
  for (int d = 0; d < 3; ++d) {
    z[d] = log(u[d]) - log1p(-u[d]);
    ld -= log(u[d]) + log1p(-u[d]);
  }
  for (int c = 0; c < FL_NC; ++c) {
    int nin, nt, cin[2], tr[2];
    fl_coupling(c, &nin, cin, &nt, tr);
    fl_tape t;
    double in[2] = {z[cin[0]], z[cin[1]]};
    fl_mlp(P, c, nin, in, &t);
    for (int j = 0; j < nt; ++j) {
      double s = FL_S * tanh(t.o[j] / FL_S);
      z[tr[j]] = z[tr[j]] * exp(s) + t.o[nt + j];
      ld += s;
    }
  }
  for (int d = 0; d < 3; ++d) {
    v[d] = 1.0 / (1.0 + exp(-z[d]));
    ld += log(v[d]) + log1p(-v[d]);
  }
  *logJ = ld;
}

/* gradient of sum_p (cv_p . v_p + cJ_p lnJ_p) with respect to the parameters, accumulated */
static void fl_backward_point(const float* P, const double u[3], const double cv[3], double cJ, double* G)
{
  double z[3];
  fl_tape tape[FL_NC];
  for (int d = 0; d < 3; ++d) z[d] = log(u[d]) - log1p(-u[d]);
  for (int c = 0; c < FL_NC; ++c) {
    int nin, nt, cin[2], tr[2];
    fl_coupling(c, &nin, cin, &nt, tr);
    for (int d = 0; d < 3; ++d) tape[c].zin[d] = z[d];
    double in[2] = {z[cin[0]], z[cin[1]]};
    fl_mlp(P, c, nin, in, &tape[c]);
    for (int j = 0; j < nt; ++j) {
      double s = FL_S * tanh(tape[c].o[j] / FL_S);
      z[tr[j]] = z[tr[j]] * exp(s) + tape[c].o[nt + j];
    }
  }
  double dz[3];
  for (int d = 0; d < 3; ++d) {
    double v = 1.0 / (1.0 + exp(-z[d]));
    dz[d] = cv[d] * v * (1.0 - v) + cJ * (1.0 - 2.0 * v);
  }
  for (int c = FL_NC - 1; c >= 0; --c) {
    int nin, nt, cin[2], tr[2];
    fl_coupling(c, &nin, cin, &nt, tr);
    const fl_tape* t = &tape[c];
    const float* W1 = P + c * FL_PER + FL_W1;
    const float* W2 = P + c * FL_PER + FL_W2;
    const float* W3 = P + c * FL_PER + FL_W3;
    double* g = G + c * FL_PER;
    double dO[4] = {0, 0, 0, 0}, dzT[2] = {0, 0};
    for (int j = 0; j < nt; ++j) {
      double th = tanh(t->o[j] / FL_S), s = FL_S * th, e = exp(s);
      int d = tr[j];
      double ds = dz[d] * t->zin[d] * e + cJ;
      dO[j] = ds * (1.0 - th * th);
      dO[nt + j] = dz[d];
      dzT[j] = dz[d] * e;
    }
    double dh2[64], dh1[64], dx[2] = {0, 0};
    for (int j = 0; j < 4; ++j) {
      g[FL_B3 + j] += dO[j];
      for (int k = 0; k < 64; ++k) g[FL_W3 + k * 8 + j] += t->h2[k] * dO[j];
    }
    for (int k = 0; k < 64; ++k) {
      double a = 0.0;
      for (int j = 0; j < 4; ++j) a += dO[j] * bf16r(W3[k * 8 + j]);
      dh2[k] = t->h2[k] > 0 ? a : 0.0;
    }
    for (int j = 0; j < 64; ++j) {
      g[FL_B2 + j] += dh2[j];
      for (int k = 0; k < 64; ++k) g[FL_W2 + k * 64 + j] += t->h1[k] * dh2[j];
    }
    for (int k = 0; k < 64; ++k) {
      double a = 0.0;
      for (int j = 0; j < 64; ++j) a += dh2[j] * bf16r(W2[k * 64 + j]);
      dh1[k] = t->h1[k] > 0 ? a : 0.0;
    }
    for (int j = 0; j < 64; ++j) {
      g[FL_B1 + j] += dh1[j];
      for (int k = 0; k < nin; ++k) g[FL_W1 + k * 64 + j] += t->x[k] * dh1[j];
    }
    for (int k = 0; k < nin; ++k)
      for (int j = 0; j < 64; ++j) dx[k] += dh1[j] * bf16r(W1[k * 64 + j]);
    for (int j = 0; j < nt; ++j) dz[tr[j]] = dzT[j];
    dz[cin[0]] += dx[0];
    if (nin > 1) dz[cin[1]] += dx[1];
  }
}

typedef struct {
  const float* P;
  const double *u, *cv, *cJ;
  int64_t i0, i1;
  double* G;
} fl_job;

static void* fl_thread(void* a)
{
  fl_job* j = (fl_job*)a;
  for (int64_t i = j->i0; i < j->i1; ++i) fl_backward_point(j->P, j->u + 3 * i, j->cv + 3 * i, j->cJ[i], j->G);
  return NULL;
}

/* G[FL_NC*FL_PER] = sum over points of the parameter gradient of cv . v + cJ lnJ */
void cpo_flow_backward_batch(const float* P, int64_t n, const double* u, const double* cv, const double* cJ,
                             double* G, int nthreads)
{
  const int NP = FL_NC * FL_PER;
  nthreads = clamp_threads(nthreads, (uint64_t)n);
  fl_job* jobs = (fl_job*)calloc((size_t)nthreads, sizeof(fl_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  int64_t per = n / nthreads, rem = n % nthreads, off = 0;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].P = P; jobs[t].u = u; jobs[t].cv = cv; jobs[t].cJ = cJ;
    jobs[t].i0 = off; off += per + (t < rem ? 1 : 0); jobs[t].i1 = off;
    jobs[t].G = (double*)calloc((size_t)NP, sizeof(double));
    pthread_create(&th[t], NULL, fl_thread, &jobs[t]);
  }
  memset(G, 0, sizeof(double) * (size_t)NP);
  for (int t = 0; t < nthreads; ++t) {
    pthread_join(th[t], NULL);
    for (int k = 0; k < NP; ++k) G[k] += jobs[t].G[k];
    free(jobs[t].G);
  }
  free(jobs);
  free(th);
}
