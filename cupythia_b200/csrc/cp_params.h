// cp_params.h -- host-side construction of the FP32 uniform parameters of the integrand.
// Everything here runs once per configuration in FP64 and is then rounded to FP32.
#pragma once
#include <math.h>
#include "cp_integrand.cuh"

// CTEQ5L parametrisation data (pythia8317/src/PartonDistributions.cc:936-1023).  The numbers
// are the published CTEQ5L fit (Lai et al., Eur.Phys.J. C12 (2000) 375), kept in the same
// [parametrisation][coefficient][power of sb1] order as the reference so a reader can compare.
namespace cp_cteq5l {
static const double QMIN[8] = {0., 0., 0., 0., 0., 0., 1.3, 4.5};
static const double ALPHA[8] = {0.2987216, 0.3407552, 0.4491863, 0.2457668,
                                0.5293999, 0.3713141, 0.03712017, 0.004952010};
static const double UT1[8] = {4.971265, 2.612618, -0.4656819, 3.862583,
                              0.1895615, 3.753257, 4.400772, 5.562568};
static const double UT2[8] = {-1.105128, -1.258304e5, -274.2390, -1.265969,
                              -3.069097, -1.113085, -1.356116, -1.801317};
static const double AM[8][9][3] = {
  {{0.5292616E+01, -0.2751910E+01, -0.2488990E+01}, {0.9714424E+00, 0.1011827E-01, -0.1023660E-01},
   {-0.1651006E+02, 0.7959721E+01, 0.8810563E+01}, {-0.1643394E+02, 0.5892854E+01, 0.9348874E+01},
   {0.3067422E+02, 0.4235796E+01, -0.5112136E+00}, {0.2352526E+02, -0.5305168E+01, -0.1169174E+02},
   {-0.1095451E+02, 0.3006577E+01, 0.5638136E+01}, {-0.1172251E+02, -0.2183624E+01, 0.4955794E+01},
   {0.1662533E-01, 0.7622870E-02, -0.4895887E-03}},
  {{0.9905300E+00, -0.4502235E+00, 0.1624441E+00}, {0.8867534E+00, 0.1630829E-01, -0.4049085E-01},
   {0.8547974E+00, 0.3336301E+00, 0.1371388E+00}, {0.2941113E+00, -0.1527905E+01, 0.2331879E+00},
   {0.3384235E+02, 0.3715315E+01, 0.8276930E+00}, {0.6230115E+01, 0.3134639E+01, -0.1729099E+01},
   {-0.1186928E+01, -0.3282460E+00, 0.1052020E+00}, {-0.8545702E+01, -0.6247947E+01, 0.3692561E+01},
   {0.1724598E-01, 0.7120465E-02, 0.4003646E-04}},
  {{0.1193572E+03, -0.3886845E+01, -0.1133965E+01}, {-0.9421449E+02, 0.3995885E+01, 0.1607363E+01},
   {0.4206383E+01, 0.2485954E+00, 0.2497468E+00}, {0.1210557E+03, -0.3015765E+01, -0.1423651E+01},
   {-0.1013897E+03, -0.7113478E+00, 0.2621865E+00}, {-0.1312404E+01, -0.9297691E+00, -0.1562531E+00},
   {0.1627137E+01, 0.4954111E+00, -0.6387009E+00}, {0.1537698E+00, -0.2487878E+00, 0.8305947E+00},
   {0.2496448E-01, 0.2457823E-02, 0.8234276E-03}},
  {{0.2647441E+02, 0.1059277E+02, -0.9176654E+00}, {0.1990636E+01, 0.8558918E-01, 0.4248667E-01},
   {-0.1476095E+02, -0.3276255E+02, 0.1558110E+01}, {-0.2966889E+01, -0.3649037E+02, 0.1195914E+01},
   {-0.1000519E+03, -0.2464635E+01, 0.1964849E+00}, {0.3718331E+02, 0.4700389E+02, -0.2772142E+01},
   {-0.1872722E+02, -0.2291189E+02, 0.1089052E+01}, {-0.1628146E+02, -0.1823993E+02, 0.2537369E+01},
   {-0.1156300E+01, -0.1280495E+00, 0.5153245E-01}},
  {{-0.6556775E+00, 0.2490190E+00, 0.3966485E-01}, {0.1305102E+01, -0.1188925E+00, -0.4600870E-02},
   {-0.2371436E+01, 0.3566814E+00, -0.2834683E+00}, {-0.6152826E+01, 0.8339877E+00, -0.7233230E+00},
   {-0.8346558E+01, 0.2892168E+01, 0.2137099E+00}, {0.1279530E+02, 0.1021114E+00, 0.5787439E+00},
   {0.5858816E+00, -0.1940375E+01, -0.4029269E+00}, {-0.2795725E+02, -0.5263392E+00, 0.1290229E+01},
   {0.0, 0.0, 0.0}},
  {{0.1580931E+01, -0.2273826E+01, -0.1822245E+01}, {0.2702644E+01, 0.6763243E+00, 0.7231586E-02},
   {-0.1857924E+02, 0.3907500E+01, 0.5850109E+01}, {-0.3044793E+02, 0.2639332E+01, 0.5566644E+01},
   {-0.4258011E+01, -0.5429244E+01, 0.4418946E+00}, {0.3465259E+02, -0.5532604E+01, -0.4904153E+01},
   {-0.1658858E+02, 0.2923275E+01, 0.2266286E+01}, {-0.1149263E+02, 0.2877475E+01, -0.7999105E+00},
   {0.0, 0.0, 0.0}},
  {{-0.8293661E+00, -0.3982375E+01, -0.6494283E-01}, {0.2754618E+01, 0.8338636E+00, -0.6885160E-01},
   {-0.1657987E+02, 0.1439143E+02, -0.6887240E+00}, {-0.2800703E+02, 0.1535966E+02, -0.7377693E+00},
   {-0.6460216E+01, -0.4783019E+01, 0.4913297E+00}, {0.3141830E+02, -0.3178031E+02, 0.7136013E+01},
   {-0.1802509E+02, 0.1862163E+02, -0.4632843E+01}, {-0.1240412E+02, 0.2565386E+02, -0.1066570E+02},
   {0.0, 0.0, 0.0}},
  {{-0.6031237E+01, 0.1992727E+01, -0.1076331E+01}, {0.2933912E+01, 0.5839674E+00, 0.7509435E-01},
   {-0.8284919E+01, 0.1488593E+01, -0.8251678E+00}, {-0.1925986E+02, 0.2805753E+01, -0.3015446E+01},
   {-0.9480483E+01, -0.9767837E+00, -0.1165544E+01}, {0.2193195E+02, -0.1788518E+02, 0.9460908E+01},
   {-0.1327377E+02, 0.1201754E+02, -0.6277844E+01}, {0.0, 0.0, 0.0},
   {0.0, 0.0, 0.0}}};
}  // namespace cp_cteq5l

// Physics configuration of the hadronic integrand, FP64.
struct CpHadConfig {
  double sqrtS, pTmin, aSmZ, kR, kF, convert2mb;
  int nQuarkIn, nQuarkNew, procMask;
};

// First-order Lambda values, StandardModel.cc:61-64 (MZ = 91.188, mc 1.5, mb 4.8, mt 171).
static inline void cp_lambdas(double aSmZ, double L[4])
{
  const double MZ = 91.188, mc = 1.5, mb = 4.8, mt = 171.0;
  double L5 = MZ * exp(-6. * M_PI / (23. * aSmZ));
  double L6 = L5 * pow(L5 / mt, 2. / 21.);
  double L4 = L5 * pow(mb / L5, 2. / 25.);
  double L3 = L4 * pow(mc / L4, 2. / 27.);
  L[0] = L3; L[1] = L4; L[2] = L5; L[3] = L6;
}

// Returns 0 on success, nonzero if the configuration is outside what the kernels support.
static inline int cp_build_had_params(const CpHadConfig& c, CpHadParams& P)
{
  using namespace cp_cteq5l;
  if (!(c.sqrtS > 0) || !(c.pTmin >= 2.0) || !(2.0 * c.pTmin < c.sqrtS) || !(c.aSmZ > 0.05) ||
      !(c.aSmZ < 0.3) || !(c.kR > 0) || !(c.kF > 0) || c.nQuarkIn != 5)
    return 1;
  for (int i = 0; i < 8; ++i) {
    CpCteqPoly& q = P.cteq[i];
    for (int k = 0; k < 3; ++k) {
      float* co = q.co[k];
      co[CP_CQ_A] = (float)(AM[i][0][k] + AM[i][1][k]);
      co[CP_CQ_B] = (float)(AM[i][3][k] - AM[i][0][k]);
      co[CP_CQ_AF1] = (float)AM[i][1][k];
      co[CP_CQ_AF2] = (float)AM[i][2][k];
      co[CP_CQ_P] = (float)((k == 0 ? 1.0 : 0.0) + 0.01 * AM[i][4][k]);
      co[CP_CQ_AF5] = (float)AM[i][5][k];
      co[CP_CQ_AF6] = (float)AM[i][6][k];
      co[CP_CQ_AF7] = (float)AM[i][7][k];
      co[CP_CQ_AF8] = (float)AM[i][8][k];
      co[CP_CQ_N] = 0.f;
    }
    q.lnAlpha = (float)log(ALPHA[i]);
    q.qlim = (float)(QMIN[i] > ALPHA[i] ? QMIN[i] : ALPHA[i]);
    q.qmin = (float)QMIN[i];
    q.ut1 = (float)UT1[i];
    q.eut2 = (float)exp(UT2[i]);
    q.useX1L = UT2[i] < -100.0 ? 1 : 0;
    // the kernels resolve these two cases per parametrisation at compile time
    if (q.useX1L != (cp_cteq_uses_x1l(i) ? 1 : 0) || (QMIN[i] > 0.0) != cp_cteq_has_qmin(i) ||
        (!cp_cteq_has_qmin(i) && !(ALPHA[i] < 1.0)))
      return 1;
  }
  double s = c.sqrtS * c.sqrtS;
  double tauMin = 4.0 * c.pTmin * c.pTmin / s;
  double lnTauMin = log(tauMin);
  if (!(lnTauMin > -80.0)) return 1;   // the range of the kernels' exp reduction (cp_exp_reduce2)
  P.lnTauMin = (float)lnTauMin;
  P.lnTauMinLo = (float)(lnTauMin - (double)P.lnTauMin);
  P.K0 = (float)(2.0 * M_PI * c.convert2mb * (-lnTauMin) / s);
  P.s = (float)s;
  P.conv = (float)c.convert2mb;
  P.kR = (float)c.kR;
  P.kF = (float)c.kF;
  double L[4];
  cp_lambdas(c.aSmZ, L);
  for (int k = 0; k < 4; ++k) P.lnL2[k] = (float)(2.0 * log(L[k]));
  P.thr2[0] = (float)(1.5 * 1.5);
  P.thr2[1] = (float)(4.8 * 4.8);
  P.thr2[2] = (float)(171.0 * 171.0);
  P.scale2Min = (float)((1.07 * L[0]) * (1.07 * L[0]));
  P.nQuarkNew = (float)c.nQuarkNew;
  for (int k = 0; k < 5; ++k) P.mask[k] = (c.procMask >> k) & 1 ? 1.f : 0.f;
  P.nfmax6 = 1;
  return 0;
}
