/*
 * cp_oracle_body.h -- the integrand of the hadronic QCD 2->2 integrator, written once
 * over a scalar type and included twice by cp_oracle.c:
 *   REAL = double          (the FP64 oracle)
 *   REAL = double complex  (complex-step differentiation: f(x + i h) = f(x) + i h f'(x) + O(h^2),
 *                           so Im f(x + i h) / h is the derivative to rounding error)
 * Branches and clamps compare real parts (RE), which is what the complex step needs.
 *
 * TEST INFRASTRUCTURE ONLY (see cp_oracle.h).
 *
 * Required macros: REAL, FN(name), RE(x), R_EXP, R_LOG, R_SQRT, R_POW.
 */

/* ---------------------------------------------------------------------------------------
 * CTEQ5L, restated from pythia8317/src/PartonDistributions.cc:922-1062 (CTEQ5L::xfUpdate).
 * The coefficient table is the published CTEQ5L parametrisation (J. Pumplin;
 * H.L. Lai et al., Eur.Phys.J. C12 (2000) 375) in the same [parametrisation][coefficient][power]
 * order; values are data, not code.
 * out = {xd, xu, xg, xubar, xdbar, xs, xc, xb}.
 * ------------------------------------------------------------------------------------- */
static void FN(cteq5l)(REAL x, REAL Q2, REAL out[8])
{
  /* clamps: PartonDistributions.cc:925-926 */
  REAL Q2c = Q2;
  if (RE(Q2c) > 1e8) Q2c = 1e8;
  if (RE(Q2c) < 1.0) Q2c = 1.0;
  REAL Q = R_SQRT(Q2c);
  REAL xc = x;
  if (RE(xc) > 1.0 - 1e-10) xc = 1.0 - 1e-10;
  if (RE(xc) < 1e-6) xc = 1e-6;

  /* derived quantities: :929-933 */
  REAL y = -R_LOG(xc);
  REAL u = R_LOG(xc / 0.00001);
  REAL x1 = 1.0 - xc;
  REAL x1L = R_LOG(1.0 - xc);
  REAL sumUbarDbar = 0.0;

  for (int i = 0; i < 8; ++i) {
    REAL answer = 0.0;
    double qlim = CTEQ5L_QMIN[i] > CTEQ5L_ALPHA[i] ? CTEQ5L_QMIN[i] : CTEQ5L_ALPHA[i];
    if (RE(Q) > qlim) {
      /* :1031-1046 */
      REAL tmp = R_LOG(Q / CTEQ5L_ALPHA[i]);
      REAL sb = R_LOG(tmp);
      REAL sb1 = sb - 1.2;
      REAL sb2 = sb1 * sb1;
      REAL af[9];
      for (int j = 0; j < 9; ++j)
        af[j] = CTEQ5L_AM[i][j][0] + sb1 * CTEQ5L_AM[i][j][1] + sb2 * CTEQ5L_AM[i][j][2];
      REAL part1 = af[1] * R_POW(y, 1.0 + 0.01 * af[4]) * (1.0 + af[8] * u);
      REAL part2 = af[0] * x1 + af[3] * xc;
      REAL part3 = xc * x1 * (af[5] + af[6] * x1 + af[7] * xc * x1);
      REAL part4 = (CTEQ5L_UT2[i] < -100.0)
                       ? CTEQ5L_UT1[i] * x1L + af[2] * x1L
                       : CTEQ5L_UT1[i] * x1L + af[2] * R_LOG(x1 + exp(CTEQ5L_UT2[i]));
      answer = xc * R_EXP(part1 + part2 + part3 + part4);
      answer *= 1.0 - CTEQ5L_QMIN[i] / Q;
    }
    /* flavour assignment: :1049-1057 */
    if (i == 0) out[0] = xc * answer;
    else if (i == 1) out[1] = xc * answer;
    else if (i == 2) out[2] = xc * answer;
    else if (i == 3) sumUbarDbar = xc * answer;
    else if (i == 4) {
      out[3] = sumUbarDbar / (1.0 + answer);
      out[4] = sumUbarDbar * answer / (1.0 + answer);
    } else if (i == 5) out[5] = xc * answer;
    else if (i == 6) out[6] = xc * answer;
    else out[7] = xc * answer;
  }
}

/* Proton x f(id): PDF::xf, pythia8317/src/PartonDistributions.cc:122-180 for a proton
 * (beamType 1: no isospin rearrangement), with the max(0, .) clamp. */
static REAL FN(xf_of)(const REAL raw[8], int id)
{
  REAL v;
  switch (id) {
    case 21: case 0: v = raw[2]; break;
    case 1: v = raw[0]; break;
    case -1: v = raw[4]; break;
    case 2: v = raw[1]; break;
    case -2: v = raw[3]; break;
    case 3: case -3: v = raw[5]; break;
    case 4: case -4: v = raw[6]; break;
    case 5: case -5: v = raw[7]; break;
    default: v = 0.0; break;
  }
  return RE(v) > 0.0 ? v : (REAL)0.0;
}

/* ---------------------------------------------------------------------------------------
 * First-order alpha_s with flavour-threshold matching:
 * AlphaStrong::init, pythia8317/src/StandardModel.cc:42-64,160-183 (MZ = 91.188 :25,
 * thresholds mc=1.5, mb=4.8, mt=171.0 :46, SAFETYMARGIN1 = 1.07 :29) and
 * AlphaStrong::alphaS :189-215 (order 1 branch), nfmax = 6.
 * ------------------------------------------------------------------------------------- */
static REAL FN(alphas)(REAL aSmZ, REAL scale2)
{
  const double MZ = 91.188, mc = 1.5, mb = 4.8, mt = 171.0;
  REAL L5 = MZ * R_EXP(-6.0 * M_PI / (23.0 * aSmZ));
  REAL L6 = L5 * R_POW(L5 / mt, 2.0 / 21.0);
  REAL L4 = L5 * R_POW(mb / L5, 2.0 / 25.0);
  REAL L3 = L4 * R_POW(mc / L4, 2.0 / 27.0);
  REAL scale2Min = (1.07 * L3) * (1.07 * L3);
  if (RE(scale2) < RE(scale2Min)) scale2 = scale2Min;
  if (RE(scale2) > mt * mt) return 12.0 * M_PI / (21.0 * R_LOG(scale2 / (L6 * L6)));
  if (RE(scale2) > mb * mb) return 12.0 * M_PI / (23.0 * R_LOG(scale2 / (L5 * L5)));
  if (RE(scale2) > mc * mc) return 12.0 * M_PI / (25.0 * R_LOG(scale2 / (L4 * L4)));
  return 12.0 * M_PI / (27.0 * R_LOG(scale2 / (L3 * L3)));
}

/* ---------------------------------------------------------------------------------------
 * Matrix elements, d(sigmaHat)/d(tHat) in GeV^-4: pythia8317/src/SigmaQCD.cc
 * ------------------------------------------------------------------------------------- */
/* Sigma2gg2gg::sigmaKin :115-129 */
static REAL FN(me_gg2gg)(REAL sH, REAL tH, REAL uH, REAL alpS)
{
  REAL sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  REAL sigTS = (9. / 4.) * (tH2 / sH2 + 2. * tH / sH + 3. + 2. * sH / tH + sH2 / tH2);
  REAL sigUS = (9. / 4.) * (uH2 / sH2 + 2. * uH / sH + 3. + 2. * sH / uH + sH2 / uH2);
  REAL sigTU = (9. / 4.) * (tH2 / uH2 + 2. * tH / uH + 3. + 2. * uH / tH + uH2 / tH2);
  REAL sigSum = sigTS + sigUS + sigTU;
  return (M_PI / sH2) * (alpS * alpS) * 0.5 * sigSum;
}
/* Sigma2gg2qqbar::sigmaKin :168-189; massless u,d,s (sH > 4 m^2 always holds for pT > 1 GeV) */
static REAL FN(me_gg2qqbar)(REAL sH, REAL tH, REAL uH, REAL alpS, int nQuarkNew)
{
  REAL sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  REAL sigTS = (1. / 6.) * uH / tH - (3. / 8.) * uH2 / sH2;
  REAL sigUS = (1. / 6.) * tH / uH - (3. / 8.) * tH2 / sH2;
  REAL sigSum = sigTS + sigUS;
  return (M_PI / sH2) * (alpS * alpS) * (double)nQuarkNew * sigSum;
}
/* Sigma2qg2qg::sigmaKin :216-226 */
static REAL FN(me_qg2qg)(REAL sH, REAL tH, REAL uH, REAL alpS)
{
  REAL sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  REAL sigTS = uH2 / tH2 - (4. / 9.) * uH / sH;
  REAL sigTU = sH2 / tH2 - (4. / 9.) * sH / uH;
  return (M_PI / sH2) * (alpS * alpS) * (sigTS + sigTU);
}
/* Sigma2qq2qq::sigmaKin :257-266 + sigmaHat :272-286 */
static REAL FN(me_qq2qq)(REAL sH, REAL tH, REAL uH, REAL alpS, int id1, int id2)
{
  REAL sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  REAL sigT = (4. / 9.) * (sH2 + uH2) / tH2;
  REAL sigU = (4. / 9.) * (sH2 + tH2) / uH2;
  REAL sigTU = -(8. / 27.) * sH2 / (tH * uH);
  REAL sigST = -(8. / 27.) * uH2 / (sH * tH);
  REAL sigSum;
  if (id2 == id1) sigSum = 0.5 * (sigT + sigU + sigTU);
  else if (id2 == -id1) sigSum = sigT + sigST;
  else sigSum = sigT;
  return (M_PI / sH2) * (alpS * alpS) * sigSum;
}
/* Sigma2qqbar2gg::sigmaKin :315-325 */
static REAL FN(me_qqbar2gg)(REAL sH, REAL tH, REAL uH, REAL alpS)
{
  REAL sH2 = sH * sH, tH2 = tH * tH, uH2 = uH * uH;
  REAL sigTS = (32. / 27.) * uH / tH - (8. / 3.) * uH2 / sH2;
  REAL sigUS = (32. / 27.) * tH / uH - (8. / 3.) * tH2 / sH2;
  return (M_PI / sH2) * (alpS * alpS) * 0.5 * (sigTS + sigUS);
}

/* ---------------------------------------------------------------------------------------
 * Sigma2Process::store2Kin (pythia8317/src/SigmaProcess.cc:846-925, massless branch)
 * followed by SigmaProcess::sigmaPDF (:423-480) for every selected process, with the
 * channel lists of SigmaProcess::initFlux (:124-193) and K factor 1:
 *   gg         : (21,21)
 *   qg         : (q,21) and (21,q) for q = -nQuarkIn..nQuarkIn, q != 0
 *   qq         : (q1,q2) for all q1,q2 != 0
 *   qqbarSame  : (q,-q)
 * Each pair term is  Kfactor * CONVERT2MB * sigmaHat(id1,id2) * pdfA * pdfB  as in
 * sigmaHatWrap (pythia8317/include/Pythia8/SigmaProcess.h:516-520).
 * ------------------------------------------------------------------------------------- */
static REAL FN(sigma_pdf)(const cpo_had_cfg* c, REAL aSmZ, REAL kR, REAL kF, REAL x1, REAL x2,
                          REAL sH, REAL tH, int mask, REAL extra[6])
{
  REAL uH = -(sH + tH);
  REAL pT2 = tH * uH / sH;
  REAL Q2Ren = pT2 * kR;
  REAL Q2Fac = pT2 * kF;
  REAL alpS = FN(alphas)(aSmZ, Q2Ren);
  REAL rawA[8], rawB[8];
  FN(cteq5l)(x1, Q2Fac, rawA);
  FN(cteq5l)(x2, Q2Fac, rawB);
  const double conv = c->convert2mb, K = 1.0;
  const int nQ = c->nQuarkIn;
  REAL sum = 0.0;

  if (mask & CPO_GG2GG) {
    REAL s = K * (conv * FN(me_gg2gg)(sH, tH, uH, alpS));
    s *= FN(xf_of)(rawA, 21);
    s *= FN(xf_of)(rawB, 21);
    sum += s;
  }
  if (mask & CPO_GG2QQBAR) {
    REAL s = K * (conv * FN(me_gg2qqbar)(sH, tH, uH, alpS, c->nQuarkNew));
    s *= FN(xf_of)(rawA, 21);
    s *= FN(xf_of)(rawB, 21);
    sum += s;
  }
  if (mask & CPO_QG2QG) {
    REAL me = FN(me_qg2qg)(sH, tH, uH, alpS);
    for (int q = -nQ; q <= nQ; ++q) {
      if (q == 0) continue;
      REAL s1 = K * (conv * me);
      s1 *= FN(xf_of)(rawA, q);
      s1 *= FN(xf_of)(rawB, 21);
      sum += s1;
      REAL s2 = K * (conv * me);
      s2 *= FN(xf_of)(rawA, 21);
      s2 *= FN(xf_of)(rawB, q);
      sum += s2;
    }
  }
  if (mask & CPO_QQ2QQ) {
    for (int q1 = -nQ; q1 <= nQ; ++q1) {
      if (q1 == 0) continue;
      for (int q2 = -nQ; q2 <= nQ; ++q2) {
        if (q2 == 0) continue;
        REAL s = K * (conv * FN(me_qq2qq)(sH, tH, uH, alpS, q1, q2));
        s *= FN(xf_of)(rawA, q1);
        s *= FN(xf_of)(rawB, q2);
        sum += s;
      }
    }
  }
  if (mask & CPO_QQBAR2GG) {
    REAL me = FN(me_qqbar2gg)(sH, tH, uH, alpS);
    for (int q = -nQ; q <= nQ; ++q) {
      if (q == 0) continue;
      REAL s = K * (conv * me);
      s *= FN(xf_of)(rawA, q);
      s *= FN(xf_of)(rawB, -q);
      sum += s;
    }
  }
  if (extra) {
    extra[0] = sum; extra[1] = alpS; extra[2] = Q2Ren; extra[3] = Q2Fac;
    extra[4] = uH; extra[5] = pT2;
  }
  return sum;
}

/* ---------------------------------------------------------------------------------------
 * Analytic base map x in [0,1]^3 -> (tau, y, z) over exactly the region Pythia samples:
 *   tau in [tauMin, 1]  (PhaseSpace::limitTau, PhaseSpace.cc:1149-1177: tauMin = max(sHatMin,
 *                        (2 pTmin)^2) / s for massless products, mHatMin = 4 GeV)
 *   |y| <= -ln(tau)/2   (PhaseSpace::limitY, :1183-1200)
 *   |z| <= sqrt(1 - pTmin^2 / p^2), p^2 = sH/4   (PhaseSpace::limitZ, :1206-1250)
 * with tau = tauMin^(1-x0), y = yMax (2 x1 - 1), z = zMax (2 x2 - 1).
 * Pythia's event weight is sigmaPDF * wtTau * wtY * wtZ (PhaseSpace.cc:1072-1074) with
 * wtTau = 1/(tau p(tau)), wtY = 1/p(y), wtZ = mHat pAbs / p(z) (:1317-1319,1434-1437,1550-1552),
 * so the density in (tau, y, z) is sigmaPDF * mHat pAbs / tau = sigmaPDF * sH / (2 tau).
 * ------------------------------------------------------------------------------------- */
static REAL FN(weight_x)(const cpo_had_cfg* c, REAL aSmZ, REAL kR, REAL pTmin, const REAL x[3],
                         REAL tyz[3])
{
  const double s = c->sqrtS * c->sqrtS;
  const double mHatMin = 4.0;
  REAL tauMin = 4.0 * pTmin * pTmin / s;
  if (RE(tauMin) < mHatMin * mHatMin / s) tauMin = mHatMin * mHatMin / s;
  REAL lnTauMin = R_LOG(tauMin);
  REAL lnTau = (1.0 - x[0]) * lnTauMin;
  REAL tau = R_EXP(lnTau);
  REAL jTau = -lnTauMin * tau;
  REAL yMax = -0.5 * lnTau;
  REAL y = yMax * (2.0 * x[1] - 1.0);
  REAL jY = 2.0 * yMax;
  REAL sH = tau * s;
  REAL p2 = 0.25 * sH;
  REAL zArg = 1.0 - pTmin * pTmin / p2;
  if (RE(zArg) < 0.0) zArg = 0.0;
  REAL zMax = R_SQRT(zArg);
  REAL z = zMax * (2.0 * x[2] - 1.0);
  REAL jZ = 2.0 * zMax;
  REAL tH = -0.5 * sH * (1.0 - z);
  REAL sqrtTau = R_SQRT(tau);
  REAL ey = R_EXP(y);
  REAL x1 = sqrtTau * ey;
  REAL x2 = sqrtTau / ey;
  if (tyz) { tyz[0] = tau; tyz[1] = y; tyz[2] = z; }
  if (RE(zMax) <= 0.0) return 0.0;
  REAL sig = FN(sigma_pdf)(c, aSmZ, kR, c->kF, x1, x2, sH, tH, c->procMask, NULL);
  REAL mHatPAbs = 0.5 * sH;
  return sig * (mHatPAbs / tau) * jTau * jY * jZ;
}
