// cp_dual.cuh -- forward-mode dual numbers and the integrand written over a scalar type, for the
// adjoint (gradient) kernel.  CpDual<N> carries a value and N tangents in FP32; every operation
// applies the chain rule exactly, so the tangents are the derivatives of the FP32 evaluation.
//
// The templated integrand below is the plain form of the same formulas as cp_had_eval
// (cp_integrand.cuh): it skips the compensated-FP32 refinements, which matter for the value at
// 1e-6 but not for gradients checked at 1e-4.  Parameters that the gradient is taken against
// enter as duals: ln tauMin (the pT_hat cut), k_ren, and ln Lambda_nf^2 (alpha_s(mZ)).
#pragma once
#include "cp_integrand.cuh"

template <int N>
struct CpDual {
  float v;
  float d[N];
};

template <int N>
CP_HD CpDual<N> cp_dconst(float v)
{
  CpDual<N> r;
  r.v = v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = 0.f;
  return r;
}
template <int N>
CP_HD CpDual<N> cp_dvar(float v, int k)
{
  CpDual<N> r = cp_dconst<N>(v);
  r.d[k] = 1.f;
  return r;
}

#define CP_DUAL_BIN(op, val, der)                                              \
  template <int N>                                                             \
  CP_HD CpDual<N> operator op(const CpDual<N>& a, const CpDual<N>& b)          \
  {                                                                            \
    CpDual<N> r;                                                               \
    r.v = val;                                                                 \
    _Pragma("unroll") for (int k = 0; k < N; ++k) r.d[k] = der;                \
    return r;                                                                  \
  }
CP_DUAL_BIN(+, a.v + b.v, a.d[k] + b.d[k])
CP_DUAL_BIN(-, a.v - b.v, a.d[k] - b.d[k])
CP_DUAL_BIN(*, a.v * b.v, fmaf(a.d[k], b.v, a.v * b.d[k]))
#undef CP_DUAL_BIN

template <int N>
CP_HD CpDual<N> operator/(const CpDual<N>& a, const CpDual<N>& b)
{
  CpDual<N> r;
  float ib = 1.f / b.v;
  r.v = a.v * ib;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
  return r;
}
template <int N> CP_HD CpDual<N> operator+(const CpDual<N>& a, float b) { CpDual<N> r = a; r.v += b; return r; }
template <int N> CP_HD CpDual<N> operator+(float b, const CpDual<N>& a) { return a + b; }
template <int N> CP_HD CpDual<N> operator-(const CpDual<N>& a, float b) { CpDual<N> r = a; r.v -= b; return r; }
template <int N>
CP_HD CpDual<N> operator-(float b, const CpDual<N>& a)
{
  CpDual<N> r;
  r.v = b - a.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int N>
CP_HD CpDual<N> operator-(const CpDual<N>& a)
{
  return 0.f - a;
}
template <int N>
CP_HD CpDual<N> operator*(const CpDual<N>& a, float b)
{
  CpDual<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b;
  return r;
}
template <int N> CP_HD CpDual<N> operator*(float b, const CpDual<N>& a) { return a * b; }
template <int N>
CP_HD CpDual<N> operator/(float a, const CpDual<N>& b)
{
  return cp_dconst<N>(a) / b;
}
template <int N> CP_HD CpDual<N> operator/(const CpDual<N>& a, float b) { return a * (1.f / b); }

// f(a) with derivative fp: r = (f(a), fp * a')
template <int N>
CP_HD CpDual<N> cp_dchain(const CpDual<N>& a, float f, float fp)
{
  CpDual<N> r;
  r.v = f;
#pragma unroll
  for (int k = 0; k < N; ++k) r.d[k] = fp * a.d[k];
  return r;
}

// scalar-generic math
CP_HD float cp_val(float a) { return a; }
template <int N> CP_HD float cp_val(const CpDual<N>& a) { return a.v; }
CP_HD float cp_exp_t(float a) { return cp_expf(a); }
CP_HD float cp_log_t(float a) { return cp_logf(a); }
CP_HD float cp_expm1_t(float a) { return cp_expm1f(a); }
CP_HD float cp_sqrt_t(float a) { return cp_sqrtf(a); }
template <int N> CP_HD CpDual<N> cp_exp_t(const CpDual<N>& a) { float e = cp_expf(a.v); return cp_dchain(a, e, e); }
template <int N> CP_HD CpDual<N> cp_log_t(const CpDual<N>& a) { return cp_dchain(a, cp_logf(a.v), 1.f / a.v); }
template <int N> CP_HD CpDual<N> cp_expm1_t(const CpDual<N>& a) { return cp_dchain(a, cp_expm1f(a.v), cp_expf(a.v)); }
template <int N>
CP_HD CpDual<N> cp_sqrt_t(const CpDual<N>& a)
{
  float s = cp_sqrtf(a.v);
  return cp_dchain(a, s, s > 0.f ? 0.5f / s : 0.f);
}
template <class T> CP_HD T cp_max0(const T& a) { return cp_val(a) > 0.f ? a : T(a * 0.f); }

// ------------------------------------------------------------------------------------------
// Integrand over a scalar type T (float or CpDual<N>).
// ------------------------------------------------------------------------------------------
template <class T>
struct CpHadParamsT {
  T lnTauMin;   // ln(4 pTmin^2 / s)
  T kR;         // renormalisation scale factor
  T lnL2[4];    // ln Lambda_nf^2, nf = 3..6
};

template <class T>
CP_HD T cp_alphas_t(const CpHadParams& P, const CpHadParamsT<T>& Q, const T& Q2in)
{
  T Q2 = Q2in;
  if (cp_val(Q2) < P.scale2Min) Q2 = Q2 * 0.f + P.scale2Min;
  T lnQ2 = cp_log_t(Q2);
  float b0;
  T lnL2;
  if (cp_val(Q2) > P.thr2[2] && P.nfmax6) { b0 = 21.f; lnL2 = Q.lnL2[3]; }
  else if (cp_val(Q2) > P.thr2[1]) { b0 = 23.f; lnL2 = Q.lnL2[2]; }
  else if (cp_val(Q2) > P.thr2[0]) { b0 = 25.f; lnL2 = Q.lnL2[1]; }
  else { b0 = 27.f; lnL2 = Q.lnL2[0]; }
  return (12.f * CP_PI_F / b0) / (lnQ2 - lnL2);
}

template <class T>
CP_HD T cp_poly_t(const CpCteqPoly& c, int f, const T& t)
{
  return (c.co[2][f] * t + c.co[1][f]) * t + c.co[0][f];
}

// the x-dependent quantities of one beam, shared by the 8 parametrisations
template <class T>
struct CpBeamT {
  T x, omx, y, u, x1L, lny;
};

template <class T>
CP_HD CpBeamT<T> cp_beam_t(const T& lnxIn)
{
  // x <= 1 - 1e-10 clamp of PartonDistributions.cc:926 (constant beyond it)
  const T lnx = cp_val(lnxIn) > -1e-10f ? T(lnxIn * 0.f - 1e-10f) : lnxIn;
  CpBeamT<T> b;
  b.x = cp_exp_t(lnx);
  b.omx = -cp_expm1_t(lnx);
  b.y = -lnx;
  b.u = lnx + 11.512925465f;
  b.x1L = cp_log_t(b.omx);
  b.lny = cp_log_t(b.y);
  return b;
}

template <class T>
CP_HD T cp_cteq_answer_t(const CpCteqPoly& c, const T& sb1, const T& invQ, const CpBeamT<T>& b)
{
  const T& x = b.x;
  const T& omx = b.omx;
  const T& u = b.u;
  const T& x1L = b.x1L;
  T A = cp_poly_t(c, CP_CQ_A, sb1), B = cp_poly_t(c, CP_CQ_B, sb1), af1 = cp_poly_t(c, CP_CQ_AF1, sb1);
  T af2 = cp_poly_t(c, CP_CQ_AF2, sb1), p = cp_poly_t(c, CP_CQ_P, sb1), af5 = cp_poly_t(c, CP_CQ_AF5, sb1);
  T af6 = cp_poly_t(c, CP_CQ_AF6, sb1), af7 = cp_poly_t(c, CP_CQ_AF7, sb1), af8 = cp_poly_t(c, CP_CQ_AF8, sb1);
  T ym1 = cp_expm1_t(p * b.lny);
  T U = af8 * u + 1.f;
  T part3 = x * omx * (af5 + af6 * omx + af7 * x * omx);
  T L = c.useX1L ? x1L : cp_log_t(omx + c.eut2);
  T e = A + B * x + af1 * af8 * u + af1 * ym1 * U + part3 + c.ut1 * x1L + af2 * L;
  T qfac = 1.f - c.qmin * invQ;
  return x * cp_exp_t(e) * qfac;
}

template <class T>
CP_HD void cp_cteq_pair_t(const CpCteqPoly* cteq, T Q2, T lnxA, T lnxB, T fa[8], T fb[8])
{
  if (cp_val(Q2) > 1e8f) Q2 = Q2 * 0.f + 1e8f;
  if (cp_val(Q2) < 1.f) Q2 = Q2 * 0.f + 1.f;
  const float lnxMin = -13.815510558f;
  if (cp_val(lnxA) < lnxMin) lnxA = lnxA * 0.f + lnxMin;
  if (cp_val(lnxB) < lnxMin) lnxB = lnxB * 0.f + lnxMin;
  T Q = cp_sqrt_t(Q2);
  T lnQ = 0.5f * cp_log_t(Q2);
  T invQ = 1.f / Q;
  // once per beam rather than once per parametrisation and beam: the same operations on the same
  // values (the host build gives bit-identical results; on the device the compiler may contract a
  // different product into an FMA, a last-bit difference).  12 adjoint passes of 2^22 points:
  // 38.1 -> 33.6 ms
  const CpBeamT<T> bA = cp_beam_t(lnxA), bB = cp_beam_t(lnxB);
#pragma unroll 1
  for (int i = 0; i < 8; ++i) {
    const CpCteqPoly& c = cteq[i];
    T sb1 = cp_log_t(lnQ - c.lnAlpha) - 1.2f;
    T ra, rb;
    if (cp_val(Q) > c.qlim) {
      ra = cp_cteq_answer_t(c, sb1, invQ, bA);
      rb = cp_cteq_answer_t(c, sb1, invQ, bB);
      if (i != 4) {
        ra = ra * bA.x;
        rb = rb * bB.x;
      }
    } else {
      ra = sb1 * 0.f;
      rb = sb1 * 0.f;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k == i) { fa[k] = ra; fb[k] = rb; }
  }
  T sa = fa[3], sb = fb[3], ia = 1.f / (fa[4] + 1.f), ib = 1.f / (fb[4] + 1.f);
  T ra = fa[4], rb = fb[4];
  fa[3] = sa * ia; fa[4] = sa * ra * ia;
  fb[3] = sb * ib; fb[4] = sb * rb * ib;
#pragma unroll
  for (int k = 0; k < 8; ++k) { fa[k] = cp_max0(fa[k]); fb[k] = cp_max0(fb[k]); }
}

template <class T>
CP_HD T cp_channel_sum_t(const CpHadParams& P, const T& tp, const T& up, const T* A, const T* Bq)
{
  T rt = 1.f / tp, ru = 1.f / up, tu = tp * ru, ut = up * rt;
  T sTS = (tp + 1.f) * (tp + 1.f) + (rt + 1.f) * (rt + 1.f) + 1.f;
  T sUS = (up + 1.f) * (up + 1.f) + (ru + 1.f) * (ru + 1.f) + 1.f;
  T sTU = (tu + 1.f) * (tu + 1.f) + (ut + 1.f) * (ut + 1.f) + 1.f;
  T gg2gg = 1.125f * (sTS + sUS + sTU);
  T gg2qq = P.nQuarkNew * ((1.f / 6.f) * (ut + tu) - (3.f / 8.f) * (up * up + tp * tp));
  T qg2qg = (up * up + 1.f) * (rt * rt) - (4.f / 9.f) * (up + ru);
  T qqbar2gg = 0.5f * ((32.f / 27.f) * (ut + tu) - (8.f / 3.f) * (up * up + tp * tp));
  T qqT = (4.f / 9.f) * (up * up + 1.f) * (rt * rt);
  T qqU = (4.f / 9.f) * (tp * tp + 1.f) * (ru * ru);
  T qqTU = -(8.f / 27.f) * (rt * ru);
  T qqST = -(8.f / 27.f) * (up * up) * rt;
  T QA = A[0] + A[1] + A[3] + A[4] + 2.f * (A[5] + A[6] + A[7]);
  T QB = Bq[0] + Bq[1] + Bq[3] + Bq[4] + 2.f * (Bq[5] + Bq[6] + Bq[7]);
  T Dsame = A[0] * Bq[0] + A[1] * Bq[1] + A[3] * Bq[3] + A[4] * Bq[4] +
            2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  T Dopp = A[0] * Bq[4] + A[4] * Bq[0] + A[1] * Bq[3] + A[3] * Bq[1] +
           2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  T G = A[2] * Bq[2];
  T sum = G * (P.mask[0] * gg2gg + P.mask[1] * gg2qq);
  sum = sum + P.mask[2] * qg2qg * (QA * Bq[2] + A[2] * QB);
  sum = sum + P.mask[3] * (QA * QB * qqT + Dsame * (0.5f * (qqU + qqTU - qqT)) + Dopp * qqST);
  sum = sum + P.mask[4] * Dopp * qqbar2gg;
  return sum;
}

// f * J_base at x, as a function of (x, ln tauMin, k_ren, ln Lambda^2): the plain form of cp_had_eval
template <class T>
CP_HD T cp_had_weight_t(const CpHadParams& P, const CpHadParamsT<T>& Q, const CpCteqPoly* cteq,
                        const T& x0, const T& x1, const T& x2)
{
  T lnTau = (1.f - x0) * Q.lnTauMin;
  T invTau = cp_exp_t(-lnTau);
  T tau = cp_exp_t(lnTau);
  T yMax = -0.5f * lnTau;
  T a0 = x0 * Q.lnTauMin;
  T r = cp_exp_t(a0);
  T zMax = cp_sqrt_t(-cp_expm1_t(a0));
  T omzMax = r / (zMax + 1.f);
  T omz = omzMax + 2.f * zMax * (1.f - x2);
  T opz = omzMax + 2.f * zMax * x2;
  T tp = -0.5f * omz, up = -0.5f * opz;
  T sH = tau * P.s;
  T pT2 = 0.25f * sH * omz * opz;
  T lnx1 = lnTau * (1.f - x1), lnx2 = lnTau * x1;
  T alphaS = cp_alphas_t(P, Q, Q.kR * pT2);
  T fa[8], fb[8];
  cp_cteq_pair_t(cteq, P.kF * pT2, lnx1, lnx2, fa, fb);
  T B = cp_channel_sum_t(P, tp, up, fa, fb);
  T K0 = (2.f * CP_PI_F * P.conv / P.s) * (-Q.lnTauMin);
  if (!(cp_val(zMax) > 0.f)) return B * 0.f;
  return K0 * (alphaS * alphaS) * B * yMax * zMax * invTau;
}
