// cp_integrand.cuh -- FP32 evaluation of the pp -> 2 jets hard-process integrand, shared by
// every kernel of the integrator (and compiled for the host by the accuracy probe in tests).
//
// Physics follows Pythia 8.317:
//   matrix elements      pythia8317/src/SigmaQCD.cc:115-325 (Sigma2gg2gg, gg2qqbar, qg2qg,
//                        qq2qq, qqbar2gg sigmaKin / sigmaHat)
//   channel sums         pythia8317/src/SigmaProcess.cc:124-193 (initFlux) and :423-480
//                        (sigmaPDF); CONVERT2MB :24
//   scales               pythia8317/src/SigmaProcess.cc:846-925 (store2Kin, massless branch)
//   alpha_s              pythia8317/src/StandardModel.cc:189-215 (first order)
//   CTEQ5L               pythia8317/src/PartonDistributions.cc:922-1062
//   region and Jacobian  pythia8317/src/PhaseSpace.cc:1149-1250 (limitTau/Y/Z), :1072-1074
//
// FP32 conditioning.  The formulas are evaluated in algebraically identical forms that keep
// FP32 accurate to ~1e-6 relative:
//   * 1 - z and 1 + z come from the complement of the zMax bound, 1 - zMax = r / (1 + zMax),
//     r = pT^2_min / p^2 = tauMin / tau = exp(x0 ln tauMin), never from a rounded z;
//   * ln x1 = ln tau (1 - v), ln x2 = ln tau v (v the rapidity variable), so x = exp(ln x)
//     and 1 - x = -expm1(ln x) are both accurate and CTEQ5L's y = -ln x needs no log; ln tau and
//     ln x are carried as FP32 (hi, lo) pairs (error-free TwoSum / FMA products);
//   * in CTEQ5L's exponent af0 (1-x) + af3 x + af1 y^p (1 + af8 u), whose O(100) terms cancel
//     for the gluon, the constant parts are pre-combined in FP64 on the host:
//       A = af0 + af1, B = af3 - af0, C = af1 af8, and y^p = 1 + expm1(p ln y), giving
//       exponent = A + B x + C u + af1 expm1(p ln y) (1 + af8 u) + part3 + part4,
//     summed in FP32 with the products' FMA residuals carried in a second float, and
//     exp(hi + lo) = exp(hi) (1 + lo).  The additions' own rounding errors (TwoSum) and the
//     residual of p ln y are not carried: measured on 720k points against the FP64 oracle they
//     move the largest relative weight error from 5.7e-6 to 6.5e-6, for about 310 fewer FP32
//     instructions per point;
//   * matrix elements are written in tHat/sHat and uHat/sHat with all terms of one sign.
#pragma once
#include <stdint.h>
#include <math.h>
#include <string.h>

#if defined(__CUDACC__)
#define CP_HD __host__ __device__ __forceinline__
#else
#define CP_HD static inline
#endif

#ifndef CP_PI_F
#define CP_PI_F 3.14159265358979f
#endif

// ------------------------------------------------------------------------------------------
// Uniform parameters of the hadronic integrand (built on the host in FP64, stored in FP32).
// ------------------------------------------------------------------------------------------
// the nine polynomials of a parametrisation, in the order of CpCteqPoly::co
enum { CP_CQ_A, CP_CQ_B, CP_CQ_AF1, CP_CQ_AF2, CP_CQ_P, CP_CQ_AF5, CP_CQ_AF6, CP_CQ_AF7, CP_CQ_AF8, CP_CQ_N };

// 160 bytes, 16-byte aligned.  The production, VEGAS and record-builder kernels read the records
// from their own parameters (CpHadParams::cteq, constant memory, __grid_constant__): 2.6% faster
// accept kernel than ten 128-bit shared-memory loads per record and point.  Kernels with a
// staged copy read it as 128-bit shared-memory loads.
struct alignas(16) CpCteqPoly {
  // per parametrisation i: co[k][f] = coefficient of sb1^k in polynomial f (CP_CQ_*), sb1 =
  // ln ln(Q/alpha_i) - 1.2.  The pairs (A, B), (af1, af2), (p, af5), (af6, af7) sit side by side
  // at even offsets (co[k][9] pads each power to 10 floats), so one two-lane FMA evaluates a pair.
  float co[3][10];
  float lnAlpha;  // ln(alpha_i)
  float qlim;     // max(Qmin_i, alpha_i)
  float qmin;     // Qmin_i
  float ut1;      // ut1_i
  float eut2;     // exp(ut2_i)
  int   useX1L;   // ut2_i < -100: part4 uses ln(1 - x) twice
  int   pad[4];
};
static_assert(sizeof(CpCteqPoly) == 160, "coefficient record layout");

struct CpHadParams {
  CpCteqPoly cteq[8];
  float lnTauMin;     // ln(tauMin), tauMin = 4 pTmin^2 / s
  float lnTauMinLo;   // ln(tauMin) - lnTauMin (FP64 residual)
  float K0;           // 2 pi CONVERT2MB (-ln tauMin) / s : w = K0 alpha_s^2 B yMax zMax / tau
  float conv;         // CONVERT2MB
  float s;            // sqrt(s)^2
  float kR, kF;       // muR^2 = kR pT^2, muF^2 = kF pT^2
  float lnL2[4];      // ln Lambda_nf^2, nf = 3, 4, 5, 6
  float thr2[3];      // mc^2, mb^2, mt^2
  float scale2Min;    // (1.07 Lambda_3)^2
  float nQuarkNew;    // HardQCD:nQuarkNew
  float mask[5];      // gg2gg, gg2qqbar, qg2qg, qq2qq, qqbar2gg switches (0 or 1)
  int   nfmax6;       // 1 if nf = 6 above mt
};

// Math on the host is libm.  On the device sqrt and the remaining exp calls are CUDA's accurate
// single-precision functions, and the natural logarithm is the hardware base-2 approximation
// times ln 2 (__logf; the accept kernel runs 17% faster than with the accurate logf).  What the
// integrand needs of a logarithm is a small ABSOLUTE error (about 1e-7): each
// one enters an exponent (CTEQ5L), a product with an O(1) coefficient, or alpha_s's denominator
// ln(Q^2 / Lambda^2) >= ln(50 GeV^2 / Lambda_5^2) here.  Measured against the FP64 oracle over
// 2^20 points on the uniform and an adapted grid and 2^18 at four parameter-range corners, the
// largest per-point weight error is 6.7e-6 with __logf and 6.7e-6 with logf (with cp_exp_cteq
// below as well: 7.3e-6).  The expm1 of CTEQ5L's y^p, the beams' x and 1 - x and the bound's
// r and 1 - r come from this file's own two-lane reduction (cp_exp_reduce2; the accept kernel
// 11.5% faster than with expf / expm1f), and the divisions whose last bit does not matter from
// a refined reciprocal (cp_rcp; 0.9% more): largest per-point weight error 7.6e-6, measured as
// above.
CP_HD float cp_expf(float x) { return expf(x); }
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float cp_logf(float x) { return __logf(x); }
#else
CP_HD float cp_logf(float x) { return logf(x); }
#endif
CP_HD float cp_expm1f(float x) { return expm1f(x); }
// exp of the CTEQ5L exponent on the device: the hardware base-2 approximation (__expf), relative
// error about 2^-22 + |x| 2^-24 for exponents of a few units; the accept kernel a further 3%
// faster, the largest per-point weight error 7.3e-6 (measured as above)
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float cp_exp_cteq(float x) { return __expf(x); }
#else
CP_HD float cp_exp_cteq(float x) { return expf(x); }
#endif
CP_HD float cp_sqrtf(float x) { return sqrtf(x); }
CP_HD float cp_fmaf(float a, float b, float c) { return fmaf(a, b, c); }
// a / b for a sub-ulp correction term a: the quotient's last bits do not reach the result, so
// the device takes the fast division (about 2 ulp) instead of the IEEE one
CP_HD float cp_div_correction(float a, float b)
{
#if defined(__CUDA_ARCH__)
  return __fdividef(a, b);
#else
  return a / b;
#endif
}
// 1 / b where the quotient need not be correctly rounded: on the device the fast reciprocal
// (__fdividef(1, b): within 2 ulp for 2^-126 <= |b| <= 2^126) refined by one Newton-Raphson step
// y + y (1 - b y), which leaves about 1 ulp, in place of the IEEE division; IEEE division on the
// host
CP_HD float cp_rcp(float b)
{
#if defined(__CUDA_ARCH__)
  const float y = __fdividef(1.f, b);
  return cp_fmaf(y, cp_fmaf(-b, y, 1.f), y);
#else
  return 1.f / b;
#endif
}
// polynomial f of a coefficient record at t (Horner, FMA)
CP_HD float cp_cq_poly(const CpCteqPoly& c, int f, float t)
{
  return cp_fmaf(cp_fmaf(c.co[2][f], t, c.co[1][f]), t, c.co[0][f]);
}

// ------------------------------------------------------------------------------------------
// alpha_s(Q2) at first order with threshold matching (StandardModel.cc:189-215).
// ------------------------------------------------------------------------------------------
CP_HD float cp_alphas(const CpHadParams& P, float Q2)
{
  if (Q2 < P.scale2Min) Q2 = P.scale2Min;
  float lnQ2 = cp_logf(Q2);
  float b0, lnL2;
  if (Q2 > P.thr2[2] && P.nfmax6) { b0 = 21.f; lnL2 = P.lnL2[3]; }
  else if (Q2 > P.thr2[1]) { b0 = 23.f; lnL2 = P.lnL2[2]; }
  else if (Q2 > P.thr2[0]) { b0 = 25.f; lnL2 = P.lnL2[1]; }
  else { b0 = 27.f; lnL2 = P.lnL2[0]; }
  return (12.f * CP_PI_F) * cp_rcp(b0 * (lnQ2 - lnL2));
}

// Error-free transformations on FP32 (Knuth TwoSum, FMA TwoProd) used to carry the few
// quantities whose FP32 rounding would otherwise be amplified (ln tau, ln x, the CTEQ5L exponent).
CP_HD void cp_twosum(float a, float b, float& s, float& e)
{
  s = a + b;
  float bp = s - a;
  e = (a - (s - bp)) + (b - bp);
}

// Two-lane FP32 arithmetic for the two beams: on sm_100 one packed instruction (FADD2 / FMUL2 /
// FFMA2) does both lanes, each lane rounded exactly like the scalar operation; on the host, two
// scalar operations.
struct CpF2 {
  float x, y;
};
CP_HD CpF2 cp_f2(float a, float b) { CpF2 r; r.x = a; r.y = b; return r; }
CP_HD CpF2 cp_f2s(float a) { return cp_f2(a, a); }
#if defined(__CUDA_ARCH__)
__device__ __forceinline__ float2 cp_tof2(CpF2 a) { return make_float2(a.x, a.y); }
__device__ __forceinline__ CpF2 cp_fromf2(float2 a) { return cp_f2(a.x, a.y); }
CP_HD CpF2 cp_add2(CpF2 a, CpF2 b) { return cp_fromf2(__fadd2_rn(cp_tof2(a), cp_tof2(b))); }
CP_HD CpF2 cp_sub2(CpF2 a, CpF2 b) { return cp_fromf2(__fadd2_rn(cp_tof2(a), make_float2(-b.x, -b.y))); }
CP_HD CpF2 cp_mul2(CpF2 a, CpF2 b) { return cp_fromf2(__fmul2_rn(cp_tof2(a), cp_tof2(b))); }
CP_HD CpF2 cp_fma2(CpF2 a, CpF2 b, CpF2 c) { return cp_fromf2(__ffma2_rn(cp_tof2(a), cp_tof2(b), cp_tof2(c))); }
#else
CP_HD CpF2 cp_add2(CpF2 a, CpF2 b) { return cp_f2(a.x + b.x, a.y + b.y); }
CP_HD CpF2 cp_sub2(CpF2 a, CpF2 b) { return cp_f2(a.x - b.x, a.y - b.y); }
CP_HD CpF2 cp_mul2(CpF2 a, CpF2 b) { return cp_f2(a.x * b.x, a.y * b.y); }
CP_HD CpF2 cp_fma2(CpF2 a, CpF2 b, CpF2 c) { return cp_f2(fmaf(a.x, b.x, c.x), fmaf(a.y, b.y, c.y)); }
#endif
CP_HD int cp_bits(float f)
{
#if defined(__CUDA_ARCH__)
  return __float_as_int(f);
#else
  int i;
  memcpy(&i, &f, 4);
  return i;
#endif
}
CP_HD float cp_from_bits(int i)
{
#if defined(__CUDA_ARCH__)
  return __int_as_float(i);
#else
  float f;
  memcpy(&f, &i, 4);
  return f;
#endif
}

// e^a and e^a - 1 in both lanes, from the textbook reduction e^a = 2^k e^r:
//   k = rint(a / ln 2), r = a - k ln 2 with |r| <= ln 2 / 2 (ln 2 split into a head of 16
//   significant bits, so that k * head is exact for |k| < 2^8, and the head's remainder);
//   q = e^r - 1 = r + r^2 (1/2! + r/3! + ... + r^5/7!), Horner in FMAs (truncation r^8/8! <
//   1.6e-8 relative at |r| = ln 2 / 2);
//   e^a = 2^k q + 2^k and e^a - 1 = 2^k q + (2^k - 1), where 2^k and 2^k - 1 (|k| <= 24) are
//   exact and the last FMA rounds once.
// k comes from the FMA a log2(e) + 1.5 * 2^23, which rounds the exact product to an integer kept
// in the low mantissa bits; shifting those bits left by 23 places k in the exponent field.  For a
// in [-87, 87] every 2^k is a normal float; the callers' arguments lie well inside: CTEQ5L's
// p ln y in [-32.1, 3.7] (p in [-0.03, 1.40] over its table for Q >= 1, ln y in [-23.1, 2.7]),
// ln x in [ln 1e-6, 0], and x0 ln tauMin in [ln tauMin, 0] with ln tauMin > -80, which
// cp_build_had_params checks.  Near a = 0 (k = 0) e^a - 1 is the
// polynomial alone, accurate relative to itself; elsewhere both results are within about 2 u
// (u = 2^-24; measured over 2e7 arguments against FP64: 2.0 u relative for |a| < ln 2 / 2, 1.9 u of
// max(|e^a - 1|, 1) elsewhere; libm's expm1f 1.3 and 1.4; tests/test_fp32_formulation.py holds
// it to 2.5 u over the callers' argument ranges).  Every operation is a
// two-lane FP32 operation (FFMA2 / FMUL2 / FADD2 on the device), rounded per lane as the scalar
// one, so the host build gives the device's result bit for bit.
CP_HD void cp_exp_reduce2(CpF2 a, CpF2& s, CpF2& q)
{
  const float LOG2E = 1.44269504088896341f;
  const float LN2_HI = 0.693145751953125f;          // ln 2 to 16 significant bits
  const float LN2_LO = 1.42860682030941723e-6f;     // ln 2 - LN2_HI
  const float RND = 12582912.f;                     // 1.5 * 2^23
  const CpF2 kf = cp_fma2(a, cp_f2s(LOG2E), cp_f2s(RND));
  const CpF2 k = cp_sub2(kf, cp_f2s(RND));
  CpF2 r = cp_fma2(k, cp_f2s(-LN2_HI), a);
  r = cp_fma2(k, cp_f2s(-LN2_LO), r);
  q = cp_fma2(cp_f2s(1.f / 5040.f), r, cp_f2s(1.f / 720.f));
  q = cp_fma2(q, r, cp_f2s(1.f / 120.f));
  q = cp_fma2(q, r, cp_f2s(1.f / 24.f));
  q = cp_fma2(q, r, cp_f2s(1.f / 6.f));
  q = cp_fma2(q, r, cp_f2s(0.5f));
  q = cp_fma2(cp_mul2(q, r), r, r);
  const int SHIFT_ONE = 127 << 23;
  s = cp_f2(cp_from_bits((int)((unsigned)cp_bits(kf.x) << 23) + SHIFT_ONE),
            cp_from_bits((int)((unsigned)cp_bits(kf.y) << 23) + SHIFT_ONE));
}
// cp_rcp in both lanes
CP_HD CpF2 cp_rcp2(CpF2 b)
{
#if defined(__CUDA_ARCH__)
  const CpF2 y = cp_f2(__fdividef(1.f, b.x), __fdividef(1.f, b.y));
  return cp_fma2(y, cp_fma2(cp_f2(-b.x, -b.y), y, cp_f2s(1.f)), y);
#else
  return cp_f2(1.f / b.x, 1.f / b.y);
#endif
}
CP_HD CpF2 cp_expm1_2(CpF2 a)
{
  CpF2 s, q;
  cp_exp_reduce2(a, s, q);
  return cp_fma2(s, q, cp_sub2(s, cp_f2s(1.f)));
}

// x-dependent quantities of one beam, from ln x = lnx + lnxLo (<= 0, lnxLo a sub-ulp correction)
struct CpBeamX {
  float x, omx, lny, uh, ul, x1L;
};

// lnx clamped to the x clamp of PartonDistributions.cc:926 (ln 1e-6); e1 = e^lnx, om = 1 - e^lnx
CP_HD CpBeamX cp_beam_x(float lnx, float lnxLo, float e1, float om)
{
  CpBeamX b;
  float x = cp_fmaf(e1, lnxLo, e1);
  float omx = cp_fmaf(-x, lnxLo, om);
  if (omx < 1e-10f) { omx = 1e-10f; x = 1.f - 1e-10f; lnx = -1e-10f; lnxLo = 0.f; }
  float y = -lnx;                        // y = -ln x, correction -lnxLo
  b.lny = cp_logf(y) - cp_div_correction(lnxLo, y);
  // u = ln(x / 1e-5) = ln x + ln 1e5 as a (hi, lo) pair
  const float LN1E5_HI = 11.512925148f, LN1E5_LO = 3.1696e-07f;
  cp_twosum(lnx, LN1E5_HI, b.uh, b.ul);
  b.ul += LN1E5_LO + lnxLo;
  b.x1L = cp_logf(omx);
  b.x = x;
  b.omx = omx;
  return b;
}

// both beams: x = e^lnx and 1 - x = -(e^lnx - 1) from one two-lane reduction (lnx <= 0, so
// 2^k <= 1 and 1 - 2^k is exact)
CP_HD void cp_beams_x(float lnxA, float lnxAL, float lnxB, float lnxBL, CpBeamX& A, CpBeamX& B)
{
  const float lnxMin = -13.815510558f;   // ln 1e-6
  if (lnxA < lnxMin) { lnxA = lnxMin; lnxAL = 0.f; }
  if (lnxB < lnxMin) { lnxB = lnxMin; lnxBL = 0.f; }
  CpF2 s, q;
  cp_exp_reduce2(cp_f2(lnxA, lnxB), s, q);
  const CpF2 e1 = cp_fma2(s, q, s);
  const CpF2 om = cp_fma2(cp_f2(-s.x, -s.y), q, cp_sub2(cp_f2s(1.f), s));
  A = cp_beam_x(lnxA, lnxAL, e1.x, om.x);
  B = cp_beam_x(lnxB, lnxBL, e1.y, om.y);
}

// Q-dependent coefficients of parametrisation i, shared by both beams
struct CpCteqQ {
  float A, B, af1, af2, p, af5, af6, af7, af8, qfac;
};

// Parametrisations whose part4 uses ln(1 - x) twice (ut2 < -100), and those with a threshold
// Qmin > 0.  The others have alpha_i < 1 <= Q, so their factor (1 - Qmin/Q) is exactly 1.
// cp_build_had_params checks both against the coefficient tables.
CP_HD constexpr bool cp_cteq_uses_x1l(int i) { return i == 1 || i == 2; }
CP_HD constexpr bool cp_cteq_has_qmin(int i) { return i >= 6; }

// hq = cp_cteq_has_qmin(i)
CP_HD CpCteqQ cp_cteq_coef(const CpCteqPoly& c, float lnQ, float Q, float invQ, bool hq)
{
  CpCteqQ q;
  float sb1 = cp_logf(lnQ - c.lnAlpha) - 1.2f;
  // four pairs in two-lane FMAs (each lane rounded as the scalar FMA), af8 alone
  const CpF2 t = cp_f2s(sb1);
  CpF2 v[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const CpF2 c0 = cp_f2(c.co[0][2 * j], c.co[0][2 * j + 1]), c1 = cp_f2(c.co[1][2 * j], c.co[1][2 * j + 1]);
    const CpF2 c2 = cp_f2(c.co[2][2 * j], c.co[2][2 * j + 1]);
    v[j] = cp_fma2(cp_fma2(c2, t, c1), t, c0);
  }
  q.A = v[0].x; q.B = v[0].y;
  q.af1 = v[1].x; q.af2 = v[1].y;
  q.p = v[2].x; q.af5 = v[2].y;
  q.af6 = v[3].x; q.af7 = v[3].y;
  q.af8 = cp_cq_poly(c, CP_CQ_AF8, sb1);
  q.qfac = hq ? ((Q > c.qlim) ? (1.f - c.qmin * invQ) : 0.f) : 1.f;
  return q;
}

// "answer" of xfUpdate (PartonDistributions.cc:1031-1046) for one parametrisation, for both
// beams at once (lane x: beam A, lane y: beam B): x exp(exponent) (1 - Qmin/Q), with
//   exponent = A + B x + C u + af1 (y^p - 1) U + part3 + ut1 ln(1-x) + af2 L,  C = af1 af8,
// summed with the products' FMA residuals kept in a second float, and exp(hi + lo) =
// exp(hi) (1 + lo).  Every product, residual and sum runs in two-lane arithmetic, the
// transcendentals per lane.  ux = cp_cteq_uses_x1l(i).
CP_HD CpF2 cp_cteq_answer2(const CpCteqPoly& c, const CpCteqQ& a, const CpBeamX& bA, const CpBeamX& bB, bool ux)
{
  const CpF2 lny = cp_f2(bA.lny, bB.lny), x = cp_f2(bA.x, bB.x), omx = cp_f2(bA.omx, bB.omx);
  const CpF2 uh = cp_f2(bA.uh, bB.uh), ul = cp_f2(bA.ul, bB.ul), x1L = cp_f2(bA.x1L, bB.x1L);
  const CpF2 p = cp_f2s(a.p);
  const CpF2 ah = cp_mul2(p, lny);
  const CpF2 ym1 = cp_expm1_2(ah);
  const CpF2 U = cp_fma2(cp_f2s(a.af8), uh, cp_f2s(1.f));
  const CpF2 xo = cp_mul2(x, omx);
  const CpF2 part3 = cp_mul2(xo, cp_fma2(cp_f2s(a.af7), xo, cp_fma2(cp_f2s(a.af6), omx, cp_f2s(a.af5))));
  const CpF2 L = ux ? x1L : cp_f2(cp_logf(bA.omx + c.eut2), cp_logf(bB.omx + c.eut2));
  const float Ch = a.af1 * a.af8, Cl = cp_fmaf(a.af1, a.af8, -Ch);
  const CpF2 ch = cp_f2s(Ch);
  const CpF2 t3 = cp_mul2(ch, uh);
  const CpF2 t3l = cp_fma2(cp_f2s(Cl), uh, cp_fma2(ch, ul, cp_fma2(ch, uh, cp_f2(-t3.x, -t3.y))));
  const CpF2 qv = cp_mul2(cp_f2s(a.af1), ym1);
  const CpF2 t4 = cp_mul2(qv, U), t4l = cp_fma2(qv, U, cp_f2(-t4.x, -t4.y));
  const CpF2 Bv = cp_f2s(a.B);
  const CpF2 t2 = cp_mul2(Bv, x), t2l = cp_fma2(Bv, x, cp_f2(-t2.x, -t2.y));
  const CpF2 u1 = cp_f2s(c.ut1);
  const CpF2 t6 = cp_mul2(u1, x1L), t6l = cp_fma2(u1, x1L, cp_f2(-t6.x, -t6.y));
  const CpF2 a2 = cp_f2s(a.af2);
  const CpF2 t7 = cp_mul2(a2, L), t7l = cp_fma2(a2, L, cp_f2(-t7.x, -t7.y));
  const CpF2 el = cp_add2(cp_add2(t2l, t3l), cp_add2(cp_add2(t4l, t6l), t7l));
  const CpF2 eh = cp_add2(cp_add2(cp_add2(cp_f2s(a.A), t3), cp_add2(t4, t2)), cp_add2(part3, cp_add2(t6, t7)));
  const CpF2 ex = cp_f2(cp_exp_cteq(eh.x), cp_exp_cteq(eh.y));
  return cp_mul2(cp_mul2(x, cp_fma2(ex, el, ex)), cp_f2s(a.qfac));
}

// one coefficient record in 128-bit loads (on the device, from constant or shared memory; a
// plain copy on the host)
CP_HD CpCteqPoly cp_load_poly(const CpCteqPoly* p)
{
#if defined(__CUDA_ARCH__)
  CpCteqPoly c;
  const float4* src = reinterpret_cast<const float4*>(p);
  float4* dst = reinterpret_cast<float4*>(&c);
#pragma unroll
  for (int j = 0; j < (int)(sizeof(CpCteqPoly) / 16); ++j) dst[j] = src[j];
  return c;
#else
  return *p;
#endif
}

// CTEQ5L of a proton for both beams at one factorisation scale (PDF::xf + CTEQ5L::xfUpdate):
// fa, fb = {xd, xu, xg, xubar, xdbar, xs, xc, xb}, from the coefficient records `cteq` (the
// kernel's parameters or a shared-memory copy).  UNROLL = 8 unrolls the 8 parametrisations, so the per-i
// structure (the ln(1 - x) and Qmin cases, the dbar/ubar ratio, which register a result lands in)
// is resolved at compile time: about 8% fewer cycles in the integrand kernels than the rolled
// loop.  UNROLL = 1 keeps the rolled loop where code size or registers matter more (the second
// and third evaluations of the scale-variation path).
template <int UNROLL = 8>
CP_HD void cp_cteq_pair(const CpCteqPoly* cteq, float Q2, float lnxA, float lnxAL, float lnxB,
                        float lnxBL, float fa[8], float fb[8])
{
  // Q2 clamp of PartonDistributions.cc:925
  if (Q2 > 1e8f) Q2 = 1e8f;
  if (Q2 < 1.f) Q2 = 1.f;
  const float Q = cp_sqrtf(Q2);
  const float lnQ = 0.5f * cp_logf(Q2);
  const float invQ = cp_rcp(Q);
  CpBeamX A, B;
  cp_beams_x(lnxA, lnxAL, lnxB, lnxBL, A, B);
#pragma unroll UNROLL
  for (int i = 0; i < 8; ++i) {
    const CpCteqPoly c = cp_load_poly(cteq + i);
    const CpCteqQ a = cp_cteq_coef(c, lnQ, Q, invQ, cp_cteq_has_qmin(i));
    const CpF2 r = cp_cteq_answer2(c, a, A, B, cp_cteq_uses_x1l(i));
    float ra = r.x, rb = r.y;
    // parametrisation 4 is the dbar/ubar ratio; the others are x * answer
    if (i != 4) { ra *= A.x; rb *= B.x; }
#pragma unroll
    for (int k = 0; k < 8; ++k)
      if (k == i) { fa[k] = ra; fb[k] = rb; }
  }
  // ubar and dbar from (ubar + dbar) and dbar/ubar: PartonDistributions.cc:1053-1054
  const CpF2 iab = cp_rcp2(cp_f2(1.f + fa[4], 1.f + fb[4]));
  const float ia = iab.x, ib = iab.y;
  float sa = fa[3], sb = fb[3];
  fa[3] = sa * ia; fa[4] = sa * fa[4] * ia;
  fb[3] = sb * ib; fb[4] = sb * fb[4] * ib;
  // max(0, .) of PDF::xf (PartonDistributions.cc:133-180)
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    fa[k] = fa[k] > 0.f ? fa[k] : 0.f;
    fb[k] = fb[k] > 0.f ? fb[k] : 0.f;
  }
}

// ------------------------------------------------------------------------------------------
// Channel sum B = sum over processes and pairs of bracket(t', u') * xfA * xfB, where
//   dsigma/dtHat = pi alpha_s^2 / sH^2 * bracket,   t' = tH/sH, u' = uH/sH.
// ------------------------------------------------------------------------------------------
struct CpBrackets {
  float gg2gg, gg2qqbar, qg2qg, qqbar2gg, qqT, qqU, qqTU, qqST;
};

CP_HD void cp_brackets(const CpHadParams& P, float tp, float up, CpBrackets& b)
{
  const CpF2 rtu = cp_rcp2(cp_f2(tp, up));
  float rt = rtu.x, ru = rtu.y, tu = tp * ru, ut = up * rt;
  // Sigma2gg2gg::sigmaKin: each 9/4 (a^2 + 2a + 3 + 2/a + 1/a^2) = 9/4 ((a+1)^2 + (1/a+1)^2 + 1)
  float sTS = (tp + 1.f) * (tp + 1.f) + (rt + 1.f) * (rt + 1.f) + 1.f;
  float sUS = (up + 1.f) * (up + 1.f) + (ru + 1.f) * (ru + 1.f) + 1.f;
  float sTU = (tu + 1.f) * (tu + 1.f) + (ut + 1.f) * (ut + 1.f) + 1.f;
  b.gg2gg = 0.5f * 2.25f * (sTS + sUS + sTU);
  // Sigma2gg2qqbar::sigmaKin
  b.gg2qqbar = P.nQuarkNew * ((1.f / 6.f) * (ut + tu) - (3.f / 8.f) * (up * up + tp * tp));
  // Sigma2qg2qg::sigmaKin
  b.qg2qg = (up * up + 1.f) * (rt * rt) - (4.f / 9.f) * (up + ru);
  // Sigma2qqbar2gg::sigmaKin
  b.qqbar2gg = 0.5f * ((32.f / 27.f) * (ut + tu) - (8.f / 3.f) * (up * up + tp * tp));
  // Sigma2qq2qq::sigmaKin terms
  b.qqT = (4.f / 9.f) * (1.f + up * up) * (rt * rt);
  b.qqU = (4.f / 9.f) * (1.f + tp * tp) * (ru * ru);
  b.qqTU = -(8.f / 27.f) * (rt * ru);
  b.qqST = -(8.f / 27.f) * (up * up) * rt;
}

CP_HD float cp_channel_sum(const float mask[5], const CpBrackets& b, const float A[8], const float Bq[8])
{
  // flavour sums over q = +-1..+-5 (s, c, b enter twice: quark = antiquark)
  float QA = A[0] + A[1] + A[3] + A[4] + 2.f * (A[5] + A[6] + A[7]);
  float QB = Bq[0] + Bq[1] + Bq[3] + Bq[4] + 2.f * (Bq[5] + Bq[6] + Bq[7]);
  float Dsame = A[0] * Bq[0] + A[1] * Bq[1] + A[3] * Bq[3] + A[4] * Bq[4] +
                2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  float Dopp = A[0] * Bq[4] + A[4] * Bq[0] + A[1] * Bq[3] + A[3] * Bq[1] +
               2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  float G = A[2] * Bq[2];
  float sum = G * (mask[0] * b.gg2gg + mask[1] * b.gg2qqbar);
  sum += mask[2] * b.qg2qg * (QA * Bq[2] + A[2] * QB);
  // Sigma2qq2qq::sigmaHat: identical 1/2 (T + U + TU), q qbar T + ST, otherwise T
  sum += mask[3] * (QA * QB * b.qqT + Dsame * (0.5f * (b.qqU + b.qqTU - b.qqT)) + Dopp * b.qqST);
  sum += mask[4] * Dopp * b.qqbar2gg;
  return sum;
}

// ------------------------------------------------------------------------------------------
// Weight f * J_base of a point x in [0,1]^3 (x0 -> tau, x1 -> y, x2 -> z), in mb.
// cp_had_eval keeps the pieces the event record needs (PDFs, brackets, kinematics); kernels
// that only need w call cp_had_weight and the compiler drops the rest.
// ------------------------------------------------------------------------------------------
struct CpKin {
  float tau, yMax, zMax, sH, omz, opz, lnx1, lnx2, pT2, alphaS;
  float lnx1L, lnx2L;   // sub-ulp corrections of ln x1, ln x2
};

struct CpPoint {
  CpKin k;
  CpBrackets b;
  float fa[8], fb[8];
  float scale;   // K0 alpha_s^2 yMax zMax / tau: w = scale * channel sum
};

// Weight and state of the point x.  With `pdf` (the 16 values fa[8], fb[8] an earlier evaluation
// of the same point stored) the CTEQ5L evaluation is skipped.
CP_HD float cp_had_eval(const CpHadParams& P, const CpCteqPoly* cteq, float x0, float x1, float x2,
                        CpPoint& pt, const float* pdf = nullptr)
{
  // ln tau = (1 - x0) ln tauMin as a (hi, lo) pair: both factors carry their rounding
  float omx0, omx0l;
  cp_twosum(1.f, -x0, omx0, omx0l);
  float lnTau = omx0 * P.lnTauMin;
  float lnTauL = cp_fmaf(omx0, P.lnTauMin, -lnTau) + omx0 * P.lnTauMinLo + omx0l * P.lnTauMin;
  float eT = cp_expf(lnTau);
  float tau = cp_fmaf(eT, lnTauL, eT);
  float eI = cp_expf(-lnTau);
  float invTau = cp_fmaf(-eI, lnTauL, eI);
  float yMax = -0.5f * lnTau;
  // r = pT^2_min / p^2 = tauMin / tau and 1 - r (without cancellation) from one reduction
  CpF2 rs, rq;
  cp_exp_reduce2(cp_f2s(x0 * P.lnTauMin), rs, rq);
  float r = cp_fmaf(rs.x, rq.x, rs.x);
  float zMax = cp_sqrtf(cp_fmaf(-rs.x, rq.x, 1.f - rs.x));   // sqrt(1 - r)
  float omzMax = r * cp_rcp(1.f + zMax);         // 1 - zMax
  float omz = cp_fmaf(2.f * zMax, 1.f - x2, omzMax);   // 1 - z
  float opz = cp_fmaf(2.f * zMax, x2, omzMax);         // 1 + z
  float tp = -0.5f * omz, up = -0.5f * opz;
  float sH = tau * P.s;
  float pT2 = 0.25f * sH * omz * opz;
  // ln x1 = ln tau (1 - v), ln x2 = ln tau v, each as (hi, lo)
  float omv, omvl;
  cp_twosum(1.f, -x1, omv, omvl);
  float lnx1 = lnTau * omv;
  float lnx1L = cp_fmaf(lnTau, omv, -lnx1) + lnTauL * omv + lnTau * omvl;
  float lnx2 = lnTau * x1;
  float lnx2L = cp_fmaf(lnTau, x1, -lnx2) + lnTauL * x1;
  float alphaS = cp_alphas(P, P.kR * pT2);
  if (pdf) {
#pragma unroll
    for (int k = 0; k < 8; ++k) { pt.fa[k] = pdf[k]; pt.fb[k] = pdf[8 + k]; }
  } else {
    cp_cteq_pair(cteq, P.kF * pT2, lnx1, lnx1L, lnx2, lnx2L, pt.fa, pt.fb);
  }
  cp_brackets(P, tp, up, pt.b);
  float B = cp_channel_sum(P.mask, pt.b, pt.fa, pt.fb);
  pt.k.tau = tau; pt.k.yMax = yMax; pt.k.zMax = zMax; pt.k.sH = sH; pt.k.omz = omz;
  pt.k.opz = opz; pt.k.lnx1 = lnx1; pt.k.lnx2 = lnx2; pt.k.pT2 = pT2; pt.k.alphaS = alphaS;
  pt.k.lnx1L = lnx1L; pt.k.lnx2L = lnx2L;
  pt.scale = (zMax > 0.f) ? P.K0 * (alphaS * alphaS) * yMax * zMax * invTau : 0.f;
  return pt.scale * B;
}

// Scale-variation ratios of an evaluated point, the 7-point variation of mu_R and mu_F around
// the nominal scales (mu^2 = k pT^2, SigmaProcess::store2Kin, pythia8317/src/SigmaProcess.cc:
// 906-922): out = w(muR', muF') / w(muR, muF) for (muR', muF') / (muR, muF) = (2, 1), (1/2, 1),
// (1, 2), (1, 1/2), (2, 2), (1/2, 1/2).  The brackets carry no scale, alpha_s^2 carries mu_R and
// the two PDFs mu_F, so a mu_R ratio is (alpha_s' / alpha_s)^2 and a mu_F ratio the channel sum
// with CTEQ5L at the varied scale over the nominal one; the combined points are the products.
CP_HD void cp_scale_ratios(const CpHadParams& P, const CpCteqPoly* cteq, const CpPoint& pt, float out[6])
{
  const float B0 = cp_channel_sum(P.mask, pt.b, pt.fa, pt.fb);
  if (!(B0 > 0.f) || !(pt.k.alphaS > 0.f)) {
#pragma unroll
    for (int j = 0; j < 6; ++j) out[j] = 1.f;
    return;
  }
  const float f2[2] = {4.f, 0.25f};
  float rR[2], rF[2];
#pragma unroll 1
  for (int j = 0; j < 2; ++j) {
    const float a = cp_alphas(P, P.kR * f2[j] * pt.k.pT2) / pt.k.alphaS;
    rR[j] = a * a;
    float fa[8], fb[8];
    cp_cteq_pair<1>(cteq, P.kF * f2[j] * pt.k.pT2, pt.k.lnx1, pt.k.lnx1L, pt.k.lnx2, pt.k.lnx2L, fa, fb);
    rF[j] = cp_channel_sum(P.mask, pt.b, fa, fb) / B0;
  }
  out[0] = rR[0]; out[1] = rR[1]; out[2] = rF[0]; out[3] = rF[1];
  out[4] = rR[0] * rF[0]; out[5] = rR[1] * rF[1];
}

CP_HD float cp_had_weight(const CpHadParams& P, const CpCteqPoly* cteq, float x0, float x1, float x2,
                          CpKin* kin)
{
  CpPoint pt;
  float w = cp_had_eval(P, cteq, x0, x1, x2, pt);
  if (kin) *kin = pt.k;
  return w;
}

// ------------------------------------------------------------------------------------------
// Philox-4x32-10 (Salmon et al., SC'11) and the point -> words layout used everywhere:
//   key = (seed lo, seed hi), counter = (point lo, point hi, iteration, stream).
// Words 0..2 drive the three map dimensions, word 3 the unweighting accept draw.
// ------------------------------------------------------------------------------------------
CP_HD void cp_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                     uint32_t out[4])
{
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
#if defined(__CUDA_ARCH__)
    uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
    uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

CP_HD void cp_point_words(uint64_t seed, uint64_t point, uint32_t iter, uint32_t stream, uint32_t w[4])
{
  cp_philox((uint32_t)point, (uint32_t)(point >> 32), iter, stream, (uint32_t)seed,
            (uint32_t)(seed >> 32), w);
}

// 24-bit uniform in [0, 1): exact in FP32 and FP64
CP_HD float cp_u24(uint32_t w) { return (float)(w >> 8) * (1.f / 16777216.f); }

// VEGAS bin and in-bin fraction of a 24-bit word, in integer arithmetic (exact everywhere)
CP_HD void cp_bin_frac(uint32_t w, int nb, int& bin, float& frac)
{
  uint32_t m = (w >> 8) * (uint32_t)nb;      // < 2^24 * nb <= 2^31 for nb <= 128
  bin = (int)(m >> 24);
  frac = (float)(m & 0xFFFFFFu) * (1.f / 16777216.f);
}

// ------------------------------------------------------------------------------------------
// Unweighted event record (the 64-byte cp_event of the C ABI).
// Flavour choice follows SigmaProcess::pickInState (pythia8317/src/SigmaProcess.cc:486-508):
// a process with probability proportional to its share of the channel sum, then an incoming
// pair in initFlux order (SigmaProcess.cc:124-193) with probability proportional to its
// pdfSigma; outgoing flavours follow each process's setIdColAcol (SigmaQCD.cc:135-342):
// gg -> gg and q qbar -> g g give 21 21, gg -> q qbar gives q = 1 + int(nQuarkNew u), q qbar,
// qg -> qg and qq -> qq keep the incoming flavours.
// ------------------------------------------------------------------------------------------
struct CpEventRec {
  int16_t id[4];
  float pz_in[2];
  float p3[4];
  float p4[4];
  float weight;
  float pt_hat;
  uint16_t process;
  uint16_t colour;
  uint32_t point;
};

// x f(id) from the raw array {d, u, g, ubar, dbar, s, c, b}
CP_HD float cp_xf_id(const float f[8], int id)
{
  switch (id) {
    case 1: return f[0];
    case 2: return f[1];
    case -1: return f[4];
    case -2: return f[3];
    case 3: case -3: return f[5];
    case 4: case -4: return f[6];
    case 5: case -5: return f[7];
    default: return f[2];
  }
}

CP_HD float cp_qq_pair_bracket(const CpBrackets& b, int id1, int id2)
{
  if (id2 == id1) return 0.5f * (b.qqT + b.qqU + b.qqTU);
  if (id2 == -id1) return b.qqT + b.qqST;
  return b.qqT;
}

// Process shares at one point: {gg2gg, gg2qqbar, qg2qg, qq2qq, qqbar2gg}
CP_HD void cp_process_shares(const float mask[5], const CpBrackets& b, const float* A, const float* Bq, float c[5])
{
  float QA = A[0] + A[1] + A[3] + A[4] + 2.f * (A[5] + A[6] + A[7]);
  float QB = Bq[0] + Bq[1] + Bq[3] + Bq[4] + 2.f * (Bq[5] + Bq[6] + Bq[7]);
  float Dsame = A[0] * Bq[0] + A[1] * Bq[1] + A[3] * Bq[3] + A[4] * Bq[4] +
                2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  float Dopp = A[0] * Bq[4] + A[4] * Bq[0] + A[1] * Bq[3] + A[3] * Bq[1] +
               2.f * (A[5] * Bq[5] + A[6] * Bq[6] + A[7] * Bq[7]);
  float G = A[2] * Bq[2];
  c[0] = mask[0] * G * b.gg2gg;
  c[1] = mask[1] * G * b.gg2qqbar;
  c[2] = mask[2] * b.qg2qg * (QA * Bq[2] + A[2] * QB);
  c[3] = mask[3] * (QA * QB * b.qqT + Dsame * (0.5f * (b.qqU + b.qqTU - b.qqT)) + Dopp * b.qqST);
  c[4] = mask[4] * Dopp * b.qqbar2gg;
}

// pickInState of process k (0..4 = codes 111..115; SigmaProcess.cc:486-508) with uniform r1 and
// the outgoing flavours of its setIdColAcol (new flavour of g g -> q qbar from r3,
// SigmaQCD.cc:173): id = (in a, in b, out 3, out 4).
CP_HD void cp_pick_pair(const CpHadParams& P, int k, const CpPoint& pt, float r1, float r3, int id[4])
{
  const float* A = pt.fa;
  const float* B = pt.fb;
  int a = 21, bb = 21;
  if (k == 2) {
    // (q, g) and (g, q) for q = -5..5, q != 0, in initFlux order
    float tot2 = 0.f;
    for (int q = -5; q <= 5; ++q)
      if (q) tot2 += cp_xf_id(A, q) * B[2] + A[2] * cp_xf_id(B, q);
    float u = r1 * tot2;
    a = -5; bb = 21;
    for (int q = -5; q <= 5; ++q) {
      if (!q) continue;
      float s1 = cp_xf_id(A, q) * B[2];
      if (u < s1) { a = q; bb = 21; break; }
      u -= s1;
      float s2 = A[2] * cp_xf_id(B, q);
      if (u < s2) { a = 21; bb = q; break; }
      u -= s2;
      a = 21; bb = q;   // rounding fall-through keeps the last pair
    }
  } else if (k == 3) {
    // pickInState over the 100 (q1, q2) pairs in initFlux order, walked row by row: the row
    // total A(q1) sum_q2 B(q2) br(q1, q2) from the three bracket classes first, then the pair
    // inside the chosen row
    const float brS = 0.5f * (pt.b.qqU + pt.b.qqTU + pt.b.qqT), brO = pt.b.qqT + pt.b.qqST, brT = pt.b.qqT;
    const float SB = B[0] + B[1] + B[3] + B[4] + 2.f * (B[5] + B[6] + B[7]);
    float row[10], tot2 = 0.f;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      const int q = i < 5 ? i - 5 : i - 4;
      row[i] = cp_xf_id(A, q) * (brT * SB + (brS - brT) * cp_xf_id(B, q) + (brO - brT) * cp_xf_id(B, -q));
      tot2 += row[i];
    }
    float u = r1 * tot2;
    int ir = 9;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      if (ir == 9 && i < 9) {
        if (u < row[i]) ir = i;
        else u -= row[i];
      }
    }
    const int q1 = ir < 5 ? ir - 5 : ir - 4;
    const float a1 = cp_xf_id(A, q1);
    a = q1; bb = 5;
    bool done = false;
#pragma unroll
    for (int i = 0; i < 10; ++i) {
      const int q2 = i < 5 ? i - 5 : i - 4;
      if (!done) {
        const float s = a1 * cp_xf_id(B, q2) * (q2 == q1 ? brS : (q2 == -q1 ? brO : brT));
        bb = q2;
        if (u < s) done = true;
        else u -= s;
      }
    }
  } else if (k == 4) {
    float tot2 = 0.f;
    for (int q = -5; q <= 5; ++q)
      if (q) tot2 += cp_xf_id(A, q) * cp_xf_id(B, -q);
    float u = r1 * tot2;
    a = 5; bb = -5;
    for (int q = -5; q <= 5; ++q) {
      if (!q) continue;
      float s = cp_xf_id(A, q) * cp_xf_id(B, -q);
      a = q; bb = -q;
      if (u < s) break;
      u -= s;
    }
  }
  id[0] = a; id[1] = bb;
  if (k == 0 || k == 4) { id[2] = 21; id[3] = 21; }
  else if (k == 1) {
    int qn = 1 + (int)(P.nQuarkNew * r3);
    if (qn > (int)P.nQuarkNew) qn = (int)P.nQuarkNew;
    id[2] = qn; id[3] = -qn;
  } else { id[2] = a; id[3] = bb; }
}

// Picks (process, id1, id2, id3, id4) from uniforms r0 (process), r1 (pair), r3 (new flavour).
CP_HD void cp_pick_flavours(const CpHadParams& P, const CpPoint& pt, float r0, float r1, float r3,
                            int& code, int id[4])
{
  float c[5];
  cp_process_shares(P.mask, pt.b, pt.fa, pt.fb, c);
  float tot = c[0] + c[1] + c[2] + c[3] + c[4];
  float t = r0 * tot;
  int k = 0;
  while (k < 4 && (t >= c[k] || c[k] <= 0.f)) { t -= c[k]; ++k; }
  if (c[k] <= 0.f) { k = 0; while (k < 4 && !(c[k] > 0.f)) ++k; }
  code = 111 + k;
  cp_pick_pair(P, k, pt, r1, r3, id);
}

// Colour flow of the process's setIdColAcol (pythia8317/src/SigmaQCD.cc: Sigma2gg2gg :135-148,
// Sigma2gg2qqbar :195-205, Sigma2qg2qg :232-244, Sigma2qq2qq :292-304, Sigma2qqbar2gg
// :331-342): the topology is drawn with rc in proportion to its kinematic term, the gg -> gg
// orientation with rs.  Encoded as: bits 0-1 topology index (order of the setColAcol calls in
// the source), bit 2 swapColAcol applied, bit 3 swapCol1234 applied.  tp = tHat/sHat,
// up = uHat/sHat; common factors of the terms are dropped.
CP_HD uint32_t cp_colour_flow(int code, const int id[4], float tp, float up, float rc, float rs)
{
#if defined(__CUDA_ARCH__)
  const float rt = __frcp_rn(tp), ru = __frcp_rn(up);
#else
  const float rt = 1.f / tp, ru = 1.f / up;
#endif
  uint32_t topo = 0, swapCA = 0, swap12 = 0;
  if (code == 111) {
    const float tu = tp * ru, ut = up * rt;
    const float a = (tp + 1.f) * (tp + 1.f) + (rt + 1.f) * (rt + 1.f) + 1.f;
    const float b = (up + 1.f) * (up + 1.f) + (ru + 1.f) * (ru + 1.f) + 1.f;
    const float c = (tu + 1.f) * (tu + 1.f) + (ut + 1.f) * (ut + 1.f) + 1.f;
    const float r = (a + b + c) * rc;
    topo = r < a ? 0u : (r < a + b ? 1u : 2u);
    swapCA = rs > 0.5f ? 1u : 0u;
  } else if (code == 112) {
    const float a = (1.f / 6.f) * up * rt - 0.375f * up * up;
    const float b = (1.f / 6.f) * tp * ru - 0.375f * tp * tp;
    topo = (a + b) * rc < a ? 0u : 1u;
  } else if (code == 113) {
    const float a = (up * rt) * (up * rt) - (4.f / 9.f) * up;
    const float b = rt * rt - (4.f / 9.f) * ru;
    topo = (a + b) * rc < a ? 0u : 1u;
    swap12 = id[0] == 21 ? 1u : 0u;
    swapCA = (id[0] < 0 || id[1] < 0) ? 1u : 0u;
  } else if (code == 114) {
    topo = id[0] * id[1] > 0 ? 0u : 1u;
    if (id[1] == id[0]) {
      const float T = (1.f + up * up) * rt * rt, U = (1.f + tp * tp) * ru * ru;
      if ((T + U) * rc > T) topo = 2u;
    }
    swapCA = id[0] < 0 ? 1u : 0u;
  } else {
    const float a = (32.f / 27.f) * up * rt - (8.f / 3.f) * up * up;
    const float b = (32.f / 27.f) * tp * ru - (8.f / 3.f) * tp * tp;
    topo = (a + b) * rc < a ? 0u : 1u;
    swapCA = id[0] < 0 ? 1u : 0u;
  }
  return topo | (swapCA << 2) | (swap12 << 3);
}

// Colour draws from the low bytes of the record block (the picks use the high 24 bits of each
// word): rc, 24 bits from bytes 0 of words 0..2; rs, 8 bits from byte 0 of word 3.
CP_HD float cp_colour_rc(const uint32_t w[4])
{
  return (float)((w[0] & 0xFFu) | ((w[1] & 0xFFu) << 8) | ((w[2] & 0xFFu) << 16)) * (1.f / 16777216.f);
}
CP_HD float cp_colour_rs(const uint32_t w[4]) { return (float)(w[3] & 0xFFu) * (1.f / 256.f); }

// Lab-frame four-momenta: parton 3 at cos(theta*) = z from beam A, azimuth phi; boost by the
// rapidity y = (ln x1 - ln x2)/2 of the parton system (massless, PhaseSpace.cc 2 -> 2 kinematics).
CP_HD void cp_make_event(const CpHadParams& P, const CpPoint& pt, float r0, float r1, float r2,
                         float r3, float rc, float rs, float weight, uint32_t point, CpEventRec& ev)
{
  int code, id[4];
  cp_pick_flavours(P, pt, r0, r1, r3, code, id);
  for (int k = 0; k < 4; ++k) ev.id[k] = (int16_t)id[k];
  const CpKin& k = pt.k;
  ev.colour = (uint16_t)cp_colour_flow(code, id, -0.5f * k.omz, -0.5f * k.opz, rc, rs);
  float eBeam = 0.5f * cp_sqrtf(P.s);
  float x1 = cp_expf(k.lnx1), x2 = cp_expf(k.lnx2);
  ev.pz_in[0] = eBeam * x1;
  ev.pz_in[1] = -eBeam * x2;
  float pstar = 0.5f * cp_sqrtf(k.sH);
  float z = 0.5f * (k.opz - k.omz);
  float sinT = cp_sqrtf(k.omz * k.opz);
  float pT = pstar * sinT;
  // azimuth phi = 2 pi r2: sin and cos of pi (2 r2), without the argument reduction of sincosf
  float sphi, cphi;
#if defined(__CUDA_ARCH__)
  sincospif(2.f * r2, &sphi, &cphi);
#else
  sphi = (float)sin(6.283185307179586 * (double)r2); cphi = (float)cos(6.283185307179586 * (double)r2);
#endif
  float pzs = pstar * z;
  float y = 0.5f * (k.lnx1 - k.lnx2);
  float ey = cp_expf(y);
#if defined(__CUDA_ARCH__)
  float iey = __frcp_rn(ey);   // correctly rounded 1 / e^y
#else
  float iey = 1.f / ey;
#endif
  float ch = 0.5f * (ey + iey), sh = 0.5f * (ey - iey);
  ev.p3[0] = pT * cphi; ev.p3[1] = pT * sphi;
  ev.p3[2] = pzs * ch + pstar * sh; ev.p3[3] = pstar * ch + pzs * sh;
  ev.p4[0] = -pT * cphi; ev.p4[1] = -pT * sphi;
  ev.p4[2] = -pzs * ch + pstar * sh; ev.p4[3] = pstar * ch - pzs * sh;
  ev.weight = weight;
  ev.pt_hat = cp_sqrtf(k.pT2);
  ev.process = (uint16_t)code;
  ev.point = point;
}
