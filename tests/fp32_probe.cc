// fp32_probe.cc -- host build of the device integrand header (cupythia_b200/csrc/cp_integrand.cuh)
// used by the CPU test suite to check the FP32 formulation against the FP64 oracle without a GPU.
#include "../cupythia_b200/csrc/cp_params.h"
#include "../cupythia_b200/csrc/cp_dual.cuh"

extern "C" {
int probe_had_weights(double sqrtS, double pTmin, double aSmZ, double kR, double kF, double conv,
                      int procMask, const float* x, int n, float* out)
{
  CpHadConfig c{sqrtS, pTmin, aSmZ, kR, kF, conv, 5, 3, procMask};
  CpHadParams P;
  if (cp_build_had_params(c, P)) return 1;
  for (int i = 0; i < n; ++i) out[i] = cp_had_weight(P, P.cteq, x[3 * i], x[3 * i + 1], x[3 * i + 2], nullptr);
  return 0;
}
int probe_pdf(double aSmZ, float lnx, float Q2, float* out8)
{
  CpHadConfig c{13000., 20., aSmZ, 1., 1., 0.389380, 5, 3, 31};
  CpHadParams P;
  if (cp_build_had_params(c, P)) return 1;
  float other[8];
  cp_cteq_pair(P.cteq, Q2, lnx, 0.f, lnx, 0.f, out8, other);
  return 0;
}
// value and derivatives (d/dx0, d/dx1, d/dx2, d/dalpha_s(mZ), d/dk_ren, d/dpT_hat_min) of f * J_base
// at one point, from the dual-number integrand of the adjoint kernel
int probe_had_grad(double sqrtS, double pTmin, double aSmZ, double kR, const float* x, double* out7)
{
  CpHadConfig c{sqrtS, pTmin, aSmZ, kR, 1.0, 0.389380, 5, 3, 31};
  CpHadParams P;
  if (cp_build_had_params(c, P)) return 1;
  typedef CpDual<6> D;
  CpHadParamsT<D> Q;
  Q.lnTauMin = cp_dconst<6>((float)log(4.0 * pTmin * pTmin / (sqrtS * sqrtS)));
  Q.lnTauMin.d[5] = (float)(2.0 / pTmin);
  Q.kR = cp_dconst<6>((float)kR);
  Q.kR.d[4] = 1.f;
  const double b0[4] = {27.0, 25.0, 23.0, 21.0};
  for (int k = 0; k < 4; ++k) {
    Q.lnL2[k] = cp_dconst<6>(P.lnL2[k]);
    Q.lnL2[k].d[3] = (float)(12.0 * M_PI / (b0[k] * aSmZ * aSmZ));
  }
  D w = cp_had_weight_t<D>(P, Q, P.cteq, cp_dvar<6>(x[0], 0), cp_dvar<6>(x[1], 1), cp_dvar<6>(x[2], 2));
  out7[0] = w.v;
  for (int k = 0; k < 6; ++k) out7[1 + k] = w.d[k];
  return 0;
}
void probe_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t* out)
{
  cp_philox(c0, c1, c2, c3, k0, k1, out);
}
// cp_build_had_params' verdict on a configuration (0: the kernels support it)
int probe_build_params(double sqrtS, double pTmin, double aSmZ)
{
  CpHadConfig c{sqrtS, pTmin, aSmZ, 1.0, 1.0, 0.389380, 5, 3, 31};
  CpHadParams P;
  return cp_build_had_params(c, P);
}
// the integrand's two-lane exp reduction: e^a and e^a - 1 of n arguments (pairs of lanes)
void probe_exp_reduce(const float* a, int n, float* e, float* em1)
{
  for (int i = 0; i < n; i += 2) {
    const float a1 = i + 1 < n ? a[i + 1] : 0.f;
    CpF2 s, q;
    cp_exp_reduce2(cp_f2(a[i], a1), s, q);
    const CpF2 ex = cp_fma2(s, q, s), m1 = cp_expm1_2(cp_f2(a[i], a1));
    e[i] = ex.x; em1[i] = m1.x;
    if (i + 1 < n) { e[i + 1] = ex.y; em1[i + 1] = m1.y; }
  }
}
}
