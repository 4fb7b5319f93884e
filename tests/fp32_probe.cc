// fp32_probe.cc -- host build of the device integrand header (cupythia_b200/csrc/cp_integrand.cuh)
// used by the CPU test suite to check the FP32 formulation against the FP64 oracle without a GPU.
#include "../cupythia_b200/csrc/cp_params.h"

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
void probe_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, uint32_t* out)
{
  cp_philox(c0, c1, c2, c3, k0, k1, out);
}
}
