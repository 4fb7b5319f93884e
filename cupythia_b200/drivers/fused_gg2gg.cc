// fused_gg2gg -- stage driver of the fused resident g g -> g g Monte Carlo
// (cuPythia/03_fused_resident_me/fused_gg2gg.cu:83-123): the same argv, output lines,
// validation and exit codes, over the C-ABI.  The GPU estimate uses the reference's SplitMix64
// per-thread streams (1024 x 256 threads, trialsPerThread draws each, seed 0xABCDEF01) and is
// checked against Simpson's rule (2e6 intervals) of the same integrand.
//   Run: fused_gg2gg [trialsPerThread=4000]
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t kPer = drv_arg(argc, argv, 1, 4000);
  const uint64_t threads = 1024ull * 256;
  const double sqrtS = 100.0, alphaS = 0.118, cMax = 0.9, conv = 0.3893793721;
  const uint64_t seed = 0xABCDEF01ull;
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  cp_result r;
  DRV_CK(h, cp_partonic_splitmix(h, sqrtS, alphaS, cMax, conv, seed, threads, 1, &r));   // warm-up
  const auto g0 = DrvClock::now();
  DRV_CK(h, cp_partonic_splitmix(h, sqrtS, alphaS, cMax, conv, seed, threads, kPer, &r));
  const auto g1 = DrvClock::now();
  const double gpuMs = drv_ms(g0, g1);
  const double total = (double)threads * (double)kPer;
  const double ref = drv_simpson_gg2gg(2000000, sqrtS, alphaS, cMax, conv);
  const double rel = fabs(r.sigma - ref) / ref;
  printf("FUSED resident g g -> g g  (sHat=(100 GeV)^2, alphaS=0.118, |cos theta|<%.1f), B200 sm_100a\n", cMax);
  printf("  Simpson quadrature  sigma = %.6e mb   (deterministic reference)\n", ref);
  printf("  GPU fused MC        sigma = %.6e mb   relerr=%.2e  (%.3e trials, %.2f ms)\n", r.sigma, rel, total, gpuMs);
  printf("  GPU rate = %.3e/s\n", total / (gpuMs / 1000.0));
  const bool ok = rel < 2e-3;
  printf("VALIDATION: %s (GPU MC vs deterministic quadrature, relerr < 2e-3)\n", ok ? "PASS" : "FAIL");
  cp_destroy(h);
  return ok ? 0 : 2;
}
