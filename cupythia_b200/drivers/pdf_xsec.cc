// pdf_xsec -- stage driver of the PDF-convoluted hadronic cross section
// (cuPythia/pipeline/pdf_xsec.cu:49-110): same argv (trials per thread of a 1024 x 256 launch),
// VALIDATION line and exit codes.  Computes sigma(pp -> 2 jets, pT_hat > 20 GeV, 13 TeV, CTEQ5L,
// alpha_s(mZ) = 0.13 first order) on a 10-iteration adapted VEGAS grid and checks it against
// stock Pythia 8.317's sigmaGen for the same settings, 0.7674 +- 0.0009 mb (ProcessLevel run of
// the reference's Pythia), within five combined standard errors.
//   Run: pdf_xsec [trialsPerThread=64]
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t kPer = drv_arg(argc, argv, 1, 64);
  const uint64_t n = 1024ull * 256 * kPer;
  const double pythiaSigma = 0.7674, pythiaErr = 0.0009;
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  DRV_CK(h, cp_set_point_offset(h, drv_shard_offset()));
  cp_result per[10], comb;
  const auto t0 = DrvClock::now();
  DRV_CK(h, cp_integrate(h, 10, n, 1.5, 3, per, &comb));
  const auto t1 = DrvClock::now();
  const double pull = (comb.sigma - pythiaSigma) / sqrt(comb.sigma_err * comb.sigma_err + pythiaErr * pythiaErr);
  printf("PDF convolution -> hadronic cross section (13 TeV pp, 5 HardQCD processes, pT-hat>%.0f GeV, CTEQ5L)\n",
         cfg.pt_hat_min);
  printf("  hadronic sigma (GPU, FP32 integrand, FP64 sums) = %.6e +- %.1e mb   (10 x %.3e points, %.1f ms)\n",
         comb.sigma, comb.sigma_err, (double)n, drv_ms(t0, t1));
  printf("  Pythia 8.317 sigmaGen (same settings)           = %.4e +- %.1e mb   pull = %.2f\n", pythiaSigma, pythiaErr,
         pull);
  const bool ok = fabs(pull) < 5.0 && comb.n_bad == 0;
  printf("VALIDATION: %s (hadronic sigma matches Pythia within 5 combined standard errors)\n", ok ? "PASS" : "FAIL");
  cp_destroy(h);
  return ok ? 0 : 2;
}
