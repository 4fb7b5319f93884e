// vegas -- stage driver of VEGAS importance sampling (cuPythia/11_vegas_importance/vegas.cu:95-
// 130): same argv (samples per thread of a 256 x 256 launch), twelve iterations, the
// efficiency of the first (uniform) grid against the adapted one, VALIDATION line and exit
// codes.  The integrand is this library's hadronic one (pp -> 2 jets, 13 TeV, the five HardQCD
// processes, 3 x 50 bins) instead of the reference's one-dimensional partonic gg -> gg; the
// integral is checked against the uniform-grid estimate of the same points (no quadrature of
// the 3-D hadronic integral exists), the efficiency gain as in the reference.
//   Run: vegas [samplesPerThread=2000]
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t Tper = drv_arg(argc, argv, 1, 2000);
  const int NITER = 12;
  const uint64_t n = 256ull * 256 * Tper;
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  DRV_CK(h, cp_set_point_offset(h, drv_shard_offset()));
  cp_result first, last;
  const auto t0 = DrvClock::now();
  for (int it = 0; it < NITER; ++it) {
    cp_result r;
    DRV_CK(h, cp_vegas_iteration(h, n, (uint32_t)it, 1.5, &r));
    if (it == 0) first = r;
    last = r;
  }
  const auto t1 = DrvClock::now();
  const double etaFirst = first.sigma / first.w_max, etaLast = last.sigma / last.w_max;
  const double pull = (last.sigma - first.sigma) / sqrt(last.sigma_err * last.sigma_err + first.sigma_err * first.sigma_err);
  printf("VEGAS adaptive importance sampling (pp -> 2 jets 13 TeV, 3 x %d bins, %d iters, %.3e points each, %.1f ms)\n",
         cfg.n_bins, NITER, (double)n, drv_ms(t0, t1));
  printf("  unweighting efficiency: uniform = %.2f%%  ->  VEGAS = %.2f%%   (%.1fx better)\n", 100.0 * etaFirst,
         100.0 * etaLast, etaLast / etaFirst);
  printf("  integral (VEGAS) = %.6e +- %.1e mb   uniform grid = %.6e +- %.1e mb   pull = %.2f\n", last.sigma,
         last.sigma_err, first.sigma, first.sigma_err, pull);
  const bool ok = etaLast > 1.5 * etaFirst && fabs(pull) < 5.0;
  printf("VALIDATION: %s (VEGAS raises efficiency AND integral matches the uniform-grid estimate)\n", ok ? "PASS" : "FAIL");
  cp_destroy(h);
  return ok ? 0 : 2;
}
