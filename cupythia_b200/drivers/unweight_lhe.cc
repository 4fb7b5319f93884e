// unweight_lhe -- stage driver of GPU unweighting + Les Houches output
// (cuPythia/07_unweighting_lhe/unweight_lhe.cu:105-150): same argv (trials per thread of a
// 1024 x 256 launch), output lines, VALIDATION line and exit codes, writing events.lhe (the
// first 1000 unweighted events, every process with its own colour flow).  Checks: the measured
// efficiency n_accepted / n plus the overweight excess equals <w> / w_max of the same pass, the
// unweighted cross section w_max (sum of event weights) / n equals the weighted one, and the
// file holds 1000 events.
//   Run: unweight_lhe [trialsPerThread=4000]   (writes events.lhe)
#include <vector>
#include <cuda_runtime.h>
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t nPer = drv_arg(argc, argv, 1, 4000);
  const uint64_t n = 1024ull * 256 * nPer;
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  cp_result per[10], comb;
  DRV_CK(h, cp_integrate(h, 10, 1 << 24, 1.5, 3, per, &comb));
  DRV_CK(h, cp_set_point_offset(h, drv_shard_offset()));
  double wmax = 0;
  DRV_CK(h, cp_weight_quantile(h, 0.999, &wmax));
  const uint64_t cap = (uint64_t)(1.5 * n * comb.sigma / wmax) + 4096;
  cp_event* d_rec = nullptr;
  if (cudaMalloc(&d_rec, sizeof(cp_event) * cap) != cudaSuccess) {
    printf("CUDA error: allocation of %llu records failed\n", (unsigned long long)cap);
    return 1;
  }
  cp_unweight_result u;
  const auto t0 = DrvClock::now();
  DRV_CK(h, cp_unweight(h, n, 7, d_rec, cap, &u));
  const auto t1 = DrvClock::now();
  const uint64_t nl = u.n_accepted < 1000 ? u.n_accepted : 1000;
  std::vector<cp_event> rec(nl);
  if (cudaMemcpy(rec.data(), d_rec, sizeof(cp_event) * nl, cudaMemcpyDeviceToHost) != cudaSuccess) {
    printf("CUDA error: copy back failed\n");
    return 1;
  }
  DRV_CK(h, cp_write_lhef(&cfg, rec.data(), nl, u.sigma, u.sigma_err, "events.lhe"));
  const double etaCheck = u.sigma / u.w_max;
  const double rel = fabs(u.sigma_unweighted - u.sigma) / u.sigma;
  printf("GPU unweighting (pp -> 2 jets, 5 HardQCD processes) + Les Houches output\n");
  printf("  trials                 = %.3e   w_max = %.4e mb (99.9th percentile)   %.2f ms\n", (double)n, u.w_max,
         drv_ms(t0, t1));
  printf("  unweighting efficiency = %.2f%%   (cross-check <w>/w_max = %.2f%%)   overweight events = %llu\n",
         100.0 * u.eta, 100.0 * etaCheck, (unsigned long long)u.n_overweight);
  printf("  sigma (unweighted MC)  = %.6e mb   weighted = %.6e +- %.1e mb   relerr = %.2e\n", u.sigma_unweighted,
         u.sigma, u.sigma_err, rel);
  printf("  wrote %llu unweighted events -> events.lhe (Les Houches Event File 3.0)\n", (unsigned long long)nl);
  // with w_max below the largest weight, <w>/w_max exceeds the acceptance by the overweight
  // excess sum (w - w_max)+ / (n w_max) = sigma_unweighted / w_max - eta
  const double excess = u.sigma_unweighted / u.w_max - u.eta;
  const bool ok = fabs(u.eta + excess - etaCheck) < 1e-3 && excess >= 0 && rel < 2e-3 && nl == 1000;
  printf("VALIDATION: %s (eta == <w>/w_max, unweighted sigma == weighted sigma, LHE written)\n", ok ? "PASS" : "FAIL");
  cudaFree(d_rec);
  cp_destroy(h);
  return ok ? 0 : 2;
}
