// generate -- stage driver of the device-resident parton-level generator
// (cuPythia/pipeline/generate.cu:80-127): same argv (number of events), VALIDATION line and
// exit codes.  Adapts the grid (10 x 2^24 points), sets w_max to the 99.9th percentile, runs
// production passes of 2^27 points until nEvents unweighted events exist in device memory,
// and reports the rate.  The renormalisation-scale band (mu_R = 2x .. 0.5x, the reference's
// reweighting) comes from the same points on handles with k_ren = 4 and 0.25 (common random
// numbers).  Checks: unweighted sigma == weighted sigma, the count reached, the band brackets 0.
//   Run: generate [nEvents=4000000]
#include <vector>
#include <cuda_runtime.h>
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t nEv = drv_arg(argc, argv, 1, 4000000);
  const uint64_t pass = 1ull << 27;
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  cp_result per[10], comb;
  DRV_CK(h, cp_integrate(h, 10, 1 << 24, 1.5, 3, per, &comb));
  DRV_CK(h, cp_set_point_offset(h, drv_shard_offset()));
  double wmax = 0;
  DRV_CK(h, cp_weight_quantile(h, 0.999, &wmax));
  const uint64_t cap = nEv + (uint64_t)(1.5 * pass * comb.sigma / wmax) + 4096;
  cp_event* d_rec = nullptr;
  if (cudaMalloc(&d_rec, sizeof(cp_event) * cap) != cudaSuccess) {
    printf("CUDA error: allocation of %llu records failed\n", (unsigned long long)cap);
    return 1;
  }
  uint64_t have = 0, points = 0;
  double sw = 0, sw2 = 0, su = 0;
  const auto t0 = DrvClock::now();
  for (uint32_t it = 100; have < nEv; ++it) {
    cp_unweight_result u;
    DRV_CK(h, cp_unweight(h, pass, it, d_rec + have, cap - have, &u));
    have += u.n_accepted;
    points += pass;
    const double w = 1.0 / (u.sigma_err * u.sigma_err);
    sw += w * u.sigma;
    sw2 += w;
    su += u.sigma_unweighted * pass;
  }
  const auto t1 = DrvClock::now();
  const double sig = sw / sw2, err = 1.0 / sqrt(sw2), sigU = su / points;
  // scale band on the adapted grid, same points (iteration 90)
  double grid[3 * (CP_MAX_BINS + 1)];
  DRV_CK(h, cp_grid_get(h, grid));
  double band[2] = {0, 0};
  cp_result nom;
  DRV_CK(h, cp_vegas_iteration(h, 1 << 24, 90, 0.0, &nom));
  DRV_CK(h, cp_grid_set(h, grid));
  const double kr[2] = {4.0, 0.25};
  for (int k = 0; k < 2; ++k) {
    cp_config c2 = cfg;
    c2.k_ren = kr[k];
    cp_handle* h2 = nullptr;
    DRV_CK(h2, cp_create(&c2, &h2));
    DRV_CK(h2, cp_set_point_offset(h2, drv_shard_offset()));
    DRV_CK(h2, cp_grid_set(h2, grid));
    cp_result r2;
    DRV_CK(h2, cp_vegas_iteration(h2, 1 << 24, 90, 0.0, &r2));
    band[k] = r2.sigma / nom.sigma - 1.0;
    cp_destroy(h2);
  }
  const double ms = drv_ms(t0, t1);
  printf("Device-resident parton-level generator: %llu events, draw->map->ME x PDF->unweight->compact\n",
         (unsigned long long)have);
  printf("  weighted sigma  = %.6e +- %.1e mb   unweighted = %.6e mb   relerr = %.2e\n", sig, err, sigU,
         fabs(sigU - sig) / sig);
  printf("  scale band      = [%+.1f%%, %+.1f%%]  (mu_R = 2x .. 0.5x)\n", 100.0 * band[0], 100.0 * band[1]);
  printf("  unweighting eff = %.2f%%   %.3e points in %.1f ms -> %.3e events/s\n", 100.0 * have / (double)points,
         (double)points, ms, have / (ms / 1e3));
  const bool ok = have >= nEv && fabs(sigU - sig) / sig < 2e-3 && band[0] < 0 && band[1] > 0;
  printf("VALIDATION: %s (unweighted sigma == weighted sigma + scale band brackets the nominal + count reached)\n",
         ok ? "PASS" : "FAIL");
  cudaFree(d_rec);
  cp_destroy(h);
  return ok ? 0 : 2;
}
