// cub_compaction -- stage driver of the accepted-event compaction
// (cuPythia/10_cub_compaction/cub_compaction.cu:59-100): same argv (number of candidates),
// VALIDATION line and exit codes.  The reference flags candidates and runs a library
// DeviceSelect; here the production pass compacts on the device as it accepts (per-block counts,
// one scan, records in point order like DeviceSelect's).  Validation: the number of records
// equals an independent recount of u w_max < w over the same points (weights from
// cp_point_weights, u from the Philox words), up to FP32 evaluation differences of 1 in 10^5,
// and the records' point indices increase strictly (distinct, in point order).
//   Run: cub_compaction [nCandidates=16777216]
#include <algorithm>
#include <vector>
#include <cuda_runtime.h>
#include "drv.h"

int main(int argc, char** argv)
{
  const uint64_t n = drv_arg(argc, argv, 1, 1ull << 24);
  const uint64_t off = drv_shard_offset();
  cp_config cfg;
  cp_config_default(&cfg);
  cp_handle* h = nullptr;
  DRV_CK(h, cp_create(&cfg, &h));
  cp_result per[6], comb;
  DRV_CK(h, cp_integrate(h, 6, 1 << 22, 1.5, 2, per, &comb));
  DRV_CK(h, cp_set_point_offset(h, off));
  cp_result r;
  DRV_CK(h, cp_vegas_iteration(h, n, 40, 0.0, &r));
  double wmax = 0;
  DRV_CK(h, cp_weight_quantile(h, 0.999, &wmax));
  cp_event* d_rec = nullptr;
  float* d_w = nullptr;
  uint32_t* d_words = nullptr;
  if (cudaMalloc(&d_rec, sizeof(cp_event) * n) != cudaSuccess || cudaMalloc(&d_w, sizeof(float) * n) != cudaSuccess ||
      cudaMalloc(&d_words, sizeof(uint32_t) * 4 * n) != cudaSuccess) {
    printf("CUDA error: allocation of %llu candidates failed\n", (unsigned long long)n);
    return 1;
  }
  cp_unweight_result u;
  const auto t0 = DrvClock::now();
  DRV_CK(h, cp_unweight(h, n, 41, d_rec, n, &u));
  const auto t1 = DrvClock::now();
  // independent recount on the host
  DRV_CK(h, cp_point_weights(h, 0, n, 41, d_w, nullptr));
  DRV_CK(h, cp_philox_words(h, cfg.seed, off, n, 41, 0, d_words));
  std::vector<float> w(n);
  std::vector<uint32_t> words(4 * n);
  std::vector<cp_event> rec(u.n_accepted);
  if (cudaMemcpy(w.data(), d_w, sizeof(float) * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(words.data(), d_words, sizeof(uint32_t) * 4 * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(rec.data(), d_rec, sizeof(cp_event) * u.n_accepted, cudaMemcpyDeviceToHost) != cudaSuccess) {
    printf("CUDA error: copy back failed\n");
    return 1;
  }
  const float wm = (float)wmax;
  uint64_t recount = 0;
  for (uint64_t p = 0; p < n; ++p) {
    const float uu = (float)(words[4 * p + 3] >> 8) * (1.f / 16777216.f);
    recount += uu * wm < w[p] ? 1 : 0;
  }
  std::vector<uint32_t> pts(u.n_accepted);
  for (uint64_t i = 0; i < u.n_accepted; ++i) pts[i] = rec[i].point;
  // strictly increasing: distinct points, in the point order of the reference's selection
  const bool distinct = std::adjacent_find(pts.begin(), pts.end(), [](uint32_t a, uint32_t b) { return b <= a; }) == pts.end();
  const uint64_t diff = u.n_accepted > recount ? u.n_accepted - recount : recount - u.n_accepted;
  printf("On-device compaction of accepted events (%llu candidates, w_max = q99.9 = %.4e mb)\n",
         (unsigned long long)n, wmax);
  printf("  accepted (compacted) = %llu   independent recount = %llu   records in point order: %s\n",
         (unsigned long long)u.n_accepted, (unsigned long long)recount, distinct ? "yes" : "no");
  printf("  production pass %.2f ms  (%.3e candidates/s, %.3e records/s)\n", drv_ms(t0, t1),
         n / (drv_ms(t0, t1) / 1e3), u.n_accepted / (drv_ms(t0, t1) / 1e3));
  const bool ok = distinct && u.n_accepted > 0 && diff <= std::max<uint64_t>(2, n / 100000);
  printf("VALIDATION: %s (compacted count == independent count, records in point order)\n", ok ? "PASS" : "FAIL");
  cudaFree(d_rec);
  cudaFree(d_w);
  cudaFree(d_words);
  cp_destroy(h);
  return ok ? 0 : 2;
}
