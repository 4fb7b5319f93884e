// ref_cupythia.cc -- compiles the reference's own host/device headers as plain C++ so the
// oracle can be checked against them bit for bit (built by oracle/ref.mk into oracle/_ref/).
//
// TEST INFRASTRUCTURE ONLY.  Exposes, through a C ABI:
//   splitmix64, u01                 cuPythia/common/rng.cuh:47-57
//   gg2gg_sigma                     cuPythia/pipeline/physics.cuh:9-16
//   the CPU Monte-Carlo loop of the fused gg->gg stage, on those same functions
//   (cuPythia/03_fused_resident_me/fused_gg2gg.cu:53-62, per-thread counters of :43-46)
#define __host__
#define __device__
#include <cstdint>
#include <thread>
#include <vector>
#include "common/rng.cuh"
#include "pipeline/physics.cuh"

extern "C" {
uint64_t ref_splitmix64(uint64_t x) { return splitmix64(x); }
double ref_u01(uint64_t u) { return u01(u); }
double ref_gg2gg_sigma(double sH, double tH, double uH, double aS) { return gg2gg_sigma(sH, tH, uH, aS); }

// Sum of dsigma/dtHat over threads [t0, t1) of the reference's per-thread stream layout,
// kPer trials per thread; returns the plain sum (the stage multiplies by 2 cMax s/2 / N).
static double thread_range_sum(uint64_t seed, uint64_t t0, uint64_t t1, uint64_t kPer, double s,
                               double aS, double cMax)
{
  double sum = 0.0;
  for (uint64_t tid = t0; tid < t1; ++tid) {
    uint64_t ctr = seed + tid * 0x100000001B3ULL;
    double local = 0.0;
    for (uint64_t i = 0; i < kPer; ++i) {
      double c = (2.0 * u01(splitmix64(ctr++)) - 1.0) * cMax;
      double t = -0.5 * s * (1.0 - c);
      local += gg2gg_sigma(s, t, -s - t, aS);
    }
    sum += local;
  }
  return sum;
}

// Multi-threaded over disjoint thread ranges; partial sums combined in a fixed order.
double ref_fused_cpu_sum(uint64_t seed, uint64_t nThreads, uint64_t kPer, double s, double aS,
                         double cMax, int workers)
{
  if (workers < 1) workers = 1;
  std::vector<double> part(workers, 0.0);
  std::vector<std::thread> th;
  uint64_t per = nThreads / workers, rem = nThreads % workers, off = 0;
  for (int w = 0; w < workers; ++w) {
    uint64_t n = per + ((uint64_t)w < rem ? 1 : 0);
    th.emplace_back([&, w, off, n] { part[w] = thread_range_sum(seed, off, off + n, kPer, s, aS, cMax); });
    off += n;
  }
  double sum = 0.0;
  for (int w = 0; w < workers; ++w) { th[w].join(); sum += part[w]; }
  return sum;
}

// Sequential-counter CPU loop exactly as the stage's cpuMC (fused_gg2gg.cu:53-62), in GeV^-2.
double ref_cpuMC(uint64_t seed, uint64_t total, double s, double aS, double cMax)
{
  uint64_t ctr = seed;
  double sum = 0.0;
  for (uint64_t i = 0; i < total; ++i) {
    double c = (2.0 * u01(splitmix64(ctr++)) - 1.0) * cMax;
    double t = -0.5 * s * (1.0 - c);
    sum += gg2gg_sigma(s, t, -s - t, aS);
  }
  return (2.0 * cMax) * (s / 2.0) * (sum / (double)total);
}
}
