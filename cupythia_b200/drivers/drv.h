// drv.h -- shared plumbing of the stage drivers: C-ABI error checks with the reference's exit
// codes (1 on a CUDA/library error, 2 on a failed validation, 0 on success), the shard offset
// of the reference's multi-GPU launcher, wall-clock timing and the fixed gg -> gg quadrature.
#pragma once
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include "../../include/cupythia_b200.h"

#define DRV_CK(h, call)                                                                    \
  do {                                                                                     \
    const int rc_ = (call);                                                                \
    if (rc_ != CP_OK) {                                                                    \
      printf("cupythia_b200 error %d in %s: %s\n", rc_, #call, (h) ? cp_last_error(h) : ""); \
      return 1;                                                                            \
    }                                                                                      \
  } while (0)

// CUPYTHIA_SHARD (this process's index i) x CUPYTHIA_SHARD_N (points per shard), 0 when unset
// (cuPythia/common/rng.cuh:14-19)
static inline uint64_t drv_shard_offset()
{
  const char* si = getenv("CUPYTHIA_SHARD");
  const char* sn = getenv("CUPYTHIA_SHARD_N");
  if (!si || !sn) return 0;
  return (uint64_t)strtoull(si, nullptr, 10) * (uint64_t)strtoull(sn, nullptr, 10);
}

static inline uint64_t drv_arg(int argc, char** argv, int i, uint64_t dflt)
{
  return argc > i ? strtoull(argv[i], nullptr, 10) : dflt;
}

using DrvClock = std::chrono::steady_clock;
static inline double drv_ms(DrvClock::time_point a, DrvClock::time_point b)
{
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// Pythia Sigma2gg2gg::sigmaKin (pythia8317/src/SigmaQCD.cc:115-129) at fixed sHat, as the weight
// of cos(theta) (dt/dcos = sHat / 2), integrated by Simpson's rule over |cos| < cMax: the
// deterministic reference value of the partonic drivers (cuPythia/03_fused_resident_me/
// fused_gg2gg.cu:65-74).  Returns GeV^-2 x conv.
static inline double drv_simpson_gg2gg(int n, double sqrtShat, double alpS, double cMax, double conv)
{
  const double sH = sqrtShat * sqrtShat;
  auto dsig = [&](double c) {
    const double tH = -0.5 * sH * (1.0 - c), uH = -sH - tH;
    const double a = tH / sH, b = uH / sH, d = tH / uH;
    auto br = [](double r) { return r * r + 2.0 * r + 3.0 + 2.0 / r + 1.0 / (r * r); };
    return (M_PI / (sH * sH)) * alpS * alpS * 0.5 * (9.0 / 4.0) * (br(a) + br(b) + br(d)) * 0.5 * sH;
  };
  const double h = 2.0 * cMax / n;
  double s = 0.0;
  for (int i = 0; i <= n; ++i) {
    const double w = (i == 0 || i == n) ? 1.0 : (i % 2 ? 4.0 : 2.0);
    s += w * dsig(-cMax + i * h);
  }
  return s * h / 3.0 * conv;
}
