// pythia_plugin_check.cc -- test program of the Pythia plug-in (cupythia_b200/pythia/CpSigmaQCD.*)
// against stock Pythia 8.317 (built from the reference's sources by oracle/ref.mk).  Run by
// tests/test_gpu_pythia_plugin.py on a GPU; prints one JSON line per mode.
//   sigma <n> <seed>   n random massless 2 -> 2 points with pT > 20 GeV at 13 TeV: set2Kin on the
//                      stock Sigma2* object and on the plug-in process of the same code, then
//                      sigmaHatWrap for the incoming pairs the process accepts; largest relative
//                      difference per process
//   gen <nAcc> <seed>  ProcessLevel generation of nAcc events with the stock HardQCD processes,
//                      then with the plug-in (HardQCD:all = off, cupythia::addHardQCD), same seed;
//                      sigmaGen +- sigmaErr, tries and seconds of each, the plug-in's library calls
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "CpSigmaQCD.h"
#include "Pythia8/Pythia.h"
#include "Pythia8/SigmaQCD.h"

using namespace Pythia8;

static const char* xmldoc()
{
  const char* e = getenv("CP_PYTHIA_XMLDOC");
  return e ? e : "oracle/_ref/xmldoc";
}

static void settings(Pythia& p, bool stock, int seed)
{
  p.readString("Beams:idA = 2212");
  p.readString("Beams:idB = 2212");
  p.readString("Beams:eCM = 13000.");
  if (stock) {
    p.readString("HardQCD:gg2gg = on");
    p.readString("HardQCD:qg2qg = on");
    p.readString("HardQCD:qqbar2gg = on");
    p.readString("HardQCD:gg2qqbar = on");
    p.readString("HardQCD:qq2qq = on");
  } else {
    p.readString("HardQCD:all = off");
  }
  p.readString("PhaseSpace:pTHatMin = 20.");
  p.readString("PDF:pSet = 2");
  p.readString("SigmaProcess:alphaSvalue = 0.13");
  p.readString("SigmaProcess:alphaSorder = 1");
  p.readString("PartonLevel:all = off");
  p.readString("HadronLevel:all = off");
  p.readString("Next:numberCount = 0");
  p.readString("Print:quiet = on");
  p.readString("Random:setSeed = on");
  p.readString("Random:seed = " + std::to_string(seed));
}

static int cmd_sigma(int n, int seed)
{
  Pythia ps(xmldoc(), false), pc(xmldoc(), false);
  settings(ps, false, seed);
  settings(pc, false, seed);
  std::vector<SigmaProcessPtr> stock = {std::make_shared<Sigma2gg2gg>(), std::make_shared<Sigma2gg2qqbar>(),
                                        std::make_shared<Sigma2qg2qg>(), std::make_shared<Sigma2qq2qq>(),
                                        std::make_shared<Sigma2qqbar2gg>()};
  for (auto& s : stock) ps.addSigmaPtr(s);
  std::vector<std::shared_ptr<cupythia::CpSigma2QCD>> plug;
  auto ctx = cupythia::addHardQCD(pc, 0, &plug);
  if (!ps.init() || !pc.init()) {
    printf("{\"init\": false}\n");
    return 2;
  }
  // incoming pairs per process (Pythia ids)
  const std::vector<std::vector<std::pair<int, int>>> pairs = {
      {{21, 21}}, {{21, 21}}, {{2, 21}, {21, -1}, {-5, 21}},
      {{2, 2}, {2, -2}, {1, 2}, {-3, -3}, {-1, 4}, {5, -3}}, {{1, -1}, {-2, 2}}};
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(0.0, 1.0);
  const double s = 13000.0 * 13000.0, pTmin = 20.0;
  double worst[5] = {0, 0, 0, 0, 0};
  long npts = 0;
  for (int i = 0; i < n; ++i) {
    // tau log-uniform above (2 pTmin)^2 / s, y inside its range, cos theta inside the pT cut
    const double tauMin = 4.0 * pTmin * pTmin / s;
    const double tau = tauMin * std::pow(1.0 / tauMin, U(rng));
    const double yMax = -0.5 * std::log(tau), y = yMax * (2.0 * U(rng) - 1.0);
    const double sH = tau * s, zMax = std::sqrt(1.0 - 4.0 * pTmin * pTmin / sH);
    const double z = zMax * (2.0 * U(rng) - 1.0), tH = -0.5 * sH * (1.0 - z);
    const double x1 = std::sqrt(tau) * std::exp(y), x2 = std::sqrt(tau) * std::exp(-y);
    if (x1 >= 1.0 || x2 >= 1.0) continue;
    ++npts;
    for (int k = 0; k < 5; ++k) {
      stock[k]->set2Kin(x1, x2, sH, tH, 0., 0., 1., 1.);
      plug[k]->set2Kin(x1, x2, sH, tH, 0., 0., 1., 1.);
      for (auto& pr : pairs[k]) {
        const double a = stock[k]->sigmaHatWrap(pr.first, pr.second);
        const double b = plug[k]->sigmaHatWrap(pr.first, pr.second);
        const double r = std::fabs(b - a) / std::fabs(a);
        if (r > worst[k]) worst[k] = r;
      }
    }
  }
  printf("{\"points\": %ld, \"calls\": %ld, \"max_rel\": [%.3e, %.3e, %.3e, %.3e, %.3e]}\n", npts, ctx->calls(),
         worst[0], worst[1], worst[2], worst[3], worst[4]);
  return 0;
}

static int cmd_gen(long nAcc, int seed)
{
  double sig[2], err[2], sec[2];
  long tried[2], acc[2], calls = 0;
  for (int pass = 0; pass < 2; ++pass) {
    Pythia p(xmldoc(), false);
    settings(p, pass == 0, seed);
    std::shared_ptr<cupythia::CpContext> ctx;
    if (pass == 1) ctx = cupythia::addHardQCD(p, 0);
    if (!p.init()) {
      printf("{\"init\": false, \"pass\": %d}\n", pass);
      return 2;
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (long i = 0; i < nAcc; ++i) p.next();
    sec[pass] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    sig[pass] = p.info.sigmaGen();
    err[pass] = p.info.sigmaErr();
    tried[pass] = p.info.nTried();
    acc[pass] = p.info.nAccepted();
    if (ctx) calls = ctx->calls();
  }
  printf("{\"stock\": {\"sigma_mb\": %.9g, \"sigma_err_mb\": %.4g, \"tried\": %ld, \"accepted\": %ld, \"seconds\": %.3f}, "
         "\"plugin\": {\"sigma_mb\": %.9g, \"sigma_err_mb\": %.4g, \"tried\": %ld, \"accepted\": %ld, \"seconds\": %.3f, "
         "\"library_calls\": %ld}}\n",
         sig[0], err[0], tried[0], acc[0], sec[0], sig[1], err[1], tried[1], acc[1], sec[1], calls);
  return 0;
}

int main(int argc, char** argv)
{
  if (argc >= 4 && !strcmp(argv[1], "sigma")) return cmd_sigma(atoi(argv[2]), atoi(argv[3]));
  if (argc >= 4 && !strcmp(argv[1], "gen")) return cmd_gen(atol(argv[2]), atoi(argv[3]));
  fprintf(stderr, "usage: pythia_plugin_check sigma <n> <seed> | gen <nAccepted> <seed>\n");
  return 1;
}
