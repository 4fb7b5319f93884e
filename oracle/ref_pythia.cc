// ref_pythia.cc -- driver over the reference's own Pythia 8.317 code (built by oracle/ref.mk).
//
// TEST INFRASTRUCTURE ONLY: it produces golden vectors for the oracle and is the timed CPU
// reference arm of bench.py.  It calls stock Pythia through its public API:
//   pdf    <x> <Q2> ...                 CTEQ5L xf for ids -5..5, 21   (PDF::xf, PartonDistributions.cc:122)
//   alphas <aSmZ> <Q2> ...              first-order AlphaStrong       (StandardModel.cc:42-252)
//   sigma  <file>                       per process set2Kin + sigmaKin + sigmaPDF on lines
//                                       "x1 x2 sH tH"                (SigmaProcess.cc:423-480,846-925)
//   gen    <nAccepted> <seed> <threads> [pTmin] [aSmZ]
//                                       ProcessLevel-only HardQCD generation, one Pythia per thread,
//                                       prints tried/accepted, the seconds of generation alone
//                                       (after every thread's init), the init seconds, sigmaGen +- sigmaErr
//   lhef   <file> [shower]              reads a Les Houches Event File back (Beams:frameType = 4);
//                                       with shower = 1 also showers (MPI off) and hadronizes every
//                                       event, which needs a valid colour flow; prints counts and
//                                       the largest total four-momentum imbalance
// Settings follow the hadronic dijet configuration: pp at 13 TeV, HardQCD gg2gg, qg2qg,
// qqbar2gg, gg2qqbar, qq2qq on, PhaseSpace:pTHatMin = 20, PDF:pSet = 2 (CTEQ5L),
// SigmaProcess:alphaSvalue = 0.13 at first order, parton and hadron levels off.
#include "Pythia8/Pythia.h"
#include "Pythia8/SigmaQCD.h"
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <thread>
#include <vector>
#include <unistd.h>
#include <libgen.h>
#include <climits>

using namespace Pythia8;

static std::string xmlDir()
{
  const char* env = getenv("CP_PYTHIA_XMLDOC");
  if (env) return env;
  char buf[PATH_MAX];
  ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  if (n <= 0) return "xmldoc";
  buf[n] = 0;
  return std::string(dirname(buf)) + "/xmldoc";
}

static void configure(Pythia& p, double pTmin, double aSmZ, bool processes, int seed)
{
  p.readString("Beams:idA = 2212");
  p.readString("Beams:idB = 2212");
  p.readString("Beams:eCM = 13000.");
  if (processes) {
    p.readString("HardQCD:gg2gg = on");
    p.readString("HardQCD:qg2qg = on");
    p.readString("HardQCD:qqbar2gg = on");
    p.readString("HardQCD:gg2qqbar = on");
    p.readString("HardQCD:qq2qq = on");
  }
  p.readString("PhaseSpace:pTHatMin = " + std::to_string(pTmin));
  p.readString("PDF:pSet = 2");
  p.readString("SigmaProcess:alphaSvalue = " + std::to_string(aSmZ));
  p.readString("SigmaProcess:alphaSorder = 1");
  p.readString("PartonLevel:all = off");
  p.readString("HadronLevel:all = off");
  p.readString("Next:numberCount = 0");
  p.readString("Print:quiet = on");
  p.readString("Random:setSeed = on");
  p.readString("Random:seed = " + std::to_string(seed));
}

static int cmd_pdf(int argc, char** argv)
{
  CTEQ5L pdf(2212);
  for (int i = 0; i + 1 < argc; i += 2) {
    double x = atof(argv[i]), Q2 = atof(argv[i + 1]);
    printf("%.17g %.17g", x, Q2);
    const int ids[11] = {-5, -4, -3, -2, -1, 1, 2, 3, 4, 5, 21};
    for (int k = 0; k < 11; ++k) printf(" %.17g", pdf.xf(ids[k], x, Q2));
    printf("\n");
  }
  return 0;
}

static int cmd_alphas(int argc, char** argv)
{
  AlphaStrong a;
  a.init(atof(argv[0]), 1, 6, false);
  for (int i = 1; i < argc; ++i) printf("%.17g %.17g\n", atof(argv[i]), a.alphaS(atof(argv[i])));
  return 0;
}

static int cmd_sigma(const char* path)
{
  Pythia p(xmlDir(), false);
  configure(p, 20.0, 0.13, false, 1);
  std::vector<SigmaProcessPtr> procs = {
      std::make_shared<Sigma2gg2gg>(), std::make_shared<Sigma2gg2qqbar>(),
      std::make_shared<Sigma2qg2qg>(), std::make_shared<Sigma2qq2qq>(),
      std::make_shared<Sigma2qqbar2gg>()};
  for (auto& s : procs) p.addSigmaPtr(s);
  if (!p.init()) { fprintf(stderr, "pythia init failed\n"); return 1; }
  std::ifstream in(path);
  double x1, x2, sH, tH;
  while (in >> x1 >> x2 >> sH >> tH) {
    printf("%.17g %.17g %.17g %.17g", x1, x2, sH, tH);
    for (auto& s : procs) {
      s->set2Kin(x1, x2, sH, tH, 0., 0., 1., 1.);
      double sp = s->sigmaPDF();
      printf(" %.17g", sp);
    }
    printf(" %.17g %.17g\n", procs[0]->alphaSRen(), procs[0]->Q2Ren());
  }
  return 0;
}

struct GenResult { long tried = 0, accepted = 0; double sigma = 0, err = 0; };

// Every worker constructs and initialises its own Pythia (including the sigma_max scan of
// PhaseSpace::setupSampling), then waits until all workers are ready; the clock runs only around
// the Pythia::next() loops, so the timed region is event generation alone, as on the GPU side
// (where adaptation and training are outside the timed region too).  The initialisation time is
// reported separately ("init_seconds", the slowest worker's).
static int cmd_gen(long nAcc, int seed, int threads, double pTmin, double aSmZ)
{
  std::vector<GenResult> res(threads);
  std::vector<double> initT(threads, 0.0);
  std::mutex mu;
  std::condition_variable cv;
  int ready = 0;
  bool go = false;
  auto worker = [&](int t) {
    const auto i0 = std::chrono::steady_clock::now();
    Pythia p(xmlDir(), false);
    configure(p, pTmin, aSmZ, true, seed + t);
    const bool ok = p.init();
    initT[t] = std::chrono::duration<double>(std::chrono::steady_clock::now() - i0).count();
    {
      std::unique_lock<std::mutex> lock(mu);
      ++ready;
      cv.notify_all();
      cv.wait(lock, [&] { return go; });
    }
    if (!ok) return;
    long per = nAcc / threads + (t < nAcc % threads ? 1 : 0);
    for (long i = 0; i < per; ++i) p.next();
    res[t].tried = p.info.nTried();
    res[t].accepted = p.info.nAccepted();
    res[t].sigma = p.info.sigmaGen();
    res[t].err = p.info.sigmaErr();
  };
  std::vector<std::thread> th;
  for (int t = 0; t < threads; ++t) th.emplace_back(worker, t);
  std::chrono::steady_clock::time_point t0;
  {
    std::unique_lock<std::mutex> lock(mu);
    cv.wait(lock, [&] { return ready == threads; });
    t0 = std::chrono::steady_clock::now();
    go = true;
  }
  cv.notify_all();
  for (auto& x : th) x.join();
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  long tried = 0, acc = 0;
  double wsum = 0, w2 = 0, initMax = 0;
  for (int t = 0; t < threads; ++t) {
    const GenResult& r = res[t];
    tried += r.tried;
    acc += r.accepted;
    if (r.err > 0) { wsum += r.sigma / (r.err * r.err); w2 += 1.0 / (r.err * r.err); }
    if (initT[t] > initMax) initMax = initT[t];
  }
  double sig = w2 > 0 ? wsum / w2 : 0, err = w2 > 0 ? 1.0 / sqrt(w2) : 0;
  printf("{\"tried\": %ld, \"accepted\": %ld, \"seconds\": %.6f, \"init_seconds\": %.6f, \"threads\": %d, "
         "\"sigma_mb\": %.8g, \"sigma_err_mb\": %.8g}\n",
         tried, acc, sec, initMax, threads, sig, err);
  return 0;
}

static int cmd_lhef(const char* path, int shower)
{
  Pythia p(xmlDir(), false);
  p.readString("Beams:frameType = 4");
  p.settings.word("Beams:LHEF", path);
  p.readString("PDF:pSet = 2");
  if (shower) {
    p.readString("PartonLevel:MPI = off");
  } else {
    p.readString("PartonLevel:all = off");
    p.readString("HadronLevel:all = off");
  }
  p.readString("Next:numberCount = 0");
  if (!getenv("CP_PYTHIA_VERBOSE")) p.readString("Print:quiet = on");
  if (!p.init()) {
    printf("{\"init\": false}\n");
    return 2;
  }
  const double eTot = p.info.eA() + p.info.eB();
  long nOk = 0, nAbort = 0, nCode[5] = {0, 0, 0, 0, 0};
  double maxImb = 0.0;
  for (;;) {
    if (!p.next()) {
      if (p.info.atEndOfFile()) break;
      if (++nAbort > 1000) break;
      continue;
    }
    ++nOk;
    const int code = p.info.codeSub();
    if (code >= 111 && code <= 115) ++nCode[code - 111];
    double px = 0, py = 0, pz = 0, e = 0;
    const Event& ev = shower ? p.event : p.process;
    for (int i = 0; i < ev.size(); ++i)
      if (ev[i].isFinal()) { px += ev[i].px(); py += ev[i].py(); pz += ev[i].pz(); e += ev[i].e(); }
    double imb = fabs(px) + fabs(py) + (shower ? fabs(pz) + fabs(e - eTot) : 0.0);
    if (imb > maxImb) maxImb = imb;
  }
  printf("{\"init\": true, \"read\": %ld, \"aborted\": %ld, \"max_imbalance_gev\": %.6g, "
         "\"by_code\": [%ld, %ld, %ld, %ld, %ld], \"sigma_gen_mb\": %.8g, \"e_cm\": %.8g}\n",
         nOk, nAbort, maxImb, nCode[0], nCode[1], nCode[2], nCode[3], nCode[4], p.info.sigmaGen(), eTot);
  return 0;
}

int main(int argc, char** argv)
{
  if (argc < 2) { fprintf(stderr, "usage: pythia_ref pdf|alphas|sigma|gen ...\n"); return 1; }
  if (!strcmp(argv[1], "pdf")) return cmd_pdf(argc - 2, argv + 2);
  if (!strcmp(argv[1], "alphas")) return cmd_alphas(argc - 2, argv + 2);
  if (!strcmp(argv[1], "sigma") && argc > 2) return cmd_sigma(argv[2]);
  if (!strcmp(argv[1], "lhef") && argc > 2) return cmd_lhef(argv[2], argc > 3 ? atoi(argv[3]) : 0);
  if (!strcmp(argv[1], "gen") && argc > 4)
    return cmd_gen(atol(argv[2]), atoi(argv[3]), atoi(argv[4]), argc > 5 ? atof(argv[5]) : 20.0,
                   argc > 6 ? atof(argv[6]) : 0.13);
  fprintf(stderr, "bad arguments\n");
  return 1;
}
