// CpSigmaQCD.h -- Pythia 8 plug-in: the five HardQCD 2 -> 2 processes with their matrix elements
// evaluated by the cupythia_b200 library through its C ABI (include/cupythia_b200.h).
//
// Each class derives from Pythia8::Sigma2Process and carries the name(), code() and inFlux() of
// the stock process it replaces (pythia8317/include/Pythia8/SigmaQCD.h:188-352):
//   111 g g -> g g (gg), 112 g g -> q qbar (uds) (gg), 113 q g -> q g (qg),
//   114 q q(bar)' -> q q(bar)' (qq), 115 q qbar -> g g (qqbarSame).
// Pythia keeps everything around the matrix element: phase-space sampling, its own PDFs in
// sigmaPDF, pickInState, the sigma_max bookkeeping and the event record.  Per trial,
// set2Kin -> store2Kin (Pythia) -> sigmaKin() sends (x1, x2, sHat, tHat) to the library at
// Pythia's FP64 (cp_set2kin_batch_f64: uHat, pT^2, scales, first-order alpha_s) and receives dsigmaHat/dtHat
// (cp_sigma_kin_batch; for 114 the three flavour cases of sigmaHat(id1, id2) from
// cp_sigma_hat_batch), which sigmaHat() returns for the pair Pythia asks for.  setIdColAcol()
// calls the library's cp_set_id_col_acol with Pythia's own random numbers, drawn where the stock
// classes draw them (pythia8317/src/SigmaQCD.cc:135-342), so a run consumes Pythia's random
// stream exactly as the stock processes do.
//
// A batch of one point per call: this is the drop-in path for a Pythia program, one GPU round
// trip per trial; the batched entry points of the library are the throughput path.
//
// Usage (HardQCD processes of the stock library switched off):
//   Pythia8::Pythia pythia;
//   pythia.readString("HardQCD:all = off");
//   auto ctx = cupythia::addHardQCD(pythia);     // five processes sharing one library handle
//   pythia.init();  ...  pythia.next();
#ifndef CUPYTHIA_B200_CP_SIGMA_QCD_H
#define CUPYTHIA_B200_CP_SIGMA_QCD_H

#include <memory>
#include <string>
#include <vector>

#include "Pythia8/Pythia.h"
#include "Pythia8/SigmaProcess.h"
#include "cupythia_b200.h"

namespace cupythia {

// The library handle shared by the processes of one Pythia instance, with a one-point device
// batch.  Configured once, from the Pythia settings, by the first process whose initProc runs.
class CpContext {
 public:
  explicit CpContext(int device = 0) : device_(device) {}
  ~CpContext();
  CpContext(const CpContext&) = delete;
  CpContext& operator=(const CpContext&) = delete;

  // Reads the settings the library depends on; false (with the reason in why) for settings it
  // does not cover: SigmaProcess:alphaSorder != 1, StandardModel:alphaSnfmax != 6, scale choices
  // other than pT^2 for massless 2 -> 2 (renormScale2, factorScale2 >= 4), PDFinProcess:nQuarkIn
  // != 5, or a CUDA / library failure.
  bool configure(Pythia8::Settings& settings, std::string& why);
  bool ready() const { return h_ != nullptr; }
  // dsigmaHat/dtHat (GeV^-4) of process `code` at (x1, x2, sHat, tHat); for 114 the three cases
  // (id2 == id1, id2 == -id1, other); false on a library error.
  bool sigma(int code, double x1, double x2, double sH, double tH, double out[3]);
  int nQuarkNew() const { return cfg_.n_quark_new; }
  long calls() const { return calls_; }

 private:
  int device_;
  cp_config cfg_{};
  cp_handle* h_ = nullptr;
  double* d_ = nullptr;  // device: x1, x2, sH, tH (FP64), then the three FP32 outputs
  bool tried_ = false;
  std::string why_;
  long calls_ = 0;
};

class CpSigma2QCD : public Pythia8::Sigma2Process {
 public:
  CpSigma2QCD(int code, std::shared_ptr<CpContext> ctx) : code_(code), ctx_(std::move(ctx)) {}

  void initProc() override;
  // Pythia's channel set-up of inFlux(); false (Pythia's init fails) when the library could not
  // be configured, with the reason in Pythia's log
  bool initFlux() override { return ctx_->ready() && Sigma2Process::initFlux(); }
  void sigmaKin() override;
  double sigmaHat() override;
  void setIdColAcol() override;

  std::string name() const override;
  int code() const override { return code_; }
  std::string inFlux() const override;

 private:
  int code_;
  std::shared_ptr<CpContext> ctx_;
  double sig_[3] = {0., 0., 0.};
  double rFlavour_ = 0.;   // g g -> q qbar: the new flavour's draw, taken in sigmaKin as Pythia does
};

// Adds the five processes (codes 111 .. 115) to `pythia` with addSigmaPtr, sharing one context
// on CUDA device `device`; returns the context (its calls() counts the library round trips) and,
// with `procs`, the five process objects in code order.
std::shared_ptr<CpContext> addHardQCD(Pythia8::Pythia& pythia, int device = 0,
                                      std::vector<std::shared_ptr<CpSigma2QCD>>* procs = nullptr);

}  // namespace cupythia

#endif
