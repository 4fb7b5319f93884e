// CpSigmaQCD.cc -- the Pythia 8 plug-in of the HardQCD 2 -> 2 processes over the cupythia_b200
// C ABI (see CpSigmaQCD.h).
#include "CpSigmaQCD.h"

#include <cuda_runtime.h>

namespace cupythia {

CpContext::~CpContext()
{
  if (d_) cudaFree(d_);
  if (h_) cp_destroy(h_);
}

bool CpContext::configure(Pythia8::Settings& s, std::string& why)
{
  if (tried_) {
    why = why_;
    return h_ != nullptr;
  }
  tried_ = true;
  if (s.mode("SigmaProcess:alphaSorder") != 1) why_ = "SigmaProcess:alphaSorder must be 1 (first-order running)";
  else if (s.mode("StandardModel:alphaSnfmax") != 6) why_ = "StandardModel:alphaSnfmax must be 6";
  else if (s.mode("SigmaProcess:renormScale2") >= 4 || s.mode("SigmaProcess:factorScale2") >= 4)
    why_ = "SigmaProcess:renormScale2 and factorScale2 must choose pT^2 (values 1..3) for massless 2 -> 2";
  else if (s.mode("PDFinProcess:nQuarkIn") != 5) why_ = "PDFinProcess:nQuarkIn must be 5";
  if (!why_.empty()) {
    why = why_;
    return false;
  }
  cp_config_default(&cfg_);
  cfg_.sqrt_s = s.parm("Beams:eCM");
  cfg_.pt_hat_min = s.parm("PhaseSpace:pTHatMin");
  cfg_.alphas_mz = s.parm("SigmaProcess:alphaSvalue");
  cfg_.k_ren = s.parm("SigmaProcess:renormMultFac");
  cfg_.k_fac = s.parm("SigmaProcess:factorMultFac");
  cfg_.n_quark_new = s.mode("HardQCD:nQuarkNew");
  cfg_.device = device_;
  // the library checks pT_hat_min >= 2 GeV for its phase-space map, which this path does not use
  if (cfg_.pt_hat_min < 2.0) cfg_.pt_hat_min = 2.0;
  cp_handle* h = nullptr;
  int rc = cp_create(&cfg_, &h);
  if (rc != CP_OK) {
    why_ = "cp_create failed (status " + std::to_string(rc) + ")";
  } else if (cudaSetDevice(device_) != cudaSuccess || cudaMalloc(&d_, 6 * sizeof(double)) != cudaSuccess) {
    why_ = "device buffer allocation failed";
    cp_destroy(h);
  } else {
    h_ = h;
  }
  why = why_;
  return h_ != nullptr;
}

bool CpContext::sigma(int code, double x1, double x2, double sH, double tH, double out[3])
{
  if (!h_) return false;
  ++calls_;
  const double in[4] = {x1, x2, sH, tH};
  float res[3] = {0.f, 0.f, 0.f};
  float* out_dev = reinterpret_cast<float*>(d_ + 4);
  if (cudaMemcpy(d_, in, sizeof in, cudaMemcpyHostToDevice) != cudaSuccess) return false;
  if (cp_set2kin_batch_f64(h_, d_, d_ + 1, d_ + 2, d_ + 3, 1) != CP_OK) return false;
  if (code == 114) {
    if (cp_sigma_hat_batch(h_, 114, 1, 1, out_dev) != CP_OK || cp_sigma_hat_batch(h_, 114, 1, -1, out_dev + 1) != CP_OK ||
        cp_sigma_hat_batch(h_, 114, 1, 2, out_dev + 2) != CP_OK)
      return false;
  } else if (cp_sigma_kin_batch(h_, code, out_dev) != CP_OK) {
    return false;
  }
  if (cudaMemcpy(res, out_dev, sizeof res, cudaMemcpyDeviceToHost) != cudaSuccess) return false;
  for (int k = 0; k < 3; ++k) out[k] = res[k];
  return true;
}

void CpSigma2QCD::initProc()
{
  std::string why;
  if (!ctx_->configure(*settingsPtr, why))
    loggerPtr->errorMsg("CpSigma2QCD::initProc", "cupythia_b200 plug-in unavailable", why, true);
}

void CpSigma2QCD::sigmaKin()
{
  // g g -> q qbar draws its new flavour here (Sigma2gg2qqbar::sigmaKin, SigmaQCD.cc:168-172)
  if (code_ == 112) rFlavour_ = rndmPtr->flat();
  if (!ctx_->sigma(code_, x1Save, x2Save, sH, tH, sig_)) {
    sig_[0] = sig_[1] = sig_[2] = 0.;
    loggerPtr->errorMsg("CpSigma2QCD::sigmaKin", "cupythia_b200 call failed; cross section set to zero");
  }
}

double CpSigma2QCD::sigmaHat()
{
  if (code_ != 114) return sig_[0];
  // Sigma2qq2qq::sigmaHat (SigmaQCD.cc:272-286): identical quarks, quark-antiquark of one
  // flavour, or different flavours
  return id2 == id1 ? sig_[0] : (id2 == -id1 ? sig_[1] : sig_[2]);
}

void CpSigma2QCD::setIdColAcol()
{
  // Pythia's draws, in the order and number of the stock setIdColAcol
  double rColour = 0., rSwap = 0.;
  if (code_ == 111) {
    rColour = rndmPtr->flat();
    rSwap = rndmPtr->flat();
  } else if (code_ == 114) {
    if (id2 == id1) rColour = rndmPtr->flat();
  } else {
    rColour = rndmPtr->flat();
  }
  int ids[4], col[4], acol[4];
  if (cp_set_id_col_acol(code_, id1, id2, tH / sH, uH / sH, ctx_->nQuarkNew(), rFlavour_, rColour, rSwap, ids, col,
                         acol) != CP_OK) {
    loggerPtr->errorMsg("CpSigma2QCD::setIdColAcol", "cupythia_b200 rejected the incoming pair");
    setId(id1, id2, id1, id2);
    setColAcol();
    return;
  }
  setId(ids[0], ids[1], ids[2], ids[3]);
  setColAcol(col[0], acol[0], col[1], acol[1], col[2], acol[2], col[3], acol[3]);
}

std::string CpSigma2QCD::name() const
{
  switch (code_) {
    case 111: return "g g -> g g";
    case 112: return "g g -> q qbar (uds)";
    case 113: return "q g -> q g";
    case 114: return "q q(bar)' -> q q(bar)'";
    default: return "q qbar -> g g";
  }
}

std::string CpSigma2QCD::inFlux() const
{
  switch (code_) {
    case 111: case 112: return "gg";
    case 113: return "qg";
    case 114: return "qq";
    default: return "qqbarSame";
  }
}

std::shared_ptr<CpContext> addHardQCD(Pythia8::Pythia& pythia, int device,
                                      std::vector<std::shared_ptr<CpSigma2QCD>>* procs)
{
  auto ctx = std::make_shared<CpContext>(device);
  for (int code = 111; code <= 115; ++code) {
    auto p = std::make_shared<CpSigma2QCD>(code, ctx);
    pythia.addSigmaPtr(p);
    if (procs) procs->push_back(p);
  }
  return ctx;
}

}  // namespace cupythia
