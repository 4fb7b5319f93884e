// cp_api.cu -- handles, errors, the counter-RNG surface, the batched SigmaProcess surface and
// the partonic gg -> gg kernels.
#include <math.h>
#include <string.h>
#include "cp_internal.cuh"

int cp_had_launch_shape(cp_handle* h);

// ------------------------------------------------------------------------------------------
// errors and scratch
// ------------------------------------------------------------------------------------------
int cp_fail(cp_handle* h, int code, const std::string& msg)
{
  if (h) h->err = msg;
  return code;
}

int cp_fail_cuda(cp_handle* h, cudaError_t e, const char* what)
{
  if (h) h->err = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? CP_ERR_NOMEM : CP_ERR_CUDA;
}

int cp_ensure_slots(cp_handle* h, size_t doubles)
{
  if (doubles <= h->slots_cap) return CP_OK;
  if (h->d_slots) {
    CP_CUDA(h, cudaStreamSynchronize(h->stream));
    CP_CUDA(h, cudaFree(h->d_slots));
    h->d_slots = nullptr;
  }
  CP_CUDA(h, cudaMalloc(&h->d_slots, doubles * sizeof(double)));
  h->slots_cap = doubles;
  return CP_OK;
}

int cp_ensure_iters(cp_handle* h, int n)
{
  if (n <= h->iters_cap) return CP_OK;
  if (h->d_iters) {
    CP_CUDA(h, cudaStreamSynchronize(h->stream));
    CP_CUDA(h, cudaFree(h->d_iters));
    h->d_iters = nullptr;
  }
  CP_CUDA(h, cudaMalloc(&h->d_iters, sizeof(CpIterDev) * (size_t)n));
  h->iters_cap = n;
  return CP_OK;
}

static int ensure_kin(cp_handle* h, int64_t n)
{
  if (n <= h->kin_cap) return CP_OK;
  float** bufs[8] = {&h->d_x1, &h->d_x2, &h->d_sH, &h->d_tH, &h->d_uH, &h->d_as, &h->d_q2r, &h->d_q2f};
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  for (auto b : bufs) {
    if (*b) CP_CUDA(h, cudaFree(*b));
    *b = nullptr;
  }
  for (auto b : bufs) CP_CUDA(h, cudaMalloc(b, sizeof(float) * (size_t)n));
  h->kin_cap = n;
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// handles
// ------------------------------------------------------------------------------------------
extern "C" int cp_abi_version(void) { return CP_ABI_VERSION; }

extern "C" int cp_config_default(cp_config* c)
{
  if (!c) return CP_ERR_INVALID;
  memset(c, 0, sizeof *c);
  c->sqrt_s = 13000.0;
  c->pt_hat_min = 20.0;
  c->alphas_mz = 0.13;
  c->k_ren = 1.0;
  c->k_fac = 1.0;
  c->convert2mb = 0.389380;
  c->n_quark_in = 5;
  c->n_quark_new = 3;
  c->proc_mask = CP_PROC_ALL;
  c->n_bins = 50;
  c->device = 0;
  c->seed = 42;
  return CP_OK;
}

static int apply_config(cp_handle* h, const cp_config* c)
{
  if (c->n_bins < 2 || c->n_bins > CP_MAX_BINS)
    return cp_fail(h, CP_ERR_INVALID, "n_bins must be in [2, 128]");
  if ((c->proc_mask & ~CP_PROC_ALL) || c->proc_mask == 0)
    return cp_fail(h, CP_ERR_INVALID, "proc_mask must be a nonzero OR of CP_PROC_*");
  CpHadConfig hc{c->sqrt_s, c->pt_hat_min, c->alphas_mz, c->k_ren, c->k_fac, c->convert2mb,
                 c->n_quark_in, c->n_quark_new, c->proc_mask};
  if (cp_build_had_params(hc, h->P))
    return cp_fail(h, CP_ERR_INVALID,
                   "unsupported configuration (need pT_hat_min >= 2 GeV, 2 pT_hat_min < sqrt_s, "
                   "0.05 < alphas_mz < 0.3, positive scale factors, n_quark_in == 5)");
  h->cfg = *c;
  h->nb = c->n_bins;
  return CP_OK;
}

extern "C" int cp_create(const cp_config* cfg, cp_handle** out)
{
  if (!out) return CP_ERR_INVALID;
  *out = nullptr;
  cp_config def;
  cp_config_default(&def);
  if (!cfg) cfg = &def;
  cp_handle* h = new cp_handle();
  int rc = apply_config(h, cfg);
  if (rc) { delete h; return rc; }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) { delete h; return CP_ERR_CUDA; }
  if (cfg->device < 0 || cfg->device >= ndev) { delete h; return CP_ERR_INVALID; }
  h->device = cfg->device;
  CpDeviceGuard guard(h->device);
  int cur = -1;
  if (cudaGetDevice(&cur) != cudaSuccess || cur != h->device) { delete h; return CP_ERR_CUDA; }
  cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device);
  bool ok = cudaMalloc(&h->d_edges, sizeof(double) * 3 * (CP_MAX_BINS + 1)) == cudaSuccess &&
            cudaMalloc(&h->d_red, sizeof(double) * (CP_SLOT_HEAD + 3 * CP_MAX_BINS)) == cudaSuccess &&
            cudaMalloc(&h->d_qhist, sizeof(unsigned long long) * CP_QBINS) == cudaSuccess &&
            cudaMalloc(&h->d_wmax, sizeof(double) * 2) == cudaSuccess &&
            cudaMalloc(&h->d_counter, sizeof(unsigned long long) * 2) == cudaSuccess &&
            cudaMemset(h->d_wmax, 0, sizeof(double) * 2) == cudaSuccess &&
            cudaMalloc(&h->d_cteq, sizeof(CpCteqPoly) * 8) == cudaSuccess &&
            cudaMemcpy(h->d_cteq, h->P.cteq, sizeof(CpCteqPoly) * 8, cudaMemcpyHostToDevice) == cudaSuccess;
  if (!ok || cp_had_launch_shape(h) != CP_OK || cp_ensure_iters(h, 16) != CP_OK) {
    cp_destroy(h);
    return CP_ERR_NOMEM;
  }
  rc = cp_grid_reset(h);
  if (rc) { cp_destroy(h); return rc; }
  *out = h;
  return CP_OK;
}

extern "C" int cp_destroy(cp_handle* h)
{
  if (!h) return CP_OK;
  CpDeviceGuard guard(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  if (h->gen_copy) cudaStreamSynchronize(h->gen_copy);
  for (cudaEvent_t e : h->tpool) cudaEventDestroy(e);
  for (int k = 0; k < CP_GEN_BUFS; ++k) {
    if (h->gen_counted[k]) cudaEventDestroy(h->gen_counted[k]);
    if (h->gen_copied[k]) cudaEventDestroy(h->gen_copied[k]);
  }
  if (h->gen_copy) cudaStreamDestroy(h->gen_copy);
  if (h->h_gen_cnt) cudaFreeHost(h->h_gen_cnt);
  void* bufs[] = {h->d_edges, h->d_slots, h->d_red, h->d_iters, h->d_x1, h->d_x2, h->d_sH,
                  h->d_tH, h->d_uH, h->d_as, h->d_q2r, h->d_q2f, h->d_qhist, h->d_wmax, h->d_counter, h->d_cteq, h->d_flow, h->d_flow_pk,
                  h->d_flow_bias, h->d_flow_buf, h->d_flow_tc, h->d_flow_status, h->d_flow_ticket, h->d_pdfbuf,
                  h->d_gen_stage, h->d_gen_red, h->d_gen_cnt, h->d_ftrain, h->d_tails, h->d_bmask,
                  h->d_rsum, h->d_roff, h->d_unw_red};
  for (void* b : bufs)
    if (b) cudaFree(b);
  delete h;
  return CP_OK;
}

extern "C" const char* cp_last_error(const cp_handle* h) { return h ? h->err.c_str() : "null handle"; }

// Offset of this handle's point indices (cuPythia/common/rng.cuh:5-19: shard i of M points per
// shard works on the global points [i M, i M + count)); every pass then draws the Philox block of
// global point offset + p, so shards are disjoint and their union is the single-device run.
extern "C" int cp_set_point_offset(cp_handle* h, uint64_t offset)
{
  CP_CHECK_HANDLE(h);
  h->point_offset = offset;
  return CP_OK;
}

extern "C" int cp_set_stream(cp_handle* h, void* s)
{
  CP_CHECK_HANDLE(h);
  h->stream = (cudaStream_t)s;
  return CP_OK;
}

extern "C" int cp_synchronize(cp_handle* h)
{
  CP_CHECK_HANDLE(h);
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_device_sm_count(cp_handle* h, int* n)
{
  CP_CHECK_HANDLE(h);
  if (!n) return CP_ERR_INVALID;
  *n = h->num_sms;
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// grid
// ------------------------------------------------------------------------------------------
extern "C" int cp_grid_reset(cp_handle* h)
{
  CP_CHECK_HANDLE(h);
  double e[3 * (CP_MAX_BINS + 1)];
  for (int d = 0; d < 3; ++d)
    for (int k = 0; k <= h->nb; ++k) e[d * (h->nb + 1) + k] = (double)k / (double)h->nb;
  return cp_grid_set(h, e);
}

extern "C" int cp_grid_set(cp_handle* h, const double* e)
{
  CP_CHECK_HANDLE(h);
  if (!e) return cp_fail(h, CP_ERR_INVALID, "cp_grid_set: null edges");
  const int nb = h->nb;
  for (int d = 0; d < 3; ++d) {
    const double* ed = e + d * (nb + 1);
    if (ed[0] != 0.0 || ed[nb] != 1.0) return cp_fail(h, CP_ERR_INVALID, "grid must span [0, 1]");
    for (int k = 0; k < nb; ++k)
      if (!(ed[k + 1] > ed[k])) return cp_fail(h, CP_ERR_INVALID, "grid edges must increase");
  }
  CP_CUDA(h, cudaMemcpyAsync(h->d_edges, e, sizeof(double) * 3 * (nb + 1), cudaMemcpyHostToDevice,
                             h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_grid_get(cp_handle* h, double* e)
{
  CP_CHECK_HANDLE(h);
  if (!e) return cp_fail(h, CP_ERR_INVALID, "cp_grid_get: null edges");
  CP_CUDA(h, cudaMemcpyAsync(e, h->d_edges, sizeof(double) * 3 * (h->nb + 1), cudaMemcpyDeviceToHost,
                             h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// counter RNG surface
// ------------------------------------------------------------------------------------------
__global__ void k_philox_words(uint64_t seed, uint64_t p0, uint64_t n, uint32_t iter, uint32_t stream,
                               uint4* out)
{
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t w[4];
    cp_point_words(seed, p0 + i, iter, stream, w);
    out[i] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

__device__ __forceinline__ double cp_u01(uint64_t u) { return (double)(u >> 11) * (1.0 / 9007199254740992.0); }

__global__ void k_splitmix(uint64_t seed, uint64_t nthr, uint64_t kper, double* out)
{
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nthr;
       t += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t ctr = seed + t * 0x100000001B3ULL;
    for (uint64_t i = 0; i < kper; ++i) out[t * kper + i] = cp_u01(cp_splitmix64(ctr++));
  }
}

__global__ void k_event_keys(uint64_t base, uint64_t e0, uint64_t n, uint64_t* out)
{
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = cp_splitmix64(base ^ ((e0 + i) * 0x9E3779B97F4A7C15ULL));
}

static int grid_for(cp_handle* h, uint64_t n)
{
  uint64_t b = (n + 255) / 256;
  uint64_t cap = (uint64_t)h->num_sms * 32;
  return (int)(b < cap ? (b > 0 ? b : 1) : cap);
}

extern "C" int cp_philox_words(cp_handle* h, uint64_t seed, uint64_t p0, uint64_t n, uint32_t iter,
                               uint32_t stream, uint32_t* out)
{
  CP_CHECK_HANDLE(h);
  if (n && !out) return cp_fail(h, CP_ERR_INVALID, "cp_philox_words: null output");
  if (((uintptr_t)out & 15) != 0) return cp_fail(h, CP_ERR_INVALID, "cp_philox_words: output must be 16-byte aligned");
  if (!n) return CP_OK;
  k_philox_words<<<grid_for(h, n), 256, 0, h->stream>>>(seed, p0, n, iter, stream, (uint4*)out);
  CP_LAUNCH_CHECK(h, "k_philox_words");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_splitmix_uniforms(cp_handle* h, uint64_t seed, uint64_t nthr, uint64_t kper, double* out)
{
  CP_CHECK_HANDLE(h);
  if (nthr && kper && !out) return cp_fail(h, CP_ERR_INVALID, "cp_splitmix_uniforms: null output");
  if (!nthr || !kper) return CP_OK;
  k_splitmix<<<grid_for(h, nthr), 256, 0, h->stream>>>(seed, nthr, kper, out);
  CP_LAUNCH_CHECK(h, "k_splitmix");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_event_keys(cp_handle* h, uint64_t base, uint64_t e0, uint64_t n, uint64_t* out)
{
  CP_CHECK_HANDLE(h);
  if (n && !out) return cp_fail(h, CP_ERR_INVALID, "cp_event_keys: null output");
  if (!n) return CP_OK;
  k_event_keys<<<grid_for(h, n), 256, 0, h->stream>>>(base, e0, n, out);
  CP_LAUNCH_CHECK(h, "k_event_keys");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// SigmaProcess surface
// ------------------------------------------------------------------------------------------
__global__ void k_set2kin(const CpHadParams P, int64_t n, const float* __restrict__ sH,
                          const float* __restrict__ tH, float* uH, float* as, float* q2r, float* q2f)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float s = sH[i], t = tH[i], u = -(s + t);
    float pT2 = t * u / s;
    float qr = P.kR * pT2, qf = P.kF * pT2;
    uH[i] = u;
    q2r[i] = qr;
    q2f[i] = qf;
    as[i] = cp_alphas(P, qr);
  }
}

// The same from FP64 kinematics (what Pythia's set2Kin receives): uHat = -(sHat + tHat) and
// pT^2 = tHat uHat / sHat are formed in FP64 and only then rounded, so a small |uHat| (a large
// sHat near the pT cut, where the FP32 sum of sHat and tHat would cancel) keeps its precision.
__global__ void k_set2kin_f64(const CpHadParams P, int64_t n, const double* __restrict__ x1d,
                              const double* __restrict__ x2d, const double* __restrict__ sHd,
                              const double* __restrict__ tHd, float* x1, float* x2, float* sH, float* tH,
                              float* uH, float* as, float* q2r, float* q2f)
{
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double s = sHd[i], t = tHd[i], u = -(s + t);
    const float pT2 = (float)(t * u / s);
    const float qr = P.kR * pT2, qf = P.kF * pT2;
    x1[i] = (float)x1d[i];
    x2[i] = (float)x2d[i];
    sH[i] = (float)s;
    tH[i] = (float)t;
    uH[i] = (float)u;
    q2r[i] = qr;
    q2f[i] = qf;
    as[i] = cp_alphas(P, qr);
  }
}

// which: 0 = sigmaKin of code (flavour independent), 1 = sigmaHat(id1, id2), 2 = sigmaPDF(mask)
__global__ void k_sigma(const CpHadParams P, const CpCteqPoly* cteq_g, int64_t n, int which, int code,
                        int id1, int id2, int mask, const float* __restrict__ x1,
                        const float* __restrict__ x2, const float* __restrict__ sH,
                        const float* __restrict__ tH, const float* __restrict__ uH,
                        const float* __restrict__ as, const float* __restrict__ q2f, float* out)
{
  __shared__ CpCteqPoly cteq[8];
  cp_stage_cteq(cteq, cteq_g);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float s = sH[i], t = tH[i], u = uH[i];
    float tp = t / s, up = u / s;
    CpBrackets b;
    cp_brackets(P, tp, up, b);
    float a = as[i];
    float pref = CP_PI_F * (a * a) / (s * s);   // dsigma/dtHat = pref * bracket
    float v;
    if (which == 2) {
      float m[5];
      for (int k = 0; k < 5; ++k) m[k] = (mask >> k) & 1 ? 1.f : 0.f;
      float fa[8], fb[8];
      cp_cteq_pair<1>(cteq, q2f[i], logf(x1[i]), 0.f, logf(x2[i]), 0.f, fa, fb);
      v = P.conv * pref * cp_channel_sum(m, b, fa, fb);
    } else {
      float br = 0.f;
      if (code == 111) br = b.gg2gg;
      else if (code == 112) br = b.gg2qqbar;
      else if (code == 113) br = b.qg2qg;
      else if (code == 115) br = b.qqbar2gg;
      else if (code == 114) {
        if (id2 == id1) br = 0.5f * (b.qqT + b.qqU + b.qqTU);
        else if (id2 == -id1) br = b.qqT + b.qqST;
        else br = b.qqT;
      }
      v = pref * br;
    }
    out[i] = v;
  }
}

// pickInState + setIdColAcol of one process over the stored batch: per point the uniforms
// r = (pair, new flavour, colour topology, gg -> gg orientation); PDFs at Q2Fac of the batch.
__global__ void k_pick_state(const CpHadParams P, const CpCteqPoly* cteq_g, int64_t n, int k,
                             const float* __restrict__ x1, const float* __restrict__ x2,
                             const float* __restrict__ sH, const float* __restrict__ tH,
                             const float* __restrict__ uH, const float* __restrict__ q2f,
                             const float4* __restrict__ r,
                             short4* __restrict__ ids, uint16_t* __restrict__ colour)
{
  __shared__ CpCteqPoly cteq[8];
  cp_stage_cteq(cteq, cteq_g);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float s = sH[i], t = tH[i], u = uH[i];
    const float tp = t / s, up = u / s;
    CpPoint pt;
    cp_brackets(P, tp, up, pt.b);
    cp_cteq_pair<1>(cteq, q2f[i], logf(x1[i]), 0.f, logf(x2[i]), 0.f, pt.fa, pt.fb);
    const float4 ri = r[i];
    int id[4];
    cp_pick_pair(P, k, pt, ri.x, ri.y, id);
    ids[i] = make_short4((short)id[0], (short)id[1], (short)id[2], (short)id[3]);
    colour[i] = (uint16_t)cp_colour_flow(111 + k, id, tp, up, ri.z, ri.w);
  }
}

__global__ void k_pdf(const CpCteqPoly* cteq_g, int64_t n, const float* __restrict__ x,
                      const float* __restrict__ q2, float* out)
{
  __shared__ CpCteqPoly cteq[8];
  cp_stage_cteq(cteq, cteq_g);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float f[8], g[8];
    float lx = logf(x[i]);
    cp_cteq_pair<1>(cteq, q2[i], lx, 0.f, lx, 0.f, f, g);
    // id order -5..-1, 1..5, 21; f = {d, u, g, ubar, dbar, s, c, b}
    float* o = out + 11 * i;
    o[0] = f[7]; o[1] = f[6]; o[2] = f[5]; o[3] = f[3]; o[4] = f[4];
    o[5] = f[0]; o[6] = f[1]; o[7] = f[5]; o[8] = f[6]; o[9] = f[7]; o[10] = f[2];
  }
}

extern "C" int cp_set2kin_batch(cp_handle* h, const float* x1, const float* x2, const float* sH,
                                const float* tH, int64_t n)
{
  CP_CHECK_HANDLE(h);
  if (n < 0 || (n > 0 && (!x1 || !x2 || !sH || !tH)))
    return cp_fail(h, CP_ERR_INVALID, "cp_set2kin_batch: bad arguments");
  int rc = ensure_kin(h, n > 0 ? n : 1);
  if (rc) return rc;
  h->kin_n = n;
  if (!n) return CP_OK;
  size_t bytes = sizeof(float) * (size_t)n;
  CP_CUDA(h, cudaMemcpyAsync(h->d_x1, x1, bytes, cudaMemcpyDeviceToDevice, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(h->d_x2, x2, bytes, cudaMemcpyDeviceToDevice, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(h->d_sH, sH, bytes, cudaMemcpyDeviceToDevice, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(h->d_tH, tH, bytes, cudaMemcpyDeviceToDevice, h->stream));
  k_set2kin<<<grid_for(h, n), 256, 0, h->stream>>>(h->P, n, h->d_sH, h->d_tH, h->d_uH, h->d_as, h->d_q2r, h->d_q2f);
  CP_LAUNCH_CHECK(h, "k_set2kin");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_set2kin_batch_f64(cp_handle* h, const double* x1, const double* x2, const double* sH,
                                    const double* tH, int64_t n)
{
  CP_CHECK_HANDLE(h);
  if (n < 0 || (n > 0 && (!x1 || !x2 || !sH || !tH)))
    return cp_fail(h, CP_ERR_INVALID, "cp_set2kin_batch_f64: bad arguments");
  int rc = ensure_kin(h, n > 0 ? n : 1);
  if (rc) return rc;
  h->kin_n = n;
  if (!n) return CP_OK;
  k_set2kin_f64<<<grid_for(h, n), 256, 0, h->stream>>>(h->P, n, x1, x2, sH, tH, h->d_x1, h->d_x2, h->d_sH, h->d_tH,
                                                       h->d_uH, h->d_as, h->d_q2r, h->d_q2f);
  CP_LAUNCH_CHECK(h, "k_set2kin_f64");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

static int sigma_launch(cp_handle* h, int which, int code, int id1, int id2, int mask, float* out)
{
  if (h->kin_n == 0) return CP_OK;
  if (!out) return cp_fail(h, CP_ERR_INVALID, "null output");
  k_sigma<<<grid_for(h, h->kin_n), 256, 0, h->stream>>>(h->P, h->d_cteq, h->kin_n, which, code, id1, id2, mask,
                                                         h->d_x1, h->d_x2, h->d_sH, h->d_tH, h->d_uH,
                                                         h->d_as, h->d_q2f, out);
  CP_LAUNCH_CHECK(h, "k_sigma");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_sigma_kin_batch(cp_handle* h, int code, float* out)
{
  CP_CHECK_HANDLE(h);
  if (code != 111 && code != 112 && code != 113 && code != 115)
    return cp_fail(h, CP_ERR_INVALID,
                   "cp_sigma_kin_batch: codes 111, 112, 113, 115 (114 depends on the flavour pair: "
                   "use cp_sigma_hat_batch)");
  return sigma_launch(h, 0, code, 0, 0, 0, out);
}

extern "C" int cp_sigma_hat_batch(cp_handle* h, int code, int id1, int id2, float* out)
{
  CP_CHECK_HANDLE(h);
  if (code < 111 || code > 115) return cp_fail(h, CP_ERR_INVALID, "cp_sigma_hat_batch: code 111..115");
  return sigma_launch(h, 1, code, id1, id2, 0, out);
}

extern "C" int cp_sigma_pdf_batch(cp_handle* h, int mask, float* out)
{
  CP_CHECK_HANDLE(h);
  if ((mask & ~CP_PROC_ALL) || !mask) return cp_fail(h, CP_ERR_INVALID, "cp_sigma_pdf_batch: bad mask");
  return sigma_launch(h, 2, 0, 0, 0, mask, out);
}

extern "C" int cp_pick_state_batch(cp_handle* h, int code, const float* r_dev, int16_t* ids_dev, uint16_t* colour_dev)
{
  CP_CHECK_HANDLE(h);
  if (code < 111 || code > 115) return cp_fail(h, CP_ERR_INVALID, "cp_pick_state_batch: code 111..115");
  if (!h->kin_n) return CP_OK;
  if (!r_dev || !ids_dev || !colour_dev || ((uintptr_t)r_dev & 15) || ((uintptr_t)ids_dev & 7))
    return cp_fail(h, CP_ERR_INVALID, "cp_pick_state_batch: r (16-byte aligned) and ids (8-byte aligned) required");
  k_pick_state<<<grid_for(h, h->kin_n), 256, 0, h->stream>>>(h->P, h->d_cteq, h->kin_n, code - 111, h->d_x1, h->d_x2,
                                                             h->d_sH, h->d_tH, h->d_uH, h->d_q2f,
                                                             reinterpret_cast<const float4*>(r_dev),
                                                             reinterpret_cast<short4*>(ids_dev), colour_dev);
  CP_LAUNCH_CHECK(h, "k_pick_state");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_scales_batch(cp_handle* h, float* as, float* q2r, float* q2f)
{
  CP_CHECK_HANDLE(h);
  size_t bytes = sizeof(float) * (size_t)h->kin_n;
  if (!h->kin_n) return CP_OK;
  if (as) CP_CUDA(h, cudaMemcpyAsync(as, h->d_as, bytes, cudaMemcpyDeviceToDevice, h->stream));
  if (q2r) CP_CUDA(h, cudaMemcpyAsync(q2r, h->d_q2r, bytes, cudaMemcpyDeviceToDevice, h->stream));
  if (q2f) CP_CUDA(h, cudaMemcpyAsync(q2f, h->d_q2f, bytes, cudaMemcpyDeviceToDevice, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_pdf_batch(cp_handle* h, const float* x, const float* q2, int64_t n, float* out)
{
  CP_CHECK_HANDLE(h);
  if (n < 0 || (n > 0 && (!x || !q2 || !out))) return cp_fail(h, CP_ERR_INVALID, "cp_pdf_batch: bad arguments");
  if (!n) return CP_OK;
  k_pdf<<<grid_for(h, n), 256, 0, h->stream>>>(h->d_cteq, n, x, q2, out);
  CP_LAUNCH_CHECK(h, "k_pdf");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// partonic gg -> gg, FP64 (cuPythia/03_fused_resident_me/fused_gg2gg.cu:28-51)
// ------------------------------------------------------------------------------------------
struct PartonicArgs {
  double s, aS, cMax, scale;  // scale = (2 cMax)(s/2) conv
  uint64_t seed, p0, n;       // Philox mode: points; SplitMix mode: reference threads
  uint64_t kper;              // SplitMix mode: draws per reference thread
  double* slots;              // gridDim.x * 4
  double* w_out;
};

// Sigma2gg2gg::sigmaKin (pythia8317/src/SigmaQCD.cc:115-129; pipeline/physics.cuh:9-16) for a fixed
// s-hat.  With s + t + u = 0 the three brackets sigTS + sigUS + sigTU sum to
// (9/2) (3 - t u / s^2 - s u / t^2 - s t / u^2), the textbook form of the g g -> g g matrix element,
// which takes one FP64 reciprocal (of t u; 1/t = u / (t u), 1/u = t / (t u)) and about half the
// operations of the bracket form.  With u = -s - t rounded as the reference rounds it, the two
// forms agree to 1.1e-15 relative over |cos theta| < 0.9.  The prefactor (pi / s^2) alpha_s^2 / 2
// is the same for every draw and is formed once.
struct CpGG2GG {
  double s, is2, pre, cMax;
  __device__ __forceinline__ CpGG2GG(double s_, double aS, double cMax_) : s(s_), cMax(cMax_)
  {
    const double is = 1.0 / s;
    is2 = is * is;
    pre = M_PI * is * is * (aS * aS) * 0.5 * 4.5;
  }
  // dsigma/dt at cos theta = (2 u01 - 1) cMax
  __device__ __forceinline__ double operator()(double u01) const
  {
    const double c = (2.0 * u01 - 1.0) * cMax;
    const double tH = -0.5 * s * (1.0 - c), uH = -s - tH;
    const double tu = tH * uH, itu = 1.0 / tu;
    const double it = uH * itu, iu = tH * itu;
    return pre * (3.0 - tu * is2 - (s * uH) * (it * it) - (s * tH) * (iu * iu));
  }
};

__device__ __forceinline__ double cp_philox_u01_d(uint64_t seed, uint64_t point)
{
  uint32_t wd[4];
  cp_point_words(seed, point, 0, 0, wd);
  const uint64_t v = ((uint64_t)wd[1] << 32) | wd[0];
  return (double)(v >> 11) * (1.0 / 9007199254740992.0);
}

// MODE 0: Philox sums over points; 1: SplitMix64 sums over the reference's (thread, draw) pairs;
// 2: Philox per-point weights.  Sums are of dsigma/dt; each block scales its slot by `scale`.
template <int MODE>
__global__ void __launch_bounds__(CP_THREADS, 5) k_partonic(const PartonicArgs a)
{
  __shared__ double sRed[CP_WARPS][3];
  const CpGG2GG f(a.s, a.aS, a.cMax);
  double s1 = 0.0, s2 = 0.0, wm = 0.0;
  const uint64_t nthr = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t t = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
  if (MODE == 1) {
    // the reference's thread i makes draws k = 0 .. kper-1 from counter seed + i 0x100000001B3 + k
    // (cuPythia/03_fused_resident_me/fused_gg2gg.cu:43-50); the n kper pairs are split into
    // equal contiguous shares, so every thread here does the same number of draws
    const uint64_t total = a.n * a.kper, q = total / nthr, rem = total % nthr;
    const uint64_t w0 = q * t + (t < rem ? t : rem), cnt = q + (t < rem ? 1 : 0);
    uint64_t i = w0 / a.kper, k = w0 - i * a.kper;
    uint64_t ctr = a.seed + i * 0x100000001B3ULL + k;
    for (uint64_t w = 0; w < cnt; ++w) {
      const double v = f(cp_u01(cp_splitmix64(ctr)));
      s1 += v; s2 += v * v; wm = fmax(wm, v);
      if (++k == a.kper) { k = 0; ++i; ctr = a.seed + i * 0x100000001B3ULL; }
      else ++ctr;
    }
  } else {
    for (uint64_t i = t; i < a.n; i += nthr) {
      const double v = f(cp_philox_u01_d(a.seed, a.p0 + i));
      if (MODE == 2) { a.w_out[i] = v * a.scale; continue; }
      s1 += v; s2 += v * v; wm = fmax(wm, v);
    }
  }
  if (MODE == 2) return;
  s1 = cp_warp_sum_d(s1);
  s2 = cp_warp_sum_d(s2);
  wm = cp_warp_max_d(wm);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { sRed[warp][0] = s1; sRed[warp][1] = s2; sRed[warp][2] = wm; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b1 = 0, b2 = 0, bm = 0;
    for (int k = 0; k < CP_WARPS; ++k) { b1 += sRed[k][0]; b2 += sRed[k][1]; bm = fmax(bm, sRed[k][2]); }
    double* slot = a.slots + 4 * (size_t)blockIdx.x;
    slot[0] = b1 * a.scale; slot[1] = b2 * (a.scale * a.scale); slot[2] = bm * a.scale; slot[3] = 0.0;
  }
}

static int partonic_run(cp_handle* h, int mode, PartonicArgs a, uint64_t npoints, cp_result* out)
{
  if (!(a.s > 0) || !(a.cMax > 0) || !(a.cMax < 1)) return cp_fail(h, CP_ERR_INVALID, "partonic: bad kinematics");
  // one wave of resident blocks: the per-thread shares are equal, so nothing waits on a tail
  int per_sm = 0;
  const cudaError_t oe = mode == 0 ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_partonic<0>, CP_THREADS, 0)
                                   : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_partonic<1>, CP_THREADS, 0);
  if (oe != cudaSuccess || per_sm < 1) per_sm = 4;
  const int blocks = h->num_sms * per_sm;
  int rc = cp_ensure_slots(h, (size_t)blocks * 4);
  if (rc) return rc;
  a.slots = h->d_slots;
  if (mode == 0) k_partonic<0><<<blocks, CP_THREADS, 0, h->stream>>>(a);
  else k_partonic<1><<<blocks, CP_THREADS, 0, h->stream>>>(a);
  CP_LAUNCH_CHECK(h, "k_partonic");
  k_reduce_slots<0><<<1, 4 * 32, 0, h->stream>>>(h->d_slots, blocks, 4, h->d_red);
  CP_LAUNCH_CHECK(h, "k_reduce_slots");
  double red[4];
  CP_CUDA(h, cudaMemcpyAsync(red, h->d_red, sizeof red, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (out) {
    double n = (double)npoints, mean = red[0] / n, var = (red[1] / n - mean * mean) / (n - 1.0);
    out->sigma = mean;
    out->sigma_err = sqrt(var > 0 ? var : 0);
    out->sum_w = red[0]; out->sum_w2 = red[1]; out->w_max = red[2];
    out->n_points = npoints; out->n_bad = 0;
    out->eta = red[2] > 0 ? mean / red[2] : 0;
  }
  return CP_OK;
}

extern "C" int cp_partonic_integrate(cp_handle* h, double sqrt_shat, double alphas, double cmax,
                                     double conv, uint64_t seed, uint64_t n, cp_result* out)
{
  CP_CHECK_HANDLE(h);
  if (n < 2) return cp_fail(h, CP_ERR_INVALID, "n_points < 2");
  double s = sqrt_shat * sqrt_shat;
  PartonicArgs a{s, alphas, cmax, (2.0 * cmax) * (s / 2.0) * conv, seed, 0, n, 0, nullptr, nullptr};
  return partonic_run(h, 0, a, n, out);
}

extern "C" int cp_partonic_splitmix(cp_handle* h, double sqrt_shat, double alphas, double cmax,
                                    double conv, uint64_t seed, uint64_t nthr, uint64_t kper,
                                    cp_result* out)
{
  CP_CHECK_HANDLE(h);
  if (kper && nthr > UINT64_MAX / kper) return cp_fail(h, CP_ERR_INVALID, "too many draws");
  if (nthr * kper < 2) return cp_fail(h, CP_ERR_INVALID, "too few draws");
  double s = sqrt_shat * sqrt_shat;
  PartonicArgs a{s, alphas, cmax, (2.0 * cmax) * (s / 2.0) * conv, seed, 0, nthr, kper, nullptr, nullptr};
  return partonic_run(h, 1, a, nthr * kper, out);
}

extern "C" int cp_partonic_weights(cp_handle* h, double sqrt_shat, double alphas, double cmax,
                                   double conv, uint64_t seed, uint64_t p0, uint64_t n, double* w)
{
  CP_CHECK_HANDLE(h);
  if (n && !w) return cp_fail(h, CP_ERR_INVALID, "null output");
  if (!n) return CP_OK;
  double s = sqrt_shat * sqrt_shat;
  PartonicArgs a{s, alphas, cmax, (2.0 * cmax) * (s / 2.0) * conv, seed, p0, n, 0, nullptr, w};
  k_partonic<2><<<grid_for(h, n), CP_THREADS, 0, h->stream>>>(a);
  CP_LAUNCH_CHECK(h, "k_partonic");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}
