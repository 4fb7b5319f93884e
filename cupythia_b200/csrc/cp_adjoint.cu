// cp_adjoint.cu -- gradients of the VEGAS estimator: d sigma and d Var[w] with respect to the
// 3 x (n_bins + 1) grid edges, alpha_s(mZ), the renormalisation-scale factor and the pT_hat cut.
// The reference has no derivative code; this is the added adjoint of the integrator.
//
// Each point is evaluated once in forward mode with 6 tangents (x0, x1, x2, alpha_s(mZ), k_ren,
// pT_hat_min) over the same counter draws as the forward pass, so the result is the exact
// derivative of the estimator at fixed random numbers (common random numbers).  With
// w = f(x(u; e); theta) * prod_d nb (e_{d,b+1} - e_{d,b}) and x_d = e_{d,b} + frac_d (e_{d,b+1} - e_{d,b}):
//   dw/de_{d,b}   = -w / Delta_d + (df/dx_d) J (1 - frac_d)
//   dw/de_{d,b+1} =  w / Delta_d + (df/dx_d) J frac_d
// accumulated per bin (lower- and upper-edge parts, plain and w-weighted) in deterministic
// warp-private shared-memory histograms, then FP64 block slots, then the fixed-order reduction.
// sigma = <w>, Var = <w^2> - <w>^2, d sigma = <dw>, d Var = 2 <w dw> - 2 <w> <dw>.
// With a moment order p != 2 (cp_vegas_gradient_objective) the same pass gives the gradient of
// the relative p-th moment R_p = <w^p> / <w>^p instead: w^(p-1) takes the place of w in the
// weighted sums, and the record's var entry becomes (R_p - 1) sigma^2, so var / sigma^2 is
// R_p - 1 (for p = 2 the relative variance, as before).
#include <vector>
#include "cp_dual.cuh"
#include "cp_internal.cuh"

#define CP_ADJ_THREADS 128
#define CP_ADJ_WARPS (CP_ADJ_THREADS / 32)
#define CP_ADJ_HEAD 10   // sum w, sum w^2, sum dw[3], sum w dw[3], max w, n_bad

struct AdjLaunch {
  uint64_t seed, point0, n;
  uint32_t iter, stream;
  int nb;
  const double* edges;
  const CpCteqPoly* cteq;
  double* slots;            // gridDim.x * (CP_ADJ_HEAD + 12 nb)
  float lnTauMin, dlnTauMin_dpt;   // ln tauMin and its pT_hat_min derivative 2 / pTmin
  float lnL2[4], dlnL2_da[4];      // ln Lambda_nf^2 and d/d alpha_s(mZ) = 12 pi / (b0 alpha_s(mZ)^2)
  float pm1;                       // moment order - 1 (1: the variance)
};

// NT = 6: tangents x0, x1, x2, alpha_s(mZ), k_ren, pT_hat_min; NT = 3: the x tangents only (the
// edge gradients and the sums of w are the same bit for bit, since tangents never mix; the
// parameter sums stay zero)
template <int NT>
__global__ void __launch_bounds__(CP_ADJ_THREADS) k_adjoint(const CpHadParams P, const AdjLaunch L)
{
  typedef CpDual<NT> D6;
  extern __shared__ float sDyn[];   // [warp][dim][4][nb]: lo, hi, w*lo, w*hi
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  __shared__ CpCteqPoly sCteq[8];
  __shared__ double sRed[CP_ADJ_WARPS][CP_ADJ_HEAD];
  const int nb = L.nb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < 3 * nb; k += CP_ADJ_THREADS) {
    int d = k / nb, b = k - d * nb;
    const double* e = L.edges + d * (nb + 1);
    sEdge[d][b] = make_float2((float)e[b], (float)(e[b + 1] - e[b]));
  }
  cp_stage_cteq(sCteq, L.cteq);
  for (int k = threadIdx.x; k < CP_ADJ_WARPS * 12 * nb; k += CP_ADJ_THREADS) sDyn[k] = 0.f;
  __syncthreads();

  CpHadParamsT<D6> Q;
  Q.lnTauMin = cp_dconst<NT>(L.lnTauMin);
  Q.kR = cp_dconst<NT>(P.kR);
  for (int k = 0; k < 4; ++k) Q.lnL2[k] = cp_dconst<NT>(L.lnL2[k]);
  if constexpr (NT == 6) {
    Q.lnTauMin.d[5] = L.dlnTauMin_dpt;
    Q.kR.d[4] = 1.f;
    for (int k = 0; k < 4; ++k) Q.lnL2[k].d[3] = L.dlnL2_da[k];
  }

  const float nbf = (float)nb;
  const uint64_t stride = (uint64_t)gridDim.x * CP_ADJ_THREADS;
  const uint64_t gtid = (uint64_t)blockIdx.x * CP_ADJ_THREADS + threadIdx.x;
  const uint64_t rounds = (L.n + stride - 1) / stride;
  float acc[8], cmp[8];
  for (int k = 0; k < 8; ++k) { acc[k] = 0.f; cmp[k] = 0.f; }
  float wmax = 0.f;
  uint32_t nbad = 0;
  float* my = sDyn + warp * 12 * nb;

  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t p = r * stride + gtid;
    int bin[3] = {0, 0, 0};
    float dlo[3] = {0.f, 0.f, 0.f}, dhi[3] = {0.f, 0.f, 0.f};
    float w = 0.f, wq = 0.f;   // the weight and w^(p-1)
    if (p < L.n) {
      uint32_t wd[4];
      cp_point_words(L.seed, L.point0 + p, L.iter, L.stream, wd);
      float x[3], frac[3], width[3], jv = 1.f;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        cp_bin_frac(wd[d], nb, bin[d], frac[d]);
        float2 e = sEdge[d][bin[d]];
        x[d] = fmaf(frac[d], e.y, e.x);
        width[d] = e.y;
        jv *= nbf * e.y;
      }
      D6 wb = cp_had_weight_t<D6>(P, Q, sCteq, cp_dvar<NT>(x[0], 0), cp_dvar<NT>(x[1], 1),
                                  cp_dvar<NT>(x[2], 2));
      w = wb.v * jv;
      bool ok = (w >= 0.f) && !isinf(w);
#pragma unroll
      for (int k = 0; k < NT; ++k) ok = ok && isfinite(wb.d[k]);
      if (!ok) {
        ++nbad;
        w = 0.f;
      } else {
        float dth[3] = {0.f, 0.f, 0.f};
        if constexpr (NT == 6) {
          dth[0] = wb.d[3] * jv;
          dth[1] = wb.d[4] * jv;
          dth[2] = wb.d[5] * jv;
        }
        wq = L.pm1 == 1.f ? w : powf(w, L.pm1);
        cp_kahan(acc[0], cmp[0], w);
        cp_kahan(acc[1], cmp[1], w * wq);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          cp_kahan(acc[2 + k], cmp[2 + k], dth[k]);
          cp_kahan(acc[5 + k], cmp[5 + k], wq * dth[k]);
        }
        wmax = fmaxf(wmax, w);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          float dxw = wb.d[d] * jv;
          float wid = w / width[d];
          dlo[d] = fmaf(dxw, 1.f - frac[d], -wid);
          dhi[d] = fmaf(dxw, frac[d], wid);
        }
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      float* h = my + d * 4 * nb;
      cp_warp_hist_add(h, bin[d], dlo[d]);
      cp_warp_hist_add(h + nb, bin[d], dhi[d]);
      cp_warp_hist_add(h + 2 * nb, bin[d], wq * dlo[d]);
      cp_warp_hist_add(h + 3 * nb, bin[d], wq * dhi[d]);
    }
  }
  // block reduction of the head sums, FP64 across warps in fixed order
  double v[CP_ADJ_HEAD];
  for (int k = 0; k < 8; ++k) v[k] = cp_warp_sum_d((double)acc[k] - (double)cmp[k]);
  v[8] = cp_warp_max_d((double)wmax);
  v[9] = cp_warp_sum_d((double)nbad);
  if (lane == 0)
    for (int k = 0; k < CP_ADJ_HEAD; ++k) sRed[warp][k] = v[k];
  __syncthreads();
  double* slot = L.slots + (size_t)blockIdx.x * (CP_ADJ_HEAD + 12 * nb);
  if (threadIdx.x < CP_ADJ_HEAD) {
    const int k = threadIdx.x;
    double a = 0.0;
    for (int q = 0; q < CP_ADJ_WARPS; ++q) a = (k == 8) ? fmax(a, sRed[q][k]) : a + sRed[q][k];
    slot[k] = a;
  }
  for (int k = threadIdx.x; k < 12 * nb; k += CP_ADJ_THREADS) {
    double a = 0.0;
    for (int q = 0; q < CP_ADJ_WARPS; ++q) a += (double)sDyn[q * 12 * nb + k];
    slot[CP_ADJ_HEAD + k] = a;
  }
}

// Reduced slots -> gradient record (FP64), and optionally one variance-gradient step on the
// grid: per dimension, G_b = dVar / d ln(Delta_b) of the bin widths (widening bin b shifts every
// edge above it), ln Delta_b -= lr G_b / max_b |G_b|, renormalised to span [0, 1].  The step is
// scale-free: the most sensitive bin changes its width by exp(+-lr).  One thread per dimension.
__global__ void k_adjoint_finish(const double* red, int nb, double n, double* edges, double lr, double p,
                                 double* out)   // out: sigma, var, dsig[3], dvar[3], nbad, wmax, dsig_de[3(nb+1)], dvar_de[3(nb+1)]
{
  const int d = threadIdx.x;
  const double mean = red[0] / n;
  // p = 2: Var and its gradient 2 <w dw> - 2 <w> <dw>; otherwise (R_p - 1) sigma^2 and the
  // gradient of the p-th moment, p <w^(p-1) dw> - p (<w^p> / <w>) <dw>
  const bool two = p == 2.0;
  const double mp = red[1] / n;
  const double var = two ? mp - mean * mean : (mp / pow(mean, p) - 1.0) * mean * mean;
  const double cw = two ? 2.0 : p, cm = two ? 2.0 * mean : p * mp / mean;
  if (d == 0) {
    out[0] = mean;
    out[1] = var;
    for (int k = 0; k < 3; ++k) {
      out[2 + k] = red[2 + k] / n;
      out[5 + k] = cw * red[5 + k] / n - cm * red[2 + k] / n;
    }
    out[8] = red[9];
    out[9] = red[8];
  }
  if (d >= 3) return;
  const double* h = red + CP_ADJ_HEAD + d * 4 * nb;   // lo, hi, w lo, w hi
  double* gs = out + 10 + d * (nb + 1);
  double* gv = out + 10 + 3 * (nb + 1) + d * (nb + 1);
  for (int k = 0; k <= nb; ++k) {
    double a = (k < nb ? h[k] : 0.0) + (k > 0 ? h[nb + k - 1] : 0.0);
    double aw = (k < nb ? h[2 * nb + k] : 0.0) + (k > 0 ? h[3 * nb + k - 1] : 0.0);
    gs[k] = a / n;
    gv[k] = cw * aw / n - cm * a / n;
  }
  if (!(lr > 0.0) || !(var > 0.0)) return;
  double* e = edges + d * (nb + 1);
  double lw[CP_MAX_BINS], G[CP_MAX_BINS], tail = 0.0, gmax = 0.0, tot = 0.0;
  // dVar/dDelta_b = sum_{k > b, k < nb} dVar/de_k  (edges 0 and nb are fixed)
  for (int b = nb - 1; b >= 0; --b) {
    if (b + 1 < nb) tail += gv[b + 1];
    G[b] = (e[b + 1] - e[b]) * tail;
    gmax = fabs(G[b]) > gmax ? fabs(G[b]) : gmax;
  }
  if (!(gmax > 0.0)) return;
  for (int b = 0; b < nb; ++b) lw[b] = log(e[b + 1] - e[b]) - lr * G[b] / gmax;
  double mx = lw[0];
  for (int b = 1; b < nb; ++b) mx = lw[b] > mx ? lw[b] : mx;
  for (int b = 0; b < nb; ++b) { lw[b] = exp(lw[b] - mx); tot += lw[b]; }
  double acc = 0.0;
  e[0] = 0.0;
  for (int b = 0; b < nb - 1; ++b) { acc += lw[b] / tot; e[b + 1] = acc; }
  e[nb] = 1.0;
}

// Sums of one adjoint pass over this handle's points [offset, offset + n) into sums_out
// (CP_ADJ_HEAD + 12 nb doubles: entry 8 is the largest weight, every other entry a sum).
static int adjoint_accumulate(cp_handle* h, uint64_t n, uint32_t iter, uint32_t stream, double* sums_out)
{
  CP_CHECK_HANDLE(h);
  if (n < 1) return cp_fail(h, CP_ERR_INVALID, "cp_adjoint: no points");
  const int nb = h->nb, width = CP_ADJ_HEAD + 12 * nb;
  const size_t dyn = sizeof(float) * CP_ADJ_WARPS * 12 * nb;
  // the attribute is per device: set it on every call (host-side, cheap)
  const int full = h->adj_params ? 1 : 0;
  const void* kfn = full ? reinterpret_cast<const void*>(k_adjoint<6>) : reinterpret_cast<const void*>(k_adjoint<3>);
  CP_CUDA(h, cudaFuncSetAttribute(kfn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(float) * CP_ADJ_WARPS * 12 * CP_MAX_BINS)));
  if (h->adj_per_sm_nt[full] < 0) {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kfn, CP_ADJ_THREADS, dyn) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    h->adj_per_sm_nt[full] = per_sm;
  }
  const int blocks = h->num_sms * h->adj_per_sm_nt[full];
  int rc = cp_ensure_slots(h, (size_t)blocks * width);
  if (rc) return rc;
  AdjLaunch L;
  L.seed = h->cfg.seed; L.point0 = h->point_offset; L.n = n; L.iter = iter; L.stream = stream; L.nb = nb;
  L.edges = h->d_edges; L.cteq = h->d_cteq; L.slots = h->d_slots;
  const double pt = h->cfg.pt_hat_min, s = h->cfg.sqrt_s * h->cfg.sqrt_s, a = h->cfg.alphas_mz;
  L.lnTauMin = (float)log(4.0 * pt * pt / s);
  L.pm1 = (float)(h->adj_p - 1.0);
  L.dlnTauMin_dpt = (float)(2.0 / pt);
  const double b0[4] = {27.0, 25.0, 23.0, 21.0};
  for (int k = 0; k < 4; ++k) {
    L.lnL2[k] = h->P.lnL2[k];
    L.dlnL2_da[k] = (float)(12.0 * M_PI / (b0[k] * a * a));
  }
  if (full) k_adjoint<6><<<blocks, CP_ADJ_THREADS, dyn, h->stream>>>(h->P, L);
  else k_adjoint<3><<<blocks, CP_ADJ_THREADS, dyn, h->stream>>>(h->P, L);
  CP_LAUNCH_CHECK(h, "k_adjoint");
  k_reduce_slots<0><<<(width + 7) / 8, 256, 0, h->stream>>>(h->d_slots, blocks, width, sums_out, 8);
  CP_LAUNCH_CHECK(h, "k_reduce_slots");
  return CP_OK;
}

// Gradient record over n_total points from (rank-reduced) sums, and with lr > 0 one
// variance-gradient step on the grid.
static int adjoint_finish(cp_handle* h, const double* sums, double n_total, double lr, cp_grad* g,
                          double* dsig_de, double* dvar_de)
{
  if (!(n_total >= 2.0)) return cp_fail(h, CP_ERR_INVALID, "cp_adjoint: n_points < 2");
  const int nb = h->nb;
  const size_t out_n = 10 + 6 * (nb + 1);
  double* out = nullptr;
  CP_CUDA(h, cudaMallocAsync(reinterpret_cast<void**>(&out), sizeof(double) * out_n, h->stream));
  k_adjoint_finish<<<1, 32, 0, h->stream>>>(sums, nb, n_total, h->d_edges, lr, h->adj_p, out);
  cudaError_t e = cudaGetLastError();
  std::vector<double> host(out_n, 0.0);
  if (e == cudaSuccess) e = cudaMemcpyAsync(host.data(), out, sizeof(double) * out_n, cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(out, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cp_fail_cuda(h, e, "cp_adjoint readback");
  if (g) {
    g->sigma = host[0];
    g->var = host[1];
    for (int k = 0; k < 3; ++k) { g->dsigma[k] = host[2 + k]; g->dvar[k] = host[5 + k]; }
    g->n_points = (uint64_t)n_total;
    g->n_bad = (uint64_t)host[8];
  }
  if (dsig_de) for (int k = 0; k < 3 * (nb + 1); ++k) dsig_de[k] = host[10 + k];
  if (dvar_de) for (int k = 0; k < 3 * (nb + 1); ++k) dvar_de[k] = host[10 + 3 * (nb + 1) + k];
  if (host[8] > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights or gradients were zeroed");
  return CP_OK;
}

static int adjoint_run(cp_handle* h, uint64_t n, uint32_t iter, uint32_t stream, double lr,
                       cp_grad* g, double* dsig_de, double* dvar_de)
{
  CP_CHECK_HANDLE(h);
  if (n < 2) return cp_fail(h, CP_ERR_INVALID, "cp_adjoint: n_points < 2");
  const int width = CP_ADJ_HEAD + 12 * h->nb;
  double* sums = nullptr;
  CP_CUDA(h, cudaMallocAsync(reinterpret_cast<void**>(&sums), sizeof(double) * width, h->stream));
  int rc = adjoint_accumulate(h, n, iter, stream, sums);
  if (!rc) rc = adjoint_finish(h, sums, (double)n, lr, g, dsig_de, dvar_de);
  cudaFreeAsync(sums, h->stream);
  return rc;
}

extern "C" int cp_vegas_gradient_objective(cp_handle* h, double p)
{
  CP_CHECK_HANDLE(h);
  if (!(p >= 2.0 && p <= 8.0)) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_gradient_objective: p must be in [2, 8]");
  h->adj_p = p;
  return CP_OK;
}

extern "C" int cp_adjoint_parameter_tangents(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  h->adj_params = on ? 1 : 0;
  return CP_OK;
}

extern "C" int cp_adjoint_sums_size(cp_handle* h, int* n_doubles)
{
  CP_CHECK_HANDLE(h);
  if (!n_doubles) return CP_ERR_INVALID;
  *n_doubles = CP_ADJ_HEAD + 12 * h->nb;
  return CP_OK;
}

extern "C" int cp_adjoint_accumulate(cp_handle* h, uint64_t n_points, uint32_t iter, uint32_t stream,
                                     double* sums_dev)
{
  CP_CHECK_HANDLE(h);
  if (!sums_dev) return cp_fail(h, CP_ERR_INVALID, "cp_adjoint_accumulate: null sums");
  return adjoint_accumulate(h, n_points, iter, stream, sums_dev);
}

extern "C" int cp_vegas_gradient_apply(cp_handle* h, const double* sums_dev, uint64_t n_total, double lr,
                                       cp_grad* out)
{
  CP_CHECK_HANDLE(h);
  if (!sums_dev || !(lr >= 0.0)) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_gradient_apply: bad arguments");
  return adjoint_finish(h, sums_dev, (double)n_total, lr, out, nullptr, nullptr);
}

extern "C" int cp_adjoint(cp_handle* h, uint64_t n_points, uint32_t iter, uint32_t stream,
                          cp_grad* out, double* dsigma_dedges, double* dvar_dedges)
{
  return adjoint_run(h, n_points, iter, stream, 0.0, out, dsigma_dedges, dvar_dedges);
}

extern "C" int cp_vegas_gradient_step(cp_handle* h, uint64_t n_points, uint32_t iter, double lr,
                                      cp_grad* out)
{
  if (!(lr > 0.0)) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_gradient_step: lr must be positive");
  return adjoint_run(h, n_points, iter, 0, lr, out, nullptr, nullptr);
}
