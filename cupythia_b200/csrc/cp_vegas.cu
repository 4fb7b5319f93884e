// cp_vegas.cu -- the fused hadronic VEGAS iteration and its FP64 reduction / refinement.
//
// One persistent kernel per iteration: every thread draws its points' Philox words, maps them
// through the VEGAS grid (edges staged in shared memory as FP32 (lo, width) pairs) and the
// analytic (tau, y, z) base map, evaluates the FP32 integrand in registers, and accumulates
//   sum w, sum w^2   Kahan-compensated FP32 per thread, compensated warp and block trees,
//   max w, n_bad     per thread, then warp / block,
//   sum w^2 per bin  warp-private shared-memory histograms, deterministic lane-order adds.
// Each block writes one FP64 slot; a second kernel reduces the slots in a fixed order (FP64)
// and a third refines the grid in FP64 on the device, so iterations chain on the stream
// without host round trips (the reference round-trips through the host every iteration:
// cuPythia/11_vegas_importance/vegas.cu:107-124).
#include <mutex>
#include "cp_internal.cuh"

struct HadLaunch {
  uint64_t seed, point0, n;
  uint32_t iter, stream;
  int nb;
  const double* edges;
  double* slots;   // gridDim.x * (CP_SLOT_HEAD + 3 nb)
  float* w_out;    // optional per-point weights
  float* x_out;    // optional per-point mapped x (3 per point)
  unsigned long long* qhist;   // weight histogram (CP_QBINS), integer adds
  const float4* flow;          // flow output (v, ln J) per point, or null: map the Philox words
};

template <bool WRITE>
__global__ void __launch_bounds__(CP_THREADS, CP_MIN_BLOCKS) k_had_accum(const __grid_constant__ CpHadParams P,
                                                                          const __grid_constant__ HadLaunch L)
{
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  __shared__ float sHist[CP_WARPS][3][CP_MAX_BINS];
  __shared__ float sRed[CP_WARPS][6];
  __shared__ unsigned sQ[CP_QBINS];
  const int nb = L.nb;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = threadIdx.x; k < 3 * nb; k += CP_THREADS) {
    int d = k / nb, b = k - d * nb;
    const double* e = L.edges + d * (nb + 1);
    double lo = e[b], hi = e[b + 1];
    sEdge[d][b] = make_float2((float)lo, (float)(hi - lo));
  }
  for (int k = threadIdx.x; k < CP_WARPS * 3 * CP_MAX_BINS; k += CP_THREADS)
    (&sHist[0][0][0])[k] = 0.f;
  for (int k = threadIdx.x; k < CP_QBINS; k += CP_THREADS) sQ[k] = 0u;
  __syncthreads();

  const float nbf = (float)nb;
  const uint64_t stride = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t gtid = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
  const uint64_t rounds = (L.n + stride - 1) / stride;
  float s1 = 0.f, c1 = 0.f, s2 = 0.f, c2 = 0.f, wmax = 0.f;
  uint32_t nbad = 0;
  float* myHist = &sHist[warp][0][0];

  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t p = r * stride + gtid;
    const bool active = p < L.n;
    float w = 0.f;
    int bin[3] = {0, 0, 0};
    if (active) {
      float x[3], jv = 1.f;
      uint32_t wd[4];
      cp_point_words(L.seed, L.point0 + p, L.iter, L.stream, wd);
      if (L.flow) {
        // the flow already applied the VEGAS map and its own transform: x and the total ln J
        const float4 f = L.flow[p];
        x[0] = f.x; x[1] = f.y; x[2] = f.z;
        jv = expf(f.w);
#pragma unroll
        for (int d = 0; d < 3; ++d) bin[d] = (int)(((wd[d] >> 8) * (uint32_t)nb) >> 24);
      } else {
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          float frac;
          cp_bin_frac(wd[d], nb, bin[d], frac);
          float2 e = sEdge[d][bin[d]];
          x[d] = fmaf(frac, e.y, e.x);
          jv *= nbf * e.y;
        }
      }
      w = cp_had_weight(P, P.cteq, x[0], x[1], x[2], nullptr) * jv;
      if (!(w >= 0.f) || isinf(w)) { ++nbad; w = 0.f; }
      cp_kahan(s1, c1, w);
      cp_kahan(s2, c2, w * w);
      wmax = fmaxf(wmax, w);
      int qb = cp_qbin(w);
      if (qb >= 0) atomicAdd(&sQ[qb], 1u);
      if (WRITE) {
        if (L.w_out) L.w_out[p] = w;
        if (L.x_out) { L.x_out[3 * p] = x[0]; L.x_out[3 * p + 1] = x[1]; L.x_out[3 * p + 2] = x[2]; }
      }
    }
    const float w2 = w * w;
#pragma unroll
    for (int d = 0; d < 3; ++d) cp_warp_hist_add(myHist + d * CP_MAX_BINS, bin[d], w2);
  }

  // compensated warp trees: Kahan sum s with compensation -c is the pair (s, -c)
  float h1 = s1, l1 = -c1, h2 = s2, l2 = -c2;
  cp_warp_sum_comp(h1, l1);
  cp_warp_sum_comp(h2, l2);
  float wm = cp_warp_max(wmax);
  unsigned nb_w = __reduce_add_sync(0xffffffffu, nbad);
  if (lane == 0) {
    sRed[warp][0] = h1; sRed[warp][1] = l1; sRed[warp][2] = h2; sRed[warp][3] = l2;
    sRed[warp][4] = wm; sRed[warp][5] = __uint_as_float(nb_w);
  }
  __syncthreads();
  double* slot = L.slots + (size_t)blockIdx.x * (CP_SLOT_HEAD + 3 * nb);
  if (threadIdx.x == 0) {
    // block combine in warp order, FP32 compensated, then one FP64 store
    float bh1 = 0.f, bl1 = 0.f, bh2 = 0.f, bl2 = 0.f, bm = 0.f;
    unsigned bn = 0;
    for (int k = 0; k < CP_WARPS; ++k) {
      float s, e;
      cp_two_sum(bh1, sRed[k][0], s, e); bh1 = s; bl1 += sRed[k][1] + e;
      cp_two_sum(bh2, sRed[k][2], s, e); bh2 = s; bl2 += sRed[k][3] + e;
      bm = fmaxf(bm, sRed[k][4]);
      bn += __float_as_uint(sRed[k][5]);
    }
    slot[0] = (double)bh1 + (double)bl1;
    slot[1] = (double)bh2 + (double)bl2;
    slot[2] = (double)bm;
    slot[3] = (double)bn;
  }
  for (int k = threadIdx.x; k < 3 * nb; k += CP_THREADS) {
    int d = k / nb, b = k - d * nb;
    float s = 0.f;
    for (int q = 0; q < CP_WARPS; ++q) s += sHist[q][d][b];
    slot[CP_SLOT_HEAD + k] = (double)s;
  }
  for (int k = threadIdx.x; k < CP_QBINS; k += CP_THREADS)
    if (sQ[k]) atomicAdd(&L.qhist[k], (unsigned long long)sQ[k]);
}

// Smallest bin edge w such that at most (1 - q) n of the weights lie above it (q-quantile,
// rounded up to the bin's upper edge); stored as the unweighting threshold.
__global__ void k_quantile(const unsigned long long* __restrict__ qhist, double q, double* wmax)
{
  __shared__ unsigned long long sh[CP_QBINS];
  for (int k = threadIdx.x; k < CP_QBINS; k += blockDim.x) sh[k] = qhist[k];
  __syncthreads();
  if (threadIdx.x != 0) return;
  unsigned long long tot = 0;
  for (int k = 0; k < CP_QBINS; ++k) tot += sh[k];
  double allowed = (1.0 - q) * (double)tot;
  unsigned long long above = 0;
  int b = CP_QBINS - 1;
  for (; b > 0; --b) {
    if ((double)(above + sh[b]) > allowed) break;
    above += sh[b];
  }
  wmax[0] = (double)cp_qbin_hi(b);
  wmax[1] = q;
}

// Iteration record and, if alpha > 0, Lepage's refinement of each dimension (FP64, one
// thread per dimension): smooth (1,1)/(1,1,1)/(1,1), normalise, compress
// r = ((d - 1) / ln d)^alpha, and rebin to equal shares of sum r.
__global__ void k_refine(double* edges, const double* red, int nb, double n, double alpha,
                         CpIterDev* rec)
{
  const int d = threadIdx.x;
  if (d == 0 && rec) {
    double sumw = red[0], sumw2 = red[1];
    double mean = sumw / n;
    double var = (sumw2 / n - mean * mean) / (n - 1.0);
    rec->sumw = sumw; rec->sumw2 = sumw2; rec->wmax = red[2]; rec->nbad = red[3]; rec->n = n;
    rec->sigma = mean; rec->err = sqrt(var > 0.0 ? var : 0.0);
  }
  if (!(alpha > 0.0) || d >= 3) return;
  const double* h = red + CP_SLOT_HEAD + d * nb;
  double* e = edges + d * (nb + 1);
  double sm[CP_MAX_BINS], r[CP_MAX_BINS], ne[CP_MAX_BINS + 1];
  double tot = 0.0;
  for (int i = 0; i < nb; ++i) {
    double s;
    if (i == 0) s = (h[0] + h[1]) / 2.0;
    else if (i == nb - 1) s = (h[nb - 2] + h[nb - 1]) / 2.0;
    else s = (h[i - 1] + h[i] + h[i + 1]) / 3.0;
    sm[i] = s;
    tot += s;
  }
  if (!(tot > 0.0)) return;
  double rsum = 0.0;
  for (int i = 0; i < nb; ++i) {
    double di = sm[i] / tot, ri = 0.0;
    if (di >= 1.0) ri = 1.0;
    else if (di > 0.0) ri = pow((di - 1.0) / log(di), alpha);
    r[i] = ri;
    rsum += ri;
  }
  double step = rsum / (double)nb;
  ne[0] = e[0];
  ne[nb] = e[nb];
  double acc = 0.0;
  int j = 0;
  for (int k = 1; k < nb; ++k) {
    double need = step * (double)k;
    while (j < nb - 1 && acc + r[j] < need) { acc += r[j]; ++j; }
    double frac = r[j] > 0.0 ? (need - acc) / r[j] : 0.0;
    frac = frac < 0.0 ? 0.0 : (frac > 1.0 ? 1.0 : frac);
    ne[k] = e[j] + frac * (e[j + 1] - e[j]);
  }
  for (int k = 0; k <= nb; ++k) e[k] = ne[k];
}

// FP32 integrand at caller-supplied x
__global__ void __launch_bounds__(CP_THREADS, CP_MIN_BLOCKS) k_weight_at(const CpHadParams P, const CpCteqPoly* cteq_g, const float* __restrict__ x,
                            int64_t n, float* w)
{
  __shared__ CpCteqPoly sCteq[8];
  cp_stage_cteq(sCteq, cteq_g);
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    w[i] = cp_had_weight(P, sCteq, x[3 * i], x[3 * i + 1], x[3 * i + 2], nullptr);
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
static int had_launch(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream,
                      float* w_out, float* x_out)
{
  const int width = CP_SLOT_HEAD + 3 * h->nb;
  int rc = cp_ensure_slots(h, (size_t)h->had_blocks * width);
  if (rc) return rc;
  point0 += h->point_offset;
  HadLaunch L;
  L.seed = h->cfg.seed; L.point0 = point0; L.n = n; L.iter = iter; L.stream = stream;
  L.nb = h->nb; L.edges = h->d_edges; L.slots = h->d_slots; L.w_out = w_out; L.x_out = x_out;
  L.qhist = h->d_qhist;
  L.flow = nullptr;
  if (h->flow_on) {
    rc = cp_flow_buffer(h, n);
    if (rc) return rc;
    rc = cp_flow_forward_enqueue(h, point0, n, iter, stream, h->d_flow_buf, nullptr);
    if (rc) return rc;
    L.flow = h->d_flow_buf;
  }
  CP_CUDA(h, cudaMemsetAsync(h->d_qhist, 0, sizeof(unsigned long long) * CP_QBINS, h->stream));
  h->last_n = n;
  if (w_out || x_out) k_had_accum<true><<<h->had_blocks, CP_THREADS, 0, h->stream>>>(h->P, L);
  else k_had_accum<false><<<h->had_blocks, CP_THREADS, 0, h->stream>>>(h->P, L);
  CP_LAUNCH_CHECK(h, "k_had_accum");
  const int wpb = 8;
  k_reduce_slots<0><<<(width + wpb - 1) / wpb, wpb * 32, 0, h->stream>>>(h->d_slots, h->had_blocks,
                                                                        width, h->d_red);
  CP_LAUNCH_CHECK(h, "k_reduce_slots");
  return CP_OK;
}

static void fill_result(const CpIterDev& r, cp_result* out)
{
  out->sigma = r.sigma;
  out->sigma_err = r.err;
  out->sum_w = r.sumw;
  out->sum_w2 = r.sumw2;
  out->w_max = r.wmax;
  out->n_points = (uint64_t)r.n;
  out->n_bad = (uint64_t)r.nbad;
  out->eta = r.wmax > 0 ? r.sigma / r.wmax : 0.0;
}

int cp_had_launch_shape(cp_handle* h)
{
  int per_sm = 0;
  CP_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_had_accum<false>, CP_THREADS, 0));
  if (per_sm < 1) per_sm = 1;
  h->had_blocks = h->num_sms * per_sm;
  return CP_OK;
}

extern "C" int cp_vegas_iteration(cp_handle* h, uint64_t n_points, uint32_t iter, double alpha,
                                  cp_result* out)
{
  CP_CHECK_HANDLE(h);
  if (n_points < 2) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_iteration: n_points < 2");
  int rc = cp_ensure_iters(h, 1);
  if (rc) return rc;
  rc = had_launch(h, 0, n_points, iter, 0, nullptr, nullptr);
  if (rc) return rc;
  k_refine<<<1, 32, 0, h->stream>>>(h->d_edges, h->d_red, h->nb, (double)n_points, alpha, h->d_iters);
  CP_LAUNCH_CHECK(h, "k_refine");
  CpIterDev r;
  CP_CUDA(h, cudaMemcpyAsync(&r, h->d_iters, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) return rc;
  if (out) fill_result(r, out);
  if (r.nbad > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights were zeroed");
  return CP_OK;
}

extern "C" int cp_integrate(cp_handle* h, int n_iter, uint64_t n_points, double alpha, int skip,
                            cp_result* per_iter, cp_result* combined)
{
  CP_CHECK_HANDLE(h);
  if (n_iter < 1 || n_points < 2) return cp_fail(h, CP_ERR_INVALID, "cp_integrate: bad sizes");
  int rc = cp_ensure_iters(h, n_iter);
  if (rc) return rc;
  for (int it = 0; it < n_iter; ++it) {
    rc = had_launch(h, 0, n_points, (uint32_t)it, 0, nullptr, nullptr);
    if (rc) return rc;
    k_refine<<<1, 32, 0, h->stream>>>(h->d_edges, h->d_red, h->nb, (double)n_points, alpha,
                                       h->d_iters + it);
    CP_LAUNCH_CHECK(h, "k_refine");
  }
  CpIterDev* recs = new CpIterDev[n_iter];
  cudaError_t e = cudaMemcpyAsync(recs, h->d_iters, sizeof(CpIterDev) * n_iter,
                                  cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) { delete[] recs; return cp_fail_cuda(h, e, "cp_integrate readback"); }
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) { delete[] recs; return rc; }
  double wsum = 0, w2 = 0, sw = 0, sw2 = 0, wmax = 0, nbad = 0, npts = 0;
  for (int it = 0; it < n_iter; ++it) {
    if (per_iter) fill_result(recs[it], per_iter + it);
    nbad += recs[it].nbad;
    if (it < skip) continue;
    double err = recs[it].err;
    if (err > 0) { wsum += recs[it].sigma / (err * err); w2 += 1.0 / (err * err); }
    sw += recs[it].sumw; sw2 += recs[it].sumw2; npts += recs[it].n;
    wmax = recs[it].wmax > wmax ? recs[it].wmax : wmax;
  }
  delete[] recs;
  if (combined) {
    combined->sigma = w2 > 0 ? wsum / w2 : 0;
    combined->sigma_err = w2 > 0 ? 1.0 / sqrt(w2) : 0;
    combined->sum_w = sw; combined->sum_w2 = sw2; combined->w_max = wmax;
    combined->n_points = (uint64_t)npts; combined->n_bad = (uint64_t)nbad;
    combined->eta = wmax > 0 ? combined->sigma / wmax : 0;
  }
  if (nbad > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights were zeroed");
  return CP_OK;
}

extern "C" int cp_point_weights(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter,
                                float* w_dev, float* x_dev)
{
  CP_CHECK_HANDLE(h);
  if (!w_dev && !x_dev) return cp_fail(h, CP_ERR_INVALID, "cp_point_weights: no output");
  if (n == 0) return CP_OK;
  int rc = had_launch(h, point0, n, iter, 0, w_dev, x_dev);
  if (rc) return rc;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_weight_at(cp_handle* h, const float* x, int64_t n, float* w)
{
  CP_CHECK_HANDLE(h);
  if (n < 0 || (n > 0 && (!x || !w))) return cp_fail(h, CP_ERR_INVALID, "cp_weight_at: bad args");
  if (n == 0) return CP_OK;
  int blocks = (int)((n + CP_THREADS - 1) / CP_THREADS);
  if (blocks > h->num_sms * 16) blocks = h->num_sms * 16;
  k_weight_at<<<blocks, CP_THREADS, 0, h->stream>>>(h->P, h->d_cteq, x, n, w);
  CP_LAUNCH_CHECK(h, "k_weight_at");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_last_histogram(cp_handle* h, double* out)
{
  CP_CHECK_HANDLE(h);
  if (!out) return cp_fail(h, CP_ERR_INVALID, "cp_last_histogram: null output");
  CP_CUDA(h, cudaMemcpyAsync(out, h->d_red, sizeof(double) * (CP_SLOT_HEAD + 3 * h->nb),
                             cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_weight_quantile(cp_handle* h, double q, double* w_q)
{
  CP_CHECK_HANDLE(h);
  if (!(q > 0.0 && q < 1.0)) return cp_fail(h, CP_ERR_INVALID, "cp_weight_quantile: q must be in (0, 1)");
  if (h->last_n == 0) return cp_fail(h, CP_ERR_INVALID, "cp_weight_quantile: run an iteration first");
  k_quantile<<<1, 256, 0, h->stream>>>(h->d_qhist, q, h->d_wmax);
  CP_LAUNCH_CHECK(h, "k_quantile");
  double v[2];
  CP_CUDA(h, cudaMemcpyAsync(v, h->d_wmax, sizeof v, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  h->wmax_host = v[0];   // production passes check the threshold without reading the device
  if (w_q) *w_q = v[0];
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// Distributed iteration: a pass over this handle's points into a caller buffer, and the
// refinement from sums the caller has reduced over ranks (sum over every entry except the
// maximum weight at index 2, which is reduced by max).
// ------------------------------------------------------------------------------------------
extern "C" int cp_vegas_accumulate(cp_handle* h, uint64_t n_points, uint32_t iter, double* sums_dev)
{
  CP_CHECK_HANDLE(h);
  if (n_points < 1 || !sums_dev) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_accumulate: bad arguments");
  int rc = had_launch(h, 0, n_points, iter, 0, nullptr, nullptr);
  if (rc) return rc;
  CP_CUDA(h, cudaMemcpyAsync(sums_dev, h->d_red, sizeof(double) * (CP_SLOT_HEAD + 3 * h->nb), cudaMemcpyDeviceToDevice,
                             h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) return rc;
  return CP_OK;
}

extern "C" int cp_vegas_refine_sums(cp_handle* h, const double* sums_dev, double n_total, double alpha, cp_result* out)
{
  CP_CHECK_HANDLE(h);
  if (!sums_dev || !(n_total >= 2)) return cp_fail(h, CP_ERR_INVALID, "cp_vegas_refine_sums: bad arguments");
  int rc = cp_ensure_iters(h, 1);
  if (rc) return rc;
  CP_CUDA(h, cudaMemcpyAsync(h->d_red, sums_dev, sizeof(double) * (CP_SLOT_HEAD + 3 * h->nb), cudaMemcpyDeviceToDevice,
                             h->stream));
  k_refine<<<1, 32, 0, h->stream>>>(h->d_edges, h->d_red, h->nb, n_total, alpha, h->d_iters);
  CP_LAUNCH_CHECK(h, "k_refine");
  CpIterDev r;
  CP_CUDA(h, cudaMemcpyAsync(&r, h->d_iters, sizeof r, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (out) fill_result(r, out);
  if (r.nbad > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights were zeroed");
  return CP_OK;
}

extern "C" int cp_weight_histogram(cp_handle* h, unsigned long long* hist_dev)
{
  CP_CHECK_HANDLE(h);
  if (!hist_dev) return cp_fail(h, CP_ERR_INVALID, "cp_weight_histogram: null buffer");
  if (h->last_n == 0) return cp_fail(h, CP_ERR_INVALID, "cp_weight_histogram: run a pass first");
  CP_CUDA(h, cudaMemcpyAsync(hist_dev, h->d_qhist, sizeof(unsigned long long) * CP_QBINS, cudaMemcpyDeviceToDevice,
                             h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_weight_quantile_hist(cp_handle* h, const unsigned long long* hist_dev, double q, double* w_q)
{
  CP_CHECK_HANDLE(h);
  if (!hist_dev || !(q > 0.0 && q < 1.0)) return cp_fail(h, CP_ERR_INVALID, "cp_weight_quantile_hist: bad arguments");
  k_quantile<<<1, 256, 0, h->stream>>>(hist_dev, q, h->d_wmax);
  CP_LAUNCH_CHECK(h, "k_quantile");
  double v[2];
  CP_CUDA(h, cudaMemcpyAsync(v, h->d_wmax, sizeof v, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  h->wmax_host = v[0];
  if (w_q) *w_q = v[0];
  return CP_OK;
}

// ------------------------------------------------------------------------------------------
// Allocation-free VEGAS pass.
//
// For callers that must not allocate device memory: a host program that owns every device
// allocation (a caching allocator or memory pool whose accounting a cudaMalloc behind its back
// would break), a process held to a fixed device-memory budget, or a plugin such as a Pythia
// SigmaProcess running inside someone else's event loop, which cannot create and keep a handle
// with its own buffers.  This entry point creates no handle and calls no cudaMalloc / cudaFree:
// its scratch (the per-block partial sums and the weight histogram; the CTEQ5L coefficient
// records travel in the kernel's parameters) lives in the file-scope array below, which every GPU that loads this library keeps
// until the process exits.  The first call on a device looks up the array's address and the
// launch shape (later calls only re-check the address); make that first call before any stream
// capture.
//
// Limits: the partial sums hold at most CP_NOALLOC_MAX_BLOCKS blocks of CP_SLOT_HEAD + 3 *
// CP_MAX_BINS doubles, so n_bins above CP_MAX_BINS is rejected; the grid is capped at
// CP_NOALLOC_MAX_BLOCKS blocks (296 are used on a B200).  Total: 1,622,016 bytes per device.
// Every call shares the array and it keeps the last call's contents; each call clears the
// weight histogram and rewrites every partial-sum slot it reads.  Calls that overlap on the GPU (different streams, or several host threads) race on the
// array and must not be issued; calls in one stream are ordered and safe.
// ------------------------------------------------------------------------------------------
#define CP_NOALLOC_MAX_BLOCKS 512
#define CP_NOALLOC_SLOT_DOUBLES (CP_NOALLOC_MAX_BLOCKS * (CP_SLOT_HEAD + 3 * CP_MAX_BINS))
#define CP_NOALLOC_DOUBLES (CP_QBINS + CP_NOALLOC_SLOT_DOUBLES)

static __device__ __align__(256) double cp_noalloc_scratch[CP_NOALLOC_DOUBLES];

// Per-call set-up of the shared array, on the caller's stream: a cleared weight histogram.
__global__ void k_noalloc_setup(double* base)
{
  unsigned long long* qhist = reinterpret_cast<unsigned long long*>(base);
  for (int k = threadIdx.x; k < CP_QBINS; k += blockDim.x) qhist[k] = 0ull;
}

namespace {
struct NoallocDevice {
  double* scratch = nullptr;   // device address of cp_noalloc_scratch on this device
  int blocks = 0;
};
const int CP_NOALLOC_MAX_DEVICES = 64;
NoallocDevice g_noalloc[CP_NOALLOC_MAX_DEVICES];
std::mutex g_noalloc_mutex;
}  // namespace

extern "C" int cp_vegas_pass_noalloc(const cp_config* cfg, uint64_t n_points, uint32_t iter,
                                     const double* edges_dev, double* sums_dev, void* cuda_stream)
{
  if (!cfg || !edges_dev || !sums_dev) return CP_ERR_INVALID;
  if (cfg->n_bins < 2 || cfg->n_bins > CP_MAX_BINS) return CP_ERR_INVALID;   // beyond the scratch
  if (n_points < 2) return CP_ERR_INVALID;
  if (cfg->device < 0 || cfg->device >= CP_NOALLOC_MAX_DEVICES) return CP_ERR_INVALID;
  CpHadConfig hc{cfg->sqrt_s, cfg->pt_hat_min, cfg->alphas_mz, cfg->k_ren, cfg->k_fac,
                 cfg->convert2mb, cfg->n_quark_in, cfg->n_quark_new, cfg->proc_mask};
  CpHadParams P;
  if (cp_build_had_params(hc, P) || (cfg->proc_mask & ~CP_PROC_ALL) || cfg->proc_mask == 0)
    return CP_ERR_INVALID;
  int prev = -1;
  if (cudaGetDevice(&prev) != cudaSuccess) return CP_ERR_CUDA;
  if (prev != cfg->device && cudaSetDevice(cfg->device) != cudaSuccess) return CP_ERR_CUDA;
  cudaStream_t stream = (cudaStream_t)cuda_stream;
  int rc = CP_OK;
  NoallocDevice D;
  {
    // With the device current: the array's device address (looked up on every call, so a
    // reloaded module after a device reset is picked up) and, when it is new, the launch shape.
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    NoallocDevice& G = g_noalloc[cfg->device];
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, cp_noalloc_scratch) != cudaSuccess || !ptr) {
      rc = CP_ERR_CUDA;
    } else if (ptr != G.scratch) {
      int nsm = 0, per_sm = 0;
      if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, cfg->device) != cudaSuccess ||
          cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_had_accum<false>, CP_THREADS, 0) != cudaSuccess) {
        rc = CP_ERR_CUDA;
      } else {
        const int blocks = nsm * (per_sm > 0 ? per_sm : 1);
        G.blocks = blocks < CP_NOALLOC_MAX_BLOCKS ? blocks : CP_NOALLOC_MAX_BLOCKS;
        G.scratch = (double*)ptr;
      }
    }
    D = G;
  }
  if (rc == CP_OK) {
    double* base = D.scratch;
    unsigned long long* qhist = reinterpret_cast<unsigned long long*>(base);
    double* slots = base + CP_QBINS;
    int nb = cfg->n_bins, width = CP_SLOT_HEAD + 3 * nb, max_col = 2;
    HadLaunch L;
    L.seed = cfg->seed; L.point0 = 0; L.n = n_points; L.iter = iter; L.stream = 0;
    L.nb = nb; L.edges = edges_dev;
    L.slots = slots; L.w_out = nullptr; L.x_out = nullptr; L.qhist = qhist; L.flow = nullptr;
    // Each launch's own return code is checked; an error the caller left pending from earlier,
    // unrelated work is neither reported as this call's nor cleared.
    void* a_setup[] = {&base};
    void* a_accum[] = {&P, &L};
    void* a_reduce[] = {&slots, &D.blocks, &width, &sums_dev, &max_col};
    if (cudaLaunchKernel((const void*)k_noalloc_setup, dim3(1), dim3(256), a_setup, 0, stream) != cudaSuccess ||
        cudaLaunchKernel((const void*)k_had_accum<false>, dim3(D.blocks), dim3(CP_THREADS), a_accum, 0, stream) !=
            cudaSuccess ||
        cudaLaunchKernel((const void*)k_reduce_slots<0>, dim3((width + 7) / 8), dim3(8 * 32), a_reduce, 0, stream) !=
            cudaSuccess)
      rc = CP_ERR_CUDA;
  }
  if (prev != cfg->device) cudaSetDevice(prev);
  return rc;
}
