// cp_flow.cu -- parameters, packing and the forward (sampling) kernel of the learned proposal.
#include "cp_flow.cuh"
#include "cp_internal.cuh"

// ------------------------------------------------------------------------------------------
// Xavier-uniform initialisation from the counter RNG (key = seed, counter = (index, 0, 0, 7)):
// W ~ U(-a, a), a = sqrt(6 / (fan_in + fan_out)) with the true (unpadded) fans; biases zero.
// The output layer starts at zero so the untrained flow is the identity map and the proposal
// starts from the VEGAS grid it sits on.
// ------------------------------------------------------------------------------------------
__global__ void k_flow_init(float* P, uint64_t seed)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= CP_FLOW_NPARAM) return;
  const int c = i / CP_FLOW_PER, o = i % CP_FLOW_PER;
  const CpCoupling k = cp_coupling(c);
  float v = 0.f;
  uint32_t w[4];
  cp_point_words(seed, (uint64_t)i, 0, 7, w);
  const float u = cp_u24(w[0]) * 2.f - 1.f;
  if (o < CP_FLOW_B1) {
    const int row = o / 64;
    if (row < k.nin) v = u * sqrtf(6.f / (k.nin + 64.f));
  } else if (o >= CP_FLOW_W2 && o < CP_FLOW_B2) {
    v = u * sqrtf(6.f / 128.f);
  }
  P[i] = v;
}

// FP32 master -> BF16 B fragments (forward and transposed) and staged biases; grid (coupling,
// CP_FLOW_PACK_SPLIT blocks sharing its fragments).
#define CP_FLOW_PACK_SPLIT 8
__global__ void k_flow_pack(const float* __restrict__ P, uint2* __restrict__ pk, float* __restrict__ bias)
{
  const int c = blockIdx.x;
  const float* W1 = P + c * CP_FLOW_PER + CP_FLOW_W1;
  const float* W2 = P + c * CP_FLOW_PER + CP_FLOW_W2;
  const float* W3 = P + c * CP_FLOW_PER + CP_FLOW_W3;
  uint2* q = pk + c * CP_FLOW_P_PER;
  const int t0 = blockIdx.y * blockDim.x + threadIdx.x, tstride = gridDim.y * blockDim.x;
  for (int e = t0; e < CP_FLOW_P_PER; e += tstride) {
    const int lane = e & 31, gid = lane >> 2, tig = lane & 3, f = e >> 5;
    float a0, a1, a2, a3;
    if (e < CP_FLOW_P_W2) {                       // W1 [16][64]: tile nt = f
      const int n = f * 8 + gid, k = 2 * tig;
      a0 = W1[k * 64 + n]; a1 = W1[(k + 1) * 64 + n]; a2 = W1[(k + 8) * 64 + n]; a3 = W1[(k + 9) * 64 + n];
    } else if (e < CP_FLOW_P_W3) {                // W2 [64][64]: tile (kt, nt)
      const int t = f - CP_FLOW_P_W2 / 32, kt = t / 8, nt = t % 8;
      const int n = nt * 8 + gid, k = kt * 16 + 2 * tig;
      a0 = W2[k * 64 + n]; a1 = W2[(k + 1) * 64 + n]; a2 = W2[(k + 8) * 64 + n]; a3 = W2[(k + 9) * 64 + n];
    } else if (e < CP_FLOW_P_W3T) {               // W3 [64][8]: tile kt
      const int kt = f - CP_FLOW_P_W3 / 32, n = gid, k = kt * 16 + 2 * tig;
      a0 = W3[k * 8 + n]; a1 = W3[(k + 1) * 8 + n]; a2 = W3[(k + 8) * 8 + n]; a3 = W3[(k + 9) * 8 + n];
    } else if (e < CP_FLOW_P_W2T) {               // W3^T [16 (out, padded)][64]: tile nt
      const int nt = f - CP_FLOW_P_W3T / 32, n = nt * 8 + gid, k = 2 * tig;
      a0 = W3[n * 8 + k]; a1 = W3[n * 8 + k + 1]; a2 = 0.f; a3 = 0.f;
    } else if (e < CP_FLOW_P_W1T) {               // W2^T [64 (out)][64 (in)]: tile (kt, nt)
      const int t = f - CP_FLOW_P_W2T / 32, kt = t / 8, nt = t % 8;
      const int n = nt * 8 + gid, k = kt * 16 + 2 * tig;
      a0 = W2[n * 64 + k]; a1 = W2[n * 64 + k + 1]; a2 = W2[n * 64 + k + 8]; a3 = W2[n * 64 + k + 9];
    } else {                                      // W1^T [64 (hidden)][8 (inputs)]: tile kt
      const int kt = f - CP_FLOW_P_W1T / 32, n = gid, k = kt * 16 + 2 * tig;
      a0 = W1[n * 64 + k]; a1 = W1[n * 64 + k + 1]; a2 = W1[n * 64 + k + 8]; a3 = W1[n * 64 + k + 9];
    }
    q[e] = make_uint2(cp_bf2(a0, a1), cp_bf2(a2, a3));
  }
  for (int j = t0; j < CP_FLOW_NB; j += tstride) {
    float v;
    if (j < 64) v = P[c * CP_FLOW_PER + CP_FLOW_B1 + j];
    else if (j < 128) v = P[c * CP_FLOW_PER + CP_FLOW_B2 + j - 64];
    else v = P[c * CP_FLOW_PER + CP_FLOW_B3 + j - 128];
    bias[c * CP_FLOW_NB + j] = v;
  }
}

// Forward pass over points [point0, point0 + n): Philox (stream) words 0..2 -> VEGAS map -> x_v
// -> flow -> out[p] = (x0, x1, x2, ln(VEGAS Jacobian) + ln |dx/dx_v|).
__global__ void __launch_bounds__(CP_THREADS) k_flow_fwd(const uint2* __restrict__ pk_g, const float* __restrict__ bias_g,
                                                         const double* __restrict__ edges, int nb,
                                                         uint64_t seed, uint64_t point0, uint64_t n, uint32_t iter,
                                                         uint32_t stream, float4* __restrict__ out)
{
  extern __shared__ uint2 sPk[];   // CP_FLOW_NC * CP_FLOW_P_FWD, then the biases
  float* sBias = reinterpret_cast<float*>(sPk + CP_FLOW_NC * CP_FLOW_P_FWD);
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  for (int k = threadIdx.x; k < 3 * nb; k += CP_THREADS) {
    const int d = k / nb, b = k - d * nb;
    sEdge[d][b] = make_float2((float)edges[d * (nb + 1) + b], (float)(edges[d * (nb + 1) + b + 1] - edges[d * (nb + 1) + b]));
  }
  for (int c = 0; c < CP_FLOW_NC; ++c)
    for (int e = threadIdx.x; e < CP_FLOW_P_FWD; e += CP_THREADS) sPk[c * CP_FLOW_P_FWD + e] = pk_g[c * CP_FLOW_P_PER + e];
  for (int j = threadIdx.x; j < CP_FLOW_NC * CP_FLOW_NB; j += CP_THREADS) sBias[j] = bias_g[j];
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t rounds = (n + stride - 1) / stride;
  const uint64_t gtid = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t p = r * stride + gtid;
    const bool active = p < n;
    float z[3], jv = 1.f, logdet = 0.f;
    uint32_t w[4] = {0x80000000u, 0x80000000u, 0x80000000u, 0u};
    if (active) cp_point_words(seed, point0 + p, iter, stream, w);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int bin;
      const float xv = cp_flow_vegas_in(sEdge[d], nb, w[d], jv, bin);
      logdet += cp_flow_logit(xv, z[d]);
    }
    logdet += logf(jv);
    cp_flow_couplings(sPk, sBias, z, logdet);
    float v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) logdet += cp_flow_sigmoid(z[d], v[d]);
    if (active) out[p] = make_float4(v[0], v[1], v[2], logdet);
  }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
static size_t flow_fwd_smem() { return sizeof(uint2) * CP_FLOW_NC * CP_FLOW_P_FWD + sizeof(float) * CP_FLOW_NC * CP_FLOW_NB; }

int cp_flow_ensure(cp_handle* h)
{
  if (h->d_flow) return CP_OK;
  CP_CUDA(h, cudaMalloc(&h->d_flow, sizeof(float) * CP_FLOW_NPARAM * 4));   // master, grad, m, v
  CP_CUDA(h, cudaMemsetAsync(h->d_flow, 0, sizeof(float) * CP_FLOW_NPARAM * 4, h->stream));
  CP_CUDA(h, cudaMalloc(&h->d_flow_pk, sizeof(uint2) * CP_FLOW_NC * CP_FLOW_P_PER));
  CP_CUDA(h, cudaMalloc(&h->d_flow_bias, sizeof(float) * CP_FLOW_NC * CP_FLOW_NB));
  CP_CUDA(h, cudaMalloc(&h->d_flow_ticket, sizeof(unsigned)));
  CP_CUDA(h, cudaMemsetAsync(h->d_flow_ticket, 0, sizeof(unsigned), h->stream));
  CP_CUDA(h, cudaFuncSetAttribute(k_flow_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)flow_fwd_smem()));
  return cp_flow_tc_alloc(h);
}

// The warp-level fragments (used by training and the mma.sync forward) are repacked at once; the
// tcgen05 forward's shared-memory image only when a sampling pass next needs it, so a training
// run does not repack it after every update.
int cp_flow_repack(cp_handle* h)
{
  k_flow_pack<<<dim3(CP_FLOW_NC, CP_FLOW_PACK_SPLIT), 256, 0, h->stream>>>(h->d_flow, h->d_flow_pk, h->d_flow_bias);
  CP_LAUNCH_CHECK(h, "k_flow_pack");
  h->flow_tc_stale = 1;
  return CP_OK;
}

int cp_flow_buffer(cp_handle* h, uint64_t n)
{
  if (n <= h->flow_buf_cap) return CP_OK;
  if (h->d_flow_buf) {
    CP_CUDA(h, cudaStreamSynchronize(h->stream));
    CP_CUDA(h, cudaFree(h->d_flow_buf));
    h->d_flow_buf = nullptr;
    h->d_flow_u = nullptr;
  }
  // the points' (v, ln J), then their accept draws
  CP_CUDA(h, cudaMalloc(&h->d_flow_buf, (sizeof(float4) + sizeof(float)) * n));
  h->d_flow_u = reinterpret_cast<float*>(h->d_flow_buf + n);
  h->flow_buf_cap = n;
  return CP_OK;
}

// Enqueues the flow forward for points [point0, point0 + n) into out (no synchronisation).
int cp_flow_forward_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float4* out,
                            float* uout)
{
  if (h->flow_kernel == 0) return cp_flow_tc_enqueue(h, point0, n, iter, stream, out, uout);
  if (h->flow_per_sm < 0) {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_flow_fwd, CP_THREADS, flow_fwd_smem()) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    h->flow_per_sm = per_sm;
  }
  k_flow_fwd<<<h->num_sms * h->flow_per_sm, CP_THREADS, flow_fwd_smem(), h->stream>>>(
      h->d_flow_pk, h->d_flow_bias, h->d_edges, h->nb, h->cfg.seed, point0, n, iter, stream, out);
  CP_LAUNCH_CHECK(h, "k_flow_fwd");
  return CP_OK;
}

extern "C" int cp_flow_init(cp_handle* h, uint64_t seed)
{
  CP_CHECK_HANDLE(h);
  int rc = cp_flow_ensure(h);
  if (rc) return rc;
  CP_CUDA(h, cudaMemsetAsync(h->d_flow, 0, sizeof(float) * CP_FLOW_NPARAM * 4, h->stream));
  k_flow_init<<<(CP_FLOW_NPARAM + 255) / 256, 256, 0, h->stream>>>(h->d_flow, seed);
  CP_LAUNCH_CHECK(h, "k_flow_init");
  h->flow_t = 0;
  rc = cp_flow_repack(h);
  if (rc) return rc;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_flow_num_params(void) { return CP_FLOW_NPARAM; }

extern "C" int cp_flow_get_params(cp_handle* h, float* out, int n)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised");
  if (!out || n < CP_FLOW_NPARAM) return cp_fail(h, CP_ERR_INVALID, "cp_flow_get_params: buffer too small");
  CP_CUDA(h, cudaMemcpyAsync(out, h->d_flow, sizeof(float) * CP_FLOW_NPARAM, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

extern "C" int cp_flow_set_params(cp_handle* h, const float* in, int n)
{
  CP_CHECK_HANDLE(h);
  if (!in || n != CP_FLOW_NPARAM) return cp_fail(h, CP_ERR_INVALID, "cp_flow_set_params: need cp_flow_num_params() floats");
  int rc = cp_flow_ensure(h);
  if (rc) return rc;
  CP_CUDA(h, cudaMemcpyAsync(h->d_flow, in, sizeof(float) * CP_FLOW_NPARAM, cudaMemcpyHostToDevice, h->stream));
  rc = cp_flow_repack(h);
  if (rc) return rc;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return CP_OK;
}

// Full training state: master parameters, Adam's first and second moments (the gradient slot
// between them is zero between steps and is not part of it) and the number of updates taken.
extern "C" int cp_flow_state_size(void) { return 3 * CP_FLOW_NPARAM; }

extern "C" int cp_flow_get_state(cp_handle* h, float* out, int n, int64_t* updates)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised");
  if (!out || !updates || n != 3 * CP_FLOW_NPARAM)
    return cp_fail(h, CP_ERR_INVALID, "cp_flow_get_state: need cp_flow_state_size() floats and an update count");
  const size_t P = sizeof(float) * CP_FLOW_NPARAM;
  CP_CUDA(h, cudaMemcpyAsync(out, h->d_flow, P, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(out + CP_FLOW_NPARAM, h->d_flow + 2 * CP_FLOW_NPARAM, 2 * P, cudaMemcpyDeviceToHost,
                             h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  *updates = (int64_t)h->flow_t;
  return CP_OK;
}

extern "C" int cp_flow_set_state(cp_handle* h, const float* in, int n, int64_t updates)
{
  CP_CHECK_HANDLE(h);
  if (!in || n != 3 * CP_FLOW_NPARAM || updates < 0 || updates > 0xFFFFFFFFll)
    return cp_fail(h, CP_ERR_INVALID, "cp_flow_set_state: need cp_flow_state_size() floats and 0 <= updates < 2^32");
  int rc = cp_flow_ensure(h);
  if (rc) return rc;
  const size_t P = sizeof(float) * CP_FLOW_NPARAM;
  CP_CUDA(h, cudaMemcpyAsync(h->d_flow, in, P, cudaMemcpyHostToDevice, h->stream));
  CP_CUDA(h, cudaMemsetAsync(h->d_flow + CP_FLOW_NPARAM, 0, P, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(h->d_flow + 2 * CP_FLOW_NPARAM, in + CP_FLOW_NPARAM, 2 * P, cudaMemcpyHostToDevice,
                             h->stream));
  rc = cp_flow_repack(h);
  if (rc) return rc;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  h->flow_t = (long)updates;
  return CP_OK;
}

extern "C" int cp_flow_sample(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float* out_dev)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  if (n && (!out_dev || ((uintptr_t)out_dev & 15))) return cp_fail(h, CP_ERR_INVALID, "cp_flow_sample: output must be 16-byte aligned");
  if (!n) return CP_OK;
  int rc = cp_flow_forward_enqueue(h, point0, n, iter, stream, reinterpret_cast<float4*>(out_dev), nullptr);
  if (rc) return rc;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return cp_flow_tc_status(h);
}

// Selects the flow forward kernel: 0 = tcgen05 (TMEM accumulators, default), 1 = warp-level
// mma.sync tiles (the kernel the training pass shares).
extern "C" int cp_flow_select_kernel(cp_handle* h, int which)
{
  CP_CHECK_HANDLE(h);
  if (which != 0 && which != 1) return cp_fail(h, CP_ERR_INVALID, "cp_flow_select_kernel: 0 (tcgen05) or 1 (mma.sync)");
  h->flow_kernel = which;
  return CP_OK;
}

extern "C" int cp_flow_fuse_production(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  h->flow_fuse = on ? 1 : 0;
  return CP_OK;
}

extern "C" int cp_flow_enable(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  if (on && !h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  h->flow_on = on ? 1 : 0;
  return CP_OK;
}
