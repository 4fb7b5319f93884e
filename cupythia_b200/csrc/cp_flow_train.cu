// cp_flow_train.cu -- training of the learned proposal on weights the integrator generates.
//
// Objective: the relative second moment of the weights, L = <w^2> / <w>^2 (= 1 + Var[w]/sigma^2),
// minimised over the flow parameters theta at fixed VEGAS grid (cp_flow_set_objective selects
// the relative p-th moment <w^p>/<w>^p instead, which weighs the tail of the weights more).  With w = f(x(x_v; theta)) J,
// x_v the VEGAS-mapped point (fixed by the random numbers), f the integrand and J the VEGAS
// Jacobian times |dx/dx_v|, the pathwise gradient is
//   dL/dtheta = 2/(B sigma^2) sum_points w^2 (d ln f/dx . dx/dtheta + d ln J/dtheta),
// so one step is: flow forward (saving each coupling's input) -> integrand value and d ln f/dx
// (forward-mode FP32 duals, the adjoint machinery) -> backward through sigmoid and couplings
// with each coupling's MLP recomputed on the tensor cores -> weight-gradient GEMMs on the tensor
// cores -> Adam (FP32 master weights) -> BF16 fragment repack.
#include "cp_dual.cuh"
#include "cp_flow.cuh"
#include "cp_internal.cuh"
#include "cp_tc.cuh"

int cp_flow_ensure(cp_handle* h);
int cp_flow_repack(cp_handle* h);

struct FlowTrainBufs {
  float* zs;           // [B][4][3] input z of each coupling
  float4* vj;          // [B] (v0, v1, v2, ln J)
  float4* wg;          // [B] (w, d ln F / dv)
  uint16_t* X;         // [4][B][16]  bf16 MLP inputs
  uint16_t* H1;        // [4][B][64]  bf16 post-ReLU hidden 1
  uint16_t* H2;        // [4][B][64]  bf16 post-ReLU hidden 2
  uint16_t* D1;        // [4][B][64]  bf16 d pre-activation 1
  uint16_t* D2;        // [4][B][64]  bf16 d pre-activation 2
  uint16_t* DO;        // [4][B][16]  bf16 d outputs (s_raw, t)
  double* sums;        // [2] sum w, sum w^2 of the batch
  double* loss;        // per-step relative second moment
  float* gpart;        // [CP_WG_MAXBLK][CP_FLOW_NPARAM] per-block weight and bias gradients
};

__device__ __forceinline__ float cp_bf_lo(uint32_t v) { return __uint_as_float(v << 16); }
__device__ __forceinline__ float cp_bf_hi(uint32_t v) { return __uint_as_float(v & 0xffff0000u); }

// ------------------------------------------------------------------------------------------
// 1. forward, saving the input z of every coupling
// ------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(CP_THREADS, 2) k_flow_fwd_train(const uint2* __restrict__ pk_g, const float* __restrict__ bias_g,
                                                               const double* __restrict__ edges, int nb,
                                                               uint64_t seed, uint32_t iter, uint32_t stream, uint64_t point0,
                                                               uint64_t n, float* __restrict__ zs, float4* __restrict__ vj)
{
  extern __shared__ uint2 sPk[];
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
  const int lane = threadIdx.x & 31;
  const uint64_t stride = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t rounds = (n + stride - 1) / stride;
  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t p = r * stride + (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
    const bool active = p < n;
    float z[3], jv = 1.f, logdet = 0.f;
    uint32_t w[4] = {0x80000000u, 0x80000000u, 0x80000000u, 0u};
    if (active) cp_point_words(seed, point0 + p, iter, stream, w);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int bin;
      logdet += cp_flow_logit(cp_flow_vegas_in(sEdge[d], nb, w[d], jv, bin), z[d]);
    }
    logdet += logf(jv);
#pragma unroll 1
    for (int c = 0; c < CP_FLOW_NC; ++c) {
      if (active)
        for (int d = 0; d < 3; ++d) zs[(p * CP_FLOW_NC + c) * 3 + d] = z[d];
      const CpCoupling k = cp_coupling(c);
      const float* b = sBias + c * CP_FLOW_NB;
      float o0[4], o1[4], o[4];
      cp_flow_mlp_tile(sPk + c * CP_FLOW_P_FWD, b, b + 64, b + 128, z[k.cin[0]], z[k.cin[1]], k.nin, 0, o0);
      cp_flow_mlp_tile(sPk + c * CP_FLOW_P_FWD, b, b + 64, b + 128, z[k.cin[0]], z[k.cin[1]], k.nin, 16, o1);
#pragma unroll
      for (int q = 0; q < 4; ++q) o[q] = lane >= 16 ? o1[q] : o0[q];
      for (int j = 0; j < k.nt; ++j) {
        const float s = CP_FLOW_S * tanhf(o[j] / CP_FLOW_S);
        z[k.tr[j]] = fmaf(z[k.tr[j]], expf(s), o[k.nt + j]);
        logdet += s;
      }
    }
    float v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) logdet += cp_flow_sigmoid(z[d], v[d]);
    if (active) vj[p] = make_float4(v[0], v[1], v[2], logdet);
  }
}

// ------------------------------------------------------------------------------------------
// 2. integrand value and d ln f / dx at the flow's points (3-tangent duals), batch sums
// ------------------------------------------------------------------------------------------
// Each block writes its (sum w, sum w^2) to its slot; the block that finishes last (integer
// ticket, after a fence) adds all slots in a fixed order (strided per-thread sums, the xor tree
// of each warp, the warps in order) into moments[0..1], writes the batch loss <w^2>/<w>^2 over
// n_loss points when loss != null, and re-arms the ticket.
__global__ void __launch_bounds__(128) k_flow_igrad(const CpHadParams P, const CpCteqPoly* __restrict__ cteq_g,
                                                    uint64_t n, float lnTauMin, const float4* __restrict__ vj,
                                                    float4* __restrict__ wg, double* __restrict__ slots,
                                                    unsigned* __restrict__ ticket, double* __restrict__ moments,
                                                    double n_loss, double* __restrict__ loss)
{
  __shared__ CpCteqPoly sCteq[8];
  __shared__ double sRed[4][2];
  __shared__ int sLast;
  cp_stage_cteq(sCteq, cteq_g);
  __syncthreads();
  typedef CpDual<3> D3;
  CpHadParamsT<D3> Q;
  Q.lnTauMin = cp_dconst<3>(lnTauMin);
  Q.kR = cp_dconst<3>(P.kR);
  for (int k = 0; k < 4; ++k) Q.lnL2[k] = cp_dconst<3>(P.lnL2[k]);
  double s1 = 0.0, s2 = 0.0;
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (uint64_t)gridDim.x * blockDim.x) {
    const float4 f = vj[p];
    D3 F = cp_had_weight_t<D3>(P, Q, sCteq, cp_dvar<3>(f.x, 0), cp_dvar<3>(f.y, 1), cp_dvar<3>(f.z, 2));
    float w = F.v * expf(f.w);
    float g[3] = {0.f, 0.f, 0.f};
    if (F.v > 0.f && isfinite(w)) {
      for (int d = 0; d < 3; ++d) g[d] = F.d[d] / F.v;
    } else {
      w = 0.f;
    }
    wg[p] = make_float4(w, g[0], g[1], g[2]);
    s1 += w;
    s2 += (double)w * w;
  }
  s1 = cp_warp_sum_d(s1);
  s2 = cp_warp_sum_d(s2);
  if ((threadIdx.x & 31) == 0) { sRed[threadIdx.x >> 5][0] = s1; sRed[threadIdx.x >> 5][1] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0, b = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += sRed[q][0]; b += sRed[q][1]; }
    slots[2 * blockIdx.x] = a;
    slots[2 * blockIdx.x + 1] = b;
    __threadfence();
    sLast = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!sLast) return;
  __threadfence();
  double a = 0.0, b = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
    a += __ldcg(slots + 2 * k);
    b += __ldcg(slots + 2 * k + 1);
  }
  a = cp_warp_sum_d(a);
  b = cp_warp_sum_d(b);
  __syncthreads();   // sRed is reused
  if ((threadIdx.x & 31) == 0) { sRed[threadIdx.x >> 5][0] = a; sRed[threadIdx.x >> 5][1] = b; }
  __syncthreads();
  if (threadIdx.x == 0) {
    a = 0.0;
    b = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) { a += sRed[q][0]; b += sRed[q][1]; }
    moments[0] = a;
    moments[1] = b;
    if (loss) {
      const double m = a / n_loss;
      loss[0] = (b / n_loss) / (m * m);
    }
    *ticket = 0u;
  }
}

// ------------------------------------------------------------------------------------------
// 3. backward through the couplings (MLPs recomputed), writing the GEMM operands
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_store_rowfrag(uint16_t* base, int ld, uint64_t row0, uint64_t n, int gid, int tig,
                                                 const uint32_t h[4][4])
{
  // writes a 16 x 64 bf16 tile held as A fragments (rows row0 + gid, row0 + gid + 8)
  const uint64_t ra = row0 + gid, rb = row0 + gid + 8;
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    const int c0 = 16 * kt + 2 * tig;
    if (ra < n) {
      *reinterpret_cast<uint32_t*>(base + ra * ld + c0) = h[kt][0];
      *reinterpret_cast<uint32_t*>(base + ra * ld + c0 + 8) = h[kt][2];
    }
    if (rb < n) {
      *reinterpret_cast<uint32_t*>(base + rb * ld + c0) = h[kt][1];
      *reinterpret_cast<uint32_t*>(base + rb * ld + c0 + 8) = h[kt][3];
    }
  }
}

#define CP_BWD_THREADS 256   // 8 warps; the 92 KB of staged fragments admit two blocks per SM
__global__ void __launch_bounds__(CP_BWD_THREADS, 2) k_flow_bwd(const uint2* __restrict__ pk_g, const float* __restrict__ bias_g, uint64_t n,
                                                  double n_batch, const float* __restrict__ zs, const float4* __restrict__ vj,
                                                  const float4* __restrict__ wg, const double* __restrict__ sums,
                                                  FlowTrainBufs out, float loss_p)
{
  extern __shared__ uint2 sPk[];   // all CP_FLOW_P_PER fragments of the 4 couplings, then biases
  float* sBias = reinterpret_cast<float*>(sPk + CP_FLOW_NC * CP_FLOW_P_PER);
  for (int e = threadIdx.x; e < CP_FLOW_NC * CP_FLOW_P_PER; e += blockDim.x) sPk[e] = pk_g[e];
  for (int j = threadIdx.x; j < CP_FLOW_NC * CP_FLOW_NB; j += blockDim.x) sBias[j] = bias_g[j];
  __syncthreads();
  const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
  // the batch's moments and size (all ranks' points when the batch is sharded)
  const double sig = sums[0] / n_batch;
  const float cnorm = (float)(2.0 / (n_batch * sig * sig));
  // objective <w^p>/<w>^p: dL/d ln w of a point = p (w / sigma)^p / B (p = 2: 2 w^2 / (B sigma^2))
  const float cnorm_p = (float)(loss_p / n_batch), inv_sig = (float)(1.0 / sig);
  const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
  const uint64_t rounds = (n + 32 * warps - 1) / (32 * warps);
  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t base = (r * warps + (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * 32;
    const uint64_t p = base + lane;
    const bool active = p < n;
    float dz[3] = {0.f, 0.f, 0.f}, cJ = 0.f;
    if (active) {
      const float4 f = vj[p], g = wg[p];
      cJ = loss_p == 2.f ? cnorm * g.x * g.x : cnorm_p * powf(g.x * inv_sig, loss_p);
      const float v[3] = {f.x, f.y, f.z}, gv[3] = {g.y, g.z, g.w};
      // sigmoid: dv/dz = v (1 - v); d ln(v (1 - v))/dz = 1 - 2 v
      for (int d = 0; d < 3; ++d) dz[d] = cJ * gv[d] * v[d] * (1.f - v[d]) + cJ * (1.f - 2.f * v[d]);
    }
#pragma unroll 1
    for (int c = CP_FLOW_NC - 1; c >= 0; --c) {
      const CpCoupling k = cp_coupling(c);
      const uint2* pk = sPk + c * CP_FLOW_P_PER;
      const float* b = sBias + c * CP_FLOW_NB;
      float zin[3] = {0.f, 0.f, 0.f};
      if (active)
        for (int d = 0; d < 3; ++d) zin[d] = zs[(p * CP_FLOW_NC + c) * 3 + d];
      const float in0 = zin[k.cin[0]], in1 = k.nin > 1 ? zin[k.cin[1]] : 0.f;
      const uint64_t off = (uint64_t)c * n;
#pragma unroll 1
      for (int tile = 0; tile < 2; ++tile) {
        const int tb = 16 * tile;
        const uint64_t row0 = base + tb;
        // ---- recompute the MLP forward of this tile (A fragments kept for the ReLU masks)
        float r0a = __shfl_sync(0xffffffffu, in0, tb + gid), r0b = __shfl_sync(0xffffffffu, in1, tb + gid);
        float r8a = __shfl_sync(0xffffffffu, in0, tb + gid + 8), r8b = __shfl_sync(0xffffffffu, in1, tb + gid + 8);
        uint32_t a[4] = {tig == 0 ? cp_bf2(r0a, r0b) : 0u, tig == 0 ? cp_bf2(r8a, r8b) : 0u, 0u, 0u};
        if (tig == 0) {
          if (row0 + gid < n) *reinterpret_cast<uint32_t*>(out.X + (off + row0 + gid) * 16) = a[0];
          if (row0 + gid + 8 < n) *reinterpret_cast<uint32_t*>(out.X + (off + row0 + gid + 8) * 16) = a[1];
        }
        float acc[8][4];
        uint32_t h1[4][4], h2[4][4];
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          const float b0 = b[nt * 8 + 2 * tig], b1 = b[nt * 8 + 2 * tig + 1];
          acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
          cp_mma_bf16(acc[nt], a, pk[CP_FLOW_P_W1 + nt * 32 + lane]);
        }
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          h1[kt][0] = cp_bf2(fmaxf(acc[2 * kt][0], 0.f), fmaxf(acc[2 * kt][1], 0.f));
          h1[kt][1] = cp_bf2(fmaxf(acc[2 * kt][2], 0.f), fmaxf(acc[2 * kt][3], 0.f));
          h1[kt][2] = cp_bf2(fmaxf(acc[2 * kt + 1][0], 0.f), fmaxf(acc[2 * kt + 1][1], 0.f));
          h1[kt][3] = cp_bf2(fmaxf(acc[2 * kt + 1][2], 0.f), fmaxf(acc[2 * kt + 1][3], 0.f));
        }
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          const float b0 = b[64 + nt * 8 + 2 * tig], b1 = b[64 + nt * 8 + 2 * tig + 1];
          acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
#pragma unroll
          for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(acc[nt], h1[kt], pk[CP_FLOW_P_W2 + (kt * 8 + nt) * 32 + lane]);
        }
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          h2[kt][0] = cp_bf2(fmaxf(acc[2 * kt][0], 0.f), fmaxf(acc[2 * kt][1], 0.f));
          h2[kt][1] = cp_bf2(fmaxf(acc[2 * kt][2], 0.f), fmaxf(acc[2 * kt][3], 0.f));
          h2[kt][2] = cp_bf2(fmaxf(acc[2 * kt + 1][0], 0.f), fmaxf(acc[2 * kt + 1][1], 0.f));
          h2[kt][3] = cp_bf2(fmaxf(acc[2 * kt + 1][2], 0.f), fmaxf(acc[2 * kt + 1][3], 0.f));
        }
        cp_store_rowfrag(out.H1 + off * 64, 64, row0, n, gid, tig, h1);
        cp_store_rowfrag(out.H2 + off * 64, 64, row0, n, gid, tig, h2);
        float c3[4] = {b[128 + 2 * tig], b[128 + 2 * tig + 1], b[128 + 2 * tig], b[128 + 2 * tig + 1]};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(c3, h2[kt], pk[CP_FLOW_P_W3 + kt * 32 + lane]);
        // ---- this tile's rows: outputs to the point lanes, coupling backward there
        const int rr = (lane - tb) & 15, src = 4 * (rr & 7);
        const bool hi = rr >= 8, mine = lane >= tb && lane < tb + 16;
        float o[4];
        {
          float x0 = __shfl_sync(0xffffffffu, c3[0], src), x1 = __shfl_sync(0xffffffffu, c3[1], src);
          float x2 = __shfl_sync(0xffffffffu, c3[2], src), x3 = __shfl_sync(0xffffffffu, c3[3], src);
          float y0 = __shfl_sync(0xffffffffu, c3[0], src + 1), y1 = __shfl_sync(0xffffffffu, c3[1], src + 1);
          float y2 = __shfl_sync(0xffffffffu, c3[2], src + 1), y3 = __shfl_sync(0xffffffffu, c3[3], src + 1);
          o[0] = hi ? x2 : x0; o[1] = hi ? x3 : x1; o[2] = hi ? y2 : y0; o[3] = hi ? y3 : y1;
        }
        float dO[4] = {0.f, 0.f, 0.f, 0.f};
        float dzT[2] = {0.f, 0.f};
        if (mine && active) {
          for (int j = 0; j < k.nt; ++j) {
            const float th = tanhf(o[j] / CP_FLOW_S), s = CP_FLOW_S * th, e = expf(s);
            const int d = k.tr[j];
            const float dzo = dz[d];
            const float ds = fmaf(dzo * zin[d], e, cJ);
            dO[j] = ds * (1.f - th * th);
            dO[k.nt + j] = dzo;
            dzT[j] = dzo * e;
          }
        }
        // dO as an A fragment: columns 0..3, rows gid and gid + 8
        // (a shuffle sends the value the source lane holds, so fetch all four and select here)
        float g0[4], g8[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          g0[q] = __shfl_sync(0xffffffffu, dO[q], tb + gid);
          g8[q] = __shfl_sync(0xffffffffu, dO[q], tb + gid + 8);
        }
        const bool odd = tig & 1;
        uint32_t ad[4] = {tig < 2 ? cp_bf2(odd ? g0[2] : g0[0], odd ? g0[3] : g0[1]) : 0u,
                          tig < 2 ? cp_bf2(odd ? g8[2] : g8[0], odd ? g8[3] : g8[1]) : 0u, 0u, 0u};
        if (tig < 2) {
          if (row0 + gid < n) *reinterpret_cast<uint32_t*>(out.DO + (off + row0 + gid) * 16 + 2 * tig) = ad[0];
          if (row0 + gid + 8 < n) *reinterpret_cast<uint32_t*>(out.DO + (off + row0 + gid + 8) * 16 + 2 * tig) = ad[1];
        }
        // dH2 = dO W3^T, masked by the ReLU of layer 2
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
          cp_mma_bf16(acc[nt], ad, pk[CP_FLOW_P_W3T + nt * 32 + lane]);
          const uint32_t m01 = h2[nt >> 1][(nt & 1) ? 2 : 0], m23 = h2[nt >> 1][(nt & 1) ? 3 : 1];
          if (cp_bf_lo(m01) <= 0.f) acc[nt][0] = 0.f;
          if (cp_bf_hi(m01) <= 0.f) acc[nt][1] = 0.f;
          if (cp_bf_lo(m23) <= 0.f) acc[nt][2] = 0.f;
          if (cp_bf_hi(m23) <= 0.f) acc[nt][3] = 0.f;
        }
        uint32_t d2[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          d2[kt][0] = cp_bf2(acc[2 * kt][0], acc[2 * kt][1]);
          d2[kt][1] = cp_bf2(acc[2 * kt][2], acc[2 * kt][3]);
          d2[kt][2] = cp_bf2(acc[2 * kt + 1][0], acc[2 * kt + 1][1]);
          d2[kt][3] = cp_bf2(acc[2 * kt + 1][2], acc[2 * kt + 1][3]);
        }
        cp_store_rowfrag(out.D2 + off * 64, 64, row0, n, gid, tig, d2);
        // dH1 = dH2 W2^T, masked by the ReLU of layer 1
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
          acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
          for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(acc[nt], d2[kt], pk[CP_FLOW_P_W2T + (kt * 8 + nt) * 32 + lane]);
          const uint32_t m01 = h1[nt >> 1][(nt & 1) ? 2 : 0], m23 = h1[nt >> 1][(nt & 1) ? 3 : 1];
          if (cp_bf_lo(m01) <= 0.f) acc[nt][0] = 0.f;
          if (cp_bf_hi(m01) <= 0.f) acc[nt][1] = 0.f;
          if (cp_bf_lo(m23) <= 0.f) acc[nt][2] = 0.f;
          if (cp_bf_hi(m23) <= 0.f) acc[nt][3] = 0.f;
        }
        uint32_t d1[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
          d1[kt][0] = cp_bf2(acc[2 * kt][0], acc[2 * kt][1]);
          d1[kt][1] = cp_bf2(acc[2 * kt][2], acc[2 * kt][3]);
          d1[kt][2] = cp_bf2(acc[2 * kt + 1][0], acc[2 * kt + 1][1]);
          d1[kt][3] = cp_bf2(acc[2 * kt + 1][2], acc[2 * kt + 1][3]);
        }
        cp_store_rowfrag(out.D1 + off * 64, 64, row0, n, gid, tig, d1);
        // dX = dH1 W1^T: columns 0..1 are the gradients of the two input features
        float cx[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(cx, d1[kt], pk[CP_FLOW_P_W1T + kt * 32 + lane]);
        const float e0 = __shfl_sync(0xffffffffu, cx[0], src), e1 = __shfl_sync(0xffffffffu, cx[1], src);
        const float e2 = __shfl_sync(0xffffffffu, cx[2], src), e3 = __shfl_sync(0xffffffffu, cx[3], src);
        if (mine && active) {
          const float dx0 = hi ? e2 : e0, dx1 = hi ? e3 : e1;
          for (int j = 0; j < k.nt; ++j) dz[k.tr[j]] = dzT[j];
          dz[k.cin[0]] += dx0;
          if (k.nin > 1) dz[k.cin[1]] += dx1;
        }
      }
    }
  }
}

// ------------------------------------------------------------------------------------------
// 4. weight and bias gradients of one layer shape for all couplings (blockIdx.y = coupling):
//    block b's chunk of points gives G_b[M][N] = sum_p A[p][0:M]^T B[p][0:N] on the tensor cores
//    and the bias gradient Gb_b[N] = sum_p B[p][0:N] from the same staged tiles, stored into its
//    own slot of the partial buffer (A, B bf16 row-major with leading dims M and N; M in {16, 64},
//    N in {16, 64}); k_flow_gsum then adds the slots in block order, so a training run is
//    reproducible bit for bit (no floating-point atomics).
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_ldsm_x4_t(uint32_t r[4], const void* p)
{
  const uint32_t a = (uint32_t)__cvta_generic_to_shared(p);
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]) : "r"(a));
}

#define CP_WG_ROWS 64   // points staged per iteration
#define CP_WG_MAXBLK 64 // blocks per coupling and layer (the batch is cut into at most this many chunks)

template <int M, int N>
__global__ void __launch_bounds__(128) k_flow_wgrad(const uint16_t* __restrict__ A0, const uint16_t* __restrict__ B0,
                                                    uint64_t n, float* __restrict__ part, int goff, int ldg, int nvalid,
                                                    int chunk, int bias_rel)
{
  constexpr int MT = M / 16, NT = N / 8, TPW = (MT * NT + 3) / 4;
  __shared__ __align__(16) uint16_t sA[CP_WG_ROWS * M];
  __shared__ __align__(16) uint16_t sB[CP_WG_ROWS * N];
  __shared__ float sBias[128];
  const int c = blockIdx.y;
  const uint16_t* A = A0 + (uint64_t)c * n * M;
  const uint16_t* B = B0 + (uint64_t)c * n * N;
  float* G = part + (size_t)blockIdx.x * CP_FLOW_NPARAM + c * CP_FLOW_PER + goff;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
  const int mi = lane >> 3, rw = lane & 7;
  float acc[TPW][4];
#pragma unroll
  for (int j = 0; j < TPW; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.f;
  const int bcol = threadIdx.x % N, brow0 = threadIdx.x / N;
  float bsum = 0.f;
  const uint64_t p_begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t p_end = p_begin + chunk < n ? p_begin + chunk : n;
  for (uint64_t p0 = p_begin; p0 < p_end; p0 += CP_WG_ROWS) {
    for (int e = threadIdx.x; e < CP_WG_ROWS * M / 8; e += blockDim.x) {
      const int row = e / (M / 8), col = (e % (M / 8)) * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p0 + row < p_end) v = *reinterpret_cast<const uint4*>(A + (p0 + row) * M + col);
      *reinterpret_cast<uint4*>(&sA[row * M + col]) = v;
    }
    for (int e = threadIdx.x; e < CP_WG_ROWS * N / 8; e += blockDim.x) {
      const int row = e / (N / 8), col = (e % (N / 8)) * 8;
      uint4 v = make_uint4(0, 0, 0, 0);
      if (p0 + row < p_end) v = *reinterpret_cast<const uint4*>(B + (p0 + row) * N + col);
      *reinterpret_cast<uint4*>(&sB[row * N + col]) = v;
    }
    __syncthreads();
    for (int r = brow0; r < CP_WG_ROWS; r += 128 / N) bsum += __uint_as_float(((uint32_t)sB[r * N + bcol]) << 16);
#pragma unroll
    for (int ks = 0; ks < CP_WG_ROWS / 16; ++ks) {
      const uint16_t* tA = sA + ks * 16 * M;
      const uint16_t* tB = sB + ks * 16 * N;
#pragma unroll
      for (int j = 0; j < TPW; ++j) {
        const int t = warp + 4 * j;
        if (t < MT * NT) {
          const int mt = t / NT, nt = t % NT;
          uint32_t a[4], bq[2];
          // A^T of m-tile mt: 8x8 blocks (points 0-7 | 8-15) x (m +0 | +8), delivered transposed
          cp_ldsm_x4_t(a, &tA[((mi >> 1) * 8 + rw) * M + mt * 16 + (mi & 1) * 8]);
          // B of n-tile nt: blocks (points 0-7 | 8-15) x (n tile), delivered transposed
          {
            const uint32_t ad = (uint32_t)__cvta_generic_to_shared(&tB[((mi & 1) * 8 + rw) * N + nt * 8]);
            asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                         : "=r"(bq[0]), "=r"(bq[1]) : "r"(ad));
          }
          cp_mma_bf16(acc[j], a, make_uint2(bq[0], bq[1]));
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int j = 0; j < TPW; ++j) {
    const int t = warp + 4 * j;
    if (t >= MT * NT) continue;
    const int mt = t / NT, nt = t % NT;
    const int m0 = mt * 16 + gid, n0 = nt * 8 + 2 * tig;
    if (n0 < nvalid) { G[m0 * ldg + n0] = acc[j][0]; G[(m0 + 8) * ldg + n0] = acc[j][2]; }
    if (n0 + 1 < nvalid) { G[m0 * ldg + n0 + 1] = acc[j][1]; G[(m0 + 8) * ldg + n0 + 1] = acc[j][3]; }
  }
  // the 128 / N threads of a bias column add their row sums in thread order
  sBias[threadIdx.x] = bsum;
  __syncthreads();
  if (threadIdx.x < N && threadIdx.x < nvalid) {
    float b = 0.f;
    for (int r = 0; r < 128 / N; ++r) b += sBias[r * N + threadIdx.x];
    G[bias_rel + threadIdx.x] = b;
  }
}

// ------------------------------------------------------------------------------------------
// 4'. The same weight and bias gradients on the 5th-generation tensor cores, all couplings and
//     the three layer shapes in one launch (blockIdx.y = coupling, blockIdx.z = layer).  Every
//     product has the hidden side (64 wide) as M and the other side as N:
//       layer 0: dW1^T[n][k] = sum_p D1[p][n] X[p][k]    M = 64 (n), N = 16 (k), bias b1 = sum D1
//       layer 1: dW2[k][n]   = sum_p H1[p][k] D2[p][n]   M = 64 (k), N = 64 (n), bias b2 = sum D2
//       layer 2: dW3[k][n]   = sum_p H2[p][k] DO[p][n]   M = 64 (k), N = 16 (n), bias b3 = sum DO
//     so D[M][N] += A[M][K] B[N][K]^T with K = the block's points, 64 per stage: A and B are the
//     row-major [point][feature] arrays read as MN-major operands (features contiguous).  Shared
//     memory holds them in the no-swizzle MN-major canonical layout: core matrices of 8 features
//     (16 bytes) x 8 points, 128 bytes; element (feature f, point q) of a stage at
//     (q / 8) * (F / 8) * 128 + (f / 8) * 128 + (q % 8) * 16 + (f % 8) * 2, so the descriptor's
//     stride in the feature direction (SBO) is 128 bytes and in the point direction (LBO)
//     (F / 8) * 128.  Stages are copied with cp.async (16-byte chunks, zero fill past the chunk's
//     end) into two buffers; one thread issues a stage's four K = 16 MMAs and commits them to the
//     buffer's mbarrier, which every thread waits on (bounded) before the buffer is refilled.  The
//     M = 64 accumulator occupies TMEM lanes 0-15 of each 32-lane quarter (row r in lane
//     r % 16 + 32 (r / 16)), so thread t < 16 of warp w reads row 16 w + t.  Each block writes its
//     own slot of the partial buffer; k_flow_gsum adds the slots in block order.
// ------------------------------------------------------------------------------------------
#define CP_WGT_STAGE 64   // points per stage (four K = 16 MMAs)

__device__ __forceinline__ void cp_cp_async16(uint32_t dst, const void* src, bool valid)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// one stage of F-wide rows [q0, q0 + 64) of X (row-major, leading dim F) into the MN-major layout
template <int F>
__device__ __forceinline__ void cp_wgt_stage_load(uint32_t sdst, const uint16_t* __restrict__ X, uint64_t q0,
                                                  uint64_t q_end)
{
  constexpr int CH = CP_WGT_STAGE * F / 8;   // 16-byte chunks
  for (int e = threadIdx.x; e < CH; e += blockDim.x) {
    // e = (point group, feature group, point within group): consecutive threads fill a core
    // matrix's consecutive 16-byte rows
    const int qg = e / (F / 8 * 8), fg = (e / 8) % (F / 8), r = e % 8;
    const uint64_t q = q0 + qg * 8 + r;
    const bool ok = q < q_end;
    cp_cp_async16(sdst + (uint32_t)e * 16u, X + (ok ? q : q0) * F + fg * 8, ok);
  }
}

__device__ __forceinline__ float cp_wgt_elem(const uint8_t* s, int F, int f, int q)
{
  const uint16_t v = *reinterpret_cast<const uint16_t*>(s + (q / 8) * (F / 8) * 128 + (f / 8) * 128 + (q % 8) * 16 + (f % 8) * 2);
  return __uint_as_float((uint32_t)v << 16);
}

template <int NB>
__device__ __forceinline__ void cp_wgt_layer(const uint16_t* __restrict__ A, const uint16_t* __restrict__ B, bool bias_of_a,
                                             uint64_t p_begin, uint64_t p_end, float* __restrict__ G, int layer,
                                             uint8_t* smem, uint32_t tmem, uint32_t mbar0, float* sBias,
                                             int* __restrict__ status)
{
  constexpr int ABYTES = CP_WGT_STAGE * 64 * 2, BBYTES = CP_WGT_STAGE * NB * 2;
  const uint32_t sbase = cp_smem_u32(smem);
  const uint32_t sA[2] = {sbase, sbase + ABYTES}, sB[2] = {sbase + 2 * ABYTES, sbase + 2 * ABYTES + BBYTES};
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(NB >> 3) << 17) |
                         ((uint32_t)(64 >> 4) << 24);
  const int nst = (int)((p_end - p_begin + CP_WGT_STAGE - 1) / CP_WGT_STAGE);
  const int tid = threadIdx.x;
  // bias column of this thread and its share of a stage's points (fixed order)
  constexpr int BW = 64;   // the bias side is 64 wide for layer 0 (A = D1), NB wide otherwise
  const int bw = bias_of_a ? BW : NB;
  const int bcol = tid % bw, bsplit = 128 / bw, brow0 = tid / bw;
  float bsum = 0.f;
  uint32_t phase[2] = {0u, 0u};
  volatile int abort_flag = 0;
  bool ok = true;
  cp_wgt_stage_load<64>(sA[0], A, p_begin, p_end);
  cp_wgt_stage_load<NB>(sB[0], B, p_begin, p_end);
  cp_cp_async_commit();
  for (int st = 0; st < nst; ++st) {
    const int b = st & 1;
    if (st + 1 < nst) {
      // the other buffer was read by stage st - 1's MMAs: wait for their commit before refilling
      if (st >= 1) {
        ok = ok && cp_mbar_wait_bounded(mbar0 + 8 * (1 - b), phase[1 - b], &abort_flag);
        phase[1 - b] ^= 1u;
      }
      const uint64_t q0 = p_begin + (uint64_t)(st + 1) * CP_WGT_STAGE;
      cp_wgt_stage_load<64>(sA[1 - b], A, q0, p_end);
      cp_wgt_stage_load<NB>(sB[1 - b], B, q0, p_end);
      cp_cp_async_commit();
      cp_cp_async_wait<1>();
    } else {
      cp_cp_async_wait<0>();
    }
    cp_fence_proxy_async();
    __syncthreads();
    {
      const uint8_t* sb = smem + (bias_of_a ? (b ? ABYTES : 0) : 2 * ABYTES + (b ? BBYTES : 0));
      for (int q = brow0; q < CP_WGT_STAGE; q += bsplit) bsum += cp_wgt_elem(sb, bias_of_a ? 64 : NB, bcol, q);
    }
    if (tid == 0 && ok) {
      cp_tc_fence_after();
#pragma unroll
      for (int k = 0; k < CP_WGT_STAGE / 16; ++k) {
        // K = 16 points = two point groups: +2 groups of (F / 8) core matrices
        const uint64_t da = cp_tc_desc(sA[b] + k * 2 * (64 / 8) * 128, (64 / 8) * 128, 128);
        const uint64_t db = cp_tc_desc(sB[b] + k * 2 * (NB / 8) * 128, (NB / 8) * 128, 128);
        cp_tc_mma(tmem, da, db, idesc, (st > 0 || k > 0) ? 1u : 0u);
      }
      cp_tc_commit(mbar0 + 8 * b);
    } else if (tid == 0) {
      cp_tc_commit(mbar0 + 8 * b);   // nothing issued: the barrier still completes its phase
    }
  }
  // the last stage's MMAs (and, in order, every earlier one) have completed
  const int bl = (nst - 1) & 1;
  ok = ok && cp_mbar_wait_bounded(mbar0 + 8 * bl, phase[bl], &abort_flag);
  if (nst >= 2) ok = ok && cp_mbar_wait_bounded(mbar0 + 8 * (1 - bl), phase[1 - bl], &abort_flag);
  cp_tc_fence_after();
  ok = __syncthreads_and(ok) != 0;
  if (!ok) {
    // a wait expired: record it, and before TMEM is released let every MMA this thread issued
    // complete (a fresh barrier, bounded wait)
    if (tid == 0) {
      atomicOr(status, 2);
      cp_tc_commit(mbar0 + 16);
      volatile int drain_abort = 0;
      cp_mbar_wait_bounded(mbar0 + 16, 0u, &drain_abort);
    }
    __syncthreads();
    return;
  }
  // accumulator: warp w, lane t < 16 = row 16 w + t
  const int warp = tid >> 5, lane = tid & 31, row = 16 * warp + lane;
  const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16);
#pragma unroll
  for (int half = 0; half < NB / 16; half += 2) {
    float v[32];
    if (NB == 64) {
      cp_tc_ld32(taddr + half * 16, v);
    } else {
      float v4[4];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        cp_tc_ld4(taddr + 4 * j, v4);
#pragma unroll
        for (int i = 0; i < 4; ++i) v[4 * j + i] = v4[i];
      }
    }
    if (lane < 16) {
      const int ncol = NB == 64 ? 32 : 16;
#pragma unroll
      for (int j = 0; j < ncol; ++j) {
        const int c = half * 16 + j;
        if (layer == 0) G[CP_FLOW_W1 + c * 64 + row] = v[j];                 // dW1[k = c][n = row]
        else if (layer == 1) G[CP_FLOW_W2 + row * 64 + c] = v[j];            // dW2[k = row][n = c]
        else if (c < 8) G[CP_FLOW_W3 + row * 8 + c] = v[j];                  // dW3[k = row][n = c < 8]
      }
    }
  }
  // bias: the bsplit threads of a column add their sums in thread order
  sBias[tid] = bsum;
  __syncthreads();
  const int nb_valid = layer == 2 ? 8 : 64;
  if (tid < bw && tid < nb_valid) {
    float acc = 0.f;
    for (int r = 0; r < bsplit; ++r) acc += sBias[r * bw + tid];
    G[(layer == 0 ? CP_FLOW_B1 : (layer == 1 ? CP_FLOW_B2 : CP_FLOW_B3)) + tid] = acc;
  }
}

__global__ void __launch_bounds__(128) k_flow_wgrad_tc(FlowTrainBufs t, uint64_t n, int chunk, int* __restrict__ status)
{
  // two A and two B stage buffers (32 KB), plus 8 KB so that the operand ranges of every
  // descriptor stay inside this array whichever of its two strides a layout reading applies
  __shared__ __align__(1024) uint8_t smem[2 * (CP_WGT_STAGE * 64 * 2) + 2 * (CP_WGT_STAGE * 64 * 2) + 8192];
  __shared__ float sBias[128];
  __shared__ __align__(8) uint64_t mbar[3];   // the two stage buffers' MMA commits, the drain
  __shared__ uint32_t tmem_slot;
  const int c = blockIdx.y, layer = blockIdx.z, tid = threadIdx.x;
  if (tid == 0) {
    for (int i = 0; i < 3; ++i) cp_mbar_init(cp_smem_u32(&mbar[i]), 1);
    cp_mbar_init_fence();
  }
  if ((tid >> 5) == 0) {
    cp_tc_alloc(cp_smem_u32(&tmem_slot), 64);
    cp_tc_relinquish();
  }
  cp_tc_fence_before();
  __syncthreads();
  cp_tc_fence_after();
  const uint32_t tmem = tmem_slot;
  const uint64_t p_begin = (uint64_t)blockIdx.x * chunk;
  const uint64_t p_end = p_begin + chunk < n ? p_begin + chunk : n;
  float* G = t.gpart + (size_t)blockIdx.x * CP_FLOW_NPARAM + c * CP_FLOW_PER;
  const uint64_t off = (uint64_t)c * n;
  const uint32_t mb = cp_smem_u32(&mbar[0]);
  if (p_begin < p_end) {
    if (layer == 0)
      cp_wgt_layer<16>(t.D1 + off * 64, t.X + off * 16, true, p_begin, p_end, G, 0, smem, tmem, mb, sBias, status);
    else if (layer == 1)
      cp_wgt_layer<64>(t.H1 + off * 64, t.D2 + off * 64, false, p_begin, p_end, G, 1, smem, tmem, mb, sBias, status);
    else
      cp_wgt_layer<16>(t.H2 + off * 64, t.DO + off * 16, false, p_begin, p_end, G, 2, smem, tmem, mb, sBias, status);
  }
  cp_tc_fence_before();
  __syncthreads();
  if ((tid >> 5) == 0) {
    cp_tc_fence_after();
    cp_tc_dealloc(tmem, 64);
  }
}

// G[i] += sum over the nblk block slots of the partial gradients, in block order
__global__ void k_flow_gsum(const float* __restrict__ part, int nblk, float* __restrict__ G)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= CP_FLOW_NPARAM) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += part[(size_t)b * CP_FLOW_NPARAM + i];
  G[i] += s;
}

// ------------------------------------------------------------------------------------------
// 5. Adam on the FP32 master weights (padding entries stay zero)
// ------------------------------------------------------------------------------------------
__host__ __device__ __forceinline__ bool cp_flow_param_used(int i)
{
  const int c = i / CP_FLOW_PER, o = i % CP_FLOW_PER;
  const CpCoupling k = cp_coupling(c);
  const int nout = 2 * k.nt;
  if (o < CP_FLOW_B1) return o / 64 < k.nin;
  if (o < CP_FLOW_B2) return true;
  if (o < CP_FLOW_W3) return true;
  if (o < CP_FLOW_B3) return ((o - CP_FLOW_W3) % 8) < nout;
  return (o - CP_FLOW_B3) < nout;
}

__device__ __forceinline__ void cp_flow_adam_one(int i, float g, float* __restrict__ P, float* __restrict__ Mo,
                                                 float* __restrict__ Vo, float lr, float b1t, float b2t)
{
  if (!cp_flow_param_used(i)) { P[i] = 0.f; return; }
  const float m = 0.9f * Mo[i] + 0.1f * g, v = 0.999f * Vo[i] + 0.001f * g * g;
  Mo[i] = m;
  Vo[i] = v;
  P[i] -= lr * (m / (1.f - b1t)) / (sqrtf(v / (1.f - b2t)) + 1e-8f);
}

__global__ void k_flow_adam(float* __restrict__ P, float* __restrict__ G, float* __restrict__ Mo, float* __restrict__ Vo,
                            float lr, float b1t, float b2t)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= CP_FLOW_NPARAM) return;
  const float g = G[i];
  G[i] = 0.f;
  cp_flow_adam_one(i, g, P, Mo, Vo, lr, b1t, b2t);
}

// k_flow_gsum into a cleared G followed by k_flow_adam, in one pass (a single handle's training
// loop, where no exchange of G sits between them): the same block-order sum, 0 + sum as the
// gradient, the same update, so the same parameters bit for bit; G is not touched.
__global__ void k_flow_gsum_adam(float* __restrict__ P, const float* __restrict__ part, int nblk, float* __restrict__ Mo,
                                 float* __restrict__ Vo, float lr, float b1t, float b2t)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= CP_FLOW_NPARAM) return;
  float s = 0.f;
  for (int b = 0; b < nblk; ++b) s += part[(size_t)b * CP_FLOW_NPARAM + i];
  cp_flow_adam_one(i, 0.f + s, P, Mo, Vo, lr, b1t, b2t);
}

// the batch's moments (summed over ranks) for the backward pass, and its loss <w^2> / <w>^2
__global__ void k_flow_batch_loss(const double* moments, double n, double* sums, double* loss)
{
  const double a = moments[0], b = moments[1];
  sums[0] = a;
  sums[1] = b;
  const double m = a / n;
  loss[0] = (b / n) / (m * m);
}

// ------------------------------------------------------------------------------------------
// host
// ------------------------------------------------------------------------------------------
static size_t train_bytes(uint64_t B)
{
  return B * (sizeof(float) * 12 + sizeof(float4) * 2 + 2 * CP_FLOW_NC * (16 + 64 * 4 + 16)) + 4096 +
         sizeof(float) * CP_WG_MAXBLK * CP_FLOW_NPARAM;
}

static FlowTrainBufs carve(void* base, uint64_t B)
{
  char* q = static_cast<char*>(base);
  FlowTrainBufs t;
  t.vj = reinterpret_cast<float4*>(q); q += sizeof(float4) * B;
  t.wg = reinterpret_cast<float4*>(q); q += sizeof(float4) * B;
  t.zs = reinterpret_cast<float*>(q); q += sizeof(float) * 12 * B;
  t.X = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 16 * B;
  t.H1 = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 64 * B;
  t.H2 = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 64 * B;
  t.D1 = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 64 * B;
  t.D2 = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 64 * B;
  t.DO = reinterpret_cast<uint16_t*>(q); q += 2 * CP_FLOW_NC * 16 * B;
  q = reinterpret_cast<char*>(((uintptr_t)q + 255) & ~(uintptr_t)255);
  t.sums = reinterpret_cast<double*>(q); q += 64;
  t.loss = reinterpret_cast<double*>(q); q += 64;
  t.gpart = reinterpret_cast<float*>(q);
  return t;
}

static size_t bwd_smem() { return sizeof(uint2) * CP_FLOW_NC * CP_FLOW_P_PER + sizeof(float) * CP_FLOW_NC * CP_FLOW_NB; }
static size_t fwd_smem() { return sizeof(uint2) * CP_FLOW_NC * CP_FLOW_P_FWD + sizeof(float) * CP_FLOW_NC * CP_FLOW_NB; }

// Training buffers for `count` points of a step, kept in the handle between the phases of a
// step.  A new layout (another count) starts from zeros: columns the kernels never write (the
// padding of the 16-wide operands) must read as zero.
static int train_buffers(cp_handle* h, uint64_t count, FlowTrainBufs& t)
{
  if (!h->d_ftrain || count > h->ftrain_cap) {
    if (h->d_ftrain) {
      CP_CUDA(h, cudaStreamSynchronize(h->stream));
      CP_CUDA(h, cudaFree(h->d_ftrain));
      h->d_ftrain = nullptr;
      h->ftrain_cap = 0;
    }
    CP_CUDA(h, cudaMalloc(&h->d_ftrain, train_bytes(count)));
    h->ftrain_cap = count;
    h->ftrain_count = 0;
  }
  if (count != h->ftrain_count) CP_CUDA(h, cudaMemsetAsync(h->d_ftrain, 0, train_bytes(count), h->stream));
  h->ftrain_count = count;
  t = carve(h->d_ftrain, count);
  // per-device attributes: set on every use (host-side, cheap)
  CP_CUDA(h, cudaFuncSetAttribute(k_flow_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bwd_smem()));
  CP_CUDA(h, cudaFuncSetAttribute(k_flow_fwd_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fwd_smem()));
  return CP_OK;
}

static void train_buffers_release(cp_handle* h)
{
  if (!h->d_ftrain) return;
  cudaStreamSynchronize(h->stream);
  cudaFree(h->d_ftrain);
  h->d_ftrain = nullptr;
  h->ftrain_cap = h->ftrain_count = 0;
}

// Phase 1 of a step: forward and integrand over the batch points [point0, point0 + count) at
// counter iteration `iter` (Philox stream 2); moments[0..1] = (sum w, sum w^2) over them.
static int flow_phase_moments(cp_handle* h, const FlowTrainBufs& t, uint64_t point0, uint64_t count, uint32_t iter,
                              double* moments, double* loss_dev = nullptr)
{
  k_flow_fwd_train<<<h->num_sms * 2, CP_THREADS, fwd_smem(), h->stream>>>(h->d_flow_pk, h->d_flow_bias, h->d_edges, h->nb,
                                                                           h->cfg.seed, iter, 2, point0, count, t.zs, t.vj);
  CP_LAUNCH_CHECK(h, "k_flow_fwd_train");
  const int gblk = h->num_sms * 4;
  int rc = cp_ensure_slots(h, (size_t)2 * gblk);
  if (rc) return rc;
  const float lnTauMin = (float)log(4.0 * h->cfg.pt_hat_min * h->cfg.pt_hat_min / (h->cfg.sqrt_s * h->cfg.sqrt_s));
  k_flow_igrad<<<gblk, 128, 0, h->stream>>>(h->P, h->d_cteq, count, lnTauMin, t.vj, t.wg, h->d_slots,
                                            h->d_flow_ticket, moments, (double)count, loss_dev);
  CP_LAUNCH_CHECK(h, "k_flow_igrad");
  return CP_OK;
}

// Phase 2: this handle's points' part of the gradient of the batch loss, from the batch's
// moments over n_batch points, into the gradient buffer G (cleared first); loss_dev = the loss.
// A single handle's loop passes local = true (moments already in t.sums, the loss written by
// phase 1): the per-block partial gradients are left in t.gpart for flow_phase_update_local,
// and *nblk_out receives their number.
static int flow_phase_gradient(cp_handle* h, const FlowTrainBufs& t, uint64_t count, const double* moments,
                               uint64_t n_batch, double* loss_dev, bool local = false, int* nblk_out = nullptr)
{
  if (!local) {
    k_flow_batch_loss<<<1, 1, 0, h->stream>>>(moments, (double)n_batch, t.sums, loss_dev);
    CP_LAUNCH_CHECK(h, "k_flow_batch_loss");
  }
  k_flow_bwd<<<h->num_sms * 2, CP_BWD_THREADS, bwd_smem(), h->stream>>>(h->d_flow_pk, h->d_flow_bias, count, (double)n_batch, t.zs,
                                                          t.vj, t.wg, t.sums, t, (float)h->flow_loss_p);
  CP_LAUNCH_CHECK(h, "k_flow_bwd");
  float* G = h->d_flow + CP_FLOW_NPARAM;
  // at most CP_WG_MAXBLK blocks per coupling and layer; chunks are whole multiples of the staged
  // rows.  The three launches share the grid, so together they write every entry of the
  // partial slots 0 .. nblk-1 (all of W1, b1, W2, b2, W3, b3 of every coupling).
  const uint64_t chunk = ((count + CP_WG_MAXBLK - 1) / CP_WG_MAXBLK + CP_WG_ROWS - 1) / CP_WG_ROWS * CP_WG_ROWS;
  const int nblk = (int)((count + chunk - 1) / chunk);
  if (h->flow_kernel == 0) {
    // tensor cores (tcgen05): every coupling and layer shape in one launch
    k_flow_wgrad_tc<<<dim3((unsigned)nblk, CP_FLOW_NC, 3), 128, 0, h->stream>>>(t, count, (int)chunk,
                                                                             h->d_flow_status);
    CP_LAUNCH_CHECK(h, "k_flow_wgrad_tc");
  } else {
    // warp-level mma.sync, one launch per layer shape (the cross-check path)
    const dim3 grid((unsigned)nblk, CP_FLOW_NC);
    k_flow_wgrad<16, 64><<<grid, 128, 0, h->stream>>>(t.X, t.D1, count, t.gpart, CP_FLOW_W1, 64, 64, (int)chunk,
                                                      CP_FLOW_B1 - CP_FLOW_W1);
    k_flow_wgrad<64, 64><<<grid, 128, 0, h->stream>>>(t.H1, t.D2, count, t.gpart, CP_FLOW_W2, 64, 64, (int)chunk,
                                                      CP_FLOW_B2 - CP_FLOW_W2);
    // W3 [64][8] from the 16-wide output-gradient rows (columns 8..15 are zero padding)
    k_flow_wgrad<64, 16><<<grid, 128, 0, h->stream>>>(t.H2, t.DO, count, t.gpart, CP_FLOW_W3, 8, 8, (int)chunk,
                                                      CP_FLOW_B3 - CP_FLOW_W3);
    CP_LAUNCH_CHECK(h, "k_flow_wgrad");
  }
  if (local) {
    *nblk_out = nblk;
    return CP_OK;
  }
  CP_CUDA(h, cudaMemsetAsync(G, 0, sizeof(float) * CP_FLOW_NPARAM, h->stream));
  k_flow_gsum<<<(CP_FLOW_NPARAM + 255) / 256, 256, 0, h->stream>>>(t.gpart, nblk, G);
  CP_LAUNCH_CHECK(h, "k_flow_gsum");
  return CP_OK;
}

// Phase 3: Adam step h->flow_t + 1 on the gradient in G (which it clears), BF16 repack.
static int flow_phase_update(cp_handle* h, double lr)
{
  float* G = h->d_flow + CP_FLOW_NPARAM;
  const long step = h->flow_t + 1;
  k_flow_adam<<<(CP_FLOW_NPARAM + 255) / 256, 256, 0, h->stream>>>(
      h->d_flow, G, G + CP_FLOW_NPARAM, G + 2 * CP_FLOW_NPARAM, (float)lr, (float)pow(0.9, (double)step),
      (float)pow(0.999, (double)step));
  CP_LAUNCH_CHECK(h, "k_flow_adam");
  const int rc = cp_flow_repack(h);
  if (rc) return rc;
  h->flow_t = step;
  return CP_OK;
}

// Phase 3 of a single handle's step: the block-order gradient sum and the Adam step in one kernel
// (the same parameters as k_flow_gsum + flow_phase_update), BF16 repack.
static int flow_phase_update_local(cp_handle* h, const FlowTrainBufs& t, int nblk, double lr)
{
  float* G = h->d_flow + CP_FLOW_NPARAM;
  const long step = h->flow_t + 1;
  k_flow_gsum_adam<<<(CP_FLOW_NPARAM + 255) / 256, 256, 0, h->stream>>>(
      h->d_flow, t.gpart, nblk, G + CP_FLOW_NPARAM, G + 2 * CP_FLOW_NPARAM, (float)lr, (float)pow(0.9, (double)step),
      (float)pow(0.999, (double)step));
  CP_LAUNCH_CHECK(h, "k_flow_gsum_adam");
  const int rc = cp_flow_repack(h);
  if (rc) return rc;
  h->flow_t = step;
  return CP_OK;
}

extern "C" int cp_flow_set_objective(cp_handle* h, double p)
{
  CP_CHECK_HANDLE(h);
  if (!(p >= 2.0 && p <= 8.0)) return cp_fail(h, CP_ERR_INVALID, "cp_flow_set_objective: p must be in [2, 8]");
  h->flow_loss_p = p;
  return CP_OK;
}

// Trains the flow for n_steps batches of `batch` points on the current VEGAS grid; loss_host
// (n_steps doubles, may be NULL) receives <w^2>/<w>^2 of each batch before its update.  Step s
// draws its batch at counter iteration flow_t (the number of updates so far), points 0..batch-1.
extern "C" int cp_flow_train(cp_handle* h, int n_steps, uint64_t batch, double lr, double* loss_host)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  if (n_steps < 1 || batch < 64 || batch > (1ull << 24) || (batch & 31))
    return cp_fail(h, CP_ERR_INVALID, "cp_flow_train: batch must be a multiple of 32 in [64, 2^24]");
  h->ftrain_count = 0;   // a fresh layout: the buffers start from zeros
  FlowTrainBufs t;
  int rc = train_buffers(h, batch, t);
  if (rc) return rc;
  double* losses = nullptr;
  CP_CUDA(h, cudaMalloc(&losses, sizeof(double) * (size_t)n_steps));
  for (int s = 0; s < n_steps && rc == CP_OK; ++s) {
    int nblk = 0;
    rc = flow_phase_moments(h, t, 0, batch, (uint32_t)h->flow_t, t.sums, losses + s);
    if (!rc) rc = flow_phase_gradient(h, t, batch, t.sums, batch, losses + s, true, &nblk);
    if (!rc) rc = flow_phase_update_local(h, t, nblk, lr);
  }
  cudaError_t e = cudaSuccess;
  if (!rc && loss_host) e = cudaMemcpyAsync(loss_host, losses, sizeof(double) * n_steps, cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (!rc && e != cudaSuccess) rc = cp_fail_cuda(h, e, "cp_flow_train readback");
  if (!rc) rc = cp_flow_tc_status(h);
  cudaFree(losses);
  train_buffers_release(h);
  return rc;
}

// Loss gradient of one batch without updating (for the gradient checks): grad_host receives
// cp_flow_num_params() floats (dL/dtheta of L = <w^2>/<w>^2), loss_host the batch loss.
extern "C" int cp_flow_loss_grad(cp_handle* h, uint64_t batch, uint32_t iter, float* grad_host, double* loss_host)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  if (batch < 64 || batch > (1ull << 24) || (batch & 31)) return cp_fail(h, CP_ERR_INVALID, "bad batch");
  h->ftrain_count = 0;
  FlowTrainBufs t;
  int rc = train_buffers(h, batch, t);
  if (rc) return rc;
  float* G = h->d_flow + CP_FLOW_NPARAM;
  rc = flow_phase_moments(h, t, 0, batch, iter, t.sums);
  if (!rc) rc = flow_phase_gradient(h, t, batch, t.sums, batch, t.loss);
  cudaError_t e = cudaSuccess;
  if (!rc) {
    e = cudaMemcpyAsync(grad_host, G, sizeof(float) * CP_FLOW_NPARAM, cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess && loss_host) e = cudaMemcpyAsync(loss_host, t.loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(G, 0, sizeof(float) * CP_FLOW_NPARAM, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) rc = cp_fail_cuda(h, e, "cp_flow_loss_grad readback");
  }
  if (!rc) rc = cp_flow_tc_status(h);
  train_buffers_release(h);
  return rc;
}

// ------------------------------------------------------------------------------------------
// Data-parallel training: one step in three calls, the caller summing over ranks in between.
// ------------------------------------------------------------------------------------------
extern "C" int cp_flow_step_moments(cp_handle* h, uint64_t point0, uint64_t count, double* moments_dev)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  if (count < 1 || count > (1ull << 24) || !moments_dev)
    return cp_fail(h, CP_ERR_INVALID, "cp_flow_step_moments: count must be in [1, 2^24]");
  FlowTrainBufs t;
  int rc = train_buffers(h, count, t);
  if (rc) return rc;
  return flow_phase_moments(h, t, point0, count, (uint32_t)h->flow_t, moments_dev);
}

extern "C" int cp_flow_step_gradient(cp_handle* h, const double* moments_dev, uint64_t batch_total, float* grad_dev,
                                     double* loss_host)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_ftrain || !h->ftrain_count || !moments_dev || batch_total < h->ftrain_count)
    return cp_fail(h, CP_ERR_INVALID, "cp_flow_step_gradient: call cp_flow_step_moments first (batch_total >= count)");
  FlowTrainBufs t = carve(h->d_ftrain, h->ftrain_count);
  int rc = flow_phase_gradient(h, t, h->ftrain_count, moments_dev, batch_total, t.loss);
  if (rc) return rc;
  if (grad_dev)
    CP_CUDA(h, cudaMemcpyAsync(grad_dev, h->d_flow + CP_FLOW_NPARAM, sizeof(float) * CP_FLOW_NPARAM,
                               cudaMemcpyDeviceToDevice, h->stream));
  if (loss_host) CP_CUDA(h, cudaMemcpyAsync(loss_host, t.loss, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  return cp_flow_tc_status(h);   // synchronises the stream
}

extern "C" int cp_flow_step_update(cp_handle* h, const float* grad_dev, double lr)
{
  CP_CHECK_HANDLE(h);
  if (!h->d_flow) return cp_fail(h, CP_ERR_INVALID, "flow not initialised (cp_flow_init)");
  if (!(lr > 0.0)) return cp_fail(h, CP_ERR_INVALID, "cp_flow_step_update: lr must be positive");
  if (grad_dev)
    CP_CUDA(h, cudaMemcpyAsync(h->d_flow + CP_FLOW_NPARAM, grad_dev, sizeof(float) * CP_FLOW_NPARAM,
                               cudaMemcpyDeviceToDevice, h->stream));
  return flow_phase_update(h, lr);
}
