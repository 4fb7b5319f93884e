// cp_flow.cuh -- the learned proposal: a RealNVP-style normalising flow on [0,1]^3 placed
// after the VEGAS map.  u (Philox words) -> VEGAS map -> x_v -> z = logit(x_v) -> 4 affine
// coupling layers -> x = sigmoid(z) -> base map (tau, y, z).  Each coupling conditions on some
// coordinates and moves the others: z_T <- z_T exp(s) + t, with (s_raw, t) from an MLP
// in -> 64 -> 64 -> out (ReLU), s = 4 tanh(s_raw / 4).  The point weight gains |dx/dx_v|.
// The flow sits after the VEGAS map, not before it: the VEGAS Jacobian is piecewise constant
// in its input, so a flow in front of it would see a weight that jumps at every bin edge, and
// the pathwise training gradient (which cannot see those jumps) would be biased; after the map,
// the bin of every point is fixed by its random numbers and the weight is smooth in the flow.
//
// Dense layers run on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulate); a
// warp's 32 points form two 16-row tiles, and the three layers chain in registers (the FP32
// accumulator fragment of one layer is, after BF16 packing, the A fragment of the next).
#pragma once
#include <cuda_bf16.h>
#include "cp_integrand.cuh"

#define CP_FLOW_NC 4            // coupling layers
#define CP_FLOW_H 64            // hidden width
// FP32 master parameters per coupling: W1[16][64] (input rows >= n_in are zero), b1[64],
// W2[64][64], b2[64], W3[64][8] (output columns >= n_out are zero), b3[8]
#define CP_FLOW_W1 0
#define CP_FLOW_B1 1024
#define CP_FLOW_W2 1088
#define CP_FLOW_B2 5184
#define CP_FLOW_W3 5248
#define CP_FLOW_B3 5760
#define CP_FLOW_PER 5768
#define CP_FLOW_NPARAM (CP_FLOW_NC * CP_FLOW_PER)
// packed BF16 B fragments per coupling (uint2 per lane per (ktile, ntile)):
// forward W1 (1x8 tiles), W2 (4x8), W3 (4x1); backward W3^T (1x8), W2^T (4x8), W1^T (4x1)
#define CP_FLOW_P_W1 0
#define CP_FLOW_P_W2 (8 * 32)
#define CP_FLOW_P_W3 (CP_FLOW_P_W2 + 32 * 32)
#define CP_FLOW_P_W3T (CP_FLOW_P_W3 + 4 * 32)
#define CP_FLOW_P_W2T (CP_FLOW_P_W3T + 8 * 32)
#define CP_FLOW_P_W1T (CP_FLOW_P_W2T + 32 * 32)
#define CP_FLOW_P_FWD (CP_FLOW_P_W3T)                 // forward part, uint2 per coupling
#define CP_FLOW_P_PER (CP_FLOW_P_W1T + 4 * 32)        // uint2 per coupling
#define CP_FLOW_S 4.0f          // scale soft clamp
#define CP_FLOW_NB 136          // staged biases per coupling: b1[64], b2[64], b3[8]

// coupling masks: conditioning dims and transformed dims
struct CpCoupling {
  int nin, nt;
  int cin[2];
  int tr[2];
};
__host__ __device__ __forceinline__ CpCoupling cp_coupling(int c)
{
  CpCoupling k;
  if (c == 0) { k.nin = 1; k.cin[0] = 0; k.cin[1] = 0; k.nt = 2; k.tr[0] = 1; k.tr[1] = 2; }
  else if (c == 1) { k.nin = 2; k.cin[0] = 1; k.cin[1] = 2; k.nt = 1; k.tr[0] = 0; k.tr[1] = 0; }
  else if (c == 2) { k.nin = 1; k.cin[0] = 1; k.cin[1] = 1; k.nt = 2; k.tr[0] = 0; k.tr[1] = 2; }
  else { k.nin = 2; k.cin[0] = 0; k.cin[1] = 2; k.nt = 1; k.tr[0] = 1; k.tr[1] = 1; }
  return k;
}

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t cp_bf2(float lo, float hi)
{
  __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&v);
}

__device__ __forceinline__ void cp_mma_bf16(float c[4], const uint32_t a[4], uint2 b)
{
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b.x), "r"(b.y));
}

// MLP of coupling c over one 16-row tile.  xin[r] holds the tile's input features (row r =
// lane tb + r).  Returns, in every lane, the FP32 output columns of that lane's own row in o[4]
// (meaningful when the lane belongs to the tile).  If h1s / h2s are given (training), the
// BF16-rounded post-ReLU activations of the tile are stored to them row-major [16][64].
__device__ __forceinline__ void cp_flow_mlp_tile(const uint2* __restrict__ pk, const float* __restrict__ bias1,
                                                 const float* __restrict__ bias2, const float* __restrict__ bias3,
                                                 float in0, float in1, int nin, int tb, float o[4],
                                                 uint32_t* h1s = nullptr, uint32_t* h2s = nullptr)
{
  const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
  // layer-1 A fragment: columns 0..1 hold the features of rows gid and gid + 8
  float r0a = __shfl_sync(0xffffffffu, in0, tb + gid), r0b = __shfl_sync(0xffffffffu, in1, tb + gid);
  float r8a = __shfl_sync(0xffffffffu, in0, tb + gid + 8), r8b = __shfl_sync(0xffffffffu, in1, tb + gid + 8);
  uint32_t a[4];
  a[0] = tig == 0 ? cp_bf2(r0a, nin > 1 ? r0b : 0.f) : 0u;
  a[1] = tig == 0 ? cp_bf2(r8a, nin > 1 ? r8b : 0.f) : 0u;
  a[2] = 0u;
  a[3] = 0u;
  float acc[8][4];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias1[nt * 8 + 2 * tig], b1 = bias1[nt * 8 + 2 * tig + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
    cp_mma_bf16(acc[nt], a, pk[CP_FLOW_P_W1 + nt * 32 + lane]);
  }
  uint32_t h[4][4];
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    h[kt][0] = cp_bf2(fmaxf(acc[2 * kt][0], 0.f), fmaxf(acc[2 * kt][1], 0.f));
    h[kt][1] = cp_bf2(fmaxf(acc[2 * kt][2], 0.f), fmaxf(acc[2 * kt][3], 0.f));
    h[kt][2] = cp_bf2(fmaxf(acc[2 * kt + 1][0], 0.f), fmaxf(acc[2 * kt + 1][1], 0.f));
    h[kt][3] = cp_bf2(fmaxf(acc[2 * kt + 1][2], 0.f), fmaxf(acc[2 * kt + 1][3], 0.f));
  }
  if (h1s) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      h1s[(gid * 64 + 16 * kt + 2 * tig) / 2] = h[kt][0];
      h1s[((gid + 8) * 64 + 16 * kt + 2 * tig) / 2] = h[kt][1];
      h1s[(gid * 64 + 16 * kt + 8 + 2 * tig) / 2] = h[kt][2];
      h1s[((gid + 8) * 64 + 16 * kt + 8 + 2 * tig) / 2] = h[kt][3];
    }
  }
#pragma unroll
  for (int nt = 0; nt < 8; ++nt) {
    const float b0 = bias2[nt * 8 + 2 * tig], b1 = bias2[nt * 8 + 2 * tig + 1];
    acc[nt][0] = b0; acc[nt][1] = b1; acc[nt][2] = b0; acc[nt][3] = b1;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(acc[nt], h[kt], pk[CP_FLOW_P_W2 + (kt * 8 + nt) * 32 + lane]);
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) {
    h[kt][0] = cp_bf2(fmaxf(acc[2 * kt][0], 0.f), fmaxf(acc[2 * kt][1], 0.f));
    h[kt][1] = cp_bf2(fmaxf(acc[2 * kt][2], 0.f), fmaxf(acc[2 * kt][3], 0.f));
    h[kt][2] = cp_bf2(fmaxf(acc[2 * kt + 1][0], 0.f), fmaxf(acc[2 * kt + 1][1], 0.f));
    h[kt][3] = cp_bf2(fmaxf(acc[2 * kt + 1][2], 0.f), fmaxf(acc[2 * kt + 1][3], 0.f));
  }
  if (h2s) {
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
      h2s[(gid * 64 + 16 * kt + 2 * tig) / 2] = h[kt][0];
      h2s[((gid + 8) * 64 + 16 * kt + 2 * tig) / 2] = h[kt][1];
      h2s[(gid * 64 + 16 * kt + 8 + 2 * tig) / 2] = h[kt][2];
      h2s[((gid + 8) * 64 + 16 * kt + 8 + 2 * tig) / 2] = h[kt][3];
    }
  }
  float c3[4];
  {
    const float b0 = bias3[2 * tig], b1 = bias3[2 * tig + 1];
    c3[0] = b0; c3[1] = b1; c3[2] = b0; c3[3] = b1;
  }
#pragma unroll
  for (int kt = 0; kt < 4; ++kt) cp_mma_bf16(c3, h[kt], pk[CP_FLOW_P_W3 + kt * 32 + lane]);
  // row r = lane - tb: columns 0,1 from lane 4 (r % 8), columns 2,3 from lane 4 (r % 8) + 1
  const int r = (lane - tb) & 15, src = 4 * (r & 7);
  const bool hi = r >= 8;
  float x0 = __shfl_sync(0xffffffffu, c3[0], src), x1 = __shfl_sync(0xffffffffu, c3[1], src);
  float x2 = __shfl_sync(0xffffffffu, c3[2], src), x3 = __shfl_sync(0xffffffffu, c3[3], src);
  float y0 = __shfl_sync(0xffffffffu, c3[0], src + 1), y1 = __shfl_sync(0xffffffffu, c3[1], src + 1);
  float y2 = __shfl_sync(0xffffffffu, c3[2], src + 1), y3 = __shfl_sync(0xffffffffu, c3[3], src + 1);
  o[0] = hi ? x2 : x0;
  o[1] = hi ? x3 : x1;
  o[2] = hi ? y2 : y0;
  o[3] = hi ? y3 : y1;
}

// Flow of one point per lane (all 32 lanes active): z in, z out, logdet accumulated.  pk is the
// packed-fragment array of all couplings (shared memory), bias arrays per coupling.
__device__ __forceinline__ void cp_flow_couplings(const uint2* __restrict__ pk, const float* __restrict__ biases,
                                                  float z[3], float& logdet)
{
  const int lane = threadIdx.x & 31;
#pragma unroll 1
  for (int c = 0; c < CP_FLOW_NC; ++c) {
    const CpCoupling k = cp_coupling(c);
    const uint2* p = pk + c * CP_FLOW_P_FWD;
    const float* b = biases + c * CP_FLOW_NB;   // b1[64], b2[64], b3[8]
    float in0 = z[k.cin[0]], in1 = z[k.cin[1]];
    float o0[4], o1[4];
    cp_flow_mlp_tile(p, b, b + 64, b + 128, in0, in1, k.nin, 0, o0);
    cp_flow_mlp_tile(p, b, b + 64, b + 128, in0, in1, k.nin, 16, o1);
    float o[4];
    const bool second = lane >= 16;
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = second ? o1[q] : o0[q];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (j >= k.nt) break;
      const float s = CP_FLOW_S * tanhf(o[j] / CP_FLOW_S), t = o[k.nt + j];
      const int d = k.tr[j];
      z[d] = fmaf(z[d], expf(s), t);
      logdet += s;
    }
  }
}

// VEGAS map of the flow's input: bin and in-bin fraction from the 24-bit word with a half-step
// offset, so x_v lies strictly inside (0, 1) and the logit stays finite; returns x_v and the
// bin Jacobian nb * width in jv.
__device__ __forceinline__ float cp_flow_vegas_in(const float2* edges_d, int nb, uint32_t w, float& jv, int& bin)
{
  const uint32_t m = (w >> 8) * (uint32_t)nb;
  bin = (int)(m >> 24);
  const float frac = ((float)(m & 0xFFFFFFu) + 0.5f) * (1.f / 16777216.f);
  const float2 e = edges_d[bin];
  jv *= (float)nb * e.y;
  float x = fmaf(frac, e.y, e.x);
  const float lo = 5.9604645e-8f, hi = 0.99999994f;
  return x < lo ? lo : (x > hi ? hi : x);
}

// logit input transform of one coordinate: z = ln(u / (1 - u)), returns -ln(u (1 - u))
__device__ __forceinline__ float cp_flow_logit(float u, float& z)
{
  const float lu = logf(u), l1u = log1pf(-u);
  z = lu - l1u;
  return -(lu + l1u);
}
// sigmoid output transform: v = 1 / (1 + e^-z), returns ln(v (1 - v)) = -|z| - 2 ln(1 + e^-|z|)
__device__ __forceinline__ float cp_flow_sigmoid(float z, float& v)
{
  const float e = expf(-fabsf(z));
  const float inv = 1.f / (1.f + e);
  v = z >= 0.f ? inv : e * inv;
  return -fabsf(z) - 2.f * log1pf(e);
}
#endif
