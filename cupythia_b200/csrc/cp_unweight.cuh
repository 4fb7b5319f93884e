// cp_unweight.cuh -- launch record of the production pass (draw, map, integrand, accept,
// per-block staging; then the record builder), shared by the accept kernel (cp_unweight.cu) and
// the tensor-core flow kernel's fused production form (cp_flow_tc.cu).
#pragma once
#include "cp_internal.cuh"

#define CP_UNW_SLOT 8   // sum w, sum w^2, max w, n_bad, n_acc, sum event weight, n_over, unused
#define CP_UNW_CHUNK (1ull << 24)   // points per production chunk (staging: 80 B per point)
#define CP_UNW_RANGE 32             // 32-point blocks per record-builder warp (1024 points)

struct UnwLaunch {
  uint64_t seed, point0, n;
  uint32_t iter;
  int nb;
  const double* edges;
  const double* wmax;          // device threshold
  CpEventRec* out;
  float4* pdf;                 // staging per point: fa[8], fb[8] of the accepted points (K1 -> K2)
  uint4* tails;                // staging per point: event weight and x[3] (bits), or null (no records)
  unsigned* bmask;             // accept mask of each 32-point block (bit = lane = point - 32 block)
  unsigned* rsum;              // accepted points per 1024-point range (zeroed before K1)
  const unsigned long long* roff;   // output index of the first record of each range
  uint64_t nblk, nrange;
  float* scalew;               // per record: 6 scale-variation ratios, or null
  uint64_t capacity;
  double* slots;
  const float4* flow;          // flow output (v, ln J) per in-call point, or null (K1 only)
  const float* flow_u;         // the flow forward's accept draw per in-call point, or null: K1 draws it
};

// the tensor-core flow kernel's production form over one chunk (cp_flow_tc.cu)
int cp_flow_tc_accept_enqueue(cp_handle* h, const UnwLaunch& L, int* blocks);

#if defined(__CUDACC__)
// Per-thread sums of a production pass (Kahan FP32), reduced per block into an FP64 slot.
struct CpUnwSums {
  float s1 = 0.f, c1 = 0.f, s2 = 0.f, c2 = 0.f, se = 0.f, ce = 0.f, wm = 0.f;
  uint32_t nbad = 0, nacc = 0, nover = 0;
};

// One point of the production pass, executed by all 32 lanes of a warp whose lanes hold the 32
// consecutive points p0 .. p0 + 31 of one block (p the chunk-local index, p0 a multiple of 32):
// the weight at the mapped point x with Jacobian jv, the accept test u w_max < w (u the point's
// accept draw), and the block's accept mask, the mask's popcount added to the 1024-point range's
// total (an integer atomic, exact in any order), and each accepted point's event weight,
// coordinates and PDFs packed at the front of the block's staging slots in point order.  Lanes
// with p >= L.n take part in the ballot only.
__device__ __forceinline__ void cp_unw_point(const CpHadParams& P, const CpCteqPoly* sCteq, const UnwLaunch& L,
                                             float wmax, uint64_t p, float x0, float x1, float x2, float jv,
                                             float u, CpUnwSums& S)
{
  const int lane = threadIdx.x & 31;
  bool accept = false;
  float w = 0.f;
  CpPoint pt;
  if (p < L.n) {
    w = cp_had_eval(P, sCteq, x0, x1, x2, pt) * jv;
    if (!(w >= 0.f) || isinf(w)) { ++S.nbad; w = 0.f; }
    cp_kahan(S.s1, S.c1, w);
    cp_kahan(S.s2, S.c2, w * w);
    S.wm = fmaxf(S.wm, w);
    accept = u * wmax < w;
  }
  const unsigned ball = __ballot_sync(0xffffffffu, accept);
  const uint64_t p0 = p - (uint64_t)lane;
  if (L.tails && lane == 0 && p0 < L.n) {
    L.bmask[p0 >> 5] = ball;
    if (ball) atomicAdd(&L.rsum[p0 >> 10], (unsigned)__popc(ball));   // integer sum: order-free
  }
  if (accept) {
    const float ew = w > wmax ? w / wmax : 1.f;
    ++S.nacc;
    S.nover += w > wmax ? 1u : 0u;
    cp_kahan(S.se, S.ce, ew);
    if (L.tails) {
      const uint64_t q = p0 + (uint64_t)__popc(ball & ((1u << lane) - 1u));
      // the event weight and the point's coordinates after the map (and flow): the record
      // builder starts from them, so it needs neither the map nor the flow output
      L.tails[q] = make_uint4(__float_as_uint(ew), __float_as_uint(x0), __float_as_uint(x1), __float_as_uint(x2));
      // the PDFs of the point, so that the record builder need not evaluate CTEQ5L again
      float4* f = L.pdf + 4 * q;
      f[0] = make_float4(pt.fa[0], pt.fa[1], pt.fa[2], pt.fa[3]);
      f[1] = make_float4(pt.fa[4], pt.fa[5], pt.fa[6], pt.fa[7]);
      f[2] = make_float4(pt.fb[0], pt.fb[1], pt.fb[2], pt.fb[3]);
      f[3] = make_float4(pt.fb[4], pt.fb[5], pt.fb[6], pt.fb[7]);
    }
  }
}

// The warp's sums (all lanes): sum w, sum w^2, max w, n_bad, n_acc, sum event weight, n_over.
__device__ __forceinline__ void cp_unw_warp_sums(const CpUnwSums& S, double v[7])
{
  v[0] = (double)S.s1 - (double)S.c1;
  v[1] = (double)S.s2 - (double)S.c2;
  v[2] = (double)S.wm;
  v[3] = (double)S.nbad;
  v[4] = (double)S.nacc;
  v[5] = (double)S.se - (double)S.ce;
  v[6] = (double)S.nover;
#pragma unroll
  for (int k = 0; k < 7; ++k) v[k] = (k == 2) ? cp_warp_max_d(v[k]) : cp_warp_sum_d(v[k]);
}
#endif
