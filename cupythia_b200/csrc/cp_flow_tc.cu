// cp_flow_tc.cu -- the flow forward (sampling) pass on the 5th-generation tensor cores.
//
// Same map as k_flow_fwd (Philox words -> VEGAS map -> logit -> 4 affine couplings -> sigmoid),
// with every dense layer as tcgen05.mma over 128-point tiles: B (weights) in shared memory, the
// FP32 accumulator in TMEM, A (activations) in shared memory for layers 1 and 2 and in TMEM for
// layer 3 (stored over the spent layer-2 accumulator).
//
// A production form (k_flow_accept_tc, opt-in through cp_flow_fuse_production) instantiates the
// same body and takes each finished tile on, from registers, through the integrand and the
// accept step of the production pass (the code of k_unw_accept, shared through cp_unweight.cuh),
// so no flow output is stored.  Its records equal the two-kernel path's byte for byte, but it is
// the slower of the two: a warpgroup's slots idle while its warps run the integrand, and the
// integrand's FMA-bound warps lengthen every flow step (2^27 points on B200: 19.3 ms with 4
// warpgroups at 96 registers, against 10.4 + 7.5 ms for the two kernels).
//
// Launch: one persistent CTA per SM (the shared-memory footprint admits one): 4 epilogue
// warpgroups of 128 threads and 4 issuing warps, one per warpgroup.  Each warpgroup owns two
// 128-point tiles in flight ("slots") with 64 TMEM columns and a 16 KB activation buffer each;
// thread r of the warpgroup is row r (one point) of both tiles and TMEM lane r.  An issuing warp
// does nothing but poll its warpgroup's two publish barriers and issue each slot's next layer,
// so no epilogue warp ever waits on MMA issue.  Per coupling and slot the epilogue has three steps
//   ep1: wait for layer 1, TMEM -> ReLU -> BF16 -> activation buffer, publish (layer 2 follows)
//   ep2: wait for layer 2, TMEM -> ReLU -> BF16 pairs -> TMEM columns 32..63, publish (layer 3,
//        A from TMEM, accumulates into columns 0..15)
//   ep3: wait for layer 3, read the 4 output columns, update the point, write the next
//        coupling's layer-1 input, publish (its layer 1 follows)
// and the steps of the two slots alternate, so one slot's MMAs run while the other slot's
// epilogue runs; a slot that finishes its last coupling writes its points and starts on the
// warpgroup's next pair at once, while the other slot finishes the current one.  The biases of layers 1 and 2 are part of the MMAs: layer 1 has them as input
// columns 14 and 15 (constant 1) times weight rows holding the BF16 high and low parts of the
// FP32 bias; layer 2 adds one K = 16 MMA of a constant block (columns 0 and 1 equal to 1) against
// the hi/lo bias rows (hi + lo reproduces the FP32 bias to about 2^-17 relative).  Layer 3's
// biases are added in FP32 by the coupling update: its 2 or 4 outputs per point cost as many
// adds, against one more MMA per tile step.
//
// Synchronisation is by mbarriers: each epilogue warp publishes its rows of a step (proxy fence,
// one arrival per warp on the slot's publish barrier); the issuing warp, seeing four arrivals,
// issues and commits to the slot's MMA barrier, which the epilogue warps wait on before reading
// TMEM.  Every wait is bounded (about 1 s of clock without progress); on expiry the waiting side
// raises its warpgroup's abort flag, no further MMAs are issued for it, its warps finish their
// loops without waiting, each issuing thread waits (bounded) for the MMAs it still has in flight,
// and the kernel sets *status and releases its TMEM.
#include "cp_flow.cuh"
#include "cp_internal.cuh"
#include "cp_tc.cuh"
#include "cp_unweight.cuh"

// weight image of one coupling, bytes (K-major, no swizzle; see cp_tc.cuh)
#define CP_TC_B1 0        // [N 64][K 16]: W1 rows 0..n_in-1, bias hi/lo in K 14/15
#define CP_TC_B2 2048     // [N 64][K 64]: W2
#define CP_TC_B2B 10240   // [N 64][K 16]: b2 hi/lo in K 0/1
#define CP_TC_B3 12288    // [N 16][K 64]: W3 (outputs 0..7, rest zero)
#define CP_TC_PER 14336
#define CP_TC_IMG (CP_FLOW_NC * CP_TC_PER)
#define CP_TC_HBYTES 16384                      // activation buffer of one slot: [128][64] bf16
#define CP_TC_TMEM_COLS 512                     // up to 8 slots x 64 columns
#define CP_TC_A3 32                             // slot's TMEM column of the layer-3 A operand
#define CP_TC_ONE2 0x3F803F80u                  // two BF16 ones
#define CP_TC_WG 4                              // sampling form: epilogue warpgroups per CTA
#define CP_TC_WG_ACC 4                          // production form: 20 warps, 5 per SM sub-partition -> 96 registers

// Shared-memory layout of a CTA with NWG epilogue warpgroups, bytes from the 1024-aligned base.
template <int NWG>
struct CpTcLayout {
  static constexpr int THREADS = NWG * 128 + NWG * 32;     // epilogue warpgroups + one issuing warp each
  static constexpr int ONES = CP_TC_IMG;                   // [128][16] bf16 constant block
  static constexpr int H = ONES + 4096;                    // activation buffers, two per warpgroup
  static constexpr int EDGE = H + NWG * 2 * CP_TC_HBYTES;
  static constexpr int MISC = EDGE + 3 * CP_MAX_BINS * 8;  // mbarriers, TMEM address, abort flags, final barriers
  static constexpr int B3 = MISC + 256;                    // FP32 layer-3 biases, 8 per coupling
  static constexpr int RED = B3 + 128;                     // production form: per-warp sums
  static constexpr int SMEM = RED + NWG * 4 * 7 * 8 + 1024;        // + 1024-byte base alignment slack
  static_assert(H % 1024 == 0 && RED % 16 == 0, "activation buffers and sums must stay aligned");
  static_assert(SMEM < (1 << 18), "descriptor offsets are added to the 14-bit address field");
  static_assert(SMEM <= 227 * 1024, "shared memory budget");
  static_assert(NWG <= 4 && 2 * NWG * 64 <= CP_TC_TMEM_COLS, "barrier area and TMEM columns");
};

static_assert(CP_TC_PER % 16 == 0, "coupling images are whole descriptor units");

constexpr uint32_t CP_TC_IDESC64 = cp_tc_idesc_bf16(64);
constexpr uint32_t CP_TC_IDESC16 = cp_tc_idesc_bf16(16);

// byte offset of element (row r, column k) in a K-major no-swizzle tile of R rows
__host__ __device__ __forceinline__ int cp_tc_off(int r, int k, int R) { return (k >> 3) * (R * 16) + (r >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2; }

__device__ __forceinline__ uint16_t cp_bf16_bits(float v)
{
  __nv_bfloat16 b = __float2bfloat16_rn(v);
  return *reinterpret_cast<uint16_t*>(&b);
}
__device__ __forceinline__ void cp_bf16_split(float v, uint16_t& hi, uint16_t& lo)
{
  hi = cp_bf16_bits(v);
  lo = cp_bf16_bits(v - __uint_as_float((uint32_t)hi << 16));
}

// FP32 master parameters -> the shared-memory weight image of every coupling
__global__ void k_flow_pack_tc(const float* __restrict__ P, uint8_t* __restrict__ img)
{
  const int c = blockIdx.x;
  const CpCoupling kc = cp_coupling(c);
  const float* W1 = P + c * CP_FLOW_PER + CP_FLOW_W1;
  const float* b1 = P + c * CP_FLOW_PER + CP_FLOW_B1;
  const float* W2 = P + c * CP_FLOW_PER + CP_FLOW_W2;
  const float* b2 = P + c * CP_FLOW_PER + CP_FLOW_B2;
  const float* W3 = P + c * CP_FLOW_PER + CP_FLOW_W3;
  uint8_t* q = img + c * CP_TC_PER;
  for (int e = threadIdx.x; e < CP_TC_PER / 2; e += blockDim.x) {
    uint16_t v = 0, hi, lo;
    int off;
    if (e < 1024) {                       // B1 [64][16]
      const int nn = e >> 4, k = e & 15;
      off = CP_TC_B1 + cp_tc_off(nn, k, 64);
      cp_bf16_split(b1[nn], hi, lo);
      if (k < kc.nin) v = cp_bf16_bits(W1[k * 64 + nn]);
      else if (k == 14) v = hi;
      else if (k == 15) v = lo;
    } else if (e < 5120) {                // B2 [64][64]
      const int i = e - 1024, nn = i >> 6, k = i & 63;
      off = CP_TC_B2 + cp_tc_off(nn, k, 64);
      v = cp_bf16_bits(W2[k * 64 + nn]);
    } else if (e < 6144) {                // B2B [64][16]
      const int i = e - 5120, nn = i >> 4, k = i & 15;
      off = CP_TC_B2B + cp_tc_off(nn, k, 64);
      cp_bf16_split(b2[nn], hi, lo);
      v = k == 0 ? hi : (k == 1 ? lo : (uint16_t)0);
    } else {                              // B3 [16][64]
      const int i = e - 6144, nn = i >> 6, k = i & 63;
      off = CP_TC_B3 + cp_tc_off(nn, k, 16);
      if (nn < 8) v = cp_bf16_bits(W3[k * 8 + nn]);
    }
    *reinterpret_cast<uint16_t*>(q + off) = v;
  }
}

// Elementwise transforms of the tensor-core path with the hardware approximations (lg2/ex2 and
// fast reciprocal; absolute errors of a few 1e-7 in z and ln J).  The log-Jacobian uses the same
// computed quantities as the map (z' = z e^s + t with ln J += s), so the weights stay consistent.
__device__ __forceinline__ float cp_tc_logit(float u, float& z)
{
  const float lu = __logf(u), l1u = __logf(1.f - u);
  z = lu - l1u;
  return -(lu + l1u);
}
__device__ __forceinline__ float cp_tc_sigmoid(float z, float& v)
{
  const float e = __expf(-fabsf(z));
  const float inv = __fdividef(1.f, 1.f + e);
  v = z >= 0.f ? inv : e * inv;
  return -fabsf(z) - 2.f * __logf(1.f + e);
}
// CP_FLOW_S tanh(x / CP_FLOW_S) from one exponential
__device__ __forceinline__ float cp_tc_softclamp(float x)
{
  const float a = fabsf(x) * (2.f / CP_FLOW_S);
  const float t = __expf(-a);
  return copysignf(CP_FLOW_S * __fdividef(1.f - t, 1.f + t), x);
}

struct CpTcPoint {
  float z0, z1, z2, ld;
};

__device__ __forceinline__ float cp_sel3(const CpTcPoint& t, int i) { return i == 0 ? t.z0 : (i == 1 ? t.z1 : t.z2); }

// this thread's row of the layer-1 input of coupling c: (in0, in1, 0 ... 0, 1, 1)
__device__ __forceinline__ void cp_tc_write_in(uint32_t hbuf, int row, int c, const CpTcPoint& t)
{
  const CpCoupling k = cp_coupling(c);
  const float in0 = cp_sel3(t, k.cin[0]);
  const float in1 = k.nin > 1 ? cp_sel3(t, k.cin[1]) : 0.f;
  cp_sts128(hbuf + row * 16, cp_bf2(in0, in1), 0u, 0u, 0u);
  cp_sts128(hbuf + 2048 + row * 16, 0u, 0u, 0u, CP_TC_ONE2);
}

// Descriptors are formed once per issuing thread: a = the slot's activation buffer (LBO 2048),
// ones = the constant block, b64 / b16 = the weight image base with the LBO of the N = 64 and
// N = 16 operands; an operand at byte offset o from a base adds o >> 4 to the start-address field
// (every shared address here is below 2^18, so the 14-bit field never carries).  bw = the
// coupling's image offset >> 4.
__device__ __forceinline__ void cp_tc_issue_l1(uint32_t d, uint64_t a, uint64_t b64, uint32_t bw)
{
  cp_tc_mma(d, a, b64 + bw + (CP_TC_B1 >> 4), CP_TC_IDESC64, 0u);
}
__device__ __forceinline__ void cp_tc_issue_l2(uint32_t d, uint64_t a, uint64_t ones, uint64_t b64, uint32_t bw)
{
#pragma unroll
  for (int j = 0; j < 4; ++j)
    cp_tc_mma(d, a + j * (4096 >> 4), b64 + bw + ((CP_TC_B2 + j * 2048) >> 4), CP_TC_IDESC64, j > 0 ? 1u : 0u);
  cp_tc_mma(d, ones, b64 + bw + (CP_TC_B2B >> 4), CP_TC_IDESC64, 1u);
}
// layer 3 reads its A operand (the layer-2 activations, BF16 pairs) from the slot's TMEM columns
// 32..63, where the ep2 epilogue stored them, and accumulates into columns 0..15
__device__ __forceinline__ void cp_tc_issue_l3(uint32_t d, uint64_t b16, uint32_t bw)
{
#pragma unroll
  for (int j = 0; j < 4; ++j)
    cp_tc_mma_ts(d, d + CP_TC_A3 + 8 * j, b16 + bw + ((CP_TC_B3 + j * 512) >> 4), CP_TC_IDESC16, j > 0 ? 1u : 0u);
}

// makes this warp's shared-memory writes (and its earlier TMEM reads) visible to the tensor core
// and arrives once on the slot's publish barrier (four arrivals complete a step)
__device__ __forceinline__ void cp_tc_publish(uint32_t pub)
{
  cp_fence_proxy_async();
  cp_tc_fence_before();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) cp_mbar_arrive(pub);
}

// the same for a step whose only writes went to TMEM (tcgen05.st, completed by cp_tc_wait_st)
__device__ __forceinline__ void cp_tc_publish_tmem(uint32_t pub)
{
  cp_tc_fence_before();
  __syncwarp();
  if ((threadIdx.x & 31) == 0) cp_mbar_arrive(pub);
}

// waits for the slot's MMAs (warp-uniform result)
__device__ __forceinline__ bool cp_tc_wait(uint32_t mbar, uint32_t& phase, volatile int* abort)
{
  const bool ok = cp_mbar_wait_bounded(mbar, phase, abort);
  phase ^= 1u;
  cp_tc_fence_after();
  return __all_sync(0xffffffffu, ok);
}

// TMEM [row][0:64] -> ReLU -> BF16 -> activation buffer row
__device__ __forceinline__ void cp_tc_hidden_out(uint32_t taddr, uint32_t hbuf, int row, bool ok)
{
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    float v[32];
    if (ok) {
      cp_tc_ld32(taddr + half * 32, v);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) v[j] = 0.f;
    }
#pragma unroll
    for (int kb = 0; kb < 4; ++kb)
      cp_sts128(hbuf + (half * 4 + kb) * 2048 + row * 16, cp_relu_bf2(v[8 * kb], v[8 * kb + 1]),
                cp_relu_bf2(v[8 * kb + 2], v[8 * kb + 3]), cp_relu_bf2(v[8 * kb + 4], v[8 * kb + 5]),
                cp_relu_bf2(v[8 * kb + 6], v[8 * kb + 7]));
  }
}

// TMEM [row][0:64] -> ReLU -> BF16 pairs -> TMEM [row][32:64], the A operand of layer 3 (hidden
// unit k in column 32 + k / 2).  Half 1 (columns 32..63) is loaded first and lands in columns
// 48..63, then half 0 (0..31) in 32..47: every column is loaded before it is stored over.
// Nothing is stored when the MMAs were not seen to complete.
__device__ __forceinline__ void cp_tc_hidden_to_tmem(uint32_t taddr, bool ok)
{
  if (!ok) return;
#pragma unroll
  for (int half = 1; half >= 0; --half) {
    float v[32];
    cp_tc_ld32(taddr + half * 32, v);
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) w[i] = cp_relu_bf2(v[2 * i], v[2 * i + 1]);
    cp_tc_st16(taddr + CP_TC_A3 + 16 * half, w);
  }
  cp_tc_wait_st();
}

// The kernel body.  Sampling form (ACCEPT false): each point's (v, ln J) goes to out.  Production
// form (ACCEPT true, draws of stream 0): each point goes straight on, from registers, through the
// integrand and the accept step of the production pass (cp_unw_point, the code of k_unw_accept),
// after both slots of its pair have started their next pair, and each CTA leaves its sums in its
// slot of L->slots; the record builder then runs unchanged.
template <int NWG, bool ACCEPT>
__device__ __forceinline__ void cp_flow_tc_body(const uint4* __restrict__ img_g, const float* __restrict__ params,
                                                const double* __restrict__ edges, int nb, uint64_t seed, uint64_t point0,
                                                uint64_t n, uint32_t iter, uint32_t stream, float4* __restrict__ out,
                                                float* __restrict__ uout, int* __restrict__ status, int stall,
                                                const CpHadParams* P,
                                                const UnwLaunch* L)
{
  using Lay = CpTcLayout<NWG>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  const uint32_t raw = cp_smem_u32(smem_raw);
  const uint32_t pad = ((raw + 1023u) & ~1023u) - raw;
  uint8_t* sm = smem_raw + pad;
  const uint32_t sbase = raw + pad;
  float2* sEdge = reinterpret_cast<float2*>(sm + Lay::EDGE);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(sm + Lay::MISC);   // [0, 2 NWG) MMA done, [2 NWG, 4 NWG) publish
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + Lay::MISC + 128);
  int* abort_flags = reinterpret_cast<int*>(sm + Lay::MISC + 144);
  uint64_t* fin_bar = reinterpret_cast<uint64_t*>(sm + Lay::MISC + 160);   // [NWG] issuers' final commits

  const int tid = threadIdx.x, warp = tid >> 5, wg = warp >> 2, row = tid & 127;

  for (int e = tid; e < CP_TC_IMG / 16; e += Lay::THREADS) reinterpret_cast<uint4*>(sm)[e] = img_g[e];
  for (int e = tid; e < 256; e += Lay::THREADS)
    reinterpret_cast<uint4*>(sm + Lay::ONES)[e] = e < 128 ? make_uint4(CP_TC_ONE2, 0u, 0u, 0u) : make_uint4(0u, 0u, 0u, 0u);
  float* sB3 = reinterpret_cast<float*>(sm + Lay::B3);
  if (tid < CP_FLOW_NC * 8) sB3[tid] = params[(tid >> 3) * CP_FLOW_PER + CP_FLOW_B3 + (tid & 7)];
  for (int k = tid; k < 3 * nb; k += Lay::THREADS) {
    const int d = k / nb, b = k - d * nb;
    const double lo = edges[d * (nb + 1) + b], hi = edges[d * (nb + 1) + b + 1];
    sEdge[d * CP_MAX_BINS + b] = make_float2((float)lo, (float)(hi - lo));
  }
  double* sRed = reinterpret_cast<double*>(sm + Lay::RED);   // [4 NWG warps][7]
  if (tid < NWG) abort_flags[tid] = 0;
  if (tid == 0) {
    for (int i = 0; i < 2 * NWG; ++i) {
      cp_mbar_init(cp_smem_u32(&mbar[i]), 1);
      cp_mbar_init(cp_smem_u32(&mbar[2 * NWG + i]), 4);
    }
    for (int i = 0; i < NWG; ++i) cp_mbar_init(cp_smem_u32(&fin_bar[i]), 1);
    cp_mbar_init_fence();
  }
  if (warp == 0) {
    cp_tc_alloc(cp_smem_u32(tmem_slot), CP_TC_TMEM_COLS);
    cp_tc_relinquish();
  }
  cp_fence_proxy_async();
  cp_tc_fence_before();
  __syncthreads();
  cp_tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t ones = sbase + Lay::ONES;
  const uint64_t npairs = (n + 255) / 256;
  const uint64_t stride = (uint64_t)gridDim.x * NWG;

  if (warp >= 4 * NWG) {
    // ---- issuing warps: warp 16 + g serves warpgroup g; one lane scans its two publish barriers
    const int g = warp - 4 * NWG;
    if ((tid & 31) == 0 && !stall) {     // stall: test hook, no MMA is ever issued
      const uint64_t q0 = (uint64_t)blockIdx.x * NWG + g;
      const uint64_t cnt = q0 < npairs ? (npairs - q0 + stride - 1) / stride : 0;
      uint32_t rem0 = (uint32_t)(3 * CP_FLOW_NC * cnt), rem1 = rem0, pph0 = 0, pph1 = 0;
      uint32_t lay0 = 0, lay1 = 0, bw0 = 0, bw1 = 0;   // layer and coupling image offset >> 4 per slot
      const uint32_t pub0 = cp_smem_u32(&mbar[2 * NWG + 2 * g]), pub1 = pub0 + 8;
      const uint32_t hb0 = sbase + Lay::H + (2 * g) * CP_TC_HBYTES, hb1 = hb0 + CP_TC_HBYTES;
      const uint32_t tc0 = tmem + (uint32_t)(2 * g * 64), tc1 = tc0 + 64;
      const uint32_t done0 = cp_smem_u32(&mbar[2 * g]), done1 = done0 + 8;
      volatile int* abort = abort_flags + g;
      const uint64_t ad0 = cp_tc_desc(hb0, 2048, 128), ad1 = cp_tc_desc(hb1, 2048, 128);
      const uint64_t adones = cp_tc_desc(ones, 2048, 128);
      const uint64_t b64 = cp_tc_desc(sbase, 1024, 128), b16 = cp_tc_desc(sbase, 256, 128);
      long long t0 = clock64();
      while (rem0 | rem1) {
        if (*abort) break;
        bool progress = false;
#pragma unroll
        for (int s = 0; s < 2; ++s) {
          uint32_t& rem = s ? rem1 : rem0;
          uint32_t& lay = s ? lay1 : lay0;
          uint32_t& bw = s ? bw1 : bw0;
          uint32_t& pph = s ? pph1 : pph0;
          if (!rem || !cp_mbar_test(s ? pub1 : pub0, pph)) continue;
          pph ^= 1u;
          cp_tc_fence_after();
          const uint32_t tc = s ? tc1 : tc0;
          const uint64_t ad = s ? ad1 : ad0;
          if (lay == 0) {
            cp_tc_issue_l1(tc, ad, b64, bw);
            lay = 1;
          } else if (lay == 1) {
            cp_tc_issue_l2(tc, ad, adones, b64, bw);
            lay = 2;
          } else {
            cp_tc_issue_l3(tc, b16, bw);
            lay = 0;
            bw = bw == (CP_FLOW_NC - 1) * (CP_TC_PER >> 4) ? 0u : bw + (CP_TC_PER >> 4);
          }
          cp_tc_commit(s ? done1 : done0);
          --rem;
          progress = true;
        }
        if (progress) {
          t0 = clock64();
        } else if (clock64() - t0 > CP_TC_WAIT_CYCLES) {
          *abort = 1;
          break;
        }
      }
      // After an abort MMAs may still be in flight: every one this thread issued has completed
      // (bounded wait) before the CTA releases its TMEM.
      const uint32_t fin = cp_smem_u32(&fin_bar[g]);
      cp_tc_commit(fin);
      volatile int fin_abort = 0;
      if (!cp_mbar_wait_bounded(fin, 0u, &fin_abort)) *abort = 1;
    }
    __syncwarp();
  } else {
    // ---- epilogue warpgroups
    volatile int* abort = abort_flags + wg;
    const uint32_t bar_id = 1 + wg;
    const uint32_t lane_base = (uint32_t)(32 * (warp & 3)) << 16;
    uint32_t hb[2], tc[2], mb[2], pb[2], ph[2] = {0u, 0u};
#pragma unroll
    for (int s = 0; s < 2; ++s) {
      hb[s] = sbase + Lay::H + (wg * 2 + s) * CP_TC_HBYTES;
      tc[s] = tmem + (uint32_t)((wg * 2 + s) * 64);
      mb[s] = cp_smem_u32(&mbar[wg * 2 + s]);
      pb[s] = cp_smem_u32(&mbar[2 * NWG + wg * 2 + s]);
    }
    CpTcPoint t[2];
    uint64_t p[2];
    // production form: the slots' accept draws; each slot's finished points (v, ln J), indices and
    // draws, held until both slots have started their next pair; the thread's sums
    [[maybe_unused]] float u[2];
    [[maybe_unused]] float4 fin0, fin1;
    [[maybe_unused]] uint64_t fp0 = 0, fp1 = 0;
    [[maybe_unused]] float fu0 = 0.f, fu1 = 0.f;
    [[maybe_unused]] CpUnwSums S;
    [[maybe_unused]] const float wmax = ACCEPT ? (float)L->wmax[0] : 0.f;
    // a slot's start on the pair qq: Philox words -> VEGAS map -> logit, layer-1 input, publish
    auto start = [&](int s, uint64_t qq) {
      p[s] = qq * 256 + s * 128 + row;
      uint32_t w[4] = {0x80000000u, 0x80000000u, 0x80000000u, 0u};
      if (p[s] < n) cp_point_words(seed, point0 + p[s], iter, stream, w);
      if (ACCEPT || uout) u[s] = cp_u24(w[3]);
      float jv = 1.f, ld = 0.f, z[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        int bin;
        const float xv = cp_flow_vegas_in(sEdge + d * CP_MAX_BINS, nb, w[d], jv, bin);
        ld += cp_tc_logit(xv, z[d]);
      }
      t[s].z0 = z[0]; t[s].z1 = z[1]; t[s].z2 = z[2];
      t[s].ld = ld + __logf(jv);
      cp_tc_write_in(hb[s], row, 0, t[s]);
      cp_tc_publish(pb[s]);
    };
    uint64_t q = (uint64_t)blockIdx.x * NWG + wg;
    if (q < npairs) {
      start(0, q);
      start(1, q);
    }
    for (; q < npairs; q += stride) {
      const uint64_t qn = q + stride;
      // unrolled: each coupling's input and transformed dimensions are compile-time constants
#pragma unroll
      for (int c = 0; c < CP_FLOW_NC; ++c) {
#pragma unroll
        for (int s = 0; s < 2; ++s) {           // ep1: layer-1 output -> layer 2
          const bool ok = cp_tc_wait(mb[s], ph[s], abort);
          cp_tc_hidden_out(tc[s] + lane_base, hb[s], row, ok);
          cp_tc_publish(pb[s]);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s) {           // ep2: layer-2 output -> layer 3 (A in TMEM)
          const bool ok = cp_tc_wait(mb[s], ph[s], abort);
          cp_tc_hidden_to_tmem(tc[s] + lane_base, ok);
          cp_tc_publish_tmem(pb[s]);
        }
#pragma unroll
        for (int s = 0; s < 2; ++s) {           // ep3: coupling update, next coupling's layer 1
          const bool ok = cp_tc_wait(mb[s], ph[s], abort);
          float o[4] = {0.f, 0.f, 0.f, 0.f};
          if (ok) cp_tc_ld4(tc[s] + lane_base, o);
          const CpCoupling k = cp_coupling(c);
          const float* b3 = sB3 + 8 * c;
#pragma unroll
          for (int j = 0; j < 2; ++j) {
            if (j >= k.nt) break;
            const float sc = cp_tc_softclamp(o[j] + b3[j]), sh = o[k.nt + j] + b3[k.nt + j];
            const int d = k.tr[j];
            const float zn = fmaf(cp_sel3(t[s], d), __expf(sc), sh);
            if (d == 0) t[s].z0 = zn;
            else if (d == 1) t[s].z1 = zn;
            else t[s].z2 = zn;
            t[s].ld += sc;
          }
          if (c + 1 < CP_FLOW_NC) {
            cp_tc_write_in(hb[s], row, c + 1, t[s]);
            cp_tc_publish(pb[s]);
          } else {
            // the slot's points are done: output, then the slot starts on the next pair while the
            // other slot finishes this one
            float v0, v1, v2;
            float ld = t[s].ld;
            ld += cp_tc_sigmoid(t[s].z0, v0);
            ld += cp_tc_sigmoid(t[s].z1, v1);
            ld += cp_tc_sigmoid(t[s].z2, v2);
            if constexpr (ACCEPT) {
              if (s == 0) {
                fin0 = make_float4(v0, v1, v2, ld); fp0 = p[s]; fu0 = u[s];
              } else {
                fin1 = make_float4(v0, v1, v2, ld); fp1 = p[s]; fu1 = u[s];
              }
            } else {
              if (p[s] < n) {
                out[p[s]] = make_float4(v0, v1, v2, ld);
                if (uout) uout[p[s]] = u[s];   // the accept draw, so the accept kernel need not redraw it
              }
            }
            if (qn < npairs) start(s, qn);
          }
        }
      }
      if constexpr (ACCEPT) {
        // weight, accept test and staging of the pair's two tiles while both slots' next layer-1
        // MMAs run; a loop over the slots keeps one copy of the integrand's code
#pragma unroll 1
        for (int s = 0; s < 2; ++s) {
          const float4 f = s ? fin1 : fin0;
          cp_unw_point(*P, P->cteq, *L, wmax, s ? fp1 : fp0, f.x, f.y, f.z, expf(f.w), s ? fu1 : fu0, S);
        }
      }
      if (cp_bar_wg_or(bar_id, *abort != 0)) break;
    }
    if (row == 0 && *abort) atomicOr(status, 1);
    if constexpr (ACCEPT) {
      double v[7];
      cp_unw_warp_sums(S, v);
      if ((tid & 31) == 0)
        for (int k = 0; k < 7; ++k) sRed[warp * 7 + k] = v[k];
    }
  }
  cp_tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    cp_tc_fence_after();
    cp_tc_dealloc(tmem, CP_TC_TMEM_COLS);
  }
  if constexpr (ACCEPT) {
    if (tid == 0) {   // the CTA's sums, warps in a fixed order
      double* slot = L->slots + (size_t)blockIdx.x * CP_UNW_SLOT;
      for (int k = 0; k < 7; ++k) {
        double acc = 0.0;
        for (int q = 0; q < 4 * NWG; ++q) acc = (k == 2) ? fmax(acc, sRed[q * 7 + k]) : acc + sRed[q * 7 + k];
        slot[k] = acc;
      }
      slot[7] = 0.0;
    }
  }
}

__global__ void __launch_bounds__(CpTcLayout<CP_TC_WG>::THREADS, 1)
    k_flow_fwd_tc(const uint4* __restrict__ img_g, const float* __restrict__ params, const double* __restrict__ edges,
                  int nb, uint64_t seed, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream,
                  float4* __restrict__ out, float* __restrict__ uout, int* __restrict__ status, int stall)
{
  cp_flow_tc_body<CP_TC_WG, false>(img_g, params, edges, nb, seed, point0, n, iter, stream, out, uout, status, stall,
                                   nullptr, nullptr);
}

// Production form: flow forward, integrand and accept step of the points [L.point0, L.point0 + L.n)
// in one pass (draws of stream 0, as k_unw_accept takes them), one CTA per SM.
__global__ void __launch_bounds__(CpTcLayout<CP_TC_WG_ACC>::THREADS, 1)
    k_flow_accept_tc(const uint4* __restrict__ img_g, const float* __restrict__ params,
                     const __grid_constant__ CpHadParams P, const __grid_constant__ UnwLaunch L,
                     int* __restrict__ status, int stall)
{
  cp_flow_tc_body<CP_TC_WG_ACC, true>(img_g, params, L.edges, L.nb, L.seed, L.point0, L.n, L.iter, 0u, nullptr,
                                      nullptr, status, stall, &P, &L);
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
int cp_flow_tc_repack(cp_handle* h)
{
  k_flow_pack_tc<<<CP_FLOW_NC, 256, 0, h->stream>>>(h->d_flow, h->d_flow_tc);
  CP_LAUNCH_CHECK(h, "k_flow_pack_tc");
  return CP_OK;
}

int cp_flow_tc_alloc(cp_handle* h)
{
  if (!h->d_flow_tc) CP_CUDA(h, cudaMalloc(&h->d_flow_tc, CP_TC_IMG));
  if (!h->d_flow_status) {
    CP_CUDA(h, cudaMalloc(&h->d_flow_status, sizeof(int)));
    CP_CUDA(h, cudaMemsetAsync(h->d_flow_status, 0, sizeof(int), h->stream));
  }
  CP_CUDA(h, cudaFuncSetAttribute(k_flow_fwd_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, CpTcLayout<CP_TC_WG>::SMEM));
  CP_CUDA(h, cudaFuncSetAttribute(k_flow_accept_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  CpTcLayout<CP_TC_WG_ACC>::SMEM));
  return CP_OK;
}

int cp_flow_tc_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float4* out,
                       float* uout)
{
  if (h->flow_tc_stale) {
    const int rc = cp_flow_tc_repack(h);
    if (rc) return rc;
    h->flow_tc_stale = 0;
  }
  const uint64_t pairs = (n + 255) / 256;
  const uint64_t want = (pairs + CP_TC_WG - 1) / CP_TC_WG;
  const int grid = (int)(want < (uint64_t)h->num_sms ? want : (uint64_t)h->num_sms);
  if (grid < 1) return CP_OK;
  k_flow_fwd_tc<<<grid, CpTcLayout<CP_TC_WG>::THREADS, CpTcLayout<CP_TC_WG>::SMEM, h->stream>>>(reinterpret_cast<const uint4*>(h->d_flow_tc), h->d_flow,
                                                                 h->d_edges,
                                                                 h->nb, h->cfg.seed, point0, n, iter, stream, out,
                                                                 uout, h->d_flow_status, h->flow_stall);
  CP_LAUNCH_CHECK(h, "k_flow_fwd_tc");
  return CP_OK;
}

// Enqueues the production form over the chunk L (its staging and range totals ready); *blocks =
// the CTAs launched, each of which writes its slot of L.slots.
int cp_flow_tc_accept_enqueue(cp_handle* h, const UnwLaunch& L, int* blocks)
{
  *blocks = 0;
  if (h->flow_tc_stale) {
    const int rc = cp_flow_tc_repack(h);
    if (rc) return rc;
    h->flow_tc_stale = 0;
  }
  const uint64_t pairs = (L.n + 255) / 256;
  const uint64_t want = (pairs + CP_TC_WG_ACC - 1) / CP_TC_WG_ACC;
  const int grid = (int)(want < (uint64_t)h->num_sms ? want : (uint64_t)h->num_sms);
  if (grid < 1) return CP_OK;
  using Lay = CpTcLayout<CP_TC_WG_ACC>;
  k_flow_accept_tc<<<grid, Lay::THREADS, Lay::SMEM, h->stream>>>(reinterpret_cast<const uint4*>(h->d_flow_tc),
                                                                  h->d_flow, h->P, L, h->d_flow_status, h->flow_stall);
  CP_LAUNCH_CHECK(h, "k_flow_accept_tc");
  *blocks = grid;
  return CP_OK;
}

// Reads and clears the device status of the tensor-core flow kernel, in order on the handle's
// stream (which may be a non-blocking stream): CP_ERR_TIMEOUT if a bounded wait expired since
// the last check.
int cp_flow_tc_status(cp_handle* h)
{
  if (!h->d_flow_status) return CP_OK;
  int s = 0;
  CP_CUDA(h, cudaMemcpyAsync(&s, h->d_flow_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!s) return CP_OK;
  CP_CUDA(h, cudaMemsetAsync(h->d_flow_status, 0, sizeof(int), h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  return cp_fail(h, CP_ERR_TIMEOUT, (s & 2) ? "k_flow_wgrad_tc: a tensor-core wait expired (this training step's gradient is invalid)"
                                            : "k_flow_fwd_tc / k_flow_accept_tc: a tensor-core wait expired (results of this pass are invalid)");
}

// Test hook of the failure path: with on != 0 the issuing warps issue nothing, so every bounded
// wait of the epilogue expires (about one second of clock), the kernel raises its status word and
// releases its TMEM, and the call returns CP_ERR_TIMEOUT with the context still usable.
extern "C" int cp_flow_test_stall(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  h->flow_stall = on ? 1 : 0;
  return CP_OK;
}
