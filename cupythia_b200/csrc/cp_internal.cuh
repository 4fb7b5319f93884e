// cp_internal.cuh -- handle layout, error plumbing and device helpers shared by the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string>
#include <vector>
#include <string.h>
#include "../../include/cupythia_b200.h"
#include "cp_params.h"

#define CP_THREADS 256
#ifndef CP_MIN_BLOCKS
#define CP_MIN_BLOCKS 2   // resident blocks per SM the hot kernels are compiled for
#endif
#define CP_WARPS (CP_THREADS / 32)
// per-block slot of the hadronic accumulation: sum w, sum w^2, max w, n_bad, then 3*nb hist
#define CP_SLOT_HEAD 4
// record staging buffers of cp_generate_host: chunk c computes into buffer c % CP_GEN_BUFS while
// the copies of the previous chunks drain
#define CP_GEN_BUFS 3

// Weight histogram for the unweighting threshold: bin = IEEE-754 bits of w >> 18 (8 exponent
// bits + 5 mantissa bits, monotone in w, about 2.2% wide), restricted to 2^-64 <= w < 2^64.
#define CP_QBINS 4096
#define CP_QBIN_OFFSET ((127 - 64) << 5)
__host__ __device__ __forceinline__ int cp_qbin(float w)
{
  if (!(w > 0.f)) return -1;
  uint32_t bits;
  memcpy(&bits, &w, 4);
  int b = (int)(bits >> 18) - CP_QBIN_OFFSET;
  return b < 0 ? 0 : (b >= CP_QBINS ? CP_QBINS - 1 : b);
}
// upper edge of a bin
__host__ __device__ __forceinline__ float cp_qbin_hi(int b)
{
  uint32_t bits = (uint32_t)(b + 1 + CP_QBIN_OFFSET) << 18;
  float f;
  memcpy(&f, &bits, 4);
  return f;
}

// Colour tags (1..4, 0 = none) of the four partons of a record from its process code (111..115)
// and encoded colour flow, as the process's setIdColAcol sets them (pythia8317/src/SigmaQCD.cc:
// 135-342: the topologies in the order of its setColAcol calls, then swapCol1234 (bit 3) and
// swapColAcol (bit 2)).  Returns false for a code / flow pair no process produces.  Host and
// device.
__host__ __device__ inline bool cp_colour_expand(uint16_t process, uint16_t colour, int col[4], int acol[4])
{
  // (col1, acol1, col2, acol2, col3, acol3, col4, acol4) per process and topology
  constexpr int8_t topo_tab[5][3][8] = {
      {{1, 2, 2, 3, 1, 4, 4, 3}, {1, 2, 3, 1, 3, 4, 4, 2}, {1, 2, 3, 4, 1, 4, 3, 2}},   // 111 g g -> g g
      {{1, 2, 2, 3, 1, 0, 0, 3}, {1, 2, 3, 1, 3, 0, 0, 2}, {0, 0, 0, 0, 0, 0, 0, 0}},   // 112 g g -> q qbar
      {{1, 0, 2, 1, 3, 0, 2, 3}, {1, 0, 2, 3, 2, 0, 1, 3}, {0, 0, 0, 0, 0, 0, 0, 0}},   // 113 q g -> q g
      {{1, 0, 2, 0, 2, 0, 1, 0}, {1, 0, 0, 1, 2, 0, 0, 2}, {1, 0, 2, 0, 1, 0, 2, 0}},   // 114 q q -> q q
      {{1, 0, 0, 2, 1, 3, 3, 2}, {1, 0, 0, 2, 3, 2, 1, 3}, {0, 0, 0, 0, 0, 0, 0, 0}}};  // 115 q qbar -> g g
  if (process < 111 || process > 115) return false;
  const int topo = colour & 3;
  if (topo > 2 || (topo == 2 && process != 111 && process != 114)) return false;
  int c[4], a[4];
  for (int k = 0; k < 4; ++k) {
    c[k] = topo_tab[process - 111][topo][2 * k];
    a[k] = topo_tab[process - 111][topo][2 * k + 1];
  }
  if (colour & 8) {   // swapCol1234: partons 1 <-> 2 and 3 <-> 4
    int x;
    x = c[0]; c[0] = c[1]; c[1] = x;  x = a[0]; a[0] = a[1]; a[1] = x;
    x = c[2]; c[2] = c[3]; c[3] = x;  x = a[2]; a[2] = a[3]; a[3] = x;
  }
  if (colour & 4)     // swapColAcol
    for (int k = 0; k < 4; ++k) { const int x = c[k]; c[k] = a[k]; a[k] = x; }
  for (int k = 0; k < 4; ++k) { col[k] = c[k]; acol[k] = a[k]; }
  return true;
}

// SplitMix64 finaliser (cuPythia/common/rng.cuh:47-53); host and device
__host__ __device__ __forceinline__ uint64_t cp_splitmix64(uint64_t x)
{
  x += 0x9E3779B97F4A7C15ULL;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
  return x ^ (x >> 31);
}

// Per-iteration record written by the device refinement kernel (FP64).
struct CpIterDev {
  double sumw, sumw2, wmax, nbad, n, sigma, err, pad;
};

struct cp_handle {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 0;
  cp_config cfg{};
  CpHadParams P{};
  int nb = 50;
  // VEGAS grid, FP64
  double* d_edges = nullptr;
  // CTEQ5L coefficient records (device copy of P.cteq, staged into shared memory by kernels)
  CpCteqPoly* d_cteq = nullptr;
  // scratch: per-block slots and reduced outputs
  double* d_slots = nullptr;
  size_t slots_cap = 0;           // doubles
  double* d_red = nullptr;        // CP_SLOT_HEAD + 3*CP_MAX_BINS doubles
  CpIterDev* d_iters = nullptr;   // per-iteration records
  int iters_cap = 0;
  // SigmaProcess batch state (SoA FP32)
  int64_t kin_n = 0, kin_cap = 0;
  float *d_x1 = nullptr, *d_x2 = nullptr, *d_sH = nullptr, *d_tH = nullptr;
  float *d_as = nullptr, *d_q2r = nullptr, *d_q2f = nullptr;
  float* d_uH = nullptr;          // uHat, formed at the input precision (FP64 for cp_set2kin_batch_f64)
  // launch shapes (resident blocks per SM on this handle's device; -1 until first use)
  int had_blocks = 0;
  int adj_per_sm_nt[2] = {-1, -1}, flow_per_sm = -1, unw_per_sm = -1;   // adjoint: x tangents only / all six
  int build_per_sm[2] = {-1, -1};   // record builder without / with scale weights
  // weight histogram of the last iteration and the unweighting threshold (device)
  unsigned long long* d_qhist = nullptr;   // CP_QBINS
  double wmax_host = 0.0;                  // the unweighting threshold d_wmax[0], as last set
  double* d_wmax = nullptr;                // [0] threshold used by cp_unweight, [1] quantile q
  unsigned long long* d_counter = nullptr; // accepted-event counter
  // production staging for pdfbuf_cap points (K1 -> K2): PDFs and record tails per point, accept
  // masks per 32-point block, totals and output offsets per 1024-point range; per-chunk sums
  float4* d_pdfbuf = nullptr;
  uint4* d_tails = nullptr;
  unsigned* d_bmask = nullptr;
  unsigned* d_rsum = nullptr;
  unsigned long long* d_roff = nullptr;
  uint64_t pdfbuf_cap = 0;
  double* d_unw_red = nullptr;
  uint64_t unw_red_cap = 0;
  float* scalew = nullptr;                 // caller's scale-variation weights (6 per record), or null
  uint64_t scalew_cap = 0;
  // cp_generate_host pipeline, kept between calls: CP_GEN_BUFS record staging buffers of gen_cap
  // slots each, per-chunk reductions and counters, the counters' host copy in mapped pinned
  // memory (written by a kernel, so that no count waits behind a record copy), the copy stream
  // and its events
  cp_event* d_gen_stage = nullptr;
  uint64_t gen_cap = 0;
  double* d_gen_red = nullptr;
  unsigned long long* d_gen_cnt = nullptr;
  unsigned long long* h_gen_cnt = nullptr;
  uint64_t gen_chunks_cap = 0;
  cudaStream_t gen_copy = nullptr;
  cudaEvent_t gen_counted[CP_GEN_BUFS] = {}, gen_copied[CP_GEN_BUFS] = {};
  uint64_t last_n = 0;
  // added to every point index of the integration, production and adjoint passes (sharding)
  uint64_t point_offset = 0;
  // learned proposal: FP32 master/grad/Adam moments (4 x n_param), packed BF16 fragments,
  // staged biases, per-point (v, ln J) buffer; flow_on routes the passes through the flow
  float* d_flow = nullptr;
  uint2* d_flow_pk = nullptr;
  float* d_flow_bias = nullptr;
  float4* d_flow_buf = nullptr;
  float* d_flow_u = nullptr;                // accept draws of d_flow_buf's points (same allocation)
  uint64_t flow_buf_cap = 0;
  int flow_on = 0;
  long flow_t = 0;                         // optimiser updates so far (a step's batch iteration)
  double flow_loss_p = 2.0;                // training objective <w^p>/<w>^p
  double adj_p = 2.0;                      // adjoint / variance-gradient objective: moment order
  int adj_params = 1;                      // adjoint passes carry the parameter tangents too
  // training buffers of the current step (per-point forward state and GEMM operands for
  // ftrain_count points), kept between the phases of a data-parallel step
  void* d_ftrain = nullptr;
  uint64_t ftrain_cap = 0, ftrain_count = 0;
  // tensor-core (tcgen05) forward: shared-memory weight image, bounded-wait status flag;
  // flow_kernel 0 = tcgen05 kernel, 1 = the warp-level mma.sync kernel
  uint8_t* d_flow_tc = nullptr;
  int* d_flow_status = nullptr;
  unsigned* d_flow_ticket = nullptr;       // last-block ticket of the training integrand kernel (0 between launches)
  int flow_kernel = 0;
  int flow_tc_stale = 1;                   // the tcgen05 weight image lags the master parameters
  int flow_stall = 0;                      // test hook: the tensor-core forward issues no MMA
  int flow_fuse = 0;                       // production passes: flow forward + accept in one kernel
  // optional per-kernel timing of the production pass (CUDA events on the handle's stream):
  // 0 = flow forward, 1 = accept (K1), 2 = record build (K2)
  int timing = 0;
  std::vector<cudaEvent_t> tpool;          // production timing events: 2 + 3 per chunk
  double t_ms[3] = {0, 0, 0};
  uint64_t t_launches[3] = {0, 0, 0};
  std::string err;
};

int cp_fail(cp_handle* h, int code, const std::string& msg);
int cp_fail_cuda(cp_handle* h, cudaError_t e, const char* what);
int cp_ensure_slots(cp_handle* h, size_t doubles);
int cp_ensure_iters(cp_handle* h, int n);
int cp_flow_buffer(cp_handle* h, uint64_t n);
// uout, if not null, receives each point's accept draw u24(word 3) of its Philox block when the
// tensor-core forward runs (cp_flow_writes_u); the mma.sync forward leaves it untouched.
int cp_flow_forward_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float4* out,
                            float* uout);
inline bool cp_flow_writes_u(const cp_handle* h) { return h->flow_kernel == 0; }
int cp_flow_tc_alloc(cp_handle* h);
int cp_flow_tc_repack(cp_handle* h);
int cp_flow_tc_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, uint32_t stream, float4* out,
                       float* uout);
int cp_flow_tc_status(cp_handle* h);

// Makes `dev` the calling thread's current device for the rest of the scope and restores the
// caller's device at its end, so one host thread can drive handles on several GPUs.
struct CpDeviceGuard {
  int prev = -1;
  explicit CpDeviceGuard(int dev)
  {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~CpDeviceGuard()
  {
    if (prev >= 0) cudaSetDevice(prev);
  }
  CpDeviceGuard(const CpDeviceGuard&) = delete;
  CpDeviceGuard& operator=(const CpDeviceGuard&) = delete;
};

// Entry check of every handle call (a statement at function scope): a null handle is invalid;
// otherwise the handle's device is current until the function returns.
#define CP_CHECK_HANDLE(h)             \
  if (!(h)) return CP_ERR_INVALID;     \
  CpDeviceGuard cp_device_guard_((h)->device)
#define CP_CUDA(h, call)                                        \
  do {                                                          \
    cudaError_t e_ = (call);                                    \
    if (e_ != cudaSuccess) return cp_fail_cuda((h), e_, #call); \
  } while (0)
#define CP_LAUNCH_CHECK(h, what)                                \
  do {                                                          \
    cudaError_t e_ = cudaGetLastError();                        \
    if (e_ != cudaSuccess) return cp_fail_cuda((h), e_, what);  \
  } while (0)

// ------------------------------------------------------------------------------------------
// Device helpers
// ------------------------------------------------------------------------------------------
#if defined(__CUDACC__)

// Kahan-compensated FP32 accumulation
__device__ __forceinline__ void cp_kahan(float& s, float& c, float v)
{
  float y = v - c;
  float t = s + y;
  c = (t - s) - y;
  s = t;
}

// Error-free sum (Knuth TwoSum): a + b = s + e exactly
__device__ __forceinline__ void cp_two_sum(float a, float b, float& s, float& e)
{
  s = a + b;
  float bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// Compensated warp reduction of (hi, lo) pairs; xor tree, deterministic. Result in all lanes.
__device__ __forceinline__ void cp_warp_sum_comp(float& hi, float& lo)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    float oh = __shfl_xor_sync(0xffffffffu, hi, o);
    float ol = __shfl_xor_sync(0xffffffffu, lo, o);
    // order the pair so every lane adds the same two operands in the same order
    int lane = threadIdx.x & 31;
    float a = (lane & o) ? oh : hi, b = (lane & o) ? hi : oh;
    float al = (lane & o) ? ol : lo, bl = (lane & o) ? lo : ol;
    float s, e;
    cp_two_sum(a, b, s, e);
    hi = s;
    lo = (al + bl) + e;
  }
}

__device__ __forceinline__ double cp_warp_sum_d(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double ov = __shfl_xor_sync(0xffffffffu, v, o);
    int lane = threadIdx.x & 31;
    v = (lane & o) ? (ov + v) : (v + ov);
  }
  return v;
}

__device__ __forceinline__ float cp_warp_max(float v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double cp_warp_max_d(double v)
{
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// VEGAS map of a continuous coordinate v in [0, 1] (the flow's output): bin, x, width.
__device__ __forceinline__ void cp_map_v(const float2* edges_d, int nb, float v, int& bin, float& x, float& width)
{
  const float t = v * (float)nb;
  int b = (int)t;
  b = b < 0 ? 0 : (b >= nb ? nb - 1 : b);
  float frac = t - (float)b;
  frac = frac < 0.f ? 0.f : (frac > 1.f ? 1.f : frac);
  const float2 e = edges_d[b];
  bin = b;
  x = fmaf(frac, e.y, e.x);
  width = e.y;
}

// Copies the 8 CTEQ5L coefficient records from global into shared memory (block-wide).
__device__ __forceinline__ void cp_stage_cteq(CpCteqPoly* dst, const CpCteqPoly* src)
{
  const uint32_t* s = reinterpret_cast<const uint32_t*>(src);
  uint32_t* d = reinterpret_cast<uint32_t*>(dst);
  for (int k = threadIdx.x; k < (int)(8 * sizeof(CpCteqPoly) / 4); k += blockDim.x) d[k] = s[k];
}

// Deterministic add of v into a warp-private histogram h[bin]: lanes that share a bin are
// summed in lane order by the group's lowest lane, which alone writes.  Needs all 32 lanes.
__device__ __forceinline__ void cp_warp_hist_add(float* h, int bin, float v)
{
  unsigned peers = __match_any_sync(0xffffffffu, bin);
  int lane = threadIdx.x & 31;
  int leader = __ffs(peers) - 1;
  float sum = 0.f;
  unsigned m = peers;
  while (m) {
    int l = __ffs(m) - 1;
    sum += __shfl_sync(peers, v, l);
    m &= m - 1;
  }
  if (lane == leader) h[bin] += sum;
}

// out[k] = sum over blocks of slots[b][k], or their max for k == max_col; fixed order, FP64.
// One warp per output element.
template <int UNUSED>
__global__ void k_reduce_slots(const double* __restrict__ slots, int nblocks, int width, double* out,
                               int max_col = 2)
{
  const int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (k >= width) return;
  double acc = 0.0;
  if (k == max_col) {
    for (int b = lane; b < nblocks; b += 32) acc = fmax(acc, slots[(size_t)b * width + k]);
    acc = cp_warp_max_d(acc);
  } else {
    for (int b = lane; b < nblocks; b += 32) acc += slots[(size_t)b * width + k];
    acc = cp_warp_sum_d(acc);
  }
  if (lane == 0) out[k] = acc;
}

#endif
