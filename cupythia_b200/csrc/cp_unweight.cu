// cp_unweight.cu -- production pass: unweighting and on-device compaction into 64-byte records.
//
// K1 draws, maps and evaluates each point exactly like the VEGAS pass and accepts it when
// u * w_max < w (cuPythia/07_unweighting_lhe/unweight_lhe.cu:54; overweight events w > w_max
// are kept with weight w / w_max, as Pythia keeps them, pythia8317/src/ProcessContainer.cc:
// 383-385).  Per 32-point block (one warp's points) it stores the warp's accept mask and adds
// the number accepted to its 1024-point range's total (an integer atomic: exact in any order),
// and packs the accepted points' event weights, mapped coordinates and 16 PDF values, in point
// order, at the front of the block's staging slots.  A one-block scan of the range totals gives each range's output offset, so the records
// come out in point order, exactly as the reference's library compaction orders them
// (cub::DeviceSelect::Flagged, cuPythia/10_cub_compaction/cub_compaction.cu:76-80,
// cuPythia/pipeline/generate.cu:97-104), without any block waiting on another.  K2 takes one
// range per warp, spreads its accepted points over the lanes (every lane busy), takes each one's
// point index from its block's mask, recomputes the points' kinematics and brackets from the
// staged coordinates (the PDFs come from K1 too), picks process, flavours and colour
// flow, and writes the 64-byte records as four 16-byte stores (and, on request, the 7-point
// scale-variation ratios).  Keeping the record builder out of K1 keeps K1's code small and its
// lanes converged.  Staging grows with the points of a pass, so passes run in chunks of at most
// CP_UNW_CHUNK points.
//
// Random numbers: the accept draw is word 3 of the point's Philox block (stream 0); accepted
// points draw a second block from stream 1 for the process / pair / azimuth / new-flavour picks
// (high 24 bits of words 0..3) and the colour topology / orientation (their low bytes).
#include <vector>
#include "cp_internal.cuh"

#include "cp_unweight.cuh"

static_assert(sizeof(CpEventRec) == 64, "event record must be 64 bytes");
static_assert(sizeof(CpEventRec) == sizeof(cp_event), "C ABI record layout");

struct CpMapped {
  float x[3], jv;
};

__device__ __forceinline__ CpMapped cp_map_point(const float2 (*sEdge)[CP_MAX_BINS], int nb, const uint32_t wd[4])
{
  CpMapped m;
  m.jv = 1.f;
  const float nbf = (float)nb;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int bin;
    float frac;
    cp_bin_frac(wd[d], nb, bin, frac);
    float2 e = sEdge[d][bin];
    m.x[d] = fmaf(frac, e.y, e.x);
    m.jv *= nbf * e.y;
  }
  return m;
}

// map of a point: the flow's v if present, else the Philox words
__device__ __forceinline__ CpMapped cp_map_any(const float2 (*sEdge)[CP_MAX_BINS], int nb, const uint32_t wd[4],
                                               const float4* flow, uint64_t p)
{
  if (!flow) return cp_map_point(sEdge, nb, wd);
  // the flow already applied the VEGAS map and its own transform: x and the total ln J
  CpMapped m;
  const float4 f = flow[p];
  m.x[0] = f.x; m.x[1] = f.y; m.x[2] = f.z;
  m.jv = expf(f.w);
  return m;
}

__device__ __forceinline__ void cp_stage_edges(float2 (*sEdge)[CP_MAX_BINS], const double* edges, int nb)
{
  for (int k = threadIdx.x; k < 3 * nb; k += CP_THREADS) {
    int d = k / nb, b = k - d * nb;
    const double* e = edges + d * (nb + 1);
    double lo = e[b], hi = e[b + 1];
    sEdge[d][b] = make_float2((float)lo, (float)(hi - lo));
  }
}

// K1: weight, accept; per 32-point block the accept mask (its popcount added to its range's
// total), and each accepted point's event weight, coordinates and PDFs packed at the front of the
// block's staging slots in point order; K2 builds the record from them.
// FLOW_U: the points' accept draws come from the flow forward's output (L.flow_u) instead of their
// Philox blocks; a separate instance, so the plain form's kernel carries no code for it
template <bool FLOW_U>
__global__ void __launch_bounds__(CP_THREADS, CP_MIN_BLOCKS) k_unw_accept(const __grid_constant__ CpHadParams P,
                                                                           const __grid_constant__ UnwLaunch L)
{
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  __shared__ double sRed[CP_WARPS][7];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  cp_stage_edges(sEdge, L.edges, L.nb);
  __syncthreads();
  const float wmax = (float)L.wmax[0];
  const uint64_t stride = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t gtid = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
  const uint64_t rounds = (L.n + stride - 1) / stride;
  CpUnwSums S;
  for (uint64_t r = 0; r < rounds; ++r) {
    // the warp's 32 points are one block: p - lane is a multiple of 32 (stride and block slices are)
    const uint64_t p = r * stride + gtid;
    uint32_t wd[4] = {0u, 0u, 0u, 0u};
    CpMapped m{};
    float u = 0.f;
    if (p < L.n) {
      if constexpr (FLOW_U) {
        // the flow forward drew this point's Philox block for the map and kept its accept draw
        m = cp_map_any(sEdge, L.nb, wd, L.flow, p);
        u = L.flow_u[p];
      } else {
        cp_point_words(L.seed, L.point0 + p, L.iter, 0, wd);
        m = cp_map_any(sEdge, L.nb, wd, L.flow, p);
        u = cp_u24(wd[3]);
      }
    }
    cp_unw_point(P, P.cteq, L, wmax, p, m.x[0], m.x[1], m.x[2], m.jv, u, S);
  }
  double v[7];
  cp_unw_warp_sums(S, v);
  if (lane == 0)
    for (int k = 0; k < 7; ++k) sRed[warp][k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
    double* slot = L.slots + (size_t)blockIdx.x * CP_UNW_SLOT;
    for (int k = 0; k < 7; ++k) {
      double a = 0.0;
      for (int q = 0; q < CP_WARPS; ++q) a = (k == 2) ? fmax(a, sRed[q][k]) : a + sRed[q][k];
      slot[k] = a;
    }
    slot[7] = 0.0;
  }
}

// Output offsets: roff[r] = *base_io + the records of the ranges before r; then *base_io +=
// the chunk's records.  One block of 1024 threads scans the range totals in tiles of 1024
// (coalesced loads, warp shuffles, one running carry): fixed order.
__global__ void __launch_bounds__(1024) k_unw_scan(const unsigned* __restrict__ rsum, uint64_t nrange,
                                                   unsigned long long* base_io, unsigned long long* __restrict__ roff)
{
  __shared__ unsigned long long wsum[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  unsigned long long carry = *base_io;
  for (uint64_t i0 = 0; i0 < nrange; i0 += 1024) {
    const uint64_t i = i0 + t;
    const unsigned long long v = i < nrange ? rsum[i] : 0ull;
    unsigned long long x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[w] = x;
    __syncthreads();
    if (w == 0) {
      unsigned long long z = wsum[lane];
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      wsum[lane] = z;
    }
    __syncthreads();
    if (i < nrange) roff[i] = carry + (w ? wsum[w - 1] : 0ull) + x - v;
    carry += wsum[31];
    __syncthreads();   // wsum is rewritten by the next tile
  }
  __syncthreads();     // every thread has read *base_io
  if (t == 0) *base_io = carry;
}

// K2: work units of a quarter range (8 blocks, 256 points: 65,536 per 2^24-point chunk, so the
// warps' shares differ by about 1%).  A warp loads its range's 32 block masks, scans their
// popcounts with shuffles and spreads the accepted points of its quarter over the lanes in point
// order; each lane takes its point index from its block's mask, re-evaluates the point's
// kinematics from the staged coordinates (the PDFs come from K1's staging too), picks process,
// flavours and colour flow, builds the lab-frame kinematics and stores the full 64-byte record
// at its output index.
// 4 resident blocks per SM without scale weights (64 registers), 2 with them
template <bool SCALEW>
__global__ void __launch_bounds__(CP_THREADS, SCALEW ? 2 : 4) k_unw_build(const __grid_constant__ CpHadParams P,
                                                                          const __grid_constant__ UnwLaunch L)
{
  const int lane = threadIdx.x & 31;
  const uint64_t nwarps = (uint64_t)gridDim.x * (CP_THREADS / 32);
  for (uint64_t U = ((uint64_t)blockIdx.x * CP_THREADS + threadIdx.x) >> 5; U < 4 * L.nrange; U += nwarps) {
    const uint64_t R = U >> 2;
    const int quarter = (int)(U & 3);
    const uint64_t blk = R * CP_UNW_RANGE + lane;
    const unsigned mk = blk < L.nblk ? L.bmask[blk] : 0u;
    const unsigned c = __popc(mk);
    unsigned incl = c;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += v;
    }
    const unsigned excl = incl - c;
    // this quarter's entries of the range: [first, total)
    const unsigned first = __shfl_sync(0xffffffffu, excl, 8 * quarter);
    const unsigned total = __shfl_sync(0xffffffffu, incl, 8 * quarter + 7);
    const unsigned long long base = L.roff[R];
    for (unsigned j0 = first; j0 < total; j0 += 32) {
      const unsigned j = j0 + lane;
      // this lane's entry lies in the first block whose inclusive count exceeds j
      int b = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if (__shfl_sync(0xffffffffu, incl, b + st - 1) <= j) b += st;
      const unsigned ex = __shfl_sync(0xffffffffu, excl, b);
      const unsigned mb = __shfl_sync(0xffffffffu, mk, b);
      const uint64_t k = base + j;   // output record
      if (j >= total || k >= L.capacity) continue;
      // the entry is the block's accepted point of rank r; its lane is the position of the
      // r-th set bit of the block's mask: the largest x with fewer than r + 1 set bits below x
      const unsigned r = j - ex;
      int x = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if ((unsigned)__popc(mb & ((1u << (x + st)) - 1u)) <= r) x += st;
      const uint64_t blkq = (R * CP_UNW_RANGE + b) * 32;
      const uint64_t q = blkq + r;   // staging slot
      const uint4 tail = L.tails[q];
      const uint64_t point = L.point0 + blkq + (uint64_t)x;
      uint32_t w2[4];
      cp_point_words(L.seed, point, L.iter, 1, w2);
      float pdf[16];
#pragma unroll
      for (int f = 0; f < 4; ++f) {
        const float4 v = L.pdf[4 * q + f];
        pdf[4 * f] = v.x; pdf[4 * f + 1] = v.y; pdf[4 * f + 2] = v.z; pdf[4 * f + 3] = v.w;
      }
      CpPoint pt;
      cp_had_eval(P, P.cteq, __uint_as_float(tail.y), __uint_as_float(tail.z), __uint_as_float(tail.w), pt, pdf);
      CpEventRec ev;
      cp_make_event(P, pt, cp_u24(w2[0]), cp_u24(w2[1]), cp_u24(w2[2]), cp_u24(w2[3]), cp_colour_rc(w2),
                    cp_colour_rs(w2), __uint_as_float(tail.x), (uint32_t)point, ev);
      if (SCALEW) {
        float r[6];
        cp_scale_ratios(P, P.cteq, pt, r);
        float2* sw = reinterpret_cast<float2*>(L.scalew + 6 * k);
        sw[0] = make_float2(r[0], r[1]);
        sw[1] = make_float2(r[2], r[3]);
        sw[2] = make_float2(r[4], r[5]);
      }
      const uint4* src = reinterpret_cast<const uint4*>(&ev);
      uint4* dst = reinterpret_cast<uint4*>(L.out + k);
#pragma unroll
      for (int f = 0; f < 4; ++f) dst[f] = src[f];
    }
  }
}

__global__ void k_set_wmax(double* wmax, double v) { wmax[0] = v; }

static int unw_blocks(cp_handle* h)
{
  if (h->unw_per_sm < 0) {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unw_accept<false>, CP_THREADS, 0) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    h->unw_per_sm = per_sm;
  }
  return h->num_sms * h->unw_per_sm;
}

// The record builder loops grid-stride over the records: its grid is exactly the blocks that
// are resident at once, so no second wave runs after the first.
static int build_blocks(cp_handle* h, bool scalew)
{
  int& c = h->build_per_sm[scalew ? 1 : 0];
  if (c < 0) {
    int per_sm = 1;
    const cudaError_t e = scalew ? cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unw_build<true>, CP_THREADS, 0)
                                 : cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unw_build<false>, CP_THREADS, 0);
    c = (e != cudaSuccess || per_sm < 1) ? 1 : per_sm;
  }
  return h->num_sms * c;
}

// Staging of a production chunk of n points: record tails and PDFs per point, accept masks per
// 32-point block, totals and output offsets per 1024-point range.
static int unw_staging(cp_handle* h, uint64_t n)
{
  if (n <= h->pdfbuf_cap) return CP_OK;
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  void* old[] = {h->d_pdfbuf, h->d_tails, h->d_bmask, h->d_roff, h->d_rsum};
  for (void* b : old)
    if (b) CP_CUDA(h, cudaFree(b));
  h->d_pdfbuf = nullptr; h->d_tails = nullptr; h->d_bmask = nullptr; h->d_roff = nullptr; h->d_rsum = nullptr;
  h->pdfbuf_cap = 0;
  const uint64_t nblk = (n + 31) / 32, nrange = (nblk + CP_UNW_RANGE - 1) / CP_UNW_RANGE;
  CP_CUDA(h, cudaMalloc(&h->d_pdfbuf, sizeof(float4) * 4 * n));
  CP_CUDA(h, cudaMalloc(&h->d_tails, sizeof(uint4) * n));
  CP_CUDA(h, cudaMalloc(&h->d_bmask, sizeof(unsigned) * nblk));
  CP_CUDA(h, cudaMalloc(&h->d_roff, sizeof(unsigned long long) * nrange));
  CP_CUDA(h, cudaMalloc(&h->d_rsum, sizeof(unsigned) * nrange));
  h->pdfbuf_cap = n;
  return CP_OK;
}

// Per-kernel timing events of a pass: the flow forward's pair, then 3 per chunk (before the
// accept kernel, after it, after the record builder); created on first use.
static int timing_reserve(cp_handle* h, size_t nsub)
{
  if (!h->timing) return CP_OK;
  while (h->tpool.size() < 2 + 3 * nsub) {
    cudaEvent_t e;
    CP_CUDA(h, cudaEventCreate(&e));
    h->tpool.push_back(e);
  }
  return CP_OK;
}

// Adds the kernel durations of one pass (after its last event) and counts the pass once per
// kernel that ran.
static void timing_collect(cp_handle* h, size_t nsub, bool flow, bool build)
{
  if (!h->timing || nsub == 0 || h->tpool.size() < 2 + 3 * nsub) return;
  if (cudaEventSynchronize(h->tpool[2 + 3 * nsub - 1]) != cudaSuccess) return;
  float a = 0.f;
  if (flow && cudaEventElapsedTime(&a, h->tpool[0], h->tpool[1]) == cudaSuccess) h->t_ms[0] += a;
  for (size_t c = 0; c < nsub; ++c) {
    float b = 0.f, d = 0.f;
    cudaEventElapsedTime(&b, h->tpool[2 + 3 * c], h->tpool[2 + 3 * c + 1]);
    cudaEventElapsedTime(&d, h->tpool[2 + 3 * c + 1], h->tpool[2 + 3 * c + 2]);
    h->t_ms[1] += b; h->t_ms[2] += d;
  }
  h->t_launches[0] += flow ? 1 : 0;
  h->t_launches[1] += 1;
  h->t_launches[2] += build ? 1 : 0;
}

// The flow form's production chunks run the tcgen05 kernel's production form (flow forward,
// integrand and accept step in one kernel) instead of the forward followed by k_unw_accept.
static bool fused_production(const cp_handle* h) { return h->flow_on && h->flow_kernel == 0 && h->flow_fuse; }

// Enqueue one production chunk of n <= CP_UNW_CHUNK points on h->stream (no host
// synchronisation).  Its records go to out[*base_dev ...] in point order (records at or beyond
// `capacity` are counted, not stored) and *base_dev advances by the chunk's accepted points;
// red_dst receives the chunk's sums.  With the flow on, flow_pre holds the flow output of the
// chunk's points (the caller ran the forward pass for the whole pass), or is null and the chunk
// runs its own.  tslot >= 0 records the chunk's timing events.
static int unweight_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, cp_event* out,
                            uint64_t capacity, double* red_dst, float* scalew, unsigned long long* base_dev,
                            const float4* flow_pre, const float* flow_u_pre, int tslot)
{
  if (n > CP_UNW_CHUNK) return cp_fail(h, CP_ERR_INVALID, "production chunk above CP_UNW_CHUNK points");
  const int blocks = unw_blocks(h);
  int rc = cp_ensure_slots(h, (size_t)blocks * CP_UNW_SLOT);
  if (rc) return rc;
  point0 += h->point_offset;
  UnwLaunch L;
  L.seed = h->cfg.seed; L.point0 = point0; L.n = n; L.iter = iter; L.nb = h->nb;
  L.edges = h->d_edges; L.wmax = h->d_wmax;
  L.out = reinterpret_cast<CpEventRec*>(out);
  L.capacity = capacity; L.slots = h->d_slots;
  L.pdf = nullptr; L.tails = nullptr; L.bmask = nullptr; L.roff = nullptr; L.rsum = nullptr;
  L.nblk = (n + 31) / 32;
  L.nrange = (L.nblk + CP_UNW_RANGE - 1) / CP_UNW_RANGE;
  L.scalew = scalew;
  if (capacity) {
    rc = unw_staging(h, n);
    if (rc) return rc;
    L.pdf = h->d_pdfbuf; L.tails = h->d_tails; L.bmask = h->d_bmask; L.roff = h->d_roff; L.rsum = h->d_rsum;
    CP_CUDA(h, cudaMemsetAsync(h->d_rsum, 0, sizeof(unsigned) * L.nrange, h->stream));
  }
  L.flow = nullptr;
  L.flow_u = nullptr;
  const bool fused = fused_production(h);
  if (h->flow_on && !fused) {
    if (flow_pre) {
      L.flow = flow_pre;
      L.flow_u = flow_u_pre;
    } else {
      rc = cp_flow_buffer(h, n);
      if (rc) return rc;
      float* ut = cp_flow_writes_u(h) ? h->d_flow_u : nullptr;
      rc = cp_flow_forward_enqueue(h, point0, n, iter, 0, h->d_flow_buf, ut);
      if (rc) return rc;
      L.flow = h->d_flow_buf;
      L.flow_u = ut;
    }
  }
  cudaEvent_t* ev = (h->timing && tslot >= 0 && h->tpool.size() >= 2 + 3 * (size_t)(tslot + 1)) ? &h->tpool[2 + 3 * tslot] : nullptr;
  if (ev) cudaEventRecord(ev[0], h->stream);
  int red_blocks = blocks;
  if (fused) {
    rc = cp_flow_tc_accept_enqueue(h, L, &red_blocks);
    if (rc) return rc;
  } else {
    if (L.flow_u) k_unw_accept<true><<<blocks, CP_THREADS, 0, h->stream>>>(h->P, L);
    else k_unw_accept<false><<<blocks, CP_THREADS, 0, h->stream>>>(h->P, L);
    CP_LAUNCH_CHECK(h, "k_unw_accept");
  }
  if (ev) cudaEventRecord(ev[1], h->stream);
  k_reduce_slots<0><<<1, CP_UNW_SLOT * 32, 0, h->stream>>>(h->d_slots, red_blocks, CP_UNW_SLOT, red_dst);
  CP_LAUNCH_CHECK(h, "k_reduce_slots");
  if (capacity) {
    k_unw_scan<<<1, 1024, 0, h->stream>>>(h->d_rsum, L.nrange, base_dev, h->d_roff);
    CP_LAUNCH_CHECK(h, "k_unw_scan");
    if (L.scalew) k_unw_build<true><<<build_blocks(h, true), CP_THREADS, 0, h->stream>>>(h->P, L);
    else k_unw_build<false><<<build_blocks(h, false), CP_THREADS, 0, h->stream>>>(h->P, L);
    CP_LAUNCH_CHECK(h, "k_unw_build");
  }
  if (ev) cudaEventRecord(ev[2], h->stream);
  return CP_OK;
}

// sums of the chunks of a pass: every entry added, the largest weight (entry 2) by max
static void combine_chunks(const double* hred, uint64_t nsub, double tot[8])
{
  for (int k = 0; k < 8; ++k) tot[k] = 0.0;
  for (uint64_t c = 0; c < nsub; ++c)
    for (int k = 0; k < 8; ++k) tot[k] = (k == 2) ? (hred[8 * c + k] > tot[k] ? hred[8 * c + k] : tot[k]) : tot[k] + hred[8 * c + k];
}

static void fill_unw(const double* red, double n, double wmax, cp_unweight_result* o)
{
  double mean = red[0] / n, var = (red[1] / n - mean * mean) / (n - 1.0);
  o->sigma = mean;
  o->sigma_err = sqrt(var > 0 ? var : 0);
  o->sigma_unweighted = wmax * red[5] / n;
  o->w_max = wmax;
  o->w_max_seen = red[2];
  o->n_points = (uint64_t)n;
  o->n_accepted = (uint64_t)red[4];
  o->n_overweight = (uint64_t)red[6];
  o->n_bad = (uint64_t)red[3];
  o->eta = red[4] / n;
}

extern "C" int cp_set_wmax(cp_handle* h, double w_max)
{
  CP_CHECK_HANDLE(h);
  if (!(w_max > 0)) return cp_fail(h, CP_ERR_INVALID, "cp_set_wmax: w_max must be positive");
  k_set_wmax<<<1, 1, 0, h->stream>>>(h->d_wmax, w_max);
  CP_LAUNCH_CHECK(h, "k_set_wmax");
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  h->wmax_host = w_max;
  return CP_OK;
}

extern "C" int cp_unweight(cp_handle* h, uint64_t n_points, uint32_t iter, cp_event* records_dev,
                           uint64_t capacity, cp_unweight_result* out)
{
  CP_CHECK_HANDLE(h);
  if (n_points < 2) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: n_points < 2");
  if (capacity && !records_dev) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: null records");
  if (((uintptr_t)records_dev & 15) != 0) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: records must be 16-byte aligned");
  // the threshold as cp_weight_quantile / cp_weight_quantile_hist / cp_set_wmax last set it: no
  // device read, so the host enqueues the pass while the stream's earlier work still runs
  const double wm0 = h->wmax_host;
  if (!(wm0 > 0)) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: no threshold (cp_weight_quantile or cp_set_wmax)");
  if (n_points > (1ull << 32)) return cp_fail(h, CP_ERR_INVALID, "at most 2^32 points per production call");
  if (h->scalew && capacity > h->scalew_cap)
    return cp_fail(h, CP_ERR_INVALID, "cp_unweight: record capacity exceeds the scale-weight buffer (cp_set_scale_weights)");
  // chunks of at most CP_UNW_CHUNK points; the running record count (d_counter) places each
  // chunk's records after the previous chunk's
  const uint64_t nsub = (n_points + CP_UNW_CHUNK - 1) / CP_UNW_CHUNK;
  if (nsub > h->unw_red_cap) {
    CP_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->d_unw_red) CP_CUDA(h, cudaFree(h->d_unw_red));
    h->d_unw_red = nullptr;
    h->unw_red_cap = 0;
    CP_CUDA(h, cudaMalloc(&h->d_unw_red, sizeof(double) * 8 * nsub));
    h->unw_red_cap = nsub;
  }
  int rc = timing_reserve(h, nsub);
  if (rc) return rc;
  CP_CUDA(h, cudaMemsetAsync(h->d_counter, 0, sizeof(unsigned long long), h->stream));
  // the flow forward once for the whole pass (20 B per point: (v, ln J) and the accept draw), then the chunks; the fused form
  // runs the forward inside each chunk's accept kernel
  const bool fused = fused_production(h);
  if (h->flow_on && !fused) {
    rc = cp_flow_buffer(h, n_points);
    if (rc) return rc;
    if (h->timing) cudaEventRecord(h->tpool[0], h->stream);
    rc = cp_flow_forward_enqueue(h, h->point_offset, n_points, iter, 0, h->d_flow_buf,
                                 cp_flow_writes_u(h) ? h->d_flow_u : nullptr);
    if (rc) return rc;
    if (h->timing) cudaEventRecord(h->tpool[1], h->stream);
  }
  for (uint64_t c = 0; c < nsub; ++c) {
    const uint64_t p0 = c * CP_UNW_CHUNK, n = p0 + CP_UNW_CHUNK <= n_points ? CP_UNW_CHUNK : n_points - p0;
    rc = unweight_enqueue(h, p0, n, iter, records_dev, capacity, h->d_unw_red + 8 * c, h->scalew, h->d_counter,
                          (h->flow_on && !fused) ? h->d_flow_buf + p0 : nullptr,
                          (h->flow_on && !fused && cp_flow_writes_u(h)) ? h->d_flow_u + p0 : nullptr, (int)c);
    if (rc) return rc;
  }
  std::vector<double> hred(8 * nsub, 0.0);
  unsigned long long cnt = 0;
  CP_CUDA(h, cudaMemcpyAsync(hred.data(), h->d_unw_red, sizeof(double) * 8 * nsub, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(&cnt, h->d_counter, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  timing_collect(h, nsub, h->flow_on && !fused, capacity > 0);
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) return rc;
  double red[8];
  combine_chunks(hred.data(), nsub, red);
  if (out) fill_unw(red, (double)n_points, wm0, out);
  if (cnt > capacity) return cp_fail(h, CP_ERR_CAPACITY, "cp_unweight: record buffer too small (n_accepted reported)");
  if (red[3] > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights were zeroed");
  return CP_OK;
}

// one counter, copied by a kernel into the mapped pinned host array (no copy engine involved)
__global__ void k_gen_count(const unsigned long long* __restrict__ src, unsigned long long* dst_mapped)
{
  *(volatile unsigned long long*)dst_mapped = *src;
  __threadfence_system();
}

// Buffers and streams of the host-delivery pipeline, grown on demand and kept in the handle.
static int gen_reserve(cp_handle* h, uint64_t cap, uint64_t nchunks)
{
  if (cap > h->gen_cap) {
    if (h->d_gen_stage) {
      if (h->gen_copy) CP_CUDA(h, cudaStreamSynchronize(h->gen_copy));
      CP_CUDA(h, cudaStreamSynchronize(h->stream));
      CP_CUDA(h, cudaFree(h->d_gen_stage));
      h->d_gen_stage = nullptr;
      h->gen_cap = 0;
    }
    CP_CUDA(h, cudaMalloc(&h->d_gen_stage, sizeof(cp_event) * CP_GEN_BUFS * cap));
    h->gen_cap = cap;
  }
  if (nchunks > h->gen_chunks_cap) {
    CP_CUDA(h, cudaStreamSynchronize(h->stream));
    if (h->d_gen_red) { CP_CUDA(h, cudaFree(h->d_gen_red)); h->d_gen_red = nullptr; }
    if (h->d_gen_cnt) { CP_CUDA(h, cudaFree(h->d_gen_cnt)); h->d_gen_cnt = nullptr; }
    if (h->h_gen_cnt) { CP_CUDA(h, cudaFreeHost(h->h_gen_cnt)); h->h_gen_cnt = nullptr; }
    h->gen_chunks_cap = 0;
    CP_CUDA(h, cudaMalloc(&h->d_gen_red, sizeof(double) * 8 * nchunks));
    CP_CUDA(h, cudaMalloc(&h->d_gen_cnt, sizeof(unsigned long long) * nchunks));
    CP_CUDA(h, cudaHostAlloc(&h->h_gen_cnt, sizeof(unsigned long long) * nchunks, cudaHostAllocMapped));
    h->gen_chunks_cap = nchunks;
  }
  if (!h->gen_copy) {
    CP_CUDA(h, cudaStreamCreateWithFlags(&h->gen_copy, cudaStreamNonBlocking));
    for (int b = 0; b < CP_GEN_BUFS; ++b) {
      CP_CUDA(h, cudaEventCreateWithFlags(&h->gen_counted[b], cudaEventDisableTiming));
      CP_CUDA(h, cudaEventCreateWithFlags(&h->gen_copied[b], cudaEventDisableTiming));
    }
  }
  return CP_OK;
}

// Chunked production into HOST memory.  Chunk c is computed on the handle's stream into staging
// buffer c % CP_GEN_BUFS (after that buffer's previous copy has drained); its accepted count
// reaches the host through mapped pinned memory; the host enqueues chunk c + 1 before it waits
// for that count, then enqueues chunk c's records on the copy stream.  The device therefore
// never waits for the host, the copy engine only carries records, and with copies slower than
// compute the copy stream runs back to back.  records_host should be pinned for the copies to
// overlap.  On return every copy into records_host has finished.
extern "C" int cp_generate_host(cp_handle* h, uint64_t n_points, uint32_t iter, uint64_t chunk,
                                cp_event* records_host, uint64_t capacity, cp_unweight_result* out)
{
  CP_CHECK_HANDLE(h);
  if (n_points < 2 || chunk < 2) return cp_fail(h, CP_ERR_INVALID, "cp_generate_host: bad sizes");
  if (capacity && !records_host) return cp_fail(h, CP_ERR_INVALID, "cp_generate_host: null records");
  const double wm0 = h->wmax_host;
  if (!(wm0 > 0)) return cp_fail(h, CP_ERR_INVALID, "cp_generate_host: no threshold");
  if (chunk > n_points) chunk = n_points;
  if (chunk > CP_UNW_CHUNK) chunk = CP_UNW_CHUNK;
  const uint64_t nchunks = (n_points + chunk - 1) / chunk;
  // a chunk accepts at most every point: staging slots = chunk
  int rc = gen_reserve(h, chunk, nchunks);
  if (rc) return rc;
  std::vector<double> hred(nchunks * 8, 0.0);
  uint64_t written = 0, total_acc = 0;
  cudaError_t e = cudaSuccess;
  unsigned long long* const hcnt = h->h_gen_cnt;
  unsigned long long* dcnt_mapped = nullptr;
  // records of chunk j: wait for its count, copy what fits
  auto drain = [&](uint64_t j) -> cudaError_t {
    const int b = (int)(j % CP_GEN_BUFS);
    cudaError_t x = cudaEventSynchronize(h->gen_counted[b]);
    if (x != cudaSuccess) return x;
    const unsigned long long cnt = *(volatile unsigned long long*)(hcnt + j);
    total_acc += cnt;
    uint64_t take = cnt < chunk ? cnt : chunk;
    if (written + take > capacity) take = capacity > written ? capacity - written : 0;
    if ((x = cudaStreamWaitEvent(h->gen_copy, h->gen_counted[b], 0)) != cudaSuccess) return x;
    if (take && (x = cudaMemcpyAsync(records_host + written, h->d_gen_stage + (uint64_t)b * chunk,
                                     sizeof(cp_event) * take, cudaMemcpyDeviceToHost, h->gen_copy)) != cudaSuccess)
      return x;
    written += take;
    return cudaEventRecord(h->gen_copied[b], h->gen_copy);
  };
  do {
    if ((e = cudaHostGetDevicePointer((void**)&dcnt_mapped, hcnt, 0)) != cudaSuccess) break;
    if ((e = cudaMemsetAsync(h->d_gen_cnt, 0, sizeof(unsigned long long) * nchunks, h->stream)) != cudaSuccess) break;
    for (uint64_t c = 0; c < nchunks; ++c) {
      const int b = (int)(c % CP_GEN_BUFS);
      const uint64_t p0 = c * chunk, n = (p0 + chunk <= n_points) ? chunk : n_points - p0;
      if (c >= CP_GEN_BUFS && (e = cudaStreamWaitEvent(h->stream, h->gen_copied[b], 0)) != cudaSuccess) break;
      rc = unweight_enqueue(h, p0, n, iter, h->d_gen_stage + (uint64_t)b * chunk, chunk, h->d_gen_red + 8 * c,
                            nullptr, h->d_gen_cnt + c, nullptr, nullptr, -1);
      if (rc) break;
      k_gen_count<<<1, 1, 0, h->stream>>>(h->d_gen_cnt + c, dcnt_mapped + c);
      if ((e = cudaGetLastError()) != cudaSuccess) break;
      if ((e = cudaEventRecord(h->gen_counted[b], h->stream)) != cudaSuccess) break;
      if (c >= 1 && (e = drain(c - 1)) != cudaSuccess) break;
    }
    if (e != cudaSuccess || rc) break;
    if ((e = drain(nchunks - 1)) != cudaSuccess) break;
    if ((e = cudaMemcpyAsync(hred.data(), h->d_gen_red, sizeof(double) * 8 * nchunks, cudaMemcpyDeviceToHost,
                             h->stream)) != cudaSuccess) break;
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) break;
    e = cudaStreamSynchronize(h->gen_copy);
  } while (0);
  // no copy into records_host may outlive the call, on the error paths too
  cudaStreamSynchronize(h->stream);
  cudaStreamSynchronize(h->gen_copy);
  if (e != cudaSuccess) return cp_fail_cuda(h, e, "cp_generate_host");
  if (rc) return rc;
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) return rc;
  double tot[8];
  combine_chunks(hred.data(), nchunks, tot);
  if (out) fill_unw(tot, (double)n_points, wm0, out);
  if (total_acc > capacity) return cp_fail(h, CP_ERR_CAPACITY, "cp_generate_host: record buffer too small");
  if (tot[3] > 0) return cp_fail(h, CP_ERR_NUMERIC, "non-finite or negative weights were zeroed");
  return CP_OK;
}

// Scale-variation weights of the production pass: with a buffer set, cp_unweight also writes
// 6 floats per record slot (the ratios of cp_scale_ratios) into it; null switches them off.
// cp_generate_host does not write them.
extern "C" int cp_set_scale_weights(cp_handle* h, float* weights_dev, uint64_t capacity)
{
  CP_CHECK_HANDLE(h);
  if (weights_dev && ((uintptr_t)weights_dev & 7))
    return cp_fail(h, CP_ERR_INVALID, "cp_set_scale_weights: buffer must be 8-byte aligned");
  h->scalew = weights_dev;
  h->scalew_cap = weights_dev ? capacity : 0;
  return CP_OK;
}

// Per-kernel timing of the production pass: on != 0 records CUDA events around the flow forward,
// the accept kernel (or the fused forward + accept kernel) and the record builder (plus the tiny slot reduction) on the handle's stream
// and accumulates their durations; cp_kernel_times reads and optionally resets them.
extern "C" int cp_set_kernel_timing(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  h->timing = on ? 1 : 0;
  return CP_OK;
}

extern "C" int cp_kernel_times(cp_handle* h, double* ms3, uint64_t* launches3, int reset)
{
  CP_CHECK_HANDLE(h);
  for (int k = 0; k < 3; ++k) {
    if (ms3) ms3[k] = h->t_ms[k];
    if (launches3) launches3[k] = h->t_launches[k];
    if (reset) { h->t_ms[k] = 0.0; h->t_launches[k] = 0; }
  }
  return CP_OK;
}
