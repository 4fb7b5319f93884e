// cp_unweight.cu -- production pass: unweighting and on-device compaction into 64-byte records.
//
// K1 draws, maps and evaluates each point exactly like the VEGAS pass, accepts it when
// u * w_max < w (cuPythia/07_unweighting_lhe/unweight_lhe.cu:54; overweight events w > w_max
// are kept with weight w / w_max, as Pythia keeps them, pythia8317/src/ProcessContainer.cc:
// 383-385) and reserves a slot in the dense record array (one ballot and one global atomic per
// warp); beside the slot it stores the point's 16 PDF values.  K2 then runs over the reserved
// slots only, with every lane busy, recomputes the points' kinematics and brackets (the PDFs
// come from K1), picks process, flavours and colour flow, and writes the 64-byte records as four
// 16-byte stores (and, on request, the 7-point scale-variation ratios).  Keeping the record builder
// out of K1 keeps K1's code small (its instruction-cache footprint, not arithmetic, limited the
// fused version) and its lanes converged.  The reference instead writes flags and runs a
// separate library compaction pass (cuPythia/10_cub_compaction/cub_compaction.cu:76-80,
// cuPythia/pipeline/generate.cu:97-104).
//
// Random numbers: the accept draw is word 3 of the point's Philox block (stream 0); accepted
// points draw a second block from stream 1 for the process / pair / azimuth / new-flavour picks
// (high 24 bits of words 0..3) and the colour topology / orientation (their low bytes).
#include <vector>
#include "cp_internal.cuh"

#define CP_UNW_SLOT 8   // sum w, sum w^2, max w, n_bad, n_acc, sum event weight, n_over, unused

struct UnwLaunch {
  uint64_t seed, point0, n;
  uint32_t iter;
  int nb;
  const double* edges;
  const CpCteqPoly* cteq;
  const double* wmax;          // device threshold
  CpEventRec* out;
  float4* pdf;                 // per record slot: fa[8], fb[8] of the accepted point (K1 -> K2)
  float* scalew;               // per record slot: 6 scale-variation ratios, or null
  uint64_t capacity;
  unsigned long long* counter; // events accepted so far (may exceed capacity: reported)
  double* slots;
  const float4* flow;          // flow output (v, ln J) per in-call point, or null
};

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

// K1: weight, accept, reserve a record slot (one ballot and one atomic per warp) and store the
// point's in-call index and event weight in that slot; K2 fills in the rest of the record.
__global__ void __launch_bounds__(CP_THREADS, CP_MIN_BLOCKS) k_unw_accept(const CpHadParams P, const UnwLaunch L)
{
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  __shared__ CpCteqPoly sCteq[8];
  __shared__ double sRed[CP_WARPS][7];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  cp_stage_edges(sEdge, L.edges, L.nb);
  cp_stage_cteq(sCteq, L.cteq);
  __syncthreads();
  const float wmax = (float)L.wmax[0];
  const uint64_t stride = (uint64_t)gridDim.x * CP_THREADS;
  const uint64_t gtid = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x;
  const uint64_t rounds = (L.n + stride - 1) / stride;
  float s1 = 0.f, c1 = 0.f, s2 = 0.f, c2 = 0.f, se = 0.f, ce = 0.f, wm = 0.f;
  uint32_t nbad = 0, nacc = 0, nover = 0;

  for (uint64_t r = 0; r < rounds; ++r) {
    const uint64_t p = r * stride + gtid;
    bool accept = false;
    float w = 0.f;
    CpPoint pt;
    if (p < L.n) {
      uint32_t wd[4];
      cp_point_words(L.seed, L.point0 + p, L.iter, 0, wd);
      CpMapped m = cp_map_any(sEdge, L.nb, wd, L.flow, p);
      w = cp_had_eval(P, sCteq, m.x[0], m.x[1], m.x[2], pt) * m.jv;
      if (!(w >= 0.f) || isinf(w)) { ++nbad; w = 0.f; }
      cp_kahan(s1, c1, w);
      cp_kahan(s2, c2, w * w);
      wm = fmaxf(wm, w);
      accept = cp_u24(wd[3]) * wmax < w;
    }
    const unsigned ball = __ballot_sync(0xffffffffu, accept);
    if (ball == 0u) continue;
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(L.counter, (unsigned long long)__popc(ball));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (accept) {
      const uint64_t slot = base + __popc(ball & ((1u << lane) - 1u));
      const float ew = w > wmax ? w / wmax : 1.f;
      ++nacc;
      nover += w > wmax ? 1u : 0u;
      cp_kahan(se, ce, ew);
      if (slot < L.capacity) {
        // weight, pt_hat, process, point: the last 16 bytes of the record
        uint4* dst = reinterpret_cast<uint4*>(L.out + slot) + 3;
        *dst = make_uint4(__float_as_uint(ew), 0u, 0u, (uint32_t)p);
        // the PDFs of the point, so that the record builder need not evaluate CTEQ5L again
        float4* q = L.pdf + 4 * slot;
        q[0] = make_float4(pt.fa[0], pt.fa[1], pt.fa[2], pt.fa[3]);
        q[1] = make_float4(pt.fa[4], pt.fa[5], pt.fa[6], pt.fa[7]);
        q[2] = make_float4(pt.fb[0], pt.fb[1], pt.fb[2], pt.fb[3]);
        q[3] = make_float4(pt.fb[4], pt.fb[5], pt.fb[6], pt.fb[7]);
      }
    }
  }
  double v[7] = {(double)s1 - (double)c1, (double)s2 - (double)c2, (double)wm, (double)nbad,
                 (double)nacc, (double)se - (double)ce, (double)nover};
#pragma unroll
  for (int k = 0; k < 7; ++k) v[k] = (k == 2) ? cp_warp_max_d(v[k]) : cp_warp_sum_d(v[k]);
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

// K2: dense pass over the reserved slots: re-evaluate the accepted point's kinematics (its PDFs
// come from K1's per-slot copy), pick process, flavours and colour flow, build the lab-frame
// kinematics, store the full 64-byte record.
// 4 resident blocks per SM without scale weights (64 registers), 2 with them
template <bool SCALEW>
__global__ void __launch_bounds__(CP_THREADS, SCALEW ? 2 : 4) k_unw_build(const CpHadParams P, const UnwLaunch L)
{
  __shared__ float2 sEdge[3][CP_MAX_BINS];
  __shared__ CpCteqPoly sCteq[8];
  cp_stage_edges(sEdge, L.edges, L.nb);
  cp_stage_cteq(sCteq, L.cteq);
  __syncthreads();
  const unsigned long long acc = *L.counter;
  const uint64_t nrec = acc < L.capacity ? acc : L.capacity;
  for (uint64_t k = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x; k < nrec;
       k += (uint64_t)gridDim.x * CP_THREADS) {
    const uint4 tail = reinterpret_cast<const uint4*>(L.out + k)[3];
    const uint64_t point = L.point0 + tail.w;
    uint32_t wd[4], w2[4];
    cp_point_words(L.seed, point, L.iter, 0, wd);
    cp_point_words(L.seed, point, L.iter, 1, w2);
    CpMapped m = cp_map_any(sEdge, L.nb, wd, L.flow, tail.w);
    float pdf[16];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const float4 v = L.pdf[4 * k + q];
      pdf[4 * q] = v.x; pdf[4 * q + 1] = v.y; pdf[4 * q + 2] = v.z; pdf[4 * q + 3] = v.w;
    }
    CpPoint pt;
    cp_had_eval(P, sCteq, m.x[0], m.x[1], m.x[2], pt, pdf);
    CpEventRec ev;
    cp_make_event(P, pt, cp_u24(w2[0]), cp_u24(w2[1]), cp_u24(w2[2]), cp_u24(w2[3]), cp_colour_rc(w2),
                  cp_colour_rs(w2), __uint_as_float(tail.x), (uint32_t)point, ev);
    if (SCALEW) {
      float r[6];
      cp_scale_ratios(P, sCteq, pt, r);
      float2* sw = reinterpret_cast<float2*>(L.scalew + 6 * k);
      sw[0] = make_float2(r[0], r[1]);
      sw[1] = make_float2(r[2], r[3]);
      sw[2] = make_float2(r[4], r[5]);
    }
    const uint4* src = reinterpret_cast<const uint4*>(&ev);
    uint4* dst = reinterpret_cast<uint4*>(L.out + k);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = src[q];
  }
}

__global__ void k_set_wmax(double* wmax, double v) { wmax[0] = v; }

static int unw_blocks(cp_handle* h)
{
  if (h->unw_per_sm < 0) {
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_unw_accept, CP_THREADS, 0) != cudaSuccess ||
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

// Enqueue one production pass on h->stream (no host synchronisation).
static int unweight_enqueue(cp_handle* h, uint64_t point0, uint64_t n, uint32_t iter, cp_event* out,
                            uint64_t capacity, double* red_dst, float* scalew = nullptr)
{
  const int blocks = unw_blocks(h);
  int rc = cp_ensure_slots(h, (size_t)blocks * CP_UNW_SLOT);
  if (rc) return rc;
  if (n > (1ull << 32)) return cp_fail(h, CP_ERR_INVALID, "at most 2^32 points per production call");
  point0 += h->point_offset;
  UnwLaunch L;
  L.seed = h->cfg.seed; L.point0 = point0; L.n = n; L.iter = iter; L.nb = h->nb;
  L.edges = h->d_edges; L.cteq = h->d_cteq; L.wmax = h->d_wmax;
  L.out = reinterpret_cast<CpEventRec*>(out);
  L.capacity = capacity; L.counter = h->d_counter; L.slots = h->d_slots;
  L.pdf = nullptr;
  L.scalew = scalew;
  if (capacity) {
    if (capacity > h->pdfbuf_cap) {
      if (h->d_pdfbuf) {
        CP_CUDA(h, cudaStreamSynchronize(h->stream));
        CP_CUDA(h, cudaFree(h->d_pdfbuf));
        h->d_pdfbuf = nullptr;
        h->pdfbuf_cap = 0;
      }
      CP_CUDA(h, cudaMalloc(&h->d_pdfbuf, sizeof(float4) * 4 * capacity));
      h->pdfbuf_cap = capacity;
    }
    L.pdf = h->d_pdfbuf;
  }
  L.flow = nullptr;
  if (h->timing) cudaEventRecord(h->tev[0], h->stream);
  if (h->flow_on) {
    rc = cp_flow_buffer(h, n);
    if (rc) return rc;
    rc = cp_flow_forward_enqueue(h, point0, n, iter, 0, h->d_flow_buf);
    if (rc) return rc;
    L.flow = h->d_flow_buf;
  }
  if (h->timing) cudaEventRecord(h->tev[1], h->stream);
  k_unw_accept<<<blocks, CP_THREADS, 0, h->stream>>>(h->P, L);
  CP_LAUNCH_CHECK(h, "k_unw_accept");
  if (h->timing) cudaEventRecord(h->tev[2], h->stream);
  k_reduce_slots<0><<<1, CP_UNW_SLOT * 32, 0, h->stream>>>(h->d_slots, blocks, CP_UNW_SLOT, red_dst);
  CP_LAUNCH_CHECK(h, "k_reduce_slots");
  if (capacity) {
    if (L.scalew) k_unw_build<true><<<build_blocks(h, true), CP_THREADS, 0, h->stream>>>(h->P, L);
    else k_unw_build<false><<<build_blocks(h, false), CP_THREADS, 0, h->stream>>>(h->P, L);
    CP_LAUNCH_CHECK(h, "k_unw_build");
  }
  if (h->timing) {
    cudaEventRecord(h->tev[3], h->stream);
    if (cudaEventSynchronize(h->tev[3]) == cudaSuccess) {
      float a = 0.f, b = 0.f, c = 0.f;
      cudaEventElapsedTime(&a, h->tev[0], h->tev[1]);
      cudaEventElapsedTime(&b, h->tev[1], h->tev[2]);
      cudaEventElapsedTime(&c, h->tev[2], h->tev[3]);
      h->t_ms[0] += a; h->t_ms[1] += b; h->t_ms[2] += c;
      h->t_launches[0] += h->flow_on ? 1 : 0; h->t_launches[1] += 1; h->t_launches[2] += capacity ? 1 : 0;
    }
  }
  return CP_OK;
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
  return CP_OK;
}

extern "C" int cp_unweight(cp_handle* h, uint64_t n_points, uint32_t iter, cp_event* records_dev,
                           uint64_t capacity, cp_unweight_result* out)
{
  CP_CHECK_HANDLE(h);
  if (n_points < 2) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: n_points < 2");
  if (capacity && !records_dev) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: null records");
  if (((uintptr_t)records_dev & 15) != 0) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: records must be 16-byte aligned");
  double wm[2];
  CP_CUDA(h, cudaMemcpyAsync(wm, h->d_wmax, sizeof wm, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!(wm[0] > 0)) return cp_fail(h, CP_ERR_INVALID, "cp_unweight: no threshold (cp_weight_quantile or cp_set_wmax)");
  CP_CUDA(h, cudaMemsetAsync(h->d_counter, 0, sizeof(unsigned long long), h->stream));
  if (h->scalew && capacity > h->scalew_cap)
    return cp_fail(h, CP_ERR_INVALID, "cp_unweight: record capacity exceeds the scale-weight buffer (cp_set_scale_weights)");
  int rc = unweight_enqueue(h, 0, n_points, iter, records_dev, capacity, h->d_red, h->scalew);
  if (rc) return rc;
  double red[8];
  unsigned long long cnt = 0;
  CP_CUDA(h, cudaMemcpyAsync(red, h->d_red, sizeof red, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaMemcpyAsync(&cnt, h->d_counter, sizeof cnt, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (h->flow_on && (rc = cp_flow_tc_status(h)) != CP_OK) return rc;
  if (out) fill_unw(red, (double)n_points, wm[0], out);
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
  double wm[2];
  CP_CUDA(h, cudaMemcpyAsync(wm, h->d_wmax, sizeof wm, cudaMemcpyDeviceToHost, h->stream));
  CP_CUDA(h, cudaStreamSynchronize(h->stream));
  if (!(wm[0] > 0)) return cp_fail(h, CP_ERR_INVALID, "cp_generate_host: no threshold");
  if (chunk > n_points) chunk = n_points;
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
      unsigned long long* saved = h->d_counter;
      h->d_counter = h->d_gen_cnt + c;
      rc = unweight_enqueue(h, p0, n, iter, h->d_gen_stage + (uint64_t)b * chunk, chunk, h->d_gen_red + 8 * c);
      h->d_counter = saved;
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
  double tot[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (uint64_t c = 0; c < nchunks; ++c)
    for (int k = 0; k < 8; ++k) tot[k] = (k == 2) ? (hred[8 * c + k] > tot[k] ? hred[8 * c + k] : tot[k]) : tot[k] + hred[8 * c + k];
  if (out) fill_unw(tot, (double)n_points, wm[0], out);
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
// the accept kernel and the record builder (plus the tiny slot reduction) on the handle's stream
// and accumulates their durations; cp_kernel_times reads and optionally resets them.
extern "C" int cp_set_kernel_timing(cp_handle* h, int on)
{
  CP_CHECK_HANDLE(h);
  if (on && !h->tev[0])
    for (int k = 0; k < 4; ++k) CP_CUDA(h, cudaEventCreate(&h->tev[k]));
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
