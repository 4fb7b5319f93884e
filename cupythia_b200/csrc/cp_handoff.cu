// cp_handoff.cu -- device-resident hand-off of the 64-byte event records to the reference
// pipeline's structure-of-arrays event record (cuPythia/pipeline/event.cuh:20-31), the input of
// its downstream stages (shower, hadronisation: outside this library).
#include <cmath>
#include "cp_internal.cuh"

struct HandoffLaunch {
  const cp_event* rec;
  uint64_t n, e0, seed;
  const float* ratios;
  double sqrt_kf, inv_ebeam;
  cp_device_events ev;
  int* bad;
};

// VEC4: maxPart == 4 and every per-particle array 16-byte aligned, so an event's four entries of
// a member are one 16-byte store (int) or two (double) instead of four scalar stores
template <bool VEC4>
__global__ void __launch_bounds__(CP_THREADS) k_to_device_events(const HandoffLaunch L)
{
  const cp_device_events& ev = L.ev;
  for (uint64_t i = (uint64_t)blockIdx.x * CP_THREADS + threadIdx.x; i < L.n; i += (uint64_t)gridDim.x * CP_THREADS) {
    // the record as four 16-byte loads
    cp_event r;
    const uint4* src = reinterpret_cast<const uint4*>(L.rec + i);
    uint4* dst = reinterpret_cast<uint4*>(&r);
#pragma unroll
    for (int q = 0; q < 4; ++q) dst[q] = src[q];
    int col[4], acol[4];
    if (!cp_colour_expand(r.process, r.colour, col, acol)) {
      atomicOr(L.bad, 1);
      for (int k = 0; k < 4; ++k) col[k] = acol[k] = 0;
    }
    const uint64_t e = L.e0 + i;
    const size_t b = (size_t)e * ev.maxPart;
    const double pin[2] = {(double)r.pz_in[0], (double)r.pz_in[1]};
    const float* pout[2] = {r.p3, r.p4};
    if (VEC4) {
      // the same values as the scalar path below, member by member
      auto st_d = [&](double* base, double a, double bb, double c, double d) {
        double2* q = reinterpret_cast<double2*>(base + b);
        q[0] = make_double2(a, bb);
        q[1] = make_double2(c, d);
      };
      auto st_i = [&](int* base, int a, int bb, int c, int d) { *reinterpret_cast<int4*>(base + b) = make_int4(a, bb, c, d); };
      st_d(ev.px, 0.0, 0.0, (double)r.p3[0], (double)r.p4[0]);
      st_d(ev.py, 0.0, 0.0, (double)r.p3[1], (double)r.p4[1]);
      st_d(ev.pz, pin[0], pin[1], (double)r.p3[2], (double)r.p4[2]);
      st_d(ev.e, fabs(pin[0]), fabs(pin[1]), (double)r.p3[3], (double)r.p4[3]);
      st_d(ev.m, 0.0, 0.0, 0.0, 0.0);
      st_i(ev.pdg, r.id[0], r.id[1], r.id[2], r.id[3]);
      st_i(ev.status, -21, -21, 23, 23);
      st_i(ev.col, col[0] ? 500 + col[0] : 0, col[1] ? 500 + col[1] : 0, col[2] ? 500 + col[2] : 0,
           col[3] ? 500 + col[3] : 0);
      st_i(ev.acol, acol[0] ? 500 + acol[0] : 0, acol[1] ? 500 + acol[1] : 0, acol[2] ? 500 + acol[2] : 0,
           acol[3] ? 500 + acol[3] : 0);
      st_i(ev.mo1, -1, -1, 0, 0);
      st_i(ev.mo2, -1, -1, 1, 1);
      st_i(ev.d1, -1, -1, -1, -1);
      st_i(ev.d2, -1, -1, -1, -1);
    } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const size_t j = b + k;
      if (k < 2) {
        ev.px[j] = 0.0; ev.py[j] = 0.0; ev.pz[j] = pin[k]; ev.e[j] = fabs(pin[k]);
        ev.status[j] = -21; ev.mo1[j] = -1; ev.mo2[j] = -1;
      } else {
        const float* p = pout[k - 2];
        ev.px[j] = (double)p[0]; ev.py[j] = (double)p[1]; ev.pz[j] = (double)p[2]; ev.e[j] = (double)p[3];
        ev.status[j] = 23; ev.mo1[j] = 0; ev.mo2[j] = 1;
      }
      ev.m[j] = 0.0;
      ev.pdg[j] = r.id[k];
      ev.col[j] = col[k] ? 500 + col[k] : 0;
      ev.acol[j] = acol[k] ? 500 + acol[k] : 0;
      ev.d1[j] = -1; ev.d2[j] = -1;
    }
    }
    ev.nPart[e] = 4;
    ev.seed[e] = cp_splitmix64(L.seed ^ ((uint64_t)r.point * 0x9E3779B97F4A7C15ULL));
    ev.scale[e] = L.sqrt_kf * (double)r.pt_hat;
    ev.x1[e] = fabs(pin[0]) * L.inv_ebeam;
    ev.x2[e] = fabs(pin[1]) * L.inv_ebeam;
    ev.flavA[e] = r.id[0];
    ev.flavB[e] = r.id[1];
    ev.active[e] = 1;
    const size_t wb = (size_t)e * ev.nVar;
    ev.weight[wb] = (double)r.weight;
    for (int k = 1; k < ev.nVar; ++k) ev.weight[wb + k] = (double)r.weight * (double)L.ratios[6 * i + (k - 1)];
  }
}

extern "C" int cp_records_to_device_events(cp_handle* h, const cp_event* records_dev, uint64_t n,
                                           const float* scale_ratios_dev, const cp_device_events* ev, uint64_t e0)
{
  CP_CHECK_HANDLE(h);
  if (!ev) return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: null event structure");
  if (n == 0) return CP_OK;
  if (!records_dev || ((uintptr_t)records_dev & 15))
    return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: records must be 16-byte aligned device memory");
  if (ev->maxPart < 4 || ev->nVar < 1 || ev->nVar > 7 || (ev->nVar > 1 && !scale_ratios_dev))
    return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: need maxPart >= 4 and 1 <= nVar <= 7 "
                                      "(nVar > 1 needs the scale ratios)");
  if (ev->nEvents < 0 || e0 + n > (uint64_t)ev->nEvents)
    return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: events e0 .. e0 + n - 1 exceed nEvents");
  const void* ptrs[] = {ev->px, ev->py, ev->pz, ev->e, ev->m, ev->pdg, ev->status, ev->col, ev->acol, ev->mo1,
                        ev->mo2, ev->d1, ev->d2, ev->nPart, ev->seed, ev->scale, ev->x1, ev->x2, ev->flavA,
                        ev->flavB, ev->active, ev->weight};
  for (const void* p : ptrs)
    if (!p) return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: null member array");
  int* bad = nullptr;
  CP_CUDA(h, cudaMallocAsync(reinterpret_cast<void**>(&bad), sizeof(int), h->stream));
  CP_CUDA(h, cudaMemsetAsync(bad, 0, sizeof(int), h->stream));
  HandoffLaunch L;
  L.rec = records_dev; L.n = n; L.e0 = e0; L.seed = h->cfg.seed; L.ratios = scale_ratios_dev;
  L.sqrt_kf = sqrt(h->cfg.k_fac);
  L.inv_ebeam = 2.0 / h->cfg.sqrt_s;
  L.ev = *ev;
  L.bad = bad;
  const uint64_t want = (n + CP_THREADS - 1) / CP_THREADS;
  const unsigned blocks = (unsigned)(want < (uint64_t)h->num_sms * 8 ? want : (uint64_t)h->num_sms * 8);
  bool vec4 = ev->maxPart == 4;
  const void* part[] = {ev->px, ev->py, ev->pz, ev->e, ev->m, ev->pdg, ev->status, ev->col, ev->acol, ev->mo1,
                        ev->mo2, ev->d1, ev->d2};
  for (const void* p : part) vec4 = vec4 && ((uintptr_t)p & 15) == 0;
  if (vec4) k_to_device_events<true><<<blocks, CP_THREADS, 0, h->stream>>>(L);
  else k_to_device_events<false><<<blocks, CP_THREADS, 0, h->stream>>>(L);
  cudaError_t e = cudaGetLastError();
  int hb = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
  cudaFreeAsync(bad, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return cp_fail_cuda(h, e, "cp_records_to_device_events");
  if (hb) return cp_fail(h, CP_ERR_INVALID, "cp_records_to_device_events: a record's process code or colour flow is invalid");
  return CP_OK;
}
