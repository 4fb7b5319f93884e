// cp_peak.cu -- FP32 and MUFU throughput microbenchmarks of the device, the denominators of the
// integrand's roofline (the integrand is SIMT FP32 / SFU work, neither HBM- nor tensor-bound).
#include "cp_internal.cuh"

// 8 independent FMA chains per thread: the FMA pipe, not latency, is the limit.
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b)
{
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = threadIdx.x * 1e-3f + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = fmaf(r[k], a, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 1234.5f) out[0] = s;   // keeps the chains alive
}

// 8 independent ex2.approx chains per thread (one MUFU op each)
__global__ void __launch_bounds__(256) k_mufu_peak(float* out, int iters)
{
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = -1e-3f * (threadIdx.x + k);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = exp2f(r[k]) - 1.0f;   // ex2 stays in (-1, 0]
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += r[k];
  if (s == 1234.5f) out[0] = s;
}

extern "C" int cp_measure_peaks(cp_handle* h, double* fp32_tflops, double* mufu_tops)
{
  CP_CHECK_HANDLE(h);
  float* d = nullptr;
  cudaEvent_t e0, e1;
  CP_CUDA(h, cudaMalloc(&d, sizeof(float)));
  CP_CUDA(h, cudaEventCreate(&e0));
  CP_CUDA(h, cudaEventCreate(&e1));
  const int blocks = h->num_sms * 8, threads = 256, iters = 4096;
  float best_f = 1e30f, best_m = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    float ms;
    cudaEventRecord(e0, h->stream);
    k_fma_peak<<<blocks, threads, 0, h->stream>>>(d, iters, 0.9999f, 1e-4f);
    cudaEventRecord(e1, h->stream);
    CP_CUDA(h, cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_f) best_f = ms;
    cudaEventRecord(e0, h->stream);
    k_mufu_peak<<<blocks, threads, 0, h->stream>>>(d, iters / 4);
    cudaEventRecord(e1, h->stream);
    CP_CUDA(h, cudaEventSynchronize(e1));
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && ms < best_m) best_m = ms;
  }
  CP_LAUNCH_CHECK(h, "k_peak");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  const double nthr = (double)blocks * threads;
  if (fp32_tflops) *fp32_tflops = nthr * iters * 8 * 2.0 / (best_f * 1e-3) / 1e12;
  if (mufu_tops) *mufu_tops = nthr * (iters / 4) * 8 / (best_m * 1e-3) / 1e12;
  return CP_OK;
}
