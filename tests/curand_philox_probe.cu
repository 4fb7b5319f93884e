// Test helper: Philox-4x32-10 words of cuRAND's device implementation (curand_Philox4x32_10 from
// curand_philox4x32_x.h) for key = (seed lo, seed hi) and counter = (point lo, point hi,
// iteration, stream), points point0 .. point0 + n - 1.  Prints one line of four hex words per point.
//   usage: curand_philox_probe <seed> <point0> <n> <iteration> <stream>
#include <cstdio>
#include <cstdlib>
#include <cstdint>
#include <vector>
#include <curand_kernel.h>

__global__ void k_words(uint64_t seed, uint64_t point0, int n, uint32_t iter, uint32_t stream, uint4* out)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t p = point0 + (uint64_t)i;
  const uint4 c = make_uint4((uint32_t)p, (uint32_t)(p >> 32), iter, stream);
  const uint2 k = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
  out[i] = curand_Philox4x32_10(c, k);
}

int main(int argc, char** argv)
{
  if (argc < 6) return 2;
  const uint64_t seed = strtoull(argv[1], nullptr, 0), point0 = strtoull(argv[2], nullptr, 0);
  const int n = atoi(argv[3]);
  const uint32_t iter = (uint32_t)strtoul(argv[4], nullptr, 0), stream = (uint32_t)strtoul(argv[5], nullptr, 0);
  if (n < 1 || n > (1 << 20)) return 2;
  uint4* d = nullptr;
  if (cudaMalloc(&d, sizeof(uint4) * n) != cudaSuccess) return 1;
  k_words<<<(n + 255) / 256, 256>>>(seed, point0, n, iter, stream, d);
  std::vector<uint4> h(n);
  if (cudaMemcpy(h.data(), d, sizeof(uint4) * n, cudaMemcpyDeviceToHost) != cudaSuccess) return 1;
  for (int i = 0; i < n; ++i) printf("%08x %08x %08x %08x\n", h[i].x, h[i].y, h[i].z, h[i].w);
  cudaFree(d);
  return 0;
}
