// cp_tc.cuh -- thin inline-PTX wrappers for the 5th-generation tensor cores (tcgen05: TMEM
// allocation, MMA with shared-memory descriptors, commit to an mbarrier, TMEM loads) and the
// mbarrier / named-barrier primitives around them.  sm_100a only.
//
// Operand layout used throughout: K-major, no swizzle ("interleaved" canonical layout).  A tile
// of R rows x K bf16 columns is stored as core matrices of 8 rows x 16 bytes (8 bf16), row r of
// k-block kb at byte  kb * (R / 8) * 128 + (r / 8) * 128 + (r % 8) * 16.  In a descriptor the
// stride-dimension offset (SBO) is 128 bytes (next 8 rows) and the leading-dimension offset (LBO)
// is (R / 8) * 128 bytes (next 8 columns of K); one MMA of K = 16 covers two k-blocks.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
__device__ __forceinline__ uint32_t cp_smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// shared-memory matrix descriptor: start address, LBO, SBO (bytes, multiples of 16), version 1,
// base offset 0, no swizzle
__device__ __forceinline__ uint64_t cp_tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
  return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
         (1ull << 46);
}

// instruction descriptor of kind::f16: D F32, A and B BF16, both K-major, M = 128, N = n
__host__ __device__ constexpr uint32_t cp_tc_idesc_bf16(int n)
{
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void cp_tc_alloc(uint32_t dst_smem, uint32_t ncols)
{
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(dst_smem), "r"(ncols) : "memory");
}
__device__ __forceinline__ void cp_tc_relinquish()
{
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void cp_tc_dealloc(uint32_t taddr, uint32_t ncols)
{
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void cp_tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void cp_tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes become visible to the tensor core's (async proxy) reads
__device__ __forceinline__ void cp_fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread
__device__ __forceinline__ void cp_tc_mma(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// D[tmem] (+)= A[tmem] * B[smem]^T, issued by one thread.  A in tensor memory: row r in lane r,
// BF16 element k of the row in the low (k even) or high (k odd) half of column k / 2.
__device__ __forceinline__ void cp_tc_mma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc, uint32_t accumulate)
{
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}
// the mbarrier receives one arrival when every tcgen05 operation this thread issued has completed
__device__ __forceinline__ void cp_tc_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane, waited for in the same statement so
// that no use of the registers can be scheduled before the load has landed
__device__ __forceinline__ void cp_tc_ld32(uint32_t taddr, float (&v)[32])
{
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
      "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
        "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
        "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
}
__device__ __forceinline__ void cp_tc_ld4(uint32_t taddr, float (&v)[4])
{
  uint32_t r[4];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n\t"
      "tcgen05.wait::ld.sync.aligned;\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int j = 0; j < 4; ++j) v[j] = __uint_as_float(r[j]);
}

// 16 consecutive 32-bit columns of this thread's TMEM lane from registers (not waited for)
__device__ __forceinline__ void cp_tc_st16(uint32_t taddr, const uint32_t (&r)[16])
{
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
      "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(taddr),
      "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]),
      "r"(r[8]), "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
      : "memory");
}
// every tcgen05.st of this thread has completed
__device__ __forceinline__ void cp_tc_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// relu, round to BF16 and pack: low half from lo, high half from hi
__device__ __forceinline__ uint32_t cp_relu_bf2(float lo, float hi)
{
  uint32_t d;
  asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(d) : "f"(hi), "f"(lo));
  return d;
}

__device__ __forceinline__ void cp_sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d)
{
  asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ void cp_mbar_init(uint32_t mbar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(mbar), "r"(count) : "memory");
}
__device__ __forceinline__ void cp_mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void cp_mbar_arrive(uint32_t mbar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(mbar) : "memory");
}
// non-blocking test of the phase `parity` of an mbarrier
__device__ __forceinline__ bool cp_mbar_test(uint32_t mbar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for the phase `parity` of an mbarrier (try_wait suspends the thread in hardware
// until the phase completes or a short time limit): gives up after CP_TC_WAIT_CYCLES clock cycles
// (about 1 s) or when *abort (shared, per warpgroup) is set by another thread that gave up; on
// giving up it sets *abort and returns false.
#define CP_TC_WAIT_CYCLES (1ll << 31)
__device__ __forceinline__ bool cp_mbar_try(uint32_t mbar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}\n"
      : "=r"(ok)
      : "r"(mbar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool cp_mbar_wait_bounded(uint32_t mbar, uint32_t parity, volatile int* abort)
{
  if (cp_mbar_try(mbar, parity)) return true;
  const long long t0 = clock64();
  for (uint32_t i = 0;; ++i) {
    if (cp_mbar_try(mbar, parity)) return true;
    if (*abort) return false;
    if (clock64() - t0 > CP_TC_WAIT_CYCLES || i > (1u << 28)) {
      *abort = 1;
      return false;
    }
  }
}

// named barrier over the 128 threads of one warpgroup
__device__ __forceinline__ void cp_bar_wg(uint32_t id)
{
  asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory");
}
// the same barrier with an OR-reduction of a predicate over the warpgroup
__device__ __forceinline__ bool cp_bar_wg_or(uint32_t id, bool v)
{
  uint32_t out;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %2, 0;\n\t"
      "bar.red.or.pred q, %1, 128, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(out)
      : "r"(id), "r"((uint32_t)v)
      : "memory");
  return out != 0;
}
#endif
