// Blackwell bulk-copy (TMA, non-tensor) staging helpers: global -> shared
// copies completed on an mbarrier with a transaction count.  Every wait is
// bounded: after WAIT_LIMIT failed probes the caller records a timeout in the
// device error word and leaves, instead of spinning forever.
#pragma once
#include <stdint.h>

namespace ncg {

constexpr int WAIT_LIMIT = 1 << 20;

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
      return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
      asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async_smem()
{
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arrive (count 1) and announce `bytes` of incoming transactions.
__device__ __forceinline__ void mbar_arrive_expect(uint64_t *bar, unsigned bytes)
{
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                   "r"(bytes)
                   : "memory");
}

// 1-D bulk copy global -> this CTA's shared memory.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(dst)),
          "l"(src), "r"(bytes), "r"(smem_u32(bar))
          : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
      unsigned ok;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(ok)
          : "r"(smem_u32(bar)), "r"(parity)
          : "memory");
      return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, unsigned parity)
{
      for (int it = 0; it < WAIT_LIMIT; ++it)
            if (mbar_try_wait(bar, parity)) return true;
      return false;
}

}  // namespace ncg
