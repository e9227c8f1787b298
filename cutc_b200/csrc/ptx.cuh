// ptx.cuh -- small sm_100a PTX helpers shared by the kernels: shared-memory
// addresses, mbarriers with a bounded wait, and the bulk (non-tensor) async
// copy from global to shared memory that completes on an mbarrier.
//
// Every wait here is bounded (about 2 s of %globaltimer); a caller that sees
// it expire records an error flag the host reads, waits again (bounded) for
// its own copies in flight and returns.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ctc {
namespace px {

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
    // make the initialised barrier visible to the async proxy
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arrive once and expect `bytes` of async-copy completions in this phase
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *mbar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar_addr, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t"
        ".reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t"
        "}\n"
        : "=r"(done)
        : "r"(mbar_addr), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait: gives up after limit_ns of globaltimer (~2 s by default)
// and reports false.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar_addr, uint32_t parity,
                                                  uint64_t limit_ns = 2000000000ull)
{
    uint64_t t0;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
    for (uint32_t it = 0;; ++it) {
        if (mbar_try_wait(mbar_addr, parity)) return true;
        if ((it & 1023u) == 1023u) {
            uint64_t t1;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t1));
            if (t1 - t0 > limit_ns) return false;
        }
    }
}

// Bulk copy of `bytes` (a multiple of 16; both addresses 16-byte aligned)
// from global to this CTA's shared memory, counted on `mbar`.  No
// multicast: the destination is the issuing CTA's own shared memory.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *mbar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(mbar))
                 : "memory");
}

// Bulk reduction of `bytes` FP32 values from this CTA's shared memory into
// global memory (dst += src, element-wise), tracked in the issuing thread's
// bulk async-group.  Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_reduce_add_f32(float *dst, const float *src, uint32_t bytes)
{
    asm volatile("cp.reduce.async.bulk.global.shared::cta.bulk_group.add.f32 [%0], [%1], %2;" ::"l"(dst),
                 "r"(smem_u32(src)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the issuing thread's bulk groups: all but the newest N have read their
// shared-memory sources
template <int N>
__device__ __forceinline__ void bulk_wait_read()
{
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}
// ... and have completed
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// generic-proxy writes to shared memory become visible to the async proxy
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace px
}  // namespace ctc
