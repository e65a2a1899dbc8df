// mbarrier and bulk-copy helpers shared by the TMA-staged kernels
// (inline PTX for sm_100a).  Every wait is bounded: after kWaitNs of wall
// clock it records AGAL_ERR_TIMEOUT in the caller's status word and returns
// false, so no kernel spins forever on a copy that never lands.  No multicast.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/agal_b200.h"

namespace agal {

static constexpr unsigned long long kWaitNs = 2000000000ull;   // 2 s

static __device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

static __device__ __forceinline__ unsigned long long now_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

static __device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

static __device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

static __device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

static __device__ __forceinline__ bool mbar_test(uint64_t *bar, unsigned parity)
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

// Bounded wait for the phase of the given parity to complete.
static __device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, int *status)
{
    if (mbar_test(bar, parity)) return true;
    const unsigned long long t0 = now_ns();
    while (true) {
        if (mbar_test(bar, parity)) return true;
        if (now_ns() - t0 > kWaitNs) {
            atomicExch(status, AGAL_ERR_TIMEOUT);
            return false;
        }
    }
}

// 1-D bulk copy global -> shared, completion counted on bar (no multicast).
static __device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

}  // namespace agal
