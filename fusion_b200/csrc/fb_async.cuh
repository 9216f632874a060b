// Asynchronous bulk copies into shared memory (sm_90+ bulk-copy engine, the
// untiled `cp.async.bulk` form) completed through shared-memory mbarriers,
// as inline PTX.  Only this GPU's own global memory is ever a source, and no
// copy uses cluster multicast.
//
// Waits are bounded: mbar_wait gives up after kMbarPolls polls of
// `mbarrier.try_wait` (each poll may suspend the thread for a short,
// hardware-defined time) and returns false, so a kernel can record the
// failure and end instead of hanging.
#ifndef FB_ASYNC_CUH
#define FB_ASYNC_CUH

#include <stdint.h>

namespace fb {

constexpr int kMbarPolls = 1 << 22;

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Initialise an mbarrier expecting `count` arrivals per phase, and make the
// initialisation visible to the bulk-copy engine.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces `bytes` of transaction to come.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// One arrival without transaction bytes.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Wait for the phase of parity `parity` to complete; false after kMbarPolls
// polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const uint32_t a = smem_addr(bar);
    for (int i = 0; i < kMbarPolls; ++i) {
        uint32_t done;
        asm volatile(
            "{\n"
            ".reg .pred p;\n"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n"
            "}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// `bytes` (a multiple of 16; both addresses 16-byte aligned) from global
// memory of this GPU into this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Orders this thread's earlier shared-memory accesses (generic proxy) before
// later bulk copies into the same memory (async proxy).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace fb

#endif
