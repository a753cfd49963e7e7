// Bulk (TMA) copies global -> shared memory with mbarrier completion, sm_90+ PTX.
// Plain 1D bulk copies only: no tensor maps, no cluster multicast.
#pragma once
#include <stdint.h>

namespace rt {

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive on the barrier and announce `bytes` of transactions for the current phase.
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Order earlier generic-proxy accesses of this thread before later async-proxy accesses.
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Copy `bytes` (multiple of 16; both addresses 16-byte aligned) from global to shared memory.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// Bounded wait for the completion of phase `parity` of the barrier. Returns false when the
// limit is reached (the caller records an error instead of hanging).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit = 1ll << 26)
{
    const uint32_t a = smem_u32(bar);
    for (long long it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Stage `nfloats` floats starting at global address `src` into shared memory at `dst`
// (16-byte aligned), as whole 16-byte units: the data lands at dst + returned offset
// (0..3 floats). Reads up to 12 bytes before `src` and after its end: the source allocation
// must be padded accordingly. Called by one thread; returns the offset in floats.
__device__ __forceinline__ int stage_rows_async(float* dst, const float* src, size_t nfloats,
                                                uint64_t* bar)
{
    const uintptr_t a = reinterpret_cast<uintptr_t>(src);
    const uintptr_t a0 = a & ~uintptr_t(15);
    const uintptr_t e1 = (a + nfloats * sizeof(float) + 15) & ~uintptr_t(15);
    const uint32_t total = (uint32_t)(e1 - a0);
    fence_proxy_async_smem();
    mbar_arrive_expect_tx(bar, total);
    constexpr uint32_t kChunk = 32768;
    for (uint32_t off = 0; off < total; off += kChunk) {
        const uint32_t n = total - off < kChunk ? total - off : kChunk;
        bulk_g2s(reinterpret_cast<unsigned char*>(dst) + off,
                 reinterpret_cast<const unsigned char*>(a0) + off, n, bar);
    }
    return (int)((a - a0) / sizeof(float));
}

}  // namespace rt
