// Bulk asynchronous copies from global to shared memory (cp.async.bulk, completion
// counted in bytes on an mbarrier) and bounded mbarrier waits.
//
// Every wait is bounded: if a copy has not landed after the limit, the waiter records
// the fault in the flag it is given, waits once more, and carries on (results are then
// wrong, but the kernel ends and the host can read the flag through
// vfhe_cuda_device_faults).
#pragma once
#include <stdint.h>

namespace vc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// global -> shared, `bytes` (multiple of 16, both addresses 16-byte aligned)
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

static __device__ __noinline__ void mbar_wait_slow(uint64_t* bar, uint32_t parity, int* fault) {
    for (int round = 0; round < 2; ++round) {
        for (int i = 0; i < (1 << 18); ++i)
            if (mbar_try_wait(bar, parity)) return;
        if (round == 0) atomicExch(fault, 1);
    }
}

// One inline attempt; the bounded retry loop is out of line so that it does not
// shape the caller's register allocation.
__device__ __forceinline__ void mbar_wait_bounded(uint64_t* bar, uint32_t parity, int* fault) {
    if (!mbar_try_wait(bar, parity)) mbar_wait_slow(bar, parity, fault);
}

// Orders this CTA's earlier generic accesses to shared memory before later async-proxy
// writes (a bulk copy refilling a buffer the threads have just read).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

}  // namespace vc
