// Bulk copies global -> shared memory through the tensor memory accelerator
// (cp.async.bulk, completion counted on a shared-memory mbarrier), for the
// level passes: a tile of object records is contiguous in global memory, so
// one thread moves it into shared memory with a few instructions and the CTA
// keeps tens of kilobytes in flight without holding them in registers.
//
// Source and destination must be 16-byte aligned and sizes multiples of 16
// bytes (a record is 32 bytes, record arrays are 256-byte aligned). No
// multicast: every copy lands in the issuing CTA's own shared memory.
#pragma once
#include <cstdint>

namespace mgbvh {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One arrival (the issuing thread's expect_tx) completes a phase together
// with the bytes it announced.
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t arrivals) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(arrivals) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for phase `parity` of the barrier; false if it has not completed
// after `limit` polls (each poll may suspend the thread for a short
// hardware-defined time). A bulk copy of valid global memory into the
// CTA's own shared memory depends on no other CTA, so the limit is only a
// guard against a copy that never lands.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

}  // namespace mgbvh
