// Asynchronous bulk copies between global and shared memory (sm_90+ PTX
// cp.async.bulk, no tensor map, no multicast) with mbarrier completion, and
// the engine's device error word.
//
// Every wait on an mbarrier is bounded: after WAIT_CYCLES the waiting thread
// records KERR_WAIT_TIMEOUT in g_kerr and gives up, so a kernel can never spin
// forever.  The host reads and clears g_kerr in lfts_synchronize.
#pragma once
#include <cstdint>

namespace lfts {

enum : unsigned { KERR_WAIT_TIMEOUT = 1u, KERR_MISALIGNED = 2u };

// set by kernels, read and cleared by the host (one translation unit includes this)
static __device__ unsigned int g_kerr;

constexpr long long WAIT_CYCLES = 4000000000LL;  // ~2 s at the 1.965 GHz boost clock

__device__ __forceinline__ void kerr_set(unsigned code) { atomicOr(&g_kerr, code); }

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
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

// Wait for the phase with the given parity to complete; false (and the error
// word set) when it has not completed after WAIT_CYCLES.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > WAIT_CYCLES) {
            kerr_set(KERR_WAIT_TIMEOUT);
            return false;
        }
    }
    return true;
}

// global -> shared, completion counted in bytes on bar (16-byte aligned, size % 16 == 0)
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst_smem)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// shared -> global in the calling thread's bulk group
__device__ __forceinline__ void bulk_store(void *dst, const void *src_smem, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_addr(src_smem)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// the shared-memory sources of this thread's committed bulk stores have been read
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// make this thread's generic-proxy shared-memory writes visible to bulk copies
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

}  // namespace lfts
