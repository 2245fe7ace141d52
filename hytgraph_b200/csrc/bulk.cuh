// Bulk-copy staging primitives (sm_90+ / sm_100a): cp.async.bulk global ->
// shared memory completed on an mbarrier transaction count, as used by the
// per-warp staging pipelines of the pull kernels.  Every wait is bounded by
// a clock budget; a wait that runs out reports failure to its caller, which
// sets the solve's error flag and leaves the kernel.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hyt::bulk {

#ifdef __CUDACC__

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// One arrival (the issuing lane's expect_tx) completes a phase once the
// expected bytes have landed.
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
}

// Makes barrier initialisation visible to the asynchronous (bulk-copy) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy accesses to shared memory
// before later bulk copies into it (a slot is rewritten by the next copy).
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// The arrival of the issuing lane, announcing `bytes` of copies to come
// (0: the phase completes at once).
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Copies `bytes` (a multiple of 16; both addresses 16-byte aligned) from
// this GPU's global memory into shared memory, streamed with an L2 cache
// policy; completion is counted on `bar`.
__device__ __forceinline__ void copy_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar, uint64_t pol) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
        : "memory");
}

__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Waits for the phase with the given parity, letting the hardware suspend
// the thread for up to kSuspendNs while the phase is incomplete (a parked
// warp leaves its issue slots to the others); true once the phase is done.
constexpr uint32_t kSuspendNs = 1000000;

__device__ __forceinline__ bool mbar_test_parity(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(kSuspendNs)
        : "memory");
    return ok != 0;
}

// Clock budget of one wait: about a second at B200 clocks, far beyond the
// microseconds a staged copy takes.
constexpr long long kWaitCycles = 2000000000ll;

// Waits for the phase of `bar` with the given parity to complete; false
// when the budget ran out.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    if (mbar_test_parity(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test_parity(bar, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

#endif  // __CUDACC__

}  // namespace hyt::bulk
