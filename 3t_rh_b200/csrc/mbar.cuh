// Shared-memory mbarriers (PTX mbarrier.*) with bounded waits, used by the
// ghost update (bulk-copy completion) and the interface fluxes (the hand-off
// of staged tiles between warps). Every wait gives up after a fixed number of
// try_wait rounds and returns false; the caller then records a timeout in the
// instance's error key and leaves its loop, so no warp waits without end.
#pragma once
#include <cstdint>

namespace rh3t {

constexpr int MBAR_WAIT_LIMIT = 1 << 18; // try_wait rounds (about a second) before a wait counts as timed out
constexpr int MBAR_TIMEOUT_CODE = 11;    // RH3T_ERR_DEVICE_TIMEOUT

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// one thread; `count` arrivals complete a phase
__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// after the initialising thread's mbar_init calls, before the block's barrier
__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// one arrival (release: this thread's earlier shared-memory writes are seen
// by a thread whose wait observes the phase's completion)
__device__ __forceinline__ void mbar_arrive(unsigned long long* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// bounded wait (acquire) for the completion of the phase with parity `parity`
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity) {
    const uint32_t a = smem_u32(bar);
    for (int it = 0; it < MBAR_WAIT_LIMIT; ++it) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

} // namespace rh3t
