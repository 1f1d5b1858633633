// TMA (cp.async.bulk.tensor) and mbarrier helpers for sm_100a.
//
// Loads are plain tiled loads into this CTA's shared memory; no multicast
// form is used anywhere.  Every wait on an mbarrier is bounded: after
// XR_WAIT_LIMIT polls the wait gives up, records an error code in the
// device-wide error word and returns false, so a kernel can never spin
// forever on a transfer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace xr {

constexpr unsigned XR_DEVERR_TMA_TIMEOUT = 1u;

// Poll limits of the bounded waits, per device (xr_set_wait_limits).  After
// its first poll an mbarrier wait polls with a 1 us time hint, so the default
// gives up after roughly 0.02 to 1 s; a TMA box lands in microseconds.
constexpr long long XR_WAIT_LIMIT_DEFAULT = 1ll << 20;
__device__ long long g_wait_limit = XR_WAIT_LIMIT_DEFAULT;

// Test hooks (xr_test_hooks), zero in normal use.  Bit 0: TMA producers arm
// their barriers for a box but issue no copy, so every consumer wait runs out
// with nothing in flight.  Bit 1: the ragged kernel's grid barriers expect
// one block more than the grid, so every barrier wait runs out.
constexpr unsigned XR_HOOK_TMA_STALL = 1u;
constexpr unsigned XR_HOOK_BARRIER_EXTRA = 2u;
__device__ unsigned int g_test_hooks = 0;

__device__ __forceinline__ unsigned smem_u32(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// One poll.  Without a time hint it suspends the thread until the phase
// completes or a system-dependent limit passes; with one, for at most about
// `ns` nanoseconds.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity, unsigned ns) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(ns)
        : "memory");
    return ok != 0;
}

// The rest of a wait whose first poll failed: polls of at most about a
// microsecond up to the limit, giving up early once `abort` (a CTA-wide flag
// in shared memory, or null) is set.  A wait that runs out sets the device
// error word and `abort`.
__device__ __forceinline__ bool mbar_wait_slow(uint64_t* bar, unsigned parity, volatile int* abort) {
    const long long limit = *(volatile long long*)&g_wait_limit;
    for (long long i = 1; i < limit; ++i) {
        if (abort && *abort) return false;
        if (mbar_try_wait(bar, parity, 1000u)) return true;
    }
    atomicOr(&g_device_error, XR_DEVERR_TMA_TIMEOUT);
    if (abort) *abort = 1;
    return false;
}

// Bounded wait for phase `parity` of `bar`; false when it gives up.  The
// first poll is usually the whole wait; it takes no time hint (a hinted first
// poll made the helical projection 4 % slower) and reads nothing but the
// barrier.  Only a longer wait reads the poll limit.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, volatile int* abort = nullptr) {
    if (mbar_try_wait(bar, parity)) return true;
    return mbar_wait_slow(bar, parity, abort);
}

// 4D tiled TMA load of one box into shared memory, completing on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace xr
