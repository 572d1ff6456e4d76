// async_copy.cuh -- mbarrier, bulk-copy (TMA engine, no multicast) and bounded-wait helpers shared by
// the blind-rotation and keyswitch kernels (sm_100a inline PTX).
#pragma once
#include <stdint.h>

namespace tfheb {

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Non-blocking test of a phase (never suspends the thread)
__device__ __forceinline__ bool mbar_test_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Same test, but a thread whose phase is not complete may sleep in hardware for up to hint_ns
// nanoseconds; it is woken as soon as the phase completes, so the hint bounds the polling rate,
// not the latency.
__device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t bar, uint32_t parity, uint32_t hint_ns) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// bulk global -> shared copy completing on an mbarrier (size multiple of 16, 16-byte aligned ends)
__device__ __forceinline__ void bulk_copy_g2s(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// Longest hardware sleep of one polling round of a bounded wait (50 us: far below every timeout, so
// an abort raised by another thread is seen promptly).
constexpr uint32_t kWaitSleepNs = 50000;

// Bounded wait: true when the phase completed, false on timeout or when the CTA already aborted.
// The thread whose wait runs out raises the CTA's abort flag and the launch's error word.
__device__ __forceinline__ bool wait_bounded(uint32_t bar, uint32_t parity, volatile int32_t *abort_flag,
                                             uint64_t timeout_ns, int32_t *err) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (;;) {
        if (*abort_flag) return false;
        if (mbar_try_wait_sleep(bar, parity, kWaitSleepNs)) return true;
        if (global_timer_ns() - t0 > timeout_ns) {
            *abort_flag = 1;
            atomicOr(err, 1);
            return false;
        }
    }
}

}  // namespace tfheb
