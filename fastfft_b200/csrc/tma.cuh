// TMA bulk copies (cp.async.bulk, no multicast) with mbarrier completion and bounded
// waits, used by the fused column kernel to stage whole columns in shared memory.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ffb {

constexpr int kErrTimeout = 1;
// Bounds of a barrier wait: 200 ms of %globaltimer, or this many polls, whichever ends first.
constexpr unsigned long long kWaitNs = 200ull * 1000 * 1000;
constexpr long long kWaitLimit = 1ll << 24;

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}

// Bulk global -> shared copy of `bytes` (multiple of 16; both addresses 16-byte aligned),
// completion counted on `bar`.  No multicast.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// Polls the barrier phase; returns false if it did not complete within the bounds.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
    const uint32_t a = smem_addr(bar);
    const unsigned long long t0 = global_ns();
    for (long long i = 0; i < kWaitLimit; i++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(done)
            : "r"(a), "r"(phase)
            : "memory");
        if (done) return true;
        if ((i & 1023) == 1023 && global_ns() - t0 > kWaitNs) return false;
    }
    return false;
}

// Block-uniform staging: thread 0 initialises `bar`, the caller's `issue` lambda (run by
// thread 0) starts the bulk copies for `bytes` in total, and thread 0 waits with the
// bounds.  Every thread then learns the outcome at the same barrier, so a timed-out block
// leaves as a whole (no thread is left waiting at a later __syncthreads); on success each
// thread also observes the completed phase itself (acquire).  On timeout *err is set and
// thread 0 gives the copies one more bounded wait before the block exits.
template <class Issue>
__device__ __forceinline__ bool stage_block(uint64_t* bar, int* ok_flag, uint32_t bytes, int* err, Issue issue) {
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_barrier_init();
        mbar_arrive_expect_tx(bar, bytes);
        issue();
        const bool ok = mbar_wait(bar, 0);
        *ok_flag = ok ? 1 : 0;
        if (!ok) {
            if (err) atomicExch(err, kErrTimeout);
            mbar_wait(bar, 0);
        }
    }
    __syncthreads();
    if (!*ok_flag) return false;
    mbar_wait(bar, 0);
    return true;
}

}  // namespace ffb
