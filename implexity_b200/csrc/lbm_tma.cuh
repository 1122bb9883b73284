// lbm_tma.cuh -- bulk asynchronous copies (cp.async.bulk, global -> shared)
// completed through an mbarrier, for the staged tiles of the stepping
// kernels.  sm_90+ PTX; the kernels here are compiled for sm_100a only.
//
// Every wait is bounded in time: after kWaitNs of the global timer the
// waiting thread records the failure in a device flag (the host turns it into
// LBM_E_CUDA) and keeps waiting for a second bounded period so that no copy is
// left in flight into shared memory when the block exits.  Each poll asks the
// hardware to suspend the thread until the phase completes (suspend-time
// hint), so waiting warps leave the issue slots to the computing ones instead
// of spinning.
#pragma once

#include <cstdint>

namespace lbm {

constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s per bounded period
constexpr uint32_t kSuspendHintNs = 10000000u;  // per poll; the thread wakes when the phase completes

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arrive once and announce `bytes` of transactions for the current phase.
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Plain arrival (count 1) on the current phase.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity), "r"(kSuspendHintNs)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Polls until the phase completes or limit_ns have passed since t0.
__device__ __forceinline__ bool mbar_poll_until(uint64_t* bar, uint32_t parity, uint64_t t0, uint64_t limit_ns) {
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Bounded wait for the phase with the given parity.  Returns false (and sets
// *err) if the copies did not land within the limit.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint64_t limit_ns = kWaitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    if (mbar_poll_until(bar, parity, global_ns(), limit_ns)) return true;
    if (err) atomicOr(err, 1);
    mbar_poll_until(bar, parity, global_ns(), limit_ns);
    return false;
}

// One bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned)
// from global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// One bulk copy of `bytes` (multiple of 16, both addresses 16-byte aligned)
// from this CTA's shared memory to global memory, tracked by the issuing
// thread's bulk groups.
__device__ __forceinline__ void bulk_s2g(void* dst, const void* src, uint32_t bytes) {
    asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
                 "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until every committed bulk store of this thread has read its source.
__device__ __forceinline__ void bulk_wait_read0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
// Waits until every committed bulk store of this thread has completed.
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
// Orders this thread's generic-proxy shared-memory writes before later
// async-proxy (bulk copy) reads of them.
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

}  // namespace lbm
