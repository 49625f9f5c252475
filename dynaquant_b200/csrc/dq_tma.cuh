// dq_tma.cuh — TMA tensor loads and mbarrier waits (inline PTX, sm_100a).
//
// Every wait is bounded: after its budget (kWaitCycles SM cycles unless a
// test lowered it) the caller gets false and must record DQ_ERR_TIMEOUT, let
// its own copies in flight land (waits with the full kWaitCycles budget) and
// leave; nothing here spins forever.
// No multicast form is used: every load reads this GPU's own memory into
// the issuing CTA's shared memory.
#pragma once
#include <cuda.h>
#include <cstdint>

namespace dq {

constexpr long long kWaitCycles = 4000000000LL;   // ~2 s at 2 GHz

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// makes the barrier initialisation visible to the async (TMA) proxy
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Non-blocking test of the phase with the given parity.
__device__ __forceinline__ bool mbar_test_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Budgets below this many cycles are shorter than one suspended try_wait may
// take, so they poll with test_wait instead and end on the cycle count.
constexpr long long kPollBudget = 1LL << 20;

// Bounded wait for the phase with the given parity; false once `budget` SM
// cycles have passed without it.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long budget = kWaitCycles) {
    const long long t0 = clock64();
    if (budget < kPollBudget) {
        while (!mbar_test_wait(bar, parity)) {
            if (clock64() - t0 > budget) return false;
        }
        return true;
    }
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > budget) return false;
    }
    return true;
}

// 2-D tiled TMA load of one box into shared memory, completing on `bar`.
// The innermost coordinate x must be a multiple of 16 bytes.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace dq
