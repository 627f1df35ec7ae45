// twi_ptx.cuh -- thin inline-PTX wrappers for the sm_100a features the
// propagator uses: shared-memory mbarriers and TMA tiled tensor loads
// (cp.async.bulk.tensor, no multicast anywhere in this library).
#pragma once

#include <cstdint>
#include <cuda.h>

namespace twi {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
                 : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_barrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// One bounded probe of the barrier phase.  Returns true once the phase with
// parity `parity` has completed.
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Wait at most `limit_ns` of wall time (checked every 256 probes, with a
// probe count as a second bound in case the timer does not advance);
// returns false if the phase never completes.
__device__ __forceinline__ bool mbar_wait_for(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    constexpr uint32_t kMaxProbes = 1u << 26;
    const uint64_t t0 = globaltimer_ns();
    for (uint32_t i = 0; i < kMaxProbes; ++i) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 255u) == 255u && globaltimer_ns() - t0 > limit_ns) return false;
    }
    return false;
}

// The step kernels' wait: a copy of a few tens of KB lands in microseconds,
// so two seconds only runs out when something is broken; the caller then
// raises the device error word, drains its other copies and leaves.
constexpr uint64_t kWaitLimitNs = 2000000000ull;
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    return mbar_wait_for(bar, parity, kWaitLimitNs);
}

// After a wait ran out: wait, bounded again, for the stage copies of shots
// [first, last) that this CTA issued (stage barrier j % stages, phase
// (j / stages) & 1), so that none lands in shared memory the CTA gave back.
__device__ __forceinline__ void drain_stages(uint64_t* stage_bars, int stages, int first, int last) {
    for (int j = first; j < last; ++j)
        mbar_wait_for(&stage_bars[j % stages], (uint32_t)((j / stages) & 1), kWaitLimitNs);
}

// Bring the 128-byte line holding `p` into L2 (no register result).
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.L2 [%0];" ::"l"(reinterpret_cast<uint64_t>(p)) : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* tm) {
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(tm)) : "memory");
}

// 2-D and 3-D tiled TMA loads global -> shared, completing on `bar`.  The
// innermost coordinate x must be a multiple of 4 floats (16 bytes); the
// callers only ever pass tile origins that are multiples of 4 columns.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* tm, int x, int y, int z,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

}  // namespace twi
