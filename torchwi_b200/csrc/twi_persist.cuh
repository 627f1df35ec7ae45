// twi_persist.cuh -- the work loop of persistent launches: one launch runs
// many time steps of one plan pass.
//
// Work items are (step, shot group, CTA of that group) in step-major order
// and are handed out by an atomic ticket, so a CTA only ever holds an item
// once it is running.  Before an item of step s runs, the CTA waits until
// every item of step s-1 of the same shot group has signalled completion on
// that group's counter (counters grow monotonically within a launch: step s
// may start once the counter reaches s * items_per_group).  Because an item
// waits only for items with smaller tickets, the earliest unfinished item
// always has everything it needs: the launch cannot deadlock, whatever the
// grid size and however many CTAs are resident.  Within a group the three
// rotating wavefield slots are safe: step s overwrites the slot of step
// s-3's output, which only steps s-2 and s-1 of the same group read, and
// those have finished.
//
// Every wait is bounded: after kWaitLimitNs without progress, or as soon as
// another CTA has raised the error word, the CTA raises bit 1 of the word
// and leaves; the launch then ends quickly and the host sees the error.
//
// Memory ordering: a finished item's stores are released (every thread
// fences, then one thread adds to the counter); the waiting thread acquires
// the counter and then fences between the generic and the async (TMA) proxy,
// so the tensor loads of the next item see the data; the CTA barrier that
// follows orders the other threads' plain loads after the acquire.
#pragma once

#include <cstdint>
#include <utility>

#include "twi_kernels.h"
#include "twi_ptx.cuh"

namespace twi {

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ int ld_volatile_s32(const int* p) {
    return *reinterpret_cast<const volatile int*>(p);
}

__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// One thread of the CTA: wait until *count >= target, for at most `limit_ns` of
// wall time and at most kMaxCountPolls polls (a second bound in case the
// timer does not advance).  False when the wait ran out (bit 1 of *err
// raised) or another CTA reported an error.  Polls back off from 32 ns to
// 1 µs so that CTAs waiting on one counter do not flood its L2 line.
constexpr uint32_t kMaxCountPolls = 1u << 24;
__device__ __forceinline__ bool wait_count_for(const unsigned* count, unsigned target, int* err,
                                               uint64_t limit_ns) {
    const uint64_t t0 = globaltimer_ns();
    unsigned ns = 32;
    for (uint32_t i = 0; i < kMaxCountPolls; ++i) {
        if (ld_acquire_u32(count) >= target) return true;
        if (ld_volatile_s32(err) != 0) return false;
        if ((i & 15u) == 15u && globaltimer_ns() - t0 > limit_ns) break;
        __nanosleep(ns);
        ns = ns < 1024 ? 2 * ns : 1024;
    }
    atomicOr(err, 2);
    return false;
}
__device__ __forceinline__ bool wait_count(const unsigned* count, unsigned target, int* err) {
    return wait_count_for(count, target, err, kWaitLimitNs);
}

// ---- chained launches (StepArgs::chain) ----------------------------------
// The stream's next launch, when it allows it, may start its CTAs once every
// CTA of this launch has started; from then on it takes the SM slots this
// one gives back.  Its CTAs hold none that this launch still needs, so both
// make progress; the counters below order the data.
__device__ __forceinline__ void allow_next_launch() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Body CTA index of launch CTA `cta` when the launch is chained: CTAs run
// group by group (group g's boundary CTAs, then its interior tiles), so
// the first CTAs of the next launch wait on the first groups of this one.
// The body's own order has every group's boundary CTAs first.
__device__ __forceinline__ int chain_order(const StepArgs& a, int cta, int nbc, int ngroups, int tiles) {
    if (a.chain == nullptr) return cta;
    const int per = nbc + tiles;
    const int g = cta / per, j = cta - g * per;
    return j < nbc ? g * nbc + j : nbc * ngroups + g * tiles + (j - nbc);
}

// One thread of the CTA (lane 0 of warp 1 in the interior tiles, thread 0 in
// the boundary CTAs): wait until the chain's earlier launches are done with
// shot group `grp`, then order this thread's tensor loads after their stores
// (the thread that issues the first copies fences again after the CTA
// barrier).  False when the wait ran out or another CTA raised the error
// word.
__device__ __forceinline__ bool chain_wait(const StepArgs& a, int grp) {
    if (a.chain == nullptr || a.chain_k <= 0) return true;
    const bool ok = wait_count(a.chain + grp, (unsigned)a.chain_k * (unsigned)a.chain_per_group, a.err);
    fence_proxy_async_global();
    return ok;
}

// Every thread, after the CTA's last store: release the stores and count the
// CTA as done for group `grp`.  The CTA barrier orders every thread's stores
// before thread 0's release add, and a release is cumulative, so the one add
// releases them all (the form a grid-wide barrier takes) without stalling
// thread 0 on a fence; the readers order their tensor loads after their
// acquire with their own proxy fence.
__device__ __forceinline__ void chain_done(const StepArgs& a, int grp) {
    if (a.chain == nullptr) return;
    __syncthreads();
    if (threadIdx.x == 0)
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(a.chain + grp) : "memory");
}

// Host: a launch of a chain after its first: it may start while the
// stream's previous launch is still running (programmatic stream
// serialization; the kernel's counters order the data).
template <typename Kernel, typename... Args>
cudaError_t launch_chained(Kernel kernel, int grid, int threads, size_t smem, cudaStream_t stream,
                           Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

// The persistent work loop.  `body(args, cta)` runs one CTA of a step as a
// non-persistent launch would (cta indexes the step's CTAs, boundary CTAs
// first); `nbars` mbarriers at `bars` are initialised by the body of an
// interior item and invalidated here after it.
template <typename Body>
__device__ __forceinline__ void persistent_loop(const PersistLaunch& P, uint64_t* bars, int nbars,
                                                Body body) {
    __shared__ unsigned s_ticket;
    __shared__ int s_go, s_more;   // uniform decisions, written by thread 0
    __shared__ StepArgs s_args;
    const unsigned per_step = (unsigned)P.ngroups * (unsigned)P.per_group;
    const unsigned total = per_step * (unsigned)P.nsteps;
    if (threadIdx.x == 0) s_ticket = atomicAdd(P.ticket, 1u);
    __syncthreads();
    unsigned item = s_ticket;
    while (item < total) {
        const unsigned step = item / per_step;
        const unsigned rem = item - step * per_step;
        const int grp = (int)(rem / (unsigned)P.per_group);
        const int j = (int)(rem - (unsigned)grp * (unsigned)P.per_group);
        const StepArgs* src = P.steps + step;
        if (threadIdx.x == 0) {
            s_ticket = atomicAdd(P.ticket, 1u);   // the next item, claimed early
            bool ok = ld_volatile_s32(src->err) == 0;
            if (ok && step > 0) ok = wait_count(P.count + grp, step * (unsigned)P.per_group, src->err);
            fence_proxy_async_global();
            s_go = ok ? 1 : 0;
        }
        // this step's arguments (the body's first barrier orders the copy)
        {
            const int* s = reinterpret_cast<const int*>(src);
            int* d = reinterpret_cast<int*>(&s_args);
            for (int i = threadIdx.x; i < (int)(sizeof(StepArgs) / 4); i += blockDim.x) d[i] = s[i];
        }
        __syncthreads();
        const unsigned next = s_ticket;
        if (!s_go) return;
        // boundary CTAs first, then the interior tiles, as in a one-step launch
        const int cta = j < P.nbc ? grp * P.nbc + j : P.nbc * P.ngroups + grp * (P.per_group - P.nbc) + (j - P.nbc);
        body(s_args, cta);
        fence_proxy_async_global();   // this item's stores, before any later tensor load
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            if (j >= P.nbc)
                for (int b = 0; b < nbars; ++b) mbar_inval(&bars[b]);
            s_more = ld_volatile_s32(s_args.err) == 0;
            if (s_more) atomicAdd(P.count + grp, 1u);
        }
        __syncthreads();
        if (!s_more) return;
        item = next;
    }
}

// Host: the grid of a persistent launch -- as many CTAs as can be resident
// at once on the current device (occupancy x SMs), at most one per work item.
template <typename Kernel>
cudaError_t persistent_grid(Kernel kernel, int threads, size_t smem_bytes, long long items, int* grid,
                            int max_ctas = 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem_bytes);
    if (e != cudaSuccess) return e;
    if (items < 1) return cudaErrorInvalidConfiguration;
    long long g = (long long)(per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
    if (g > items) g = items;
    if (max_ctas > 0 && g > max_ctas) g = max_ctas;
    *grid = (int)g;
    return cudaSuccess;
}

}  // namespace twi
