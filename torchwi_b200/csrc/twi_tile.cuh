// twi_tile.cuh -- small device helpers shared by the tile kernels
// (twi_step.cu, twi_backward.cu).
#pragma once

#include <cuda_runtime.h>

#include "twi_kernels.h"
#include "twi_ptx.cuh"

namespace twi {

constexpr int round32(int n) { return (n + 31) / 32 * 32; }

__device__ __forceinline__ float comp(const float4& v, int m) {
    return m == 0 ? v.x : m == 1 ? v.y : m == 2 ? v.z : v.w;
}
__device__ __forceinline__ void set_comp(float4& v, int m, float x) {
    if (m == 0) v.x = x;
    else if (m == 1) v.y = x;
    else if (m == 2) v.z = x;
    else v.w = x;
}
__device__ __forceinline__ float4 ld4(const float* p) {
    return *reinterpret_cast<const float4*>(p);
}

// Number of Keys boundary cells of one shot: the left and right ne columns of
// rows [ne, dimz-ne) and all columns of the bottom ne rows
// (td2d_cpu.cpp:116-145).
__host__ __device__ inline int boundary_cells(int order, int dimx, int dimz) {
    const int ne = order / 2;
    return 2 * ne * (dimz - 2 * ne) + ne * dimx;
}

// Row, column and inward step (offset to the next cell towards the interior)
// of boundary cell `idx` in the boundary CTAs' order: left columns, right
// columns (row by row, ne cells each), then the bottom rows.
template <int NE>
__device__ __forceinline__ void boundary_cell_at(int idx, int dimx, int dimz, int pitch, int& r,
                                                 int& c, long long& db) {
    const int side_rows = dimz - 2 * NE;
    const int n_side = 2 * NE * side_rows;
    if (idx < n_side) {
        const int side = idx / (NE * side_rows);
        const int rem = idx - side * NE * side_rows;
        r = NE + rem / NE;
        const int k = rem - (rem / NE) * NE;
        c = side == 0 ? k : dimx - NE + k;
        db = side == 0 ? 1 : -1;
    } else {
        const int j = idx - n_side;
        r = dimz - NE + j / dimx;
        c = j - (j / dimx) * dimx;
        db = -(long long)pitch;
    }
}

// Copy one job's arguments into shared memory (all threads take part, and
// the barrier at the end orders the copy before any use).
__device__ __forceinline__ void copy_args(StepArgs& dst, const StepArgs& src) {
    static_assert(sizeof(StepArgs) % 4 == 0, "StepArgs is copied in 4-byte words");
    const int* s = reinterpret_cast<const int*>(&src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(StepArgs) / 4); i += blockDim.x) d[i] = s[i];
    __syncthreads();
}

// Index of the last job whose first CTA is at or before `cta` (begin[] ascending).
template <typename Begin>
__device__ __forceinline__ int job_of(Begin begin, int njobs, int cta) {
    int lo = 0, hi = njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (begin(mid) <= cta) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// x neighbours of a lane's four columns at distance 1..NE (L[k]: column
// c-1-k, R[k]: column c+4+k), read from the staged row `row` in the haloed
// layout (the lane's first column at `cs`, a kHaloX-column halo on each
// side): two vector loads instead of shuffles, and no special case for the
// first and last lanes, whose neighbours sit in the halo.
template <int NE>
__device__ __forceinline__ void row_neighbours(const float* row, int cs, float (&L)[NE], float (&R)[NE]) {
    static_assert(NE == 1 || NE == 2 || NE == 4, "orders 2, 4 and 8");
    if constexpr (NE == 1) {
        L[0] = row[cs - 1];
        R[0] = row[cs + 4];
    } else if constexpr (NE == 2) {
        const float2 l = *reinterpret_cast<const float2*>(row + cs - 2);
        const float2 r = *reinterpret_cast<const float2*>(row + cs + 4);
        L[0] = l.y, L[1] = l.x;
        R[0] = r.x, R[1] = r.y;
    } else {
        const float4 l = ld4(row + cs - 4);
        const float4 r = ld4(row + cs + 4);
        L[0] = l.w, L[1] = l.z, L[2] = l.y, L[3] = l.x;
        R[0] = r.x, R[1] = r.y, R[2] = r.z, R[3] = r.w;
    }
}

// Shot stages consumed warp by warp.  Every warp waits for a stage's copies
// itself (all lanes, so each sees the data; the answer is warp-uniform), and
// the last of the CTA's `nwarps` warps to finish shot k with stage k % stages
// refills it.  `done[stage]` counts the warps' finishes over the CTA's shots
// and is never reset, so the last finisher of shot k reads
// (k / stages + 1) * nwarps - 1; no warp waits for another between shots.
__device__ __forceinline__ bool warp_wait_stage(uint64_t* bar, uint32_t parity) {
    return __all_sync(0xffffffffu, mbar_wait_bounded(bar, parity));
}
// True on lane 0 of the last warp done with shot k's stage: that lane issues
// the stage's next copies.  The fences order every lane's reads of the stage
// before the count, and the count before the refill.
__device__ __forceinline__ bool last_warp_done(int* done, int k, int stages, int nwarps) {
    __syncwarp();
    bool last = false;
    if ((threadIdx.x & 31) == 0) {
        __threadfence_block();
        last = atomicAdd(&done[k % stages], 1) == (k / stages + 1) * nwarps - 1;
        if (last) __threadfence_block();
    }
    return last;
}

}  // namespace twi
