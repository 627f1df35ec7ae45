// twi_step.cu -- the fused time-step kernel and its small helpers.
//
// One launch advances every shot of a batch by one time step.  A CTA owns a
// 128-column x TZ-row tile of the padded grid and a group of `spc` shots
// that share the velocity tile.  For each shot it stages u^n (with a 4-column
// / HZ-row halo) and u^{n-1} (4-column / 1-row halo) into shared memory with
// TMA, double-buffered across shots, and computes in one pass what the
// reference does with five launches and a memcpy per step
// (propagator_cpu.cpp:57-78, propagator_cuda.cu:61-80):
//   * the interior leapfrog update (orders 2/4/8),
//   * the Keys absorbing update of the left/right/bottom pads,
//   * the point source (forward) or the adjoint source on the receiver row,
//   * the receiver-row gather (forward),
//   * the virtual source -2/(v^3 dt^2) (u^{n+1} - 2u^n + u^{n-1}) (recompute),
//   * the gradient term -virt * lambda with Kahan or plain accumulation
//     (adjoint).
// Each warp streams RZ consecutive rows: a (2*NE+1)-row register window of
// float4s along z, and the x neighbours read from the staged row (two vector
// loads per row, the halo covering the first and last lanes).  Rows/columns of the pads use the
// general per-cell path.  The top NE rows are the free surface: always 0.
#include <atomic>
#include <cstdio>
#include <type_traits>

#include "twi_cell.cuh"
#include "twi_kernels.h"
#include "twi_persist.cuh"
#include "twi_ptx.cuh"
#include "twi_tile.cuh"

namespace twi {
namespace {

// CTAs per SM the launch bounds ask for: 2 rows per warp -> 5, 4 -> 4, 8 -> 2
// (the 8-row tiles are held to 2 by shared memory)
constexpr int kMinCtasPerSm(int rz) { return rz == 2 ? 5 : rz == 4 ? 4 : 2; }

template <int ORDER, int RZ, int WZ>
struct Smem {
    static constexpr int NE = ORDER / 2;
    static constexpr int TZ = RZ * WZ;
    static constexpr int HZ = zhalo(ORDER);
    static constexpr int U2_ROWS = TZ + 2 * HZ;               // u^n with halo
    static constexpr int U2_FLOATS = round32(U2_ROWS * kBoxX);
    static constexpr int U1_FLOATS = TZ * kTileX;              // u^{n-1}, no halo
    static constexpr int STAGE_FLOATS = U2_FLOATS + U1_FLOATS;
    static constexpr int V_FLOATS = TZ * kTileX;
    static constexpr int STAGES = 2;
    static constexpr int BAR_BYTES = 128;
    static constexpr size_t BYTES =
        128 /*alignment slack*/ + BAR_BYTES + size_t(V_FLOATS + STAGES * STAGE_FLOATS) * 4;
    static constexpr uint32_t U2_TX = U2_ROWS * kBoxX * 4;
    static constexpr uint32_t U1_TX = TZ * kTileX * 4;
    static constexpr uint32_t V_TX = TZ * kTileX * 4;
};

// One boundary CTA: a strided share of the Keys cells of one shot group,
// one thread per cell, for every shot of the group.  Neighbours come
// straight from the slots (L2); the interior CTAs never write these cells.
template <int ORDER, bool EXACT, int MODE>
__device__ __forceinline__ void boundary_part(const StepArgs& a, const StepDyn& d, int b, int nbc) {
    constexpr int NE = ORDER / 2;
    const int grp = b / nbc, part = b - grp * nbc;
    if (a.chain != nullptr) {
        __shared__ int sh_go;
        if (threadIdx.x == 0) sh_go = chain_wait(a, grp);
        __syncthreads();
        if (!sh_go) return;
    }
    const int s0 = grp * a.spc, s1 = min(s0 + a.spc, a.nshots);
    const int nb = boundary_cells(ORDER, a.dimx, a.dimz);
    for (int idx = part * blockDim.x + threadIdx.x; idx < nb; idx += nbc * blockDim.x) {
        int r, c;
        long long db;   // offset to the first cell inwards
        boundary_cell_at<NE>(idx, a.dimx, a.dimz, a.pitch, r, c, db);
        const long long cell = (long long)r * a.pitch + c;
        const float v = a.vel[cell];
        const float q = (MODE == kModeRecompute || MODE == kModeExaForward || MODE == kModeReverse)
                            ? virt_coef<EXACT>(v, a.cons) : 0.f;
        for (int s = s0; s < s1; ++s) {
            const float* U2 = a.fields + (long long)(d.cur_base + s * d.cur_stride) * a.slot_elems + cell;
            const float* U1 = a.fields + (long long)(d.prev_base + s * d.prev_stride) * a.slot_elems + cell;
            const float uo = U2[0], um = U1[0];
            float out;
            if constexpr (MODE == kModeReverse)   // u^{it-1} as the forward pass saved it (u^0 = 0)
                out = d.it >= 2 ? a.bnd[((long long)(d.it - 1) * a.nshots + s) * a.bnd_cells + idx] : 0.f;
            else
                out = keys_cell<EXACT>(uo, U2[db], U2[2 * db], um, U1[db], v, a.h2, a.dt2, a.hdt);
            a.fields[(long long)(d.next_base + s * d.next_stride) * a.slot_elems + cell] = out;
            if constexpr (MODE == kModeForward) {
                if (a.bnd != nullptr)
                    a.bnd[((long long)(d.it + 1) * a.nshots + s) * a.bnd_cells + idx] = out;
            }
            if constexpr (MODE == kModeReverse) {   // um holds u^{it+1}, out u^{it-1}
                a.virt_out[(long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                           (long long)r * a.virt_pitch + c] = virt_from_coef<EXACT>(q, out, uo, um);
            }
            if constexpr (MODE != kModeAdjoint && MODE != kModeReverse) {
                // a receiver row inside the bottom pad records Keys values
                if (a.frd != nullptr && r == a.rec_row[s] && c >= NE && c < NE + a.nx) {
                    const long long o = (long long)s * a.frd_stride + (long long)d.it * a.nx + (c - NE);
                    a.frd[o] = a.obs != nullptr ? __fsub_rn(out, a.obs[o]) : out;
                }
            }
            if constexpr (MODE == kModeRecompute) {
                a.virt_out[(long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                           (long long)r * a.virt_pitch + c] = virt_from_coef<EXACT>(q, um, uo, out);
            }
            if constexpr (MODE == kModeExaForward) {
                const float vt = virt_from_coef<EXACT>(q, um, uo, out);
                const long long e = (long long)s * a.slot_elems + cell;
                if (fabsf(vt) > fabsf(a.exa[e])) {
                    a.exa[e] = vt;
                    a.iexa[e] = static_cast<short>(d.it);
                }
            }
            if constexpr (MODE == kModeAdjoint) {
                // pad cells are cropped by every caller; the plain per-shot sums
                // keep them anyway so the full-grid gradient equals the reference's
                if (a.acc_mode == kAccPlainPerShot) {
                    const float vt = a.virt_in[(long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                                               (long long)r * a.virt_pitch + c];
                    float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems + cell;
                    *g = __fadd_rn(*g, grad_term<EXACT>(vt, out));
                } else if (a.acc_mode == kAccExa) {
                    const long long e = (long long)s * a.slot_elems + cell;
                    if (a.iexa[e] == d.it)
                        a.acc[(long long)(a.acc_base + s) * a.slot_elems + cell] =
                            grad_term<EXACT>(a.exa[e], out);
                }
            }
        }
    }
    chain_done(a, grp);
}

// One CTA of one job (a time step of one plan): `cta` indexes the job's CTAs,
// boundary CTAs first, then the interior tiles.  tm_u2 / tm_u1 / tm_vel may
// live in parameter space (single-plan kernel) or global memory (multi-plan
// kernel).
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ, bool PLAIN_ROWS = true>
__device__ __forceinline__ void step_body(const CUtensorMap* tm_u2p, const CUtensorMap* tm_u1p,
                                          const CUtensorMap* tm_velp, const StepArgs& a,
                                          const StepDyn& d, const int nbc, const int cta_in) {
    using S = Smem<ORDER, RZ, WZ>;
    constexpr int NE = S::NE, HZ = S::HZ, TZ = S::TZ, STAGES = S::STAGES;

    allow_next_launch();
    const int ngroups = (a.nshots + a.spc - 1) / a.spc;
    const int tiles_x = (a.dimx + kTileX - 1) / kTileX;
    const int tiles_z = (a.dimz + TZ - 1) / TZ;
    const int cta = chain_order(a, cta_in, nbc, ngroups, tiles_x * tiles_z);
    if (cta < nbc * ngroups) {
        boundary_part<ORDER, EXACT, MODE>(a, d, cta, nbc);
        return;
    }
    const int m_id = cta - nbc * ngroups;
    const int tile_x = m_id % tiles_x;
    const int tile_z = (m_id / tiles_x) % tiles_z;
    const int grp = m_id / (tiles_x * tiles_z);

    extern __shared__ unsigned char smem_raw[];
    unsigned char* sbase = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase);  // [0] velocity, [1+i] stage i
    float* vs = reinterpret_cast<float*>(sbase + S::BAR_BYTES);
    float* stage0 = vs + S::V_FLOATS;

    const int x0 = tile_x * kTileX;
    const int z0 = tile_z * TZ;
    const int s_begin = grp * a.spc;
    const int nloc = min(a.spc, a.nshots - s_begin);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    // the group's source cells, wavelet samples and receiver rows, read once
    __shared__ int sh_src_r[kMaxShotsPerCta], sh_src_c[kMaxShotsPerCta], sh_rec_r[kMaxShotsPerCta];
    __shared__ float sh_wamp[kMaxShotsPerCta];
    __shared__ int sh_done[STAGES];   // warps done with each stage (last_warp_done)
    if (threadIdx.x < STAGES) sh_done[threadIdx.x] = 0;
    if (threadIdx.x < nloc) {
        const int s = s_begin + threadIdx.x;
        sh_src_r[threadIdx.x] = MODE != kModeAdjoint ? a.src_rc[2 * s] : -1;
        sh_src_c[threadIdx.x] = MODE != kModeAdjoint ? a.src_rc[2 * s + 1] : -1;
        sh_wamp[threadIdx.x] = MODE != kModeAdjoint ? a.wav[(long long)s * a.wav_stride + d.it] : 0.f;
        sh_rec_r[threadIdx.x] = a.rec_row[s];
    }
    auto issue = [&](int k) {
        const int s = s_begin + k;
        float* st = stage0 + (k % STAGES) * S::STAGE_FLOATS;
        uint64_t* b = &bar[1 + (k % STAGES)];
        mbar_arrive_expect_tx(b, S::U2_TX + S::U1_TX);
        tma_load_3d(st, tm_u2p, x0 - kHaloX, z0 - HZ, d.cur_base + s * d.cur_stride, b);
        tma_load_3d(st + S::U2_FLOATS, tm_u1p, x0, z0, d.prev_base + s * d.prev_stride, b);
    };
    // Thread 0 sets up the stage barriers, issues the static velocity tile
    // and, when the launch waits for nothing, the first stages; meanwhile
    // lane 0 of warp 1 waits for the chain, if any, so that a chained
    // launch's field copies go out right after the CTA barrier.
    const bool chained_wait = a.chain != nullptr && a.chain_k > 0;
    __shared__ int sh_chain_ok;
    if (threadIdx.x == 0) {
        prefetch_tmap(tm_u2p);
        prefetch_tmap(tm_u1p);
        prefetch_tmap(tm_velp);
#pragma unroll
        for (int i = 0; i < 1 + STAGES; ++i) mbar_init(&bar[i], 1);
        fence_barrier_init();
        mbar_arrive_expect_tx(&bar[0], S::V_TX);
        tma_load_2d(vs, tm_velp, x0, z0, &bar[0]);
        if (!chained_wait)
            for (int k = 0; k < STAGES && k < nloc; ++k) issue(k);
    }
    if (chained_wait && threadIdx.x == 32) sh_chain_ok = chain_wait(a, grp) ? 1 : 0;
    __syncthreads();
    bool go = true;
    if (chained_wait && threadIdx.x == 0) {
        go = sh_chain_ok != 0;
        if (go) {
            fence_proxy_async_global();   // these tensor loads after warp 1's acquire
            for (int k = 0; k < STAGES && k < nloc; ++k) issue(k);
        }
    }

    const int rl0 = warp * RZ;           // first tile-local row of this warp
    const int c = x0 + 4 * lane;         // first column of this lane
    const int cs = kHaloX + 4 * lane;    // its column in the haloed u^n tile
    const bool col_ok = c < a.dimx;
    // the lane's four columns are all interior (stencil) columns
    const bool cols_interior = c >= NE && c + 3 < a.dimx - NE;
    bool cell_in[4];                     // per-cell interior column mask
#pragma unroll
    for (int m = 0; m < 4; ++m) cell_in[m] = c + m >= NE && c + m < a.dimx - NE;

    // the first shot's virtual source into L2 while the tiles load (the
    // loop below prefetches each next shot's)
    if constexpr (MODE == kModeAdjoint) {
        if (nloc > 0 && (lane & 7) == 0 &&
            (a.acc_mode == kAccKahanPerGroup || a.acc_mode == kAccPlainPerShot)) {
            const float* nb = a.virt_in + (long long)(d.virt_base + s_begin * a.virt_stride) * a.virt_slot_elems;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int r = z0 + rl0 + rr;
                if (col_ok && r < a.dimz) prefetch_l2(nb + (long long)r * a.virt_pitch + c);
            }
        }
    }

    {
        const bool ok = mbar_wait_bounded(&bar[0], 0);
        if (__syncthreads_or(!ok || !go)) {
            if (threadIdx.x == 0) {
                if (!ok) atomicOr(a.err, 1);
                if (go) drain_stages(&bar[1], STAGES, 0, min(STAGES, nloc));
            }
            return;
        }
    }
    // any warp may refill a stage later: every thread orders its tensor
    // loads after the chain's acquire (thread 0's, through the barrier above)
    if (a.chain != nullptr && a.chain_k > 0) fence_proxy_async_global();
    // per-cell constants over all shots: v*v*dt^2/h^2, and for the recompute
    // the virtual-source coefficient; v itself stays in shared memory
    float4 vvreg[RZ];
    constexpr bool kVirt = MODE == kModeRecompute || MODE == kModeExaForward || MODE == kModeReverse;
    float4 qreg[kVirt ? RZ : 1];
#pragma unroll
    for (int rr = 0; rr < RZ; ++rr) {
        const float4 v4 = ld4(vs + (rl0 + rr) * kTileX + 4 * lane);
        vvreg[rr] = make_float4(vv_of<EXACT>(v4.x, a.dtoh2), vv_of<EXACT>(v4.y, a.dtoh2),
                                vv_of<EXACT>(v4.z, a.dtoh2), vv_of<EXACT>(v4.w, a.dtoh2));
        if constexpr (kVirt) {
            // columns past the grid hold v = 0: keep their (never stored) coefficient finite
            qreg[rr] = make_float4(virt_coef<EXACT>(v4.x != 0.f ? v4.x : 1.f, a.cons),
                                   virt_coef<EXACT>(v4.y != 0.f ? v4.y : 1.f, a.cons),
                                   virt_coef<EXACT>(v4.z != 0.f ? v4.z : 1.f, a.cons),
                                   virt_coef<EXACT>(v4.w != 0.f ? v4.w : 1.f, a.cons));
        }
    }

    // Kahan accumulators of this CTA's shot group (adjoint)
    float4 gsum[MODE == kModeAdjoint ? RZ : 1], gcmp[MODE == kModeAdjoint ? RZ : 1];
    if constexpr (MODE == kModeAdjoint) {
        if (a.acc_mode == kAccKahanPerGroup) {
            const long long slot = a.acc_base + grp;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int r = z0 + rl0 + rr;
                gsum[rr] = gcmp[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (col_ok && r < a.dimz) {
                    const long long off = slot * a.slot_elems + (long long)r * a.pitch + c;
                    gsum[rr] = ld4(a.acc + off);
                    gcmp[rr] = ld4(a.acc_comp + off);
                }
            }
        }
    }

    for (int k = 0; k < nloc; ++k) {
        const int s = s_begin + k;
        const float* u2s = stage0 + (k % STAGES) * S::STAGE_FLOATS;
        const float* u1s = u2s + S::U2_FLOATS;

        const int src_r = sh_src_r[k], src_c = sh_src_c[k], rec_r = sh_rec_r[k];
        const float wamp = sh_wamp[k];

        // virtual source of this step for the warp's rows (adjoint); only the
        // virtual-source accumulations read it -- the excitation-amplitude
        // adjoint has no virt_in array at all
        float4 vin[MODE == kModeAdjoint ? RZ : 1];
        if constexpr (MODE == kModeAdjoint) {
            const bool need_vin = a.acc_mode == kAccKahanPerGroup || a.acc_mode == kAccPlainPerShot;
            const float* vbase =
                a.virt_in + (long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int r = z0 + rl0 + rr;
                vin[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (need_vin && col_ok && r < a.dimz) {
                    const float* p = vbase + (long long)r * a.virt_pitch + c;
                    if (a.virt_vec4) {
                        vin[rr] = ld4(p);
                    } else {
                        vin[rr].x = p[0];
                        if (c + 1 < a.dimx) vin[rr].y = p[1];
                        if (c + 2 < a.dimx) vin[rr].z = p[2];
                        if (c + 3 < a.dimx) vin[rr].w = p[3];
                    }
                }
            }
        }
        // the next shot's virtual source into L2 while this one computes
        // (one prefetch per 128-byte line of each warp row)
        if constexpr (MODE == kModeAdjoint) {
            if (k + 1 < nloc && (lane & 7) == 0 &&
                (a.acc_mode == kAccKahanPerGroup || a.acc_mode == kAccPlainPerShot)) {
                const float* nb = a.virt_in + (long long)(d.virt_base + (s + 1) * a.virt_stride) * a.virt_slot_elems;
#pragma unroll
                for (int rr = 0; rr < RZ; ++rr) {
                    const int r = z0 + rl0 + rr;
                    if (col_ok && r < a.dimz) prefetch_l2(nb + (long long)r * a.virt_pitch + c);
                }
            }
        }

        if (!warp_wait_stage(&bar[1 + (k % STAGES)], (k / STAGES) & 1)) {
            // the copies never landed: flag it, wait (bounded) for the copies
            // this warp may have issued, and leave
            if (lane == 0) {
                atomicOr(a.err, 1);
                drain_stages(&bar[1], STAGES, k, min(nloc, k + STAGES));
            }
            return;
        }

        float4 win[2 * NE + 1];
#pragma unroll
        for (int j = 0; j < 2 * NE; ++j) win[j] = ld4(u2s + (rl0 + HZ - NE + j) * kBoxX + cs);

        // PLAIN: every row of this warp is an interior row that holds neither the
        // source nor the receivers (neither pad nor free-surface rows), so the
        // rows run without any per-row test
        auto rows = [&](auto plain_tag) {
            constexpr bool PLAIN = decltype(plain_tag)::value;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int rl = rl0 + rr;
                const int r = z0 + rl;
                // the bottom pad rows and everything below belong to the boundary CTAs
                if (!PLAIN && r >= a.dimz - NE) break;
                win[2 * NE] = ld4(u2s + (rl + HZ + NE) * kBoxX + cs);
                const float c4[4] = {win[NE].x, win[NE].y, win[NE].z, win[NE].w};
                float L[NE], Rr[NE];   // L[k]: column c-1-k, Rr[k]: column c+4+k
                row_neighbours<NE>(u2s + (rl + HZ) * kBoxX, cs, L, Rr);
                const float4 um4 = ld4(u1s + rl * kTileX + 4 * lane);
                const float um[4] = {um4.x, um4.y, um4.z, um4.w};
                float* dst = a.fields + (long long)(d.next_base + s * d.next_stride) * a.slot_elems +
                             (long long)r * a.pitch + c;

                if (!PLAIN && r < NE) {
                    // free surface: the top rows stay zero (the reference never writes them)
                    if (col_ok) *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
                    if constexpr (MODE == kModeAdjoint) {
                        // the excitation-amplitude assignment covers every cell of the
                        // grid, these rows and their corner pad cells included
                        // (td2d_cuda.cu:197-205): -exa * 0 there
                        if (a.acc_mode == kAccExa && col_ok) {
                            const long long e0 = (long long)s * a.slot_elems + (long long)r * a.pitch + c;
                            float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems +
                                       (long long)r * a.pitch + c;
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                if (c + m < a.dimx && a.iexa[e0 + m] == d.it)
                                    g[m] = grad_term<EXACT>(a.exa[e0 + m], 0.f);
                        }
                    }
                    if constexpr (MODE == kModeRecompute || MODE == kModeReverse) {
                        if (col_ok) {
                            float vo[4];
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                vo[m] = MODE == kModeReverse
                                            ? virt_from_coef<EXACT>(comp(qreg[rr], m), 0.f, c4[m], um[m])
                                            : virt_from_coef<EXACT>(comp(qreg[rr], m), um[m], c4[m], 0.f);
                            float* p = a.virt_out +
                                       (long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                                       (long long)r * a.virt_pitch + c;
                            if (a.virt_vec4) {
                                *reinterpret_cast<float4*>(p) = make_float4(vo[0], vo[1], vo[2], vo[3]);
                            } else {
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (c + m < a.dimx) p[m] = vo[m];
                            }
                        }
                    }
                } else {
                    // One interior row.  FAST: neither the source nor the receiver
                    // row, so no per-row special case is tested; in the edge tiles
                    // the lanes holding pad columns mask their stores.
                    auto interior_row = [&](auto fast_tag) {
                        constexpr bool FAST = decltype(fast_tag)::value;
                        float out[4];
                        // backwards, u^{it+1} stands where u^{n-1} did, with the source
                        // that step `it` added taken off again
                        float ui[4] = {um[0], um[1], um[2], um[3]};
                        if constexpr (MODE == kModeReverse) {
                            if (!FAST && r == src_r && src_c >= c && src_c < c + 4) {
                                const float4 v4 = ld4(vs + rl * kTileX + 4 * lane);
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (c + m == src_c) ui[m] = __fsub_rn(um[m], injection<EXACT>(wamp, comp(v4, m), a.dt2));
                            }
                        }
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            float lf[NE], rt[NE], up[NE], dn[NE];
#pragma unroll
                            for (int dist = 1; dist <= NE; ++dist) {
                                const int jl = m - dist, jr = m + dist;
                                lf[dist - 1] = jl >= 0 ? c4[jl] : L[-jl - 1];
                                rt[dist - 1] = jr < 4 ? c4[jr] : Rr[jr - 4];
                                up[dist - 1] = comp(win[NE - dist], m);
                                dn[dist - 1] = comp(win[NE + dist], m);
                            }
                            out[m] = interior_update<ORDER, EXACT>(lf, rt, up, dn, c4[m], ui[m],
                                                                   comp(vvreg[rr], m));
                            if constexpr (MODE == kModeReverse) {
                                if (d.it < 2) out[m] = 0.f;   // u^0 = u^{-1} = 0 exactly
                            }
                        }
                        // sources land on interior cells only (validated on the host)
                        if constexpr (MODE != kModeAdjoint && MODE != kModeReverse) {
                            if (!FAST && r == src_r && src_c >= c && src_c < c + 4) {
                                const float4 v4 = ld4(vs + rl * kTileX + 4 * lane);
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (c + m == src_c)
                                        out[m] = add_injection<EXACT>(out[m], wamp, comp(v4, m), a.dt2);
                            }
                        } else if constexpr (MODE == kModeAdjoint) {
                            if (!FAST && r == rec_r) {
                                const float4 v4 = ld4(vs + rl * kTileX + 4 * lane);
                                const float* rs =
                                    a.resid + (long long)s * a.resid_stride + (long long)d.it * a.nx;
#pragma unroll
                                for (int m = 0; m < 4; ++m) {
                                    const int cc = c + m;
                                    if (cc >= NE && cc < NE + a.nx)
                                        out[m] = add_injection<EXACT>(out[m], rs[cc - NE], comp(v4, m), a.dt2);
                                }
                            }
                        }

                        // pad columns belong to the boundary CTAs: store interior cells only
                        if (cols_interior) {
                            *reinterpret_cast<float4*>(dst) = make_float4(out[0], out[1], out[2], out[3]);
                        } else {
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                if (cell_in[m]) dst[m] = out[m];
                        }

                        if constexpr (MODE != kModeAdjoint && MODE != kModeReverse) {
                            if (!FAST && a.frd != nullptr && r == rec_r) {
                                const long long o = (long long)s * a.frd_stride + (long long)d.it * a.nx;
                                float* g = a.frd + o;
                                if (a.obs != nullptr) {   // the residual, one rounding like frd - obs
                                    const float* ob = a.obs + o;
#pragma unroll
                                    for (int m = 0; m < 4; ++m) {
                                        const int cc = c + m;
                                        if (cc >= NE && cc < NE + a.nx) g[cc - NE] = __fsub_rn(out[m], ob[cc - NE]);
                                    }
                                } else {
#pragma unroll
                                    for (int m = 0; m < 4; ++m) {
                                        const int cc = c + m;
                                        if (cc >= NE && cc < NE + a.nx) g[cc - NE] = out[m];
                                    }
                                }
                            }
                        }

                        if constexpr (MODE == kModeRecompute || MODE == kModeReverse) {
                            float vo[4];
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                vo[m] = MODE == kModeReverse
                                            ? virt_from_coef<EXACT>(comp(qreg[rr], m), out[m], c4[m], um[m])
                                            : virt_from_coef<EXACT>(comp(qreg[rr], m), um[m], c4[m], out[m]);
                            float* p = a.virt_out +
                                       (long long)(d.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                                       (long long)r * a.virt_pitch + c;
                            if (cols_interior && a.virt_vec4) {
                                *reinterpret_cast<float4*>(p) = make_float4(vo[0], vo[1], vo[2], vo[3]);
                            } else {
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (cell_in[m]) p[m] = vo[m];
                            }
                        }

                        if constexpr (MODE == kModeExaForward) {
                            const long long e0 = (long long)s * a.slot_elems + (long long)r * a.pitch + c;
                            float4 ev = ld4(a.exa + e0);
                            short4 iv = *reinterpret_cast<const short4*>(a.iexa + e0);
                            bool changed = false;
#pragma unroll
                            for (int m = 0; m < 4; ++m) {
                                if (!cell_in[m]) continue;
                                const float vt = virt_from_coef<EXACT>(comp(qreg[rr], m), um[m], c4[m], out[m]);
                                if (fabsf(vt) > fabsf(comp(ev, m))) {
                                    set_comp(ev, m, vt);
                                    if (m == 0) iv.x = static_cast<short>(d.it);
                                    else if (m == 1) iv.y = static_cast<short>(d.it);
                                    else if (m == 2) iv.z = static_cast<short>(d.it);
                                    else iv.w = static_cast<short>(d.it);
                                    changed = true;
                                }
                            }
                            if (changed) {
                                if (cols_interior) {
                                    *reinterpret_cast<float4*>(a.exa + e0) = ev;
                                    *reinterpret_cast<short4*>(a.iexa + e0) = iv;
                                } else {   // pad columns belong to the boundary CTAs
                                    const short is[4] = {iv.x, iv.y, iv.z, iv.w};
#pragma unroll
                                    for (int m = 0; m < 4; ++m)
                                        if (cell_in[m]) a.exa[e0 + m] = comp(ev, m), a.iexa[e0 + m] = is[m];
                                }
                            }
                        }

                        if constexpr (MODE == kModeAdjoint) {
                            if (a.acc_mode == kAccExa) {
                                const long long e0 = (long long)s * a.slot_elems + (long long)r * a.pitch + c;
                                const short4 iv = *reinterpret_cast<const short4*>(a.iexa + e0);
                                const short is[4] = {iv.x, iv.y, iv.z, iv.w};
                                float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems +
                                           (long long)r * a.pitch + c;
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (cell_in[m] && is[m] == d.it) g[m] = grad_term<EXACT>(a.exa[e0 + m], out[m]);
                            } else if (a.acc_mode == kAccKahanPerGroup) {
                                // every column: the pairs of pad cells and of columns
                                // past the grid are never read (callers crop the pads)
#pragma unroll
                                for (int m = 0; m < 4; ++m) {
                                    float sm = comp(gsum[rr], m), cm = comp(gcmp[rr], m);
                                    kahan_add(sm, cm, grad_term<EXACT>(comp(vin[rr], m), out[m]));
                                    set_comp(gsum[rr], m, sm);
                                    set_comp(gcmp[rr], m, cm);
                                }
                            } else if (a.acc_mode == kAccPlainPerShot) {
                                float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems +
                                           (long long)r * a.pitch + c;
                                if (cols_interior) {
                                    float4 gv = ld4(g);
#pragma unroll
                                    for (int m = 0; m < 4; ++m)
                                        set_comp(gv, m, __fadd_rn(comp(gv, m),
                                                                  grad_term<EXACT>(comp(vin[rr], m), out[m])));
                                    *reinterpret_cast<float4*>(g) = gv;
                                } else {
#pragma unroll
                                    for (int m = 0; m < 4; ++m)
                                        if (cell_in[m])
                                            g[m] = __fadd_rn(g[m], grad_term<EXACT>(comp(vin[rr], m), out[m]));
                                }
                            }
                        }
                    };
                    if (PLAIN || (r != src_r && r != rec_r)) interior_row(std::true_type{});
                    else interior_row(std::false_type{});
                }
#pragma unroll
                for (int j = 0; j < 2 * NE; ++j) win[j] = win[j + 1];
            }
        };
        const int rw0 = z0 + rl0;   // first row of this warp
        if constexpr (PLAIN_ROWS) {
            if (rw0 >= NE && rw0 + RZ <= a.dimz - NE && (src_r < rw0 || src_r >= rw0 + RZ) &&
                (rec_r < rw0 || rec_r >= rw0 + RZ))
                rows(std::true_type{});
            else
                rows(std::false_type{});
        } else {
            rows(std::false_type{});
        }

        if (last_warp_done(sh_done, k, STAGES, WZ) && k + STAGES < nloc) issue(k + STAGES);
    }

    if constexpr (MODE == kModeAdjoint) {
        if (a.acc_mode == kAccKahanPerGroup) {
            const long long slot = a.acc_base + grp;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int r = z0 + rl0 + rr;
                if (col_ok && r < a.dimz) {
                    const long long off = slot * a.slot_elems + (long long)r * a.pitch + c;
                    *reinterpret_cast<float4*>(a.acc + off) = gsum[rr];
                    *reinterpret_cast<float4*>(a.acc_comp + off) = gcmp[rr];
                }
            }
        }
    }
    chain_done(a, grp);
}

template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kMinCtasPerSm(RZ))
step_kernel(const __grid_constant__ CUtensorMap tm_u2, const __grid_constant__ CUtensorMap tm_u1,
            const __grid_constant__ CUtensorMap tm_vel, const __grid_constant__ StepArgs a,
            const int nbc) {
    const StepDyn d = dyn_of(a);
    step_body<ORDER, EXACT, MODE, RZ, WZ>(&tm_u2, &tm_u1, &tm_vel, a, d, nbc, blockIdx.x);
}

// Several plans (different grids, shots, time indices) in one launch: CTA
// ranges of the jobs are contiguous and ascending; begins[i] is
// jobs[i].cta_begin in one compact array (the CTA's job is found by a binary
// search over it); the main-height tensor maps of plan p are
// tmaps[6p .. 6p+2].
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kMinCtasPerSm(RZ))
step_kernel_multi(const MultiJob* __restrict__ jobs, const int* __restrict__ begins, const int njobs,
                  const CUtensorMap* __restrict__ tmaps) {
    const int lo = job_of([&](int i) { return begins[i]; }, njobs, (int)blockIdx.x);
    const MultiJob& J = jobs[lo];
    const CUtensorMap* tm = tmaps + kMapsPerPlan * J.plan;
    // Read through a pointer into global memory, the arguments would have to
    // be re-read from there after the kernel's own global stores.  The
    // forward step copies them into registers; the recompute and adjoint
    // steps, which hold more live values, into shared memory.
    if constexpr (MODE == kModeForward) {
        const StepArgs a = J.a;
        step_body<ORDER, EXACT, MODE, RZ, WZ>(tm, tm + 1, tm + 2, a, dyn_of(a), J.nbc,
                                              blockIdx.x - J.cta_begin);
    } else {
        __shared__ StepArgs a;
        copy_args(a, J.a);
        step_body<ORDER, EXACT, MODE, RZ, WZ>(tm, tm + 1, tm + 2, a, dyn_of(a), J.nbc,
                                              blockIdx.x - J.cta_begin);
    }
}

// Persistent launches: many time steps of one plan pass in one launch
// (twi_persist.cuh), each work item running one CTA of one step.
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kMinCtasPerSm(RZ))
step_kernel_persistent(const __grid_constant__ CUtensorMap tm_u2, const __grid_constant__ CUtensorMap tm_u1,
                       const __grid_constant__ CUtensorMap tm_vel, const __grid_constant__ PersistLaunch P) {
    extern __shared__ unsigned char smem_raw[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    persistent_loop(P, bars, 1 + Smem<ORDER, RZ, WZ>::STAGES, [&](const StepArgs& a, int cta) {
        step_body<ORDER, EXACT, MODE, RZ, WZ, false>(&tm_u2, &tm_u1, &tm_vel, a, dyn_of(a), P.nbc, cta);
    });
}

// Engine launches: the CTA ranges and the per-step integers come from the
// kernel parameters, the static arguments of each request and kernel mode
// from a template resident in device memory.
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kMinCtasPerSm(RZ))
step_kernel_engine(const __grid_constant__ EngineLaunch L, const CUtensorMap* __restrict__ tmaps) {
    int lo = 0, hi = L.njobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (L.cta_begin[mid] <= (int)blockIdx.x) lo = mid;
        else hi = mid - 1;
    }
    const MultiJob& J = *L.tmpl[lo];
    const CUtensorMap* tm = tmaps + kMapsPerPlan * J.plan;
    if constexpr (MODE == kModeForward) {   // arguments copied as in step_kernel_multi
        const StepArgs a = J.a;
        step_body<ORDER, EXACT, MODE, RZ, WZ>(tm, tm + 1, tm + 2, a, L.dyn[lo], J.nbc,
                                              blockIdx.x - L.cta_begin[lo]);
    } else {
        __shared__ StepArgs a;
        copy_args(a, J.a);
        step_body<ORDER, EXACT, MODE, RZ, WZ>(tm, tm + 1, tm + 2, a, L.dyn[lo], J.nbc,
                                              blockIdx.x - L.cta_begin[lo]);
    }
}

// ---------------------------------------------------------------------------
// launch dispatch
// ---------------------------------------------------------------------------

// A launch request: one plan (tensor maps + args in parameter space) or
// several (job table + tensor maps in device memory); configure_only sets
// the kernels' attributes and launches nothing.
struct LaunchReq {
    const CUtensorMap* t2 = nullptr;
    const CUtensorMap* t1 = nullptr;
    const CUtensorMap* tv = nullptr;
    const StepArgs* a = nullptr;
    const MultiJob* jobs = nullptr;
    const int* begins = nullptr;
    int njobs = 0;
    long long nctas = 0;
    const CUtensorMap* tmaps = nullptr;
    const EngineLaunch* engine = nullptr;
    const PersistLaunch* persist = nullptr;
    bool multi = false;
    bool chained = false;   // multi: a later launch of a chain
    bool configure_only = false;
    int* occupancy = nullptr;   // set: CTAs per SM of the one-plan kernel, nothing launched
};

template <int ORDER, int RZ, int WZ>
int ctas_of(const StepArgs& a, int* nbc_out) {
    using S = Smem<ORDER, RZ, WZ>;
    const long long ngroups = (a.nshots + a.spc - 1) / a.spc;
    const int nb = boundary_cells(ORDER, a.dimx, a.dimz);
    const int nbc = (nb + kThreads * kBoundaryCellsPerThread - 1) / (kThreads * kBoundaryCellsPerThread);
    const long long tiles = (long long)((a.dimx + kTileX - 1) / kTileX) * ((a.dimz + S::TZ - 1) / S::TZ);
    if (nbc_out) *nbc_out = nbc;
    const long long n = ngroups * (nbc + tiles);
    return n > 0x7fffffffLL ? -1 : (int)n;
}

// Set the dynamic shared-memory limit of both kernels of one instantiation on
// the current device (once per device; done before any stream capture).
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
cudaError_t configure_one() {
    using S = Smem<ORDER, RZ, WZ>;
    // one bit per device; setting an attribute twice is harmless, but plans
    // may be created from several host threads
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev >= 64 || (configured.load(std::memory_order_relaxed) & (1ull << dev))) return cudaSuccess;
    e = cudaFuncSetAttribute(step_kernel<ORDER, EXACT, MODE, RZ, WZ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(step_kernel_persistent<ORDER, EXACT, MODE, RZ, WZ>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
    if (e != cudaSuccess) return e;
    if constexpr (MODE <= kModeAdjoint) {   // multi-plan kernels: modes 0-2
        e = cudaFuncSetAttribute(step_kernel_multi<ORDER, EXACT, MODE, RZ, WZ>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(step_kernel_engine<ORDER, EXACT, MODE, RZ, WZ>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
    }
    if (e == cudaSuccess) configured.fetch_or(1ull << dev, std::memory_order_relaxed);
    return e;
}

template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
cudaError_t launch_one(const LaunchReq& q, cudaStream_t stream) {
    using S = Smem<ORDER, RZ, WZ>;
    cudaError_t e = configure_one<ORDER, EXACT, MODE, RZ, WZ>();
    if (e != cudaSuccess || q.configure_only) return e;
    if (q.occupancy)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(q.occupancy, step_kernel<ORDER, EXACT, MODE, RZ, WZ>,
                                                             WZ * 32, S::BYTES);
    if (q.persist) {
        const long long items = (long long)q.persist->nsteps * q.persist->ngroups * q.persist->per_group;
        int grid = 0;
        e = persistent_grid(step_kernel_persistent<ORDER, EXACT, MODE, RZ, WZ>, WZ * 32, S::BYTES, items, &grid,
                            q.persist->max_ctas);
        if (e != cudaSuccess) return e;
        step_kernel_persistent<ORDER, EXACT, MODE, RZ, WZ>
            <<<dim3((unsigned)grid), WZ * 32, S::BYTES, stream>>>(*q.t2, *q.t1, *q.tv, *q.persist);
        return cudaGetLastError();
    }
    if (q.engine || q.multi) {
        if constexpr (MODE > kModeAdjoint) {
            return cudaErrorInvalidValue;   // excitation amplitude, reverse: single-plan launches only
        } else {
            if (q.nctas <= 0 || q.nctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
            if (q.engine)
                step_kernel_engine<ORDER, EXACT, MODE, RZ, WZ>
                    <<<dim3((unsigned)q.nctas), WZ * 32, S::BYTES, stream>>>(*q.engine, q.tmaps);
            else if (q.chained)
                return launch_chained(step_kernel_multi<ORDER, EXACT, MODE, RZ, WZ>, (int)q.nctas, WZ * 32,
                                      S::BYTES, stream, q.jobs, q.begins, q.njobs, q.tmaps);
            else
                step_kernel_multi<ORDER, EXACT, MODE, RZ, WZ>
                    <<<dim3((unsigned)q.nctas), WZ * 32, S::BYTES, stream>>>(q.jobs, q.begins, q.njobs, q.tmaps);
        }
    } else {
        int nbc = 0;
        const int n = ctas_of<ORDER, RZ, WZ>(*q.a, &nbc);
        if (n <= 0) return cudaErrorInvalidConfiguration;
        if (q.a->chain != nullptr && q.a->chain_k > 0)
            return launch_chained(step_kernel<ORDER, EXACT, MODE, RZ, WZ>, n, WZ * 32, S::BYTES, stream,
                                  *q.t2, *q.t1, *q.tv, *q.a, nbc);
        step_kernel<ORDER, EXACT, MODE, RZ, WZ>
            <<<dim3((unsigned)n), WZ * 32, S::BYTES, stream>>>(*q.t2, *q.t1, *q.tv, *q.a, nbc);
    }
    return cudaGetLastError();
}

template <int ORDER, bool EXACT, int MODE>
cudaError_t launch_shape(LaunchShape sh, const LaunchReq& q, cudaStream_t st) {
    if (sh.warps == 4 && sh.rows_per_warp == 2) return launch_one<ORDER, EXACT, MODE, 2, 4>(q, st);
    if (sh.warps == 4 && sh.rows_per_warp == 4) return launch_one<ORDER, EXACT, MODE, 4, 4>(q, st);
    if (sh.warps == 4 && sh.rows_per_warp == 8) return launch_one<ORDER, EXACT, MODE, 8, 4>(q, st);
    return cudaErrorInvalidValue;
}

template <int ORDER, bool EXACT>
cudaError_t launch_mode(StepMode mode, LaunchShape sh, const LaunchReq& q, cudaStream_t st) {
    switch (mode) {
        case kModeForward: return launch_shape<ORDER, EXACT, kModeForward>(sh, q, st);
        case kModeRecompute: return launch_shape<ORDER, EXACT, kModeRecompute>(sh, q, st);
        case kModeAdjoint: return launch_shape<ORDER, EXACT, kModeAdjoint>(sh, q, st);
        case kModeExaForward: return launch_shape<ORDER, EXACT, kModeExaForward>(sh, q, st);
        case kModeReverse: return launch_shape<ORDER, EXACT, kModeReverse>(sh, q, st);
    }
    return cudaErrorInvalidValue;
}

template <int ORDER>
cudaError_t launch_arith(bool exact, StepMode mode, LaunchShape sh, const LaunchReq& q,
                         cudaStream_t st) {
    return exact ? launch_mode<ORDER, true>(mode, sh, q, st)
                 : launch_mode<ORDER, false>(mode, sh, q, st);
}

cudaError_t launch_req(int order, bool exact, StepMode mode, LaunchShape shape, const LaunchReq& q,
                       cudaStream_t st) {
    switch (order) {
        case 2: return launch_arith<2>(exact, mode, shape, q, st);
        case 4: return launch_arith<4>(exact, mode, shape, q, st);
        case 8: return launch_arith<8>(exact, mode, shape, q, st);
    }
    return cudaErrorInvalidValue;
}

// ---------------------------------------------------------------------------
// model padding and gradient reduction (32x32 shared-memory transposes)
// ---------------------------------------------------------------------------

__global__ void pad_model_kernel(const float* __restrict__ vel, float* __restrict__ vpad, int nx,
                                 int nz, int ne, int dimx, int dimz, int pitch) {
    __shared__ float tile[32][33];
    const int r0 = blockIdx.y * 32, c0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
    // read: consecutive threads walk z (contiguous in the user layout)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int cl = ty + 8 * j;
        const int col = c0 + cl, row = r0 + tx;
        const int ix = min(max(col - ne, 0), nx - 1);
        const int iz = min(max(row - ne, 0), nz - 1);
        tile[cl][tx] = vel[(long long)ix * nz + iz];
    }
    __syncthreads();
    // write: consecutive threads walk x (contiguous in the padded layout)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int rl = ty + 8 * j;
        const int row = r0 + rl, col = c0 + tx;
        if (row < dimz && col < pitch)
            vpad[(long long)row * pitch + col] = col < dimx ? tile[tx][rl] : 0.f;
    }
}

struct IntChunk {
    int n;
    int v[2048];
};

__global__ void store_ints_kernel(int* __restrict__ dst, const __grid_constant__ IntChunk c) {
    for (int i = threadIdx.x; i < c.n; i += blockDim.x) dst[i] = c.v[i];
}

__global__ void reduce_grad_kernel(const float* __restrict__ acc, const float* __restrict__ comp,
                                   int nacc, long long slot_elems, int pitch, int ne, int nx,
                                   int nz, int kahan, float* __restrict__ out) {
    __shared__ float tile[32][33];
    const int z0 = blockIdx.y * 32, x0 = blockIdx.x * 32;
    const int tx = threadIdx.x, ty = threadIdx.y;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int zl = ty + 8 * j;
        const int iz = z0 + zl, ix = x0 + tx;
        float g = 0.f;
        if (iz < nz && ix < nx) {
            const long long off = (long long)(iz + ne) * pitch + (ix + ne);
            if (kahan) {
                float s = 0.f, cc = 0.f;
                for (int k = 0; k < nacc; ++k) {
                    kahan_add(s, cc, acc[k * slot_elems + off]);
                    kahan_add(s, cc, -comp[k * slot_elems + off]);
                }
                g = __fsub_rn(s, cc);
            } else {
                g = acc[off];
                for (int k = 1; k < nacc; ++k) g = __fadd_rn(g, acc[k * slot_elems + off]);
            }
        }
        tile[zl][tx] = g;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int xl = ty + 8 * j;
        const int ix = x0 + xl, iz = z0 + tx;
        if (ix < nx && iz < nz) out[(long long)ix * nz + iz] = tile[tx][xl];
    }
}

// residual = modelled - observed in place, one FP32 subtraction per sample
// (the bits of the forward kernel's fused residual and of torch's frd - obs).
__global__ void residual_kernel(float* __restrict__ frd, const float* __restrict__ obs, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        frd[i] = __fsub_rn(frd[i], obs[i]);
}

// Misfit, pass 1: a fixed grid of kMisfitBlocks blocks; block b sums, in
// FP64, the squares of the float4 groups b, b + grid, ... (thread-strided,
// then a fixed tree), so the result does not depend on timing.
__global__ void __launch_bounds__(256) misfit_partial_kernel(const float* __restrict__ r, long long n,
                                                             double* __restrict__ partial) {
    __shared__ double sh[256];
    double acc = 0.0;
    const long long n4 = n / 4;
    const float4* r4 = reinterpret_cast<const float4*>(r);
    for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n4; i += (long long)gridDim.x * 256) {
        const float4 v = r4[i];
        acc += (double)v.x * v.x + (double)v.y * v.y + (double)v.z * v.z + (double)v.w * v.w;
    }
    if (blockIdx.x == 0 && threadIdx.x < n - 4 * n4) {
        const double v = r[4 * n4 + threadIdx.x];
        acc += v * v;
    }
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = sh[0];
}

// Misfit, pass 2: one block adds the partial sums in a fixed order.
__global__ void __launch_bounds__(256) misfit_final_kernel(const double* __restrict__ partial, int np,
                                                           double* __restrict__ misfit) {
    __shared__ double sh[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += 256) acc += partial[i];
    sh[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) sh[threadIdx.x] += sh[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *misfit = 0.5 * sh[0];
}

}  // namespace

cudaError_t launch_misfit(const float* r, long long n, double* partial, double* misfit,
                          cudaStream_t stream) {
    if (reinterpret_cast<uintptr_t>(r) % 16 != 0) return cudaErrorMisalignedAddress;
    misfit_partial_kernel<<<kMisfitBlocks, 256, 0, stream>>>(r, n, partial);
    misfit_final_kernel<<<1, 256, 0, stream>>>(partial, kMisfitBlocks, misfit);
    return cudaGetLastError();
}

cudaError_t launch_residual(float* frd, const float* obs, long long n, cudaStream_t stream) {
    residual_kernel<<<kMisfitBlocks, 256, 0, stream>>>(frd, obs, n);
    return cudaGetLastError();
}

cudaError_t launch_step(int order, bool exact, StepMode mode, LaunchShape shape,
                        const CUtensorMap& tm_u2, const CUtensorMap& tm_u1,
                        const CUtensorMap& tm_vel, const StepArgs& a, cudaStream_t stream) {
    LaunchReq q;
    q.t2 = &tm_u2, q.t1 = &tm_u1, q.tv = &tm_vel, q.a = &a;
    return launch_req(order, exact, mode, shape, q, stream);
}

cudaError_t launch_step_multi(int order, bool exact, StepMode mode, LaunchShape shape,
                              const MultiJob* jobs, const int* begins, int njobs, long long nctas,
                              const CUtensorMap* tmaps, cudaStream_t stream, bool chained) {
    LaunchReq q;
    q.multi = true, q.jobs = jobs, q.begins = begins, q.njobs = njobs, q.nctas = nctas, q.tmaps = tmaps;
    q.chained = chained;
    return launch_req(order, exact, mode, shape, q, stream);
}

cudaError_t launch_step_persistent(int order, bool exact, StepMode mode, LaunchShape shape,
                                   const CUtensorMap& tm_u2, const CUtensorMap& tm_u1,
                                   const CUtensorMap& tm_vel, const PersistLaunch& P,
                                   cudaStream_t stream) {
    LaunchReq q;
    q.t2 = &tm_u2, q.t1 = &tm_u1, q.tv = &tm_vel, q.persist = &P;
    return launch_req(order, exact, mode, shape, q, stream);
}

cudaError_t launch_step_engine(int order, bool exact, StepMode mode, LaunchShape shape,
                               const EngineLaunch& L, long long nctas, const CUtensorMap* tmaps,
                               cudaStream_t stream) {
    LaunchReq q;
    q.engine = &L, q.nctas = nctas, q.tmaps = tmaps;
    return launch_req(order, exact, mode, shape, q, stream);
}

int step_resident_ctas(int order, bool exact, StepMode mode, LaunchShape shape) {
    int n = 0;
    LaunchReq q;
    q.occupancy = &n;
    return launch_req(order, exact, mode, shape, q, nullptr) == cudaSuccess ? n : 0;
}

int step_ctas(int order, LaunchShape shape, const StepArgs& a, int* nbc) {
    const int rz = shape.rows_per_warp;
    switch (order) {
        case 2: return rz == 8 ? ctas_of<2, 8, 4>(a, nbc) : rz == 2 ? ctas_of<2, 2, 4>(a, nbc) : ctas_of<2, 4, 4>(a, nbc);
        case 4: return rz == 8 ? ctas_of<4, 8, 4>(a, nbc) : rz == 2 ? ctas_of<4, 2, 4>(a, nbc) : ctas_of<4, 4, 4>(a, nbc);
        case 8: return rz == 8 ? ctas_of<8, 8, 4>(a, nbc) : rz == 2 ? ctas_of<8, 2, 4>(a, nbc) : ctas_of<8, 4, 4>(a, nbc);
    }
    return -1;
}

cudaError_t prepare_step(int order, bool exact, LaunchShape shape) {
    LaunchReq q;
    q.configure_only = true;
    for (StepMode m : {kModeForward, kModeRecompute, kModeAdjoint, kModeExaForward, kModeReverse}) {
        cudaError_t e = launch_req(order, exact, m, shape, q, nullptr);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_pad_model(const float* vel_user, float* vpad, int nx, int nz, int ne,
                             int dimx, int dimz, int pitch, cudaStream_t stream) {
    dim3 grid((pitch + 31) / 32, (dimz + 31) / 32);
    pad_model_kernel<<<grid, dim3(32, 8), 0, stream>>>(vel_user, vpad, nx, nz, ne, dimx, dimz, pitch);
    return cudaGetLastError();
}

cudaError_t launch_store_ints(int* dst, const int* src, int n, cudaStream_t stream) {
    IntChunk c;
    for (int off = 0; off < n; off += 2048) {
        c.n = n - off < 2048 ? n - off : 2048;
        for (int i = 0; i < c.n; ++i) c.v[i] = src[off + i];
        store_ints_kernel<<<1, 256, 0, stream>>>(dst + off, c);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_reduce_grad(const float* acc, const float* acc_comp, int nacc,
                               long long slot_elems, int pitch, int ne, int nx, int nz,
                               int kahan, float* grad_user, cudaStream_t stream) {
    dim3 grid((nx + 31) / 32, (nz + 31) / 32);
    reduce_grad_kernel<<<grid, dim3(32, 8), 0, stream>>>(acc, acc_comp, nacc, slot_elems, pitch, ne,
                                                        nx, nz, kahan, grad_user);
    return cudaGetLastError();
}

}  // namespace twi
