// twi_backward.cu -- the fused backward step of boundary-saving plans.
//
// The reference's adjoint loop (propagator_cpu.cpp:82-152) reads the virtual
// source of every step from an nt x dimxy history that its forward pass
// wrote (propagator_cpu.cpp:68-72).  A boundary-saving plan keeps only the
// Keys cells of every time level and rebuilds the forward field backwards
// in time, in the same direction as the adjoint, so one launch per step
// does both:
//   * u^{it-1} = (vv*Lap(u^it) + 2u^it) - (u^{it+1} - source_it) on the
//     interior (the forward update read backwards), the Keys cells of
//     u^{it-1} restored from the boundary buffer, the top rows zero;
//   * the virtual source of step it, q * ((u^{it-1} - 2u^it) + u^{it+1}),
//     q = -2/(dt^2 v^3), formed in registers and never stored;
//   * the lambda step it (stencil, adjoint source on the receiver row,
//     Keys on the pads, td2d_cpu.cpp:31-146);
//   * the gradient term -virt * lambda accumulated in Kahan pairs held in
//     registers across the CTA's shot group, or in plain per-shot sums.
// A CTA owns a 128-column x TZ-row tile and a group of shots; per shot it
// stages u^it and lambda^it (4-column / HZ-row halo) and u^{it+1} and
// lambda^{it+1} (no halo) with four TMA loads onto one mbarrier,
// double-buffered across the shots.  The arithmetic of each part is the
// step kernel's (twi_cell.cuh), so the result equals the reverse launch
// followed by the adjoint launch bit for bit.
#include <atomic>
#include <type_traits>

#include "twi_cell.cuh"
#include "twi_kernels.h"
#include "twi_persist.cuh"
#include "twi_ptx.cuh"
#include "twi_tile.cuh"

namespace twi {
namespace {

// 2 rows per warp: four CTAs (16 warps) per SM fit the shared memory;
// 4 rows: two.
constexpr int kBackCtasPerSm(int rz) { return rz == 2 ? 4 : 2; }

template <int ORDER, int RZ, int WZ>
struct BackSmem {
    static constexpr int NE = ORDER / 2;
    static constexpr int TZ = RZ * WZ;
    static constexpr int HZ = zhalo(ORDER);
    static constexpr int C_ROWS = TZ + 2 * HZ;                 // level it, with halo
    static constexpr int C_FLOATS = round32(C_ROWS * kBoxX);
    static constexpr int P_FLOATS = TZ * kTileX;              // level it+1, no halo
    static constexpr int FIELD_FLOATS = C_FLOATS + P_FLOATS;
    static constexpr int STAGE_FLOATS = 2 * FIELD_FLOATS;     // u, then lambda
    static constexpr int V_FLOATS = TZ * kTileX;
    static constexpr int STAGES = 2;
    static constexpr int BAR_BYTES = 128;
    static constexpr size_t BYTES =
        128 /*alignment slack*/ + BAR_BYTES + size_t(V_FLOATS + STAGES * STAGE_FLOATS) * 4;
    static constexpr uint32_t STAGE_TX = 2 * (C_ROWS * kBoxX * 4 + TZ * kTileX * 4);
    static constexpr uint32_t V_TX = TZ * kTileX * 4;
};

__device__ __forceinline__ long long slot_off(const StepArgs& a, int base, int stride, int s) {
    return (long long)(base + s * stride) * a.slot_elems;
}

// Boundary CTAs: a strided share of the Keys cells of one shot group, one
// thread per cell: u^{it-1} from the boundary buffer, the Keys update of
// lambda, and for plain per-shot sums the gradient term (Kahan sums cover the
// model cells only; every caller crops the pads).
template <int ORDER, bool EXACT>
__device__ __forceinline__ void backward_boundary(const StepArgs& a, int b, int nbc) {
    constexpr int NE = ORDER / 2;
    const int grp = b / nbc, part = b - grp * nbc;
    const int s0 = grp * a.spc, s1 = min(s0 + a.spc, a.nshots);
    const int nb = boundary_cells(ORDER, a.dimx, a.dimz);
    const bool plain = a.acc_mode == kAccPlainPerShot;
    if (a.chain != nullptr) {
        __shared__ int sh_go;
        if (threadIdx.x == 0) sh_go = chain_wait(a, grp);
        __syncthreads();
        if (!sh_go) return;
    }
    for (int idx = part * blockDim.x + threadIdx.x; idx < nb; idx += nbc * blockDim.x) {
        int r, c;
        long long db;   // offset to the first cell inwards
        boundary_cell_at<NE>(idx, a.dimx, a.dimz, a.pitch, r, c, db);
        const long long cell = (long long)r * a.pitch + c;
        const float v = a.vel[cell];
        const float q = virt_coef<EXACT>(v, a.cons);
        for (int s = s0; s < s1; ++s) {
            const float uc = a.fields[slot_off(a, a.cur_base, a.cur_stride, s) + cell];
            const float up = a.fields[slot_off(a, a.prev_base, a.prev_stride, s) + cell];
            // u^{it-1} as the forward pass saved it (u^0 = u^{-1} = 0)
            const float un =
                a.it >= 2 ? a.bnd[((long long)(a.it - 1) * a.nshots + s) * a.bnd_cells + idx] : 0.f;
            a.fields[slot_off(a, a.next_base, a.next_stride, s) + cell] = un;
            const float* L2 = a.fields + slot_off(a, a.lcur_base, a.lcur_stride, s) + cell;
            const float* L1 = a.fields + slot_off(a, a.lprev_base, a.lprev_stride, s) + cell;
            const float ln = keys_cell<EXACT>(L2[0], L2[db], L2[2 * db], L1[0], L1[db], v, a.h2,
                                              a.dt2, a.hdt);
            a.fields[slot_off(a, a.lnext_base, a.lnext_stride, s) + cell] = ln;
            if (plain) {
                float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems + cell;
                *g = __fadd_rn(*g, grad_term<EXACT>(virt_from_coef<EXACT>(q, un, uc, up), ln));
            }
        }
    }
    chain_done(a, grp);
}

// Interior update of a lane's four cells from a (2*NE+1)-row window.
template <int ORDER, bool EXACT>
__device__ __forceinline__ void update4(const float4 (&win)[ORDER + 1], const float (&c4)[4],
                                        const float (&L)[ORDER / 2], const float (&R)[ORDER / 2],
                                        const float (&older)[4], const float4& vv, float (&out)[4]) {
    constexpr int NE = ORDER / 2;
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float lf[NE], rt[NE], up[NE], dn[NE];
#pragma unroll
        for (int dist = 1; dist <= NE; ++dist) {
            const int jl = m - dist, jr = m + dist;
            lf[dist - 1] = jl >= 0 ? c4[jl] : L[-jl - 1];
            rt[dist - 1] = jr < 4 ? c4[jr] : R[jr - 4];
            up[dist - 1] = comp(win[NE - dist], m);
            dn[dist - 1] = comp(win[NE + dist], m);
        }
        out[m] = interior_update<ORDER, EXACT>(lf, rt, up, dn, c4[m], older[m], comp(vv, m));
    }
}

// One CTA of one backward step: `cta` indexes the step's CTAs, boundary
// CTAs first, then the interior tiles.
template <int ORDER, bool EXACT, int RZ, int WZ>
__device__ __forceinline__ void backward_body(const CUtensorMap* tm_c, const CUtensorMap* tm_p,
                                              const CUtensorMap* tm_vel, const StepArgs& a,
                                              const int nbc, const int cta_in) {
    using S = BackSmem<ORDER, RZ, WZ>;
    constexpr int NE = S::NE, HZ = S::HZ, TZ = S::TZ, STAGES = S::STAGES;

    allow_next_launch();
    const int ngroups = (a.nshots + a.spc - 1) / a.spc;
    const int tiles_x = (a.dimx + kTileX - 1) / kTileX;
    const int tiles_z = (a.dimz + TZ - 1) / TZ;
    const int cta = chain_order(a, cta_in, nbc, ngroups, tiles_x * tiles_z);
    if (cta < nbc * ngroups) {
        backward_boundary<ORDER, EXACT>(a, cta, nbc);
        return;
    }
    const int m_id = cta - nbc * ngroups;
    const int tile_x = m_id % tiles_x;
    const int tile_z = (m_id / tiles_x) % tiles_z;
    const int grp = m_id / (tiles_x * tiles_z);

    extern __shared__ unsigned char smem_raw[];
    unsigned char* sbase = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase);   // [0] velocity, [1+i] stage i
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
        sh_src_r[threadIdx.x] = a.src_rc[2 * s];
        sh_src_c[threadIdx.x] = a.src_rc[2 * s + 1];
        sh_rec_r[threadIdx.x] = a.rec_row[s];
        sh_wamp[threadIdx.x] = a.wav[(long long)s * a.wav_stride + a.it];
    }
    auto issue = [&](int k) {
        const int s = s_begin + k;
        float* st = stage0 + (k % STAGES) * S::STAGE_FLOATS;
        uint64_t* b = &bar[1 + (k % STAGES)];
        mbar_arrive_expect_tx(b, S::STAGE_TX);
        tma_load_3d(st, tm_c, x0 - kHaloX, z0 - HZ, a.cur_base + s * a.cur_stride, b);
        tma_load_3d(st + S::C_FLOATS, tm_p, x0, z0, a.prev_base + s * a.prev_stride, b);
        tma_load_3d(st + S::FIELD_FLOATS, tm_c, x0 - kHaloX, z0 - HZ, a.lcur_base + s * a.lcur_stride, b);
        tma_load_3d(st + S::FIELD_FLOATS + S::C_FLOATS, tm_p, x0, z0, a.lprev_base + s * a.lprev_stride, b);
    };
    // Thread 0 sets up the stage barriers, issues the static velocity tile
    // and, when the launch waits for nothing, the first stages; meanwhile
    // lane 0 of warp 1 waits for the chain, if any, so that a chained
    // launch's field copies go out right after the CTA barrier.
    const bool chained_wait = a.chain != nullptr && a.chain_k > 0;
    __shared__ int sh_chain_ok;
    if (threadIdx.x == 0) {
        prefetch_tmap(tm_c);
        prefetch_tmap(tm_p);
        prefetch_tmap(tm_vel);
#pragma unroll
        for (int i = 0; i < 1 + STAGES; ++i) mbar_init(&bar[i], 1);
        fence_barrier_init();
        mbar_arrive_expect_tx(&bar[0], S::V_TX);
        tma_load_2d(vs, tm_vel, x0, z0, &bar[0]);
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
    const int cs = kHaloX + 4 * lane;    // its column in a haloed row
    const bool col_ok = c < a.dimx;
    const bool cols_interior = c >= NE && c + 3 < a.dimx - NE;
    bool cell_in[4];                     // per-cell interior column mask
#pragma unroll
    for (int m = 0; m < 4; ++m) cell_in[m] = c + m >= NE && c + m < a.dimx - NE;
    const bool kahan = a.acc_mode == kAccKahanPerGroup;

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
    // per-cell constants over all shots: v*v*dt^2/h^2 and the virtual-source
    // coefficient (columns past the grid hold v = 0: kept finite, never stored)
    float4 vvreg[RZ], qreg[RZ];
#pragma unroll
    for (int rr = 0; rr < RZ; ++rr) {
        const float4 v4 = ld4(vs + (rl0 + rr) * kTileX + 4 * lane);
        vvreg[rr] = make_float4(vv_of<EXACT>(v4.x, a.dtoh2), vv_of<EXACT>(v4.y, a.dtoh2),
                                vv_of<EXACT>(v4.z, a.dtoh2), vv_of<EXACT>(v4.w, a.dtoh2));
        qreg[rr] = make_float4(virt_coef<EXACT>(v4.x != 0.f ? v4.x : 1.f, a.cons),
                               virt_coef<EXACT>(v4.y != 0.f ? v4.y : 1.f, a.cons),
                               virt_coef<EXACT>(v4.z != 0.f ? v4.z : 1.f, a.cons),
                               virt_coef<EXACT>(v4.w != 0.f ? v4.w : 1.f, a.cons));
    }

    // Kahan pairs of this CTA's shot group
    float4 gsum[RZ], gcmp[RZ];
#pragma unroll
    for (int rr = 0; rr < RZ; ++rr) {
        gsum[rr] = gcmp[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
        const int r = z0 + rl0 + rr;
        if (kahan && col_ok && r < a.dimz) {
            const long long off = (long long)(a.acc_base + grp) * a.slot_elems + (long long)r * a.pitch + c;
            gsum[rr] = ld4(a.acc + off);
            gcmp[rr] = ld4(a.acc_comp + off);
        }
    }

    for (int k = 0; k < nloc; ++k) {
        const int s = s_begin + k;
        const float* uc_s = stage0 + (k % STAGES) * S::STAGE_FLOATS;   // u^it, haloed
        const float* up_s = uc_s + S::C_FLOATS;                         // u^{it+1}
        const float* lc_s = uc_s + S::FIELD_FLOATS;                     // lambda^it, haloed
        const float* lp_s = lc_s + S::C_FLOATS;                         // lambda^{it+1}

        const int src_r = sh_src_r[k], src_c = sh_src_c[k], rec_r = sh_rec_r[k];
        const float wamp = sh_wamp[k];

        if (!warp_wait_stage(&bar[1 + (k % STAGES)], (k / STAGES) & 1)) {
            // the copies never landed: flag it, wait (bounded) for the copies
            // this warp may have issued, and leave
            if (lane == 0) {
                atomicOr(a.err, 1);
                drain_stages(&bar[1], STAGES, k, min(nloc, k + STAGES));
            }
            return;
        }

        float4 wu[2 * NE + 1], wl[2 * NE + 1];
#pragma unroll
        for (int j = 0; j < 2 * NE; ++j) {
            wu[j] = ld4(uc_s + (rl0 + HZ - NE + j) * kBoxX + cs);
            wl[j] = ld4(lc_s + (rl0 + HZ - NE + j) * kBoxX + cs);
        }

        float* const un_slot = a.fields + slot_off(a, a.next_base, a.next_stride, s);
        float* const ln_slot = a.fields + slot_off(a, a.lnext_base, a.lnext_stride, s);
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
                if constexpr (!PLAIN) {
                    if (r >= a.dimz - NE) break;
                }
                wu[2 * NE] = ld4(uc_s + (rl + HZ + NE) * kBoxX + cs);
                wl[2 * NE] = ld4(lc_s + (rl + HZ + NE) * kBoxX + cs);
                const long long roff = (long long)r * a.pitch + c;
                // One interior row.  FAST: neither the source nor the receiver
                // row, so no per-row special case is tested; in the edge tiles the
                // lanes holding pad columns mask their stores.
                auto interior_row = [&](auto fast_tag) {
                    constexpr bool FAST = decltype(fast_tag)::value;
                    // ---- u^{it-1}: the forward update run backwards
                    const float cu[4] = {wu[NE].x, wu[NE].y, wu[NE].z, wu[NE].w};
                    float Lu[NE], Ru[NE];
                    row_neighbours<NE>(uc_s + (rl + HZ) * kBoxX, cs, Lu, Ru);
                    const float4 up4 = ld4(up_s + rl * kTileX + 4 * lane);
                    const float up[4] = {up4.x, up4.y, up4.z, up4.w};
                    // u^{it+1} with the source that step `it` added taken off again
                    float ui[4] = {up[0], up[1], up[2], up[3]};
                    if (!FAST && r == src_r && src_c >= c && src_c < c + 4) {
                        const float4 v4 = ld4(vs + rl * kTileX + 4 * lane);
#pragma unroll
                        for (int m = 0; m < 4; ++m)
                            if (c + m == src_c) ui[m] = __fsub_rn(up[m], injection<EXACT>(wamp, comp(v4, m), a.dt2));
                    }
                    float uo[4];
                    update4<ORDER, EXACT>(wu, cu, Lu, Ru, ui, vvreg[rr], uo);
                    if (a.it < 2) {   // u^0 = u^{-1} = 0 exactly
#pragma unroll
                        for (int m = 0; m < 4; ++m) uo[m] = 0.f;
                    }

                    // ---- lambda step it
                    const float cl[4] = {wl[NE].x, wl[NE].y, wl[NE].z, wl[NE].w};
                    float Ll[NE], Rl[NE];
                    row_neighbours<NE>(lc_s + (rl + HZ) * kBoxX, cs, Ll, Rl);
                    const float4 lp4 = ld4(lp_s + rl * kTileX + 4 * lane);
                    const float lp[4] = {lp4.x, lp4.y, lp4.z, lp4.w};
                    float lo[4];
                    update4<ORDER, EXACT>(wl, cl, Ll, Rl, lp, vvreg[rr], lo);
                    if (!FAST && r == rec_r) {   // adjoint source on the receiver row
                        const float4 v4 = ld4(vs + rl * kTileX + 4 * lane);
                        const float* rs = a.resid + (long long)s * a.resid_stride + (long long)a.it * a.nx;
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const int cc = c + m;
                            if (cc >= NE && cc < NE + a.nx)
                                lo[m] = add_injection<EXACT>(lo[m], rs[cc - NE], comp(v4, m), a.dt2);
                        }
                    }

                    // pad columns belong to the boundary CTAs: store interior cells only
                    if (cols_interior) {
                        *reinterpret_cast<float4*>(un_slot + roff) = make_float4(uo[0], uo[1], uo[2], uo[3]);
                        *reinterpret_cast<float4*>(ln_slot + roff) = make_float4(lo[0], lo[1], lo[2], lo[3]);
                    } else {
#pragma unroll
                        for (int m = 0; m < 4; ++m)
                            if (cell_in[m]) un_slot[roff + m] = uo[m], ln_slot[roff + m] = lo[m];
                    }

                    // ---- gradient: -virt * lambda with the virtual source of step it
                    if (kahan) {
                        // every column: the pairs of pad cells and of columns
                        // past the grid are never read (callers crop the pads)
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const float vt = virt_from_coef<EXACT>(comp(qreg[rr], m), uo[m], cu[m], up[m]);
                            float sm = comp(gsum[rr], m), cm = comp(gcmp[rr], m);
                            kahan_add(sm, cm, grad_term<EXACT>(vt, lo[m]));
                            set_comp(gsum[rr], m, sm);
                            set_comp(gcmp[rr], m, cm);
                        }
                    } else {
                        float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems + roff;
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            if (cell_in[m]) {
                                const float vt = virt_from_coef<EXACT>(comp(qreg[rr], m), uo[m], cu[m], up[m]);
                                g[m] = __fadd_rn(g[m], grad_term<EXACT>(vt, lo[m]));
                            }
                        }
                    }
                };
                if constexpr (PLAIN) {
                    interior_row(std::true_type{});
                } else if (r < NE) {
                    // free surface: both fields stay zero (the reference never writes these rows)
                    if (col_ok) {
                        *reinterpret_cast<float4*>(un_slot + roff) = make_float4(0.f, 0.f, 0.f, 0.f);
                        *reinterpret_cast<float4*>(ln_slot + roff) = make_float4(0.f, 0.f, 0.f, 0.f);
                    }
                } else if (r != src_r && r != rec_r) {
                    interior_row(std::true_type{});
                } else {
                    interior_row(std::false_type{});
                }
#pragma unroll
                for (int j = 0; j < 2 * NE; ++j) wu[j] = wu[j + 1], wl[j] = wl[j + 1];
            }
        };
        const int rw0 = z0 + rl0;   // first row of this warp
        if (rw0 >= NE && rw0 + RZ <= a.dimz - NE && (src_r < rw0 || src_r >= rw0 + RZ) &&
            (rec_r < rw0 || rec_r >= rw0 + RZ))
            rows(std::true_type{});
        else
            rows(std::false_type{});

        if (last_warp_done(sh_done, k, STAGES, WZ) && k + STAGES < nloc) issue(k + STAGES);
    }

    if (kahan) {
#pragma unroll
        for (int rr = 0; rr < RZ; ++rr) {
            const int r = z0 + rl0 + rr;
            if (col_ok && r < a.dimz) {
                const long long off = (long long)(a.acc_base + grp) * a.slot_elems + (long long)r * a.pitch + c;
                *reinterpret_cast<float4*>(a.acc + off) = gsum[rr];
                *reinterpret_cast<float4*>(a.acc_comp + off) = gcmp[rr];
            }
        }
    }
    chain_done(a, grp);
}

template <int ORDER, bool EXACT, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kBackCtasPerSm(RZ))
backward_kernel(const __grid_constant__ CUtensorMap tm_c, const __grid_constant__ CUtensorMap tm_p,
                const __grid_constant__ CUtensorMap tm_vel, const __grid_constant__ StepArgs a,
                const int nbc) {
    backward_body<ORDER, EXACT, RZ, WZ>(&tm_c, &tm_p, &tm_vel, a, nbc, blockIdx.x);
}

// Backward steps of several plans in one launch: CTA ranges of the jobs are
// contiguous and ascending; a job reads its plan's adjoint-height tensor maps
// (tmaps[6p + 3 .. 6p + 5]).  The arguments are copied to shared memory so
// that the body does not re-read them from global memory after its stores.
template <int ORDER, bool EXACT, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kBackCtasPerSm(RZ))
backward_kernel_multi(const MultiJob* __restrict__ jobs, const int* __restrict__ begins, const int njobs,
                      const CUtensorMap* __restrict__ tmaps) {
    const int lo = job_of([&](int i) { return begins[i]; }, njobs, (int)blockIdx.x);
    const MultiJob& J = jobs[lo];
    const CUtensorMap* tm = tmaps + kMapsPerPlan * J.plan + 3;
    __shared__ StepArgs a;
    copy_args(a, J.a);
    backward_body<ORDER, EXACT, RZ, WZ>(tm, tm + 1, tm + 2, a, J.nbc, blockIdx.x - J.cta_begin);
}

// Engine launches: job ranges and per-step slots from the kernel parameters,
// the static arguments from the request's resident template.
template <int ORDER, bool EXACT, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kBackCtasPerSm(RZ))
backward_kernel_engine(const __grid_constant__ EngineLaunch L, const CUtensorMap* __restrict__ tmaps) {
    const int lo = job_of([&](int i) { return L.cta_begin[i]; }, L.njobs, (int)blockIdx.x);
    const MultiJob& J = *L.tmpl[lo];
    const CUtensorMap* tm = tmaps + kMapsPerPlan * J.plan + 3;
    __shared__ StepArgs a;
    copy_args(a, J.a);
    if (threadIdx.x == 0) apply_dyn(a, L.dyn[lo]);
    __syncthreads();
    backward_body<ORDER, EXACT, RZ, WZ>(tm, tm + 1, tm + 2, a, J.nbc, blockIdx.x - L.cta_begin[lo]);
}

// All backward steps of a pass in one launch (twi_persist.cuh).
template <int ORDER, bool EXACT, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, kBackCtasPerSm(RZ))
backward_kernel_persistent(const __grid_constant__ CUtensorMap tm_c, const __grid_constant__ CUtensorMap tm_p,
                           const __grid_constant__ CUtensorMap tm_vel, const __grid_constant__ PersistLaunch P) {
    extern __shared__ unsigned char smem_raw[];
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    persistent_loop(P, bars, 1 + BackSmem<ORDER, RZ, WZ>::STAGES, [&](const StepArgs& a, int cta) {
        backward_body<ORDER, EXACT, RZ, WZ>(&tm_c, &tm_p, &tm_vel, a, P.nbc, cta);
    });
}

template <int ORDER, int RZ, int WZ>
int back_ctas_of(const StepArgs& a, int* nbc_out) {
    using S = BackSmem<ORDER, RZ, WZ>;
    const long long ngroups = (a.nshots + a.spc - 1) / a.spc;
    const int nb = boundary_cells(ORDER, a.dimx, a.dimz);
    const int nbc = (nb + kThreads * kBoundaryCellsPerThread - 1) / (kThreads * kBoundaryCellsPerThread);
    const long long tiles = (long long)((a.dimx + kTileX - 1) / kTileX) * ((a.dimz + S::TZ - 1) / S::TZ);
    if (nbc_out) *nbc_out = nbc;
    const long long n = ngroups * (nbc + tiles);
    return n > 0x7fffffffLL ? -1 : (int)n;
}

// One launch request: a single step (tensor maps + args), a persistent pass,
// a job table or an engine launch; none of them = set the attributes only.
struct BackReq {
    const CUtensorMap* tc = nullptr;
    const CUtensorMap* tp = nullptr;
    const CUtensorMap* tv = nullptr;
    const StepArgs* a = nullptr;
    const PersistLaunch* pl = nullptr;
    const MultiJob* jobs = nullptr;
    const int* begins = nullptr;
    int njobs = 0;
    long long nctas = 0;
    const CUtensorMap* tmaps = nullptr;
    const EngineLaunch* engine = nullptr;
    bool chained = false;   // jobs: a later launch of a chain
    int* occupancy = nullptr;   // set: CTAs per SM of the one-plan kernel, nothing launched
};

template <int ORDER, bool EXACT, int RZ>
cudaError_t back_one(const BackReq& q, cudaStream_t st) {
    using S = BackSmem<ORDER, RZ, 4>;
    const CUtensorMap *tc = q.tc, *tp = q.tp, *tv = q.tv;
    const StepArgs* a = q.a;
    const PersistLaunch* pl = q.pl;
    static std::atomic<unsigned long long> configured{0};   // one bit per device
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured.load(std::memory_order_relaxed) & (1ull << dev))) {
        e = cudaFuncSetAttribute(backward_kernel<ORDER, EXACT, RZ, 4>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(backward_kernel_persistent<ORDER, EXACT, RZ, 4>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(backward_kernel_multi<ORDER, EXACT, RZ, 4>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        e = cudaFuncSetAttribute(backward_kernel_engine<ORDER, EXACT, RZ, 4>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        configured.fetch_or(1ull << dev, std::memory_order_relaxed);
    }
    if (q.occupancy)
        return cudaOccupancyMaxActiveBlocksPerMultiprocessor(q.occupancy, backward_kernel<ORDER, EXACT, RZ, 4>, 128,
                                                             S::BYTES);
    if (q.jobs || q.engine) {
        if (q.nctas <= 0 || q.nctas > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
        if (q.engine)
            backward_kernel_engine<ORDER, EXACT, RZ, 4>
                <<<dim3((unsigned)q.nctas), 128, S::BYTES, st>>>(*q.engine, q.tmaps);
        else if (q.chained)
            return launch_chained(backward_kernel_multi<ORDER, EXACT, RZ, 4>, (int)q.nctas, 128, S::BYTES, st,
                                  q.jobs, q.begins, q.njobs, q.tmaps);
        else
            backward_kernel_multi<ORDER, EXACT, RZ, 4>
                <<<dim3((unsigned)q.nctas), 128, S::BYTES, st>>>(q.jobs, q.begins, q.njobs, q.tmaps);
        return cudaGetLastError();
    }
    if (pl) {
        int grid = 0;
        e = persistent_grid(backward_kernel_persistent<ORDER, EXACT, RZ, 4>, 128, S::BYTES,
                            (long long)pl->nsteps * pl->ngroups * pl->per_group, &grid, pl->max_ctas);
        if (e != cudaSuccess) return e;
        backward_kernel_persistent<ORDER, EXACT, RZ, 4><<<dim3((unsigned)grid), 128, S::BYTES, st>>>(*tc, *tp, *tv, *pl);
        return cudaGetLastError();
    }
    if (!a) return cudaSuccess;   // configure only
    int nbc = 0;
    const int n = back_ctas_of<ORDER, RZ, 4>(*a, &nbc);
    if (n <= 0) return cudaErrorInvalidConfiguration;
    if (a->chain != nullptr && a->chain_k > 0)
        return launch_chained(backward_kernel<ORDER, EXACT, RZ, 4>, n, 128, S::BYTES, st, *tc, *tp, *tv, *a, nbc);
    backward_kernel<ORDER, EXACT, RZ, 4><<<dim3((unsigned)n), 128, S::BYTES, st>>>(*tc, *tp, *tv, *a, nbc);
    return cudaGetLastError();
}

template <int ORDER, bool EXACT>
cudaError_t back_shape(int rz, const BackReq& q, cudaStream_t st) {
    if (rz == 2) return back_one<ORDER, EXACT, 2>(q, st);
    if (rz == 4) return back_one<ORDER, EXACT, 4>(q, st);
    return cudaErrorInvalidValue;
}

cudaError_t back_dispatch(int order, bool exact, int rz, const BackReq& q, cudaStream_t st) {
    switch (order) {
        case 2: return exact ? back_shape<2, true>(rz, q, st) : back_shape<2, false>(rz, q, st);
        case 4: return exact ? back_shape<4, true>(rz, q, st) : back_shape<4, false>(rz, q, st);
        case 8: return exact ? back_shape<8, true>(rz, q, st) : back_shape<8, false>(rz, q, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

int backward_ctas(int order, int rows_per_warp, const StepArgs& a, int* nbc) {
    const bool r2 = rows_per_warp == 2;
    switch (order) {
        case 2: return r2 ? back_ctas_of<2, 2, 4>(a, nbc) : back_ctas_of<2, 4, 4>(a, nbc);
        case 4: return r2 ? back_ctas_of<4, 2, 4>(a, nbc) : back_ctas_of<4, 4, 4>(a, nbc);
        case 8: return r2 ? back_ctas_of<8, 2, 4>(a, nbc) : back_ctas_of<8, 4, 4>(a, nbc);
    }
    return -1;
}

cudaError_t launch_backward(int order, bool exact, LaunchShape shape, const CUtensorMap& tm_c,
                            const CUtensorMap& tm_p, const CUtensorMap& tm_vel, const StepArgs& a,
                            cudaStream_t stream) {
    if (shape.warps != 4) return cudaErrorInvalidValue;
    BackReq q;
    q.tc = &tm_c, q.tp = &tm_p, q.tv = &tm_vel, q.a = &a;
    return back_dispatch(order, exact, shape.rows_per_warp, q, stream);
}

cudaError_t launch_backward_persistent(int order, bool exact, LaunchShape shape, const CUtensorMap& tm_c,
                                       const CUtensorMap& tm_p, const CUtensorMap& tm_vel,
                                       const PersistLaunch& P, cudaStream_t stream) {
    if (shape.warps != 4) return cudaErrorInvalidValue;
    BackReq q;
    q.tc = &tm_c, q.tp = &tm_p, q.tv = &tm_vel, q.pl = &P;
    return back_dispatch(order, exact, shape.rows_per_warp, q, stream);
}

cudaError_t launch_backward_multi(int order, bool exact, LaunchShape shape, const MultiJob* jobs,
                                  const int* begins, int njobs, long long nctas,
                                  const CUtensorMap* tmaps, cudaStream_t stream, bool chained) {
    if (shape.warps != 4) return cudaErrorInvalidValue;
    BackReq q;
    q.jobs = jobs, q.begins = begins, q.njobs = njobs, q.nctas = nctas, q.tmaps = tmaps;
    q.chained = chained;
    return back_dispatch(order, exact, shape.rows_per_warp, q, stream);
}

cudaError_t launch_backward_engine(int order, bool exact, LaunchShape shape, const EngineLaunch& L,
                                   long long nctas, const CUtensorMap* tmaps, cudaStream_t stream) {
    if (shape.warps != 4) return cudaErrorInvalidValue;
    BackReq q;
    q.engine = &L, q.nctas = nctas, q.tmaps = tmaps;
    return back_dispatch(order, exact, shape.rows_per_warp, q, stream);
}

int backward_resident_ctas(int order, bool exact, LaunchShape shape) {
    if (shape.warps != 4) return 0;
    int n = 0;
    BackReq q;
    q.occupancy = &n;
    return back_dispatch(order, exact, shape.rows_per_warp, q, nullptr) == cudaSuccess ? n : 0;
}

cudaError_t prepare_backward(int order, bool exact, LaunchShape shape) {
    if (shape.warps != 4) return cudaErrorInvalidValue;
    return back_dispatch(order, exact, shape.rows_per_warp, BackReq{}, nullptr);
}

}  // namespace twi
