// twi_step2.cu -- two time steps per launch (temporal blocking).
//
// Every launch of twi_step.cu reads u^{n-1}, u^n and v and writes u^{n+1}:
// the DRAM traffic is one full read of two fields per time step.  This
// kernel advances each shot by TWO steps per launch, so u^{n-1} and u^n are
// read once per two steps; u^{n+1} and u^{n+2} are both written (the next
// launch needs both).  Results are bit-identical to two single steps: every
// cell is computed with the same per-cell arithmetic (twi_cell.cuh) from the
// same inputs.
//
// A CTA owns a 120-column x TZ-row output tile of one shot group:
//   step A  u^{n+1} on the tile plus a ring (4 columns each side: the 32
//           lanes x 4 columns make 128; RING = max(NE, 2) rows above and
//           below, since a Keys cell needs two cells inwards) into shared
//           memory, from u^n staged with a further NE ring (136 columns,
//           TZ + 2 RING + 2 NE rows) and u^{n-1} on the step-A region;
//   step B  u^{n+2} on the tile (lanes 1..30) from step A's buffer; lanes 0
//           and 31 hold the ring columns and feed the x neighbours through
//           shuffles.
// The ring cells are computed redundantly by neighbouring tiles (the same
// values).  Keys boundary cells, the free surface and the outside of the
// grid are handled inside the tiles -- there are no boundary CTAs -- by a
// per-cell fix-up path that only edge lanes take.
//
// Time indices: step A is time d = a.it, step B is d + 1 (forward, recompute)
// or d - 1 (adjoint, which runs backwards).  Slots: inputs prev/cur, outputs
// next (step A) and next2 (step B); the planner gives the four distinct
// slots.  The virtual-source slot of step B is virt_base + 1 (forward
// direction) or virt_base - 1 (adjoint).
#include <atomic>
#include <cstdio>

#include "twi_cell.cuh"
#include "twi_kernels.h"
#include "twi_ptx.cuh"
#include "twi_tile.cuh"

namespace twi {
namespace {

constexpr int kOutX = kTile2X;          // output columns per tile
constexpr int kRegX = 128;              // step-A columns: output + 4 each side
constexpr int kUnX = kRegX + 8;         // staged u^n columns: step A + 4 each side

template <int ORDER, int RZ, int WZ>
struct Smem2 {
    static constexpr int NE = ORDER / 2;
    static constexpr int TZ = RZ * WZ;
    static constexpr int RING = NE < 2 ? 2 : NE;             // step-A rows above / below the tile
    static constexpr int RA = TZ + 2 * RING;                 // step-A rows
    static constexpr int RN = RA + 2 * NE;                   // staged u^n rows
    static constexpr int RAW = (RA + WZ - 1) / WZ;           // step-A rows per warp
    static constexpr int UN_FLOATS = round32(RN * kUnX);
    static constexpr int UM_FLOATS = RA * kRegX;
    static constexpr int STAGE_FLOATS = UN_FLOATS + UM_FLOATS;
    static constexpr int V_FLOATS = RA * kRegX;
    static constexpr int A_FLOATS = RA * kRegX;
    static constexpr int STAGES = 2;
    static constexpr int BAR_BYTES = 128;
    static constexpr size_t BYTES = 128 /*alignment slack*/ + BAR_BYTES +
                                    size_t(V_FLOATS + A_FLOATS + STAGES * STAGE_FLOATS) * 4;
    static constexpr uint32_t UN_TX = RN * kUnX * 4;
    static constexpr uint32_t UM_TX = RA * kRegX * 4;
    static constexpr uint32_t V_TX = RA * kRegX * 4;
};


// One Keys cell from shared memory: `uo` points at u^n of the cell, `so` is
// the offset to the next cell inwards in that buffer; `um` / `sm` the same
// for u^{n-1}.  Out of line: only edge lanes call it.
template <bool EXACT>
__device__ __noinline__ float keys_smem(const float* uo, int so, const float* um, int sm, float v,
                                        float h2, float dt2, float hdt) {
    return keys_cell<EXACT>(uo[0], uo[so], uo[2 * so], um[0], um[sm], v, h2, dt2, hdt);
}

// Interior update of a lane's four cells from the register window `win`
// (rows r-NE..r+NE of the lane's columns) and the x neighbours of the centre
// row (L[k]: column c-1-k, R[k]: column c+4+k).
template <int ORDER, bool EXACT>
__device__ __forceinline__ void interior4(const float4* win, const float* L, const float* R,
                                          const float4& um4, const float4& v4, float dtoh2,
                                          float out[4]) {
    constexpr int NE = ORDER / 2;
    const float c4[4] = {win[NE].x, win[NE].y, win[NE].z, win[NE].w};
    const float um[4] = {um4.x, um4.y, um4.z, um4.w};
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        float lf[NE], rt[NE], up[NE], dn[NE];
#pragma unroll
        for (int d = 1; d <= NE; ++d) {
            const int jl = m - d, jr = m + d;
            lf[d - 1] = jl >= 0 ? c4[jl] : L[-jl - 1];
            rt[d - 1] = jr < 4 ? c4[jr] : R[jr - 4];
            up[d - 1] = comp(win[NE - d], m);
            dn[d - 1] = comp(win[NE + d], m);
        }
        out[m] = interior_update<ORDER, EXACT>(lf, rt, up, dn, c4[m], um[m],
                                               vv_of<EXACT>(comp(v4, m), dtoh2));
    }
}

// x neighbours of the centre row: shuffles, with lanes 0 / 31 reading the
// ring from shared memory when `edge_row` is given (step A), or keeping the
// (unused) shuffle result (step B, where lanes 0 and 31 store nothing).
template <int NE>
__device__ __forceinline__ void x_neighbours(const float4& c, int lane, const float* edge_row,
                                             int cs, float L[NE], float R[NE]) {
    const float c4[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
    for (int k = 0; k < NE; ++k) {
        L[k] = __shfl_up_sync(0xffffffffu, c4[3 - (k & 3)], 1 + (k >> 2));
        R[k] = __shfl_down_sync(0xffffffffu, c4[k & 3], 1 + (k >> 2));
    }
    if (edge_row != nullptr) {
        if (lane == 0) {
#pragma unroll
            for (int k = 0; k < NE; ++k) L[k] = edge_row[cs - 1 - k];
        }
        if (lane == 31) {
#pragma unroll
            for (int k = 0; k < NE; ++k) R[k] = edge_row[cs + 4 + k];
        }
    }
}

// One CTA: the tile at (x0, z0) of shot group `grp`.
template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__device__ __forceinline__ void step2_body(const CUtensorMap& tm_un, const CUtensorMap& tm_um,
                                           const CUtensorMap& tm_v, const StepArgs& a, int x0,
                                           int z0, int grp) {
    using S = Smem2<ORDER, RZ, WZ>;
    constexpr int NE = S::NE, RING = S::RING, RA = S::RA, RAW = S::RAW, STAGES = S::STAGES;
    constexpr int DIR = MODE == kModeAdjoint ? -1 : 1;
    const int s_begin = grp * a.spc;
    const int nloc = min(a.spc, a.nshots - s_begin);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tA = a.it, tB = a.it + DIR;

    extern __shared__ unsigned char smem_raw[];
    unsigned char* sbase = reinterpret_cast<unsigned char*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    uint64_t* bar = reinterpret_cast<uint64_t*>(sbase);   // [0] velocity, [1+i] stage i
    float* vs = reinterpret_cast<float*>(sbase + S::BAR_BYTES);
    float* As = vs + S::V_FLOATS;
    float* stage0 = As + S::A_FLOATS;

    if (threadIdx.x == 0) {
        prefetch_tmap(&tm_un);
        prefetch_tmap(&tm_um);
        prefetch_tmap(&tm_v);
#pragma unroll
        for (int i = 0; i < 1 + STAGES; ++i) mbar_init(&bar[i], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int k) {
        const int s = s_begin + k;
        float* st = stage0 + (k % STAGES) * S::STAGE_FLOATS;
        uint64_t* b = &bar[1 + (k % STAGES)];
        mbar_arrive_expect_tx(b, S::UN_TX + S::UM_TX);
        tma_load_3d(st, &tm_un, x0 - 8, z0 - RING - NE, a.cur_base + s * a.cur_stride, b);
        tma_load_3d(st + S::UN_FLOATS, &tm_um, x0 - 4, z0 - RING, a.prev_base + s * a.prev_stride, b);
    };
    if (threadIdx.x == 0) {
        mbar_arrive_expect_tx(&bar[0], S::V_TX);
        tma_load_2d(vs, &tm_v, x0 - 4, z0 - RING, &bar[0]);
        for (int k = 0; k < STAGES && k < nloc; ++k) issue(k);
    }

    const int c = x0 - 4 + 4 * lane;     // first column of this lane (both steps)
    const int cs = 4 + 4 * lane;         // its column in the staged u^n rows
    const int ca = 4 * lane;             // its column in the step-A rows
    const bool out_lane = lane >= 1 && lane <= 30;
    const bool cols_interior = c >= NE && c + 3 < a.dimx - NE;

    {
        const bool ok = mbar_wait_bounded(&bar[0], 0);
        if (__syncthreads_or(!ok)) {
            if (threadIdx.x == 0) {
                atomicOr(a.err, 1);
                drain_stages(&bar[1], STAGES, 0, min(STAGES, nloc));
            }
            return;
        }
    }

    // virtual-source coefficients of the lane's output cells (recompute)
    float4 qreg[MODE == kModeRecompute ? RZ : 1];
    if constexpr (MODE == kModeRecompute) {
#pragma unroll
        for (int rr = 0; rr < RZ; ++rr) {
            const float4 v4 = ld4(vs + (warp * RZ + rr + RING) * kRegX + ca);
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
                const int r = z0 + warp * RZ + rr;
                gsum[rr] = gcmp[rr] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (out_lane && ((c < a.dimx && r < a.dimz))) {
                    const long long off = slot * a.slot_elems + (long long)r * a.pitch + c;
                    gsum[rr] = ld4(a.acc + off);
                    gcmp[rr] = ld4(a.acc_comp + off);
                }
            }
        }
    }

    for (int k = 0; k < nloc; ++k) {
        const int s = s_begin + k;
        const float* un = stage0 + (k % STAGES) * S::STAGE_FLOATS;   // u^n, staged rows
        const float* um = un + S::UN_FLOATS;                          // u^{n-1}, step-A rows

        int src_r = -1, src_c = -1;
        float wA = 0.f, wB = 0.f;
        if constexpr (MODE != kModeAdjoint) {
            src_r = a.src_rc[2 * s];
            src_c = a.src_rc[2 * s + 1];
            wA = a.wav[(long long)s * a.wav_stride + tA];
            wB = a.wav[(long long)s * a.wav_stride + tB];
        }
        const int rec_r = a.rec_row[s];

        {
            const bool ok = mbar_wait_bounded(&bar[1 + (k % STAGES)], (k / STAGES) & 1);
            if (__syncthreads_or(!ok)) {
                if (threadIdx.x == 0) {
                    atomicOr(a.err, 1);
                    drain_stages(&bar[1], STAGES, k, min(nloc, k + STAGES));
                }
                return;
            }
        }

        // ---- step A: u^{n+1} on the output tile plus its NE ring ----------
        {
            const int ra0 = warp * RAW;
            // a rolled loop (the stencil rows are re-read from shared memory
            // each row) keeps the kernel's code small
#pragma unroll 1
            for (int i = 0; i < RAW; ++i) {
                const int ra = ra0 + i;
                if (ra >= RA) break;                      // warp-uniform
                float4 win[2 * NE + 1];
#pragma unroll
                for (int j = 0; j <= 2 * NE; ++j) win[j] = ld4(un + (ra + j) * kUnX + cs);
                const int r = z0 - RING + ra;
                const float* urow = un + (ra + NE) * kUnX;
                float L[NE], R[NE];
                x_neighbours<NE>(win[NE], lane, urow, cs, L, R);
                float out[4] = {0.f, 0.f, 0.f, 0.f};
                if (r >= NE && r < a.dimz) {    // warp-uniform
                    const float4 um4 = ld4(um + ra * kRegX + ca);
                    const float4 v4 = ld4(vs + ra * kRegX + ca);
                    interior4<ORDER, EXACT>(win, L, R, um4, v4, a.dtoh2, out);
                    if (!(cols_interior && r < a.dimz - NE)) {
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const int cc = c + m;
                            const float* uo = urow + cs + m;
                            const float* umc = um + ra * kRegX + ca + m;
                            if (cc < 0 || cc >= a.dimx) out[m] = 0.f;
                            else if (r >= a.dimz - NE)
                                out[m] = keys_smem<EXACT>(uo, -kUnX, umc, -kRegX, comp(v4, m), a.h2, a.dt2, a.hdt);
                            else if (cc < NE)
                                out[m] = keys_smem<EXACT>(uo, 1, umc, 1, comp(v4, m), a.h2, a.dt2, a.hdt);
                            else if (cc >= a.dimx - NE)
                                out[m] = keys_smem<EXACT>(uo, -1, umc, -1, comp(v4, m), a.h2, a.dt2, a.hdt);
                        }
                    }
                    if constexpr (MODE != kModeAdjoint) {
                        if (r == src_r && src_c >= c && src_c < c + 4) {
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                if (c + m == src_c) out[m] = add_injection<EXACT>(out[m], wA, comp(v4, m), a.dt2);
                        }
                    } else {
                        if (r == rec_r && r < a.dimz - NE) {
                            const float* rs = a.resid + (long long)s * a.resid_stride + (long long)tA * a.nx;
#pragma unroll
                            for (int m = 0; m < 4; ++m) {
                                const int cc = c + m;
                                if (cc >= NE && cc < NE + a.nx)
                                    out[m] = add_injection<EXACT>(out[m], rs[cc - NE], comp(v4, m), a.dt2);
                            }
                        }
                    }
                }
                *reinterpret_cast<float4*>(As + ra * kRegX + ca) = make_float4(out[0], out[1], out[2], out[3]);
            }
        }
        __syncthreads();   // step A complete: As holds u^{n+1}

        // ---- step B: u^{n+2} on the output tile ---------------------------
        {
            const int rb0 = warp * RZ;
            float* nextA = a.fields + (long long)(a.next_base + s * a.next_stride) * a.slot_elems;
            float* nextB = a.fields + (long long)(a.next2_base + s * a.next2_stride) * a.slot_elems;
            float4 win[2 * NE + 1];
#pragma unroll
            for (int j = 0; j < 2 * NE; ++j) win[j] = ld4(As + (rb0 + RING - NE + j) * kRegX + ca);
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int rb = rb0 + rr;
                const int r = z0 + rb;
                if (r >= a.dimz) break;            // warp-uniform
                win[2 * NE] = ld4(As + (rb + RING + NE) * kRegX + ca);
                const float4 uA = win[NE];                                      // u^{n+1}
                const float4 un4 = ld4(un + (rb + RING + NE) * kUnX + cs);      // u^n
                const float4 v4 = ld4(vs + (rb + RING) * kRegX + ca);
                float L[NE], R[NE];
                x_neighbours<NE>(uA, lane, nullptr, 0, L, R);
                float out[4] = {0.f, 0.f, 0.f, 0.f};
                if (r >= NE) {                                   // warp-uniform
                    interior4<ORDER, EXACT>(win, L, R, un4, v4, a.dtoh2, out);
                    if (!(cols_interior && r < a.dimz - NE)) {
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            const int cc = c + m;
                            const float* uo = As + (rb + RING) * kRegX + ca + m;
                            const float* umc = un + (rb + RING + NE) * kUnX + cs + m;
                            if (cc < 0 || cc >= a.dimx || !out_lane) out[m] = 0.f;
                            else if (r >= a.dimz - NE)
                                out[m] = keys_smem<EXACT>(uo, -kRegX, umc, -kUnX, comp(v4, m), a.h2, a.dt2, a.hdt);
                            else if (cc < NE)
                                out[m] = keys_smem<EXACT>(uo, 1, umc, 1, comp(v4, m), a.h2, a.dt2, a.hdt);
                            else if (cc >= a.dimx - NE)
                                out[m] = keys_smem<EXACT>(uo, -1, umc, -1, comp(v4, m), a.h2, a.dt2, a.hdt);
                        }
                    }
                    if constexpr (MODE != kModeAdjoint) {
                        if (r == src_r && src_c >= c && src_c < c + 4) {
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                if (c + m == src_c) out[m] = add_injection<EXACT>(out[m], wB, comp(v4, m), a.dt2);
                        }
                    } else {
                        if (r == rec_r && r < a.dimz - NE) {
                            const float* rs = a.resid + (long long)s * a.resid_stride + (long long)tB * a.nx;
#pragma unroll
                            for (int m = 0; m < 4; ++m) {
                                const int cc = c + m;
                                if (cc >= NE && cc < NE + a.nx)
                                    out[m] = add_injection<EXACT>(out[m], rs[cc - NE], comp(v4, m), a.dt2);
                            }
                        }
                    }
                }

                if (out_lane) {
                    const long long off = (long long)r * a.pitch + c;
                    const bool full = c + 3 < a.dimx;
                    if (full) {
                        *reinterpret_cast<float4*>(nextA + off) = uA;
                        *reinterpret_cast<float4*>(nextB + off) = make_float4(out[0], out[1], out[2], out[3]);
                    } else {
#pragma unroll
                        for (int m = 0; m < 4; ++m)
                            if (c + m < a.dimx) nextA[off + m] = comp(uA, m), nextB[off + m] = out[m];
                    }

                    if constexpr (MODE != kModeAdjoint) {
                        if (a.frd != nullptr && r == rec_r) {
                            const long long oA = (long long)s * a.frd_stride + (long long)tA * a.nx;
                            const long long oB = (long long)s * a.frd_stride + (long long)tB * a.nx;
#pragma unroll
                            for (int m = 0; m < 4; ++m) {
                                const int cc = c + m;
                                if (cc >= NE && cc < NE + a.nx) {
                                    const float fa = comp(uA, m), fb = out[m];
                                    if (a.obs != nullptr) {
                                        a.frd[oA + cc - NE] = __fsub_rn(fa, a.obs[oA + cc - NE]);
                                        a.frd[oB + cc - NE] = __fsub_rn(fb, a.obs[oB + cc - NE]);
                                    } else {
                                        a.frd[oA + cc - NE] = fa;
                                        a.frd[oB + cc - NE] = fb;
                                    }
                                }
                            }
                        }
                    }

                    if constexpr (MODE == kModeRecompute) {
                        const float4 um4 = ld4(um + (rb + RING) * kRegX + ca);     // u^{n-1}
                        float* pA = a.virt_out + (long long)(a.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                                    (long long)r * a.virt_pitch + c;
                        float* pB = a.virt_out + (long long)(a.virt_base + 1 + s * a.virt_stride) * a.virt_slot_elems +
                                    (long long)r * a.virt_pitch + c;
                        float vA[4], vB[4];
#pragma unroll
                        for (int m = 0; m < 4; ++m) {
                            vA[m] = virt_from_coef<EXACT>(comp(qreg[rr], m), comp(um4, m), comp(un4, m), comp(uA, m));
                            vB[m] = virt_from_coef<EXACT>(comp(qreg[rr], m), comp(un4, m), comp(uA, m), out[m]);
                        }
                        if (full && a.virt_vec4) {
                            *reinterpret_cast<float4*>(pA) = make_float4(vA[0], vA[1], vA[2], vA[3]);
                            *reinterpret_cast<float4*>(pB) = make_float4(vB[0], vB[1], vB[2], vB[3]);
                        } else {
#pragma unroll
                            for (int m = 0; m < 4; ++m)
                                if (c + m < a.dimx) pA[m] = vA[m], pB[m] = vB[m];
                        }
                    }

                    if constexpr (MODE == kModeAdjoint) {
                        if ((r >= NE) && a.acc_mode != kAccNone && a.acc_mode != kAccExa) {
                            const float* vinA = a.virt_in + (long long)(a.virt_base + s * a.virt_stride) * a.virt_slot_elems +
                                                (long long)r * a.virt_pitch + c;
                            const float* vinB = a.virt_in + (long long)(a.virt_base - 1 + s * a.virt_stride) * a.virt_slot_elems +
                                                (long long)r * a.virt_pitch + c;
                            float va[4] = {0.f, 0.f, 0.f, 0.f}, vb[4] = {0.f, 0.f, 0.f, 0.f};
                            if (full && a.virt_vec4) {
                                const float4 x = ld4(vinA), y = ld4(vinB);
                                va[0] = x.x, va[1] = x.y, va[2] = x.z, va[3] = x.w;
                                vb[0] = y.x, vb[1] = y.y, vb[2] = y.z, vb[3] = y.w;
                            } else {
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (c + m < a.dimx) va[m] = vinA[m], vb[m] = vinB[m];
                            }
                            if (a.acc_mode == kAccKahanPerGroup) {
                                // interior cells only (pad cells are cropped by every caller)
                                if (r < a.dimz - NE) {
#pragma unroll
                                    for (int m = 0; m < 4; ++m) {
                                        const int cc = c + m;
                                        if ((cc >= NE && cc < a.dimx - NE)) {
                                            float sm = comp(gsum[rr], m), cm = comp(gcmp[rr], m);
                                            kahan_add(sm, cm, grad_term<EXACT>(va[m], comp(uA, m)));
                                            kahan_add(sm, cm, grad_term<EXACT>(vb[m], out[m]));
                                            set_comp(gsum[rr], m, sm);
                                            set_comp(gcmp[rr], m, cm);
                                        }
                                    }
                                }
                            } else {   // plain per-shot sums over every cell below the free surface
                                float* g = a.acc + (long long)(a.acc_base + s) * a.slot_elems + off;
#pragma unroll
                                for (int m = 0; m < 4; ++m)
                                    if (c + m < a.dimx)
                                        g[m] = __fadd_rn(__fadd_rn(g[m], grad_term<EXACT>(va[m], comp(uA, m))),
                                                         grad_term<EXACT>(vb[m], out[m]));
                            }
                        }
                    }
                }
#pragma unroll
                for (int j = 0; j < 2 * NE; ++j) win[j] = win[j + 1];
            }
        }

        __syncthreads();   // every warp is done with this stage and with As
        if (threadIdx.x == 0 && k + STAGES < nloc) issue(k + STAGES);
    }

    if constexpr (MODE == kModeAdjoint) {
        if (a.acc_mode == kAccKahanPerGroup) {
            const long long slot = a.acc_base + grp;
#pragma unroll
            for (int rr = 0; rr < RZ; ++rr) {
                const int r = z0 + warp * RZ + rr;
                if (out_lane && ((c < a.dimx && r < a.dimz))) {
                    const long long off = slot * a.slot_elems + (long long)r * a.pitch + c;
                    *reinterpret_cast<float4*>(a.acc + off) = gsum[rr];
                    *reinterpret_cast<float4*>(a.acc_comp + off) = gcmp[rr];
                }
            }
        }
    }
}

template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
__global__ void __launch_bounds__(WZ * 32, ORDER == 8 ? 2 : 3)
step2_kernel(const __grid_constant__ CUtensorMap tm_un, const __grid_constant__ CUtensorMap tm_um,
             const __grid_constant__ CUtensorMap tm_v, const __grid_constant__ StepArgs a) {
    using S = Smem2<ORDER, RZ, WZ>;
    const int tiles_x = (a.dimx + kOutX - 1) / kOutX;
    const int tiles_z = (a.dimz + S::TZ - 1) / S::TZ;
    const int tile_x = blockIdx.x % tiles_x;
    const int tile_z = (blockIdx.x / tiles_x) % tiles_z;
    const int grp = blockIdx.x / (tiles_x * tiles_z);
    const int x0 = tile_x * kOutX, z0 = tile_z * S::TZ;
    step2_body<ORDER, EXACT, MODE, RZ, WZ>(tm_un, tm_um, tm_v, a, x0, z0, grp);
}

template <int ORDER, bool EXACT, int MODE, int RZ, int WZ>
cudaError_t launch2_one(const CUtensorMap& tun, const CUtensorMap& tum, const CUtensorMap& tv,
                        const StepArgs& a, bool configure_only, cudaStream_t stream) {
    using S = Smem2<ORDER, RZ, WZ>;
    // one bit per device; setting an attribute twice is harmless, but plans
    // may be created from several host threads
    static std::atomic<unsigned long long> configured{0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 64 && !(configured.load(std::memory_order_relaxed) & (1ull << dev))) {
        e = cudaFuncSetAttribute(step2_kernel<ORDER, EXACT, MODE, RZ, WZ>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(S::BYTES));
        if (e != cudaSuccess) return e;
        configured.fetch_or(1ull << dev, std::memory_order_relaxed);
    }
    if (configure_only) return cudaSuccess;
    const long long n = step2_ctas(ORDER, RZ, a);
    if (n <= 0 || n > 0x7fffffffLL) return cudaErrorInvalidConfiguration;
    step2_kernel<ORDER, EXACT, MODE, RZ, WZ><<<dim3((unsigned)n), WZ * 32, S::BYTES, stream>>>(tun, tum, tv, a);
    return cudaGetLastError();
}

template <int ORDER, bool EXACT, int MODE>
cudaError_t launch2_shape(LaunchShape sh, const CUtensorMap& tun, const CUtensorMap& tum,
                          const CUtensorMap& tv, const StepArgs& a, bool cfg, cudaStream_t st) {
    if (sh.warps == 4 && sh.rows_per_warp == 4) return launch2_one<ORDER, EXACT, MODE, 4, 4>(tun, tum, tv, a, cfg, st);
    if (sh.warps == 4 && sh.rows_per_warp == 8) return launch2_one<ORDER, EXACT, MODE, 8, 4>(tun, tum, tv, a, cfg, st);
    return cudaErrorInvalidValue;
}

template <int ORDER, bool EXACT>
cudaError_t launch2_mode(StepMode mode, LaunchShape sh, const CUtensorMap& tun, const CUtensorMap& tum,
                         const CUtensorMap& tv, const StepArgs& a, bool cfg, cudaStream_t st) {
    switch (mode) {
        case kModeForward: return launch2_shape<ORDER, EXACT, kModeForward>(sh, tun, tum, tv, a, cfg, st);
        case kModeRecompute: return launch2_shape<ORDER, EXACT, kModeRecompute>(sh, tun, tum, tv, a, cfg, st);
        case kModeAdjoint: return launch2_shape<ORDER, EXACT, kModeAdjoint>(sh, tun, tum, tv, a, cfg, st);
        default: return cudaErrorInvalidValue;   // excitation amplitude: single steps only
    }
}

cudaError_t launch2_req(int order, bool exact, StepMode mode, LaunchShape sh, const CUtensorMap& tun,
                        const CUtensorMap& tum, const CUtensorMap& tv, const StepArgs& a, bool cfg,
                        cudaStream_t st) {
    switch (order) {
        case 2: return exact ? launch2_mode<2, true>(mode, sh, tun, tum, tv, a, cfg, st)
                             : launch2_mode<2, false>(mode, sh, tun, tum, tv, a, cfg, st);
        case 4: return exact ? launch2_mode<4, true>(mode, sh, tun, tum, tv, a, cfg, st)
                             : launch2_mode<4, false>(mode, sh, tun, tum, tv, a, cfg, st);
        case 8: return exact ? launch2_mode<8, true>(mode, sh, tun, tum, tv, a, cfg, st)
                             : launch2_mode<8, false>(mode, sh, tun, tum, tv, a, cfg, st);
    }
    return cudaErrorInvalidValue;
}

}  // namespace

long long step2_ctas(int order, int rows_per_warp, const StepArgs& a) {
    const int tz = rows_per_warp * 4;
    const long long ngroups = (a.nshots + a.spc - 1) / a.spc;
    const long long tiles = (long long)((a.dimx + kTile2X - 1) / kTile2X) * ((a.dimz + tz - 1) / tz);
    (void)order;
    return ngroups * tiles;
}

int step2_box_rows(int order, int rows_per_warp, int which) {
    const int ne = order / 2, tz = rows_per_warp * 4, ring = ne < 2 ? 2 : ne;
    return which == 0 ? tz + 2 * ring + 2 * ne : tz + 2 * ring;
}

cudaError_t launch_step2(int order, bool exact, StepMode mode, LaunchShape shape,
                         const CUtensorMap& tm_un, const CUtensorMap& tm_um, const CUtensorMap& tm_v,
                         const StepArgs& a, cudaStream_t stream) {
    return launch2_req(order, exact, mode, shape, tm_un, tm_um, tm_v, a, false, stream);
}

cudaError_t prepare_step2(int order, bool exact, LaunchShape shape) {
    CUtensorMap dummy{};
    StepArgs a{};
    for (StepMode m : {kModeForward, kModeRecompute, kModeAdjoint}) {
        cudaError_t e = launch2_req(order, exact, m, shape, dummy, dummy, dummy, a, true, nullptr);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace twi
