// twi_cell.cuh -- per-cell arithmetic of the time step.
//
// Two arithmetic modes share every kernel:
//   EXACT=true  : reproduces TorchWI's CPU propagator bit for bit.  Storage
//                 is FP32; the sub-expressions that the reference evaluates
//                 in FP64 (its C++ constants are double literals,
//                 td2d_cpu.cpp:31-33, 107-108) are evaluated in FP64 here
//                 too, in the same order, and every operation uses an
//                 explicitly rounded intrinsic so nvcc cannot contract a
//                 multiply-add into an FMA.
//   EXACT=false : plain FP32 with FMA contraction and FP32 constants (fast
//                 mode; differs from the reference in the last bits).
#pragma once

#include <cuda_runtime.h>

namespace twi {

// Second-derivative weights, outermost ring first (td2d_cpu.cpp:4-5, 31-33,
// 61-66).  ring_w<O>(k) multiplies the four neighbours at distance NE-k.
template <int O>
__device__ __forceinline__ constexpr double ring_w(int k) {
    return O == 2 ? 1.0
         : O == 4 ? (k == 0 ? -0.08333333333333333 : 1.3333333333333333)
                  : (k == 0 ? -0.0017857142857142857
                   : k == 1 ? 0.025396825396825397
                   : k == 2 ? -0.2 : 1.6);
}
// Centre weight times two (exact in double).
template <int O>
__device__ __forceinline__ constexpr double centre2_w() {
    return O == 2 ? -4.0 : O == 4 ? -5.0 : -2.8472222222222223 * 2.0;
}

// Keys constants cos(pi/6)*cos(pi/12) and cos(pi/6)+cos(pi/12).
constexpr double kCosProd = 0.8365163037378079;
constexpr double kCosSum = 1.831951230073507;

// Interior update.  lf/rt/up/dn[d-1] are the u^n neighbours at distance d in
// -x, +x, -z, +z; u is u^n at the cell, um is u^{n-1}, vv = v*v*dt^2/h^2.
// Orders 4 and 8 sum each ring as (up + left + right + down) and add the
// Laplacian term before 2u - um; order 2 sums (left + up + right + down) and
// adds it after (td2d_cpu.cpp:23-26, 52-55, 90-95).
template <int O, bool EXACT>
__device__ __forceinline__ float interior_update(const float* lf, const float* rt,
                                                 const float* up, const float* dn, float u,
                                                 float um, float vv) {
    constexpr int NE = O / 2;
    if constexpr (EXACT) {
        double acc = 0.0;
#pragma unroll
        for (int k = 0; k < NE; ++k) {
            const int d = NE - k;
            float ring;
            if constexpr (O == 2)
                ring = __fadd_rn(__fadd_rn(__fadd_rn(lf[0], up[0]), rt[0]), dn[0]);
            else
                ring = __fadd_rn(__fadd_rn(__fadd_rn(up[d - 1], lf[d - 1]), rt[d - 1]),
                                 dn[d - 1]);
            const double term = __dmul_rn(ring_w<O>(k), static_cast<double>(ring));
            acc = (k == 0) ? term : __dadd_rn(acc, term);
        }
        acc = __dadd_rn(acc, __dmul_rn(centre2_w<O>(), static_cast<double>(u)));
        const float lap = __double2float_rn(acc);
        const float two_u = __fmul_rn(2.0f, u);
        if constexpr (O == 2) return __fadd_rn(__fsub_rn(two_u, um), __fmul_rn(vv, lap));
        return __fsub_rn(__fadd_rn(__fmul_rn(lap, vv), two_u), um);
    } else {
        float acc = static_cast<float>(centre2_w<O>()) * u;
#pragma unroll
        for (int k = 0; k < NE; ++k) {
            const int d = NE - k;
            acc = fmaf(static_cast<float>(ring_w<O>(k)),
                       (up[d - 1] + lf[d - 1]) + (rt[d - 1] + dn[d - 1]), acc);
        }
        return fmaf(acc, vv, 2.0f * u) - um;
    }
}

// v*v*dt^2/h^2 as the reference forms it: (v*v)*dtoh2.
template <bool EXACT>
__device__ __forceinline__ float vv_of(float v, float dtoh2) {
    if constexpr (EXACT) return __fmul_rn(__fmul_rn(v, v), dtoh2);
    return v * v * dtoh2;
}

// One Keys boundary cell (td2d_cpu.cpp:122-124 and its mirrored copies):
// a = boundary cell, b and c the next two cells inwards; uo = u^n, um =
// u^{n-1}.
template <bool EXACT>
__device__ __forceinline__ float keys_cell(float uo_a, float uo_b, float uo_c, float um_a,
                                           float um_b, float v, float h2, float dt2,
                                           float hdt) {
    if constexpr (EXACT) {
        double s = __dsub_rn(static_cast<double>(uo_a), __dmul_rn(2.0, static_cast<double>(uo_b)));
        s = __dadd_rn(s, static_cast<double>(uo_c));
        const float uxx = __double2float_rn(__ddiv_rn(s, static_cast<double>(h2)));
        const float uxt = __fdiv_rn(__fsub_rn(__fsub_rn(uo_a, um_a), __fsub_rn(uo_b, um_b)), hdt);
        const float a = __fmul_rn(__fmul_rn(-v, v), dt2);
        const double A = __ddiv_rn(static_cast<double>(a), kCosProd);
        const double B = __dmul_rn(__ddiv_rn(kCosSum, static_cast<double>(v)),
                                   static_cast<double>(uxt));
        const double C = __dadd_rn(static_cast<double>(uxx), B);
        const double r = __dsub_rn(__dadd_rn(__dmul_rn(A, C),
                                             __dmul_rn(2.0, static_cast<double>(uo_a))),
                                   static_cast<double>(um_a));
        return __double2float_rn(r);
    } else {
        const float uxx = (uo_a - 2.0f * uo_b + uo_c) / h2;
        const float uxt = ((uo_a - um_a) - (uo_b - um_b)) / hdt;
        const float a = -v * v * dt2 * static_cast<float>(1.0 / kCosProd);
        return a * (uxx + static_cast<float>(kCosSum) / v * uxt) + 2.0f * uo_a - um_a;
    }
}

// Point-source / adjoint-source increment amp*v*v*dt^2, formed left to
// right as in propagator_cpu.cpp:62 and :138.
template <bool EXACT>
__device__ __forceinline__ float injection(float amp, float v, float dt2) {
    if constexpr (EXACT) return __fmul_rn(__fmul_rn(__fmul_rn(amp, v), v), dt2);
    return amp * v * v * dt2;
}
template <bool EXACT>
__device__ __forceinline__ float add_injection(float val, float amp, float v, float dt2) {
    if constexpr (EXACT) return __fadd_rn(val, injection<EXACT>(amp, v, dt2));
    return fmaf(amp * v * v, dt2, val);
}

// Virtual source  cons/(v*v*v) * ((u^{n-1} - 2u^n) + u^{n+1})
// (propagator_cpu.cpp:68-72); cons = -2/dt^2.
template <bool EXACT>
__device__ __forceinline__ float virt_of(float um, float u, float up, float v, float cons) {
    if constexpr (EXACT) {
        const float v3 = __fmul_rn(__fmul_rn(v, v), v);
        return __fmul_rn(__fdiv_rn(cons, v3), __fadd_rn(__fsub_rn(um, __fmul_rn(2.0f, u)), up));
    }
    return cons / (v * v * v) * ((um - 2.0f * u) + up);
}

// The same virtual source split into a per-cell coefficient q = cons/(v*v*v)
// (constant over time, computed once) and the per-step product; bit-identical
// to virt_of.
template <bool EXACT>
__device__ __forceinline__ float virt_coef(float v, float cons) {
    if constexpr (EXACT) return __fdiv_rn(cons, __fmul_rn(__fmul_rn(v, v), v));
    return cons / (v * v * v);
}
template <bool EXACT>
__device__ __forceinline__ float virt_from_coef(float q, float um, float u, float up) {
    if constexpr (EXACT) return __fmul_rn(q, __fadd_rn(__fsub_rn(um, __fmul_rn(2.0f, u)), up));
    return q * ((um - 2.0f * u) + up);
}

// Gradient term  -virt * lambda  (propagator_cpu.cpp:143-144).
template <bool EXACT>
__device__ __forceinline__ float grad_term(float virt, float lam) {
    if constexpr (EXACT) return __fmul_rn(-virt, lam);
    return -virt * lam;
}

// Compensated (Kahan) accumulation  sum += x  with running compensation c.
__device__ __forceinline__ void kahan_add(float& sum, float& c, float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(sum, y);
    c = __fsub_rn(__fsub_rn(t, sum), y);
    sum = t;
}

}  // namespace twi
