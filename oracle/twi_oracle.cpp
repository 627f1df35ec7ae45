// twi_oracle.cpp -- CPU restatement of TorchWI's time-domain 2D acoustic
// propagator, used ONLY as test infrastructure (the checker for the CUDA
// path, and the "port" CPU baseline).  Nothing in the shipped library calls
// or links this file.
//
// Parity pin: the float instantiation is checked bit-for-bit against the
// reference's own CPU extension compiled from its sources (oracle/Makefile ->
// oracle/_ref/libtd2d_ref.so) and against golden vectors produced by running
// the reference `torchwi.Time2d(device='cpu')` (tests/golden/make_golden.py).
//
// Algorithm followed (paths relative to the TorchWI project root):
//   * interior leapfrog update, orders 2/4/8 ........ torchwi/propagator/td2d/td2d_cpu.cpp:6-98
//   * Keys absorbing boundary (right, left, bottom) .. td2d_cpu.cpp:101-146
//   * forward time loop, source, receivers, virt ..... propagator_cpu.cpp:5-79
//   * adjoint time loop, adjoint source, gradient .... propagator_cpu.cpp:82-152
//   * forward-only loop ............................... propagator_forward_cpu.cpp:5-71
//
// Arithmetic semantics.  The reference stores every field in FP32 but its
// expressions contain C++ double literals, so some sub-expressions are
// evaluated in FP64 and rounded back to FP32 on assignment.  The template
// parameter T is the STORAGE type: with T=float this file reproduces the
// reference's mixed float/double evaluation exactly (same operation order,
// no FMA contraction: build with -ffp-contract=off); with T=double every
// operation is FP64, which is the "FP64 CPU run of the same scheme" used to
// state each result's error.
//
// Layout: fields are [dimy][dimx], x fastest, dimx = nx + order,
// dimy = ny + order, ne = order/2 padding cells on every side.  Rows [0,ne)
// (the top pad) are never written, which makes the surface a zero (free)
// boundary; Keys runs on the left/right ne columns of rows [ne, dimy-ne) and
// on all columns of the bottom ne rows.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// Second-derivative weights (td2d_cpu.cpp:4-5, 31-33, 62-66), listed from
// the outermost ring inwards, followed by the centre weight.  The reference
// sums the rings outermost-first and adds the (centre weight * 2 * u) last.
struct Weights {
    int ne;
    double ring[4];    // ring[k] multiplies the 4 neighbours at distance ne-k
    double centre2;    // centre weight times 2 (exact in double)
};

Weights weights_for(int order) {
    Weights w{};
    if (order == 2) {
        w.ne = 1;
        w.ring[0] = 1.0;
        w.centre2 = -2.0 * 2.0;
    } else if (order == 4) {
        w.ne = 2;
        w.ring[0] = -0.08333333333333333;
        w.ring[1] = 1.3333333333333333;
        w.centre2 = -2.5 * 2.0;
    } else {
        w.ne = 4;
        w.ring[0] = -0.0017857142857142857;
        w.ring[1] = 0.025396825396825397;
        w.ring[2] = -0.2;
        w.ring[3] = 1.6;
        w.centre2 = -2.8472222222222223 * 2.0;
    }
    return w;
}

// Keys constants: cos(pi/6)*cos(pi/12) and cos(pi/6)+cos(pi/12)
// (td2d_cpu.cpp:101-108).
constexpr double kCosProd = 0.8365163037378079;
constexpr double kCosSum = 1.831951230073507;

// One interior cell of the leapfrog update.  `o2` selects the order-2 form,
// whose ring visits (left, up, right, down) and whose final update adds the
// Laplacian term last; orders 4 and 8 visit (up, left, right, down) and add
// the Laplacian term first (td2d_cpu.cpp:23-26 vs 52-55, 90-95).
template <typename T>
inline T interior_cell(const T* u1, const T* u2, const T* v, std::int64_t i,
                       std::int64_t sy, const Weights& W, T dtoh2) {
    double acc = 0.0;
    bool first = true;
    for (int k = 0; k < W.ne; ++k) {
        const std::int64_t d = W.ne - k;     // neighbour distance
        T ring;
        if (W.ne == 1) {
            ring = u2[i - 1];
            ring = ring + u2[i - sy];
            ring = ring + u2[i + 1];
            ring = ring + u2[i + sy];
        } else {
            ring = u2[i - d * sy];
            ring = ring + u2[i - d];
            ring = ring + u2[i + d];
            ring = ring + u2[i + d * sy];
        }
        const double term = W.ring[k] * static_cast<double>(ring);
        acc = first ? term : acc + term;
        first = false;
    }
    acc = acc + W.centre2 * static_cast<double>(u2[i]);
    const T lap = static_cast<T>(acc);
    const T vv = v[i] * v[i] * dtoh2;
    const T two_u = T(2) * u2[i];
    if (W.ne == 1) return (two_u - u1[i]) + vv * lap;
    return (lap * vv + two_u) - u1[i];
}

// One Keys cell (td2d_cpu.cpp:122-124 and the two mirrored copies).  `a` is
// the boundary cell, `b` and `c` are the next two cells inwards.
template <typename T>
inline T keys_cell(T uo_a, T uo_b, T uo_c, T um_a, T um_b, T v, T h2, T dt2,
                   T hdt) {
    const T uxx = static_cast<T>(
        ((static_cast<double>(uo_a) - 2.0 * static_cast<double>(uo_b)) +
         static_cast<double>(uo_c)) / static_cast<double>(h2));
    const T uxt = ((uo_a - um_a) - (uo_b - um_b)) / hdt;
    const T vvdt2 = (-v) * v * dt2;
    const double r =
        static_cast<double>(vvdt2) / kCosProd *
            (static_cast<double>(uxx) +
             kCosSum / static_cast<double>(v) * static_cast<double>(uxt)) +
        2.0 * static_cast<double>(uo_a) - static_cast<double>(um_a);
    return static_cast<T>(r);
}

template <typename T>
struct Grid {
    int order, ne, dimx, dimy, nx, ny;
    std::int64_t dimxy;
    T dt2, h2, dtoh2, hdt;
    Weights W;

    Grid(int order_, int dimx_, int dimy_, T h, T dt)
        : order(order_), dimx(dimx_), dimy(dimy_) {
        W = weights_for(order);
        ne = W.ne;
        nx = dimx - order;
        ny = dimy - order;
        dimxy = static_cast<std::int64_t>(dimx) * dimy;
        dt2 = dt * dt;
        h2 = h * h;
        dtoh2 = dt2 / h2;
        hdt = h * dt;
    }

    void interior(const T* u1, const T* u2, T* u3, const T* v) const {
#pragma omp parallel for schedule(static)
        for (int r = ne; r < ne + ny; ++r) {
            const std::int64_t row = static_cast<std::int64_t>(r) * dimx;
            for (int c = ne; c < ne + nx; ++c)
                u3[row + c] = interior_cell(u1, u2, v, row + c, dimx, W, dtoh2);
        }
    }

    void keys(const T* um, const T* uo, T* up, const T* v) const {
        const int nxne = dimx - ne, nyne = dimy - ne;
#pragma omp parallel for schedule(static)
        for (int r = ne; r < nyne; ++r) {
            const std::int64_t row = static_cast<std::int64_t>(r) * dimx;
            for (int c = nxne; c < dimx; ++c) {     // right pad, inward = -x
                const std::int64_t i = row + c;
                up[i] = keys_cell(uo[i], uo[i - 1], uo[i - 2], um[i], um[i - 1],
                                  v[i], h2, dt2, hdt);
            }
            for (int c = 0; c < ne; ++c) {          // left pad, inward = +x
                const std::int64_t i = row + c;
                up[i] = keys_cell(uo[i], uo[i + 1], uo[i + 2], um[i], um[i + 1],
                                  v[i], h2, dt2, hdt);
            }
        }
#pragma omp parallel for schedule(static)
        for (int r = nyne; r < dimy; ++r) {         // bottom pad, inward = -z
            const std::int64_t row = static_cast<std::int64_t>(r) * dimx;
            for (int c = 0; c < dimx; ++c) {
                const std::int64_t i = row + c;
                up[i] = keys_cell(uo[i], uo[i - dimx], uo[i - 2 * dimx], um[i],
                                  um[i - dimx], v[i], h2, dt2, hdt);
            }
        }
    }
};

// Cell index arithmetic of the reference: float division then truncation
// (propagator_cpu.cpp:44-48).
template <typename T>
int cell_of(T coord, T h) { return static_cast<int>(coord / h); }

template <typename T>
int forward_impl(T* frd, T* virt, const T* vel, const T* w, int order, int dimx,
                 int dimy, int nt, T h, T dt, T sx, T sy, T ry) {
    if (order != 2 && order != 4 && order != 8) return 1;
    Grid<T> g(order, dimx, dimy, h, dt);
    const int isx = cell_of(sx, h), isy = cell_of(sy, h), iry = cell_of(ry, h);
    if (isx < 0 || isy < 0 || isx >= g.nx || isy >= g.ny) return 2;
    if (iry < 0 || iry + g.ne >= dimy) return 3;
    const std::int64_t src = static_cast<std::int64_t>(isy + g.ne) * dimx + isx + g.ne;
    const std::int64_t rec = static_cast<std::int64_t>(iry + g.ne) * dimx + g.ne;
    const T cons = static_cast<T>(-2.0 / static_cast<double>(g.dt2));

    std::vector<T> buf(3 * g.dimxy, T(0));
    T* um = buf.data();
    T* uo = um + g.dimxy;
    T* up = uo + g.dimxy;
    for (int it = 0; it < nt; ++it) {
        g.interior(um, uo, up, vel);
        up[src] = up[src] + w[it] * vel[src] * vel[src] * g.dt2;
        g.keys(um, uo, up, vel);
        std::memcpy(frd + static_cast<std::int64_t>(it) * g.nx, up + rec,
                    sizeof(T) * g.nx);
        if (virt) {
            T* vt = virt + static_cast<std::int64_t>(it) * g.dimxy;
#pragma omp parallel for schedule(static)
            for (std::int64_t i = 0; i < g.dimxy; ++i) {
                const T v3 = vel[i] * vel[i] * vel[i];
                vt[i] = cons / v3 * ((um[i] - T(2) * uo[i]) + up[i]);
            }
        }
        T* t = um; um = uo; uo = up; up = t;
    }
    return 0;
}

template <typename T>
int backward_impl(T* grad, const T* virt, const T* vel, const T* resid,
                  int order, int dimx, int dimy, int nt, T h, T dt, T ry,
                  int kahan) {
    if (order != 2 && order != 4 && order != 8) return 1;
    Grid<T> g(order, dimx, dimy, h, dt);
    const int iry = cell_of(ry, h);
    if (iry < 0 || iry + g.ne >= dimy) return 3;
    const std::int64_t rec = static_cast<std::int64_t>(iry + g.ne) * dimx + g.ne;

    std::vector<T> buf(3 * g.dimxy, T(0));
    std::vector<T> comp(kahan ? g.dimxy : 0, T(0));
    T* um = buf.data();
    T* uo = um + g.dimxy;
    T* up = uo + g.dimxy;
    for (std::int64_t i = 0; i < g.dimxy; ++i) grad[i] = T(0);
    for (int it = nt - 1; it >= 0; --it) {
        g.interior(um, uo, up, vel);
        const T* rs = resid + static_cast<std::int64_t>(it) * g.nx;
        for (int c = 0; c < g.nx; ++c) {
            const std::int64_t j = rec + c;
            up[j] = up[j] + rs[c] * vel[j] * vel[j] * g.dt2;
        }
        g.keys(um, uo, up, vel);
        const T* vt = virt + static_cast<std::int64_t>(it) * g.dimxy;
        if (kahan) {
#pragma omp parallel for schedule(static)
            for (std::int64_t i = 0; i < g.dimxy; ++i) {
                const T term = (-vt[i]) * up[i];
                const T y = term - comp[i];
                const T s = grad[i] + y;
                comp[i] = (s - grad[i]) - y;
                grad[i] = s;
            }
        } else {
#pragma omp parallel for schedule(static)
            for (std::int64_t i = 0; i < g.dimxy; ++i)
                grad[i] = grad[i] + (-vt[i]) * up[i];
        }
        T* t = um; um = uo; uo = up; up = t;
    }
    return 0;
}

// Excitation-amplitude gradient (propagator_exa_cuda.cu:5-159,
// td2d_cuda.cu:182-205): the forward pass keeps, per cell, the virtual
// source of largest magnitude (strictly larger replaces; ties keep the
// earlier step) and its step index as a 16-bit integer; the adjoint pass
// assigns grad = -exa * lambda at that step.  The reference implements this
// on CUDA only; the stencil, Keys and virtual-source arithmetic here are
// those of the CPU propagator, like the rest of this file.
// cuda_order: form the virtual source as the reference's CUDA kernel writes
// it, cons/(v*v*v) * ((u^{n+1} - 2u^n) + u^{n-1}) (td2d_cuda.cu:189), instead
// of the CPU propagator's ((u^{n-1} - 2u^n) + u^{n+1})
// (propagator_cpu.cpp:70); used only to measure what that order changes.
template <typename T>
int exa_forward_impl(T* frd, T* exa, std::int16_t* iexa, const T* vel, const T* w, int order,
                     int dimx, int dimy, int nt, T h, T dt, T sx, T sy, T ry,
                     bool cuda_order = false) {
    if (order != 2 && order != 4 && order != 8) return 1;
    if (nt > 32767) return 4;
    Grid<T> g(order, dimx, dimy, h, dt);
    const int isx = cell_of(sx, h), isy = cell_of(sy, h), iry = cell_of(ry, h);
    if (isx < 0 || isy < 0 || isx >= g.nx || isy >= g.ny) return 2;
    if (iry < 0 || iry + g.ne >= dimy) return 3;
    const std::int64_t src = static_cast<std::int64_t>(isy + g.ne) * dimx + isx + g.ne;
    const std::int64_t rec = static_cast<std::int64_t>(iry + g.ne) * dimx + g.ne;
    const T cons = static_cast<T>(-2.0 / static_cast<double>(g.dt2));
    std::vector<T> buf(3 * g.dimxy, T(0));
    T* um = buf.data();
    T* uo = um + g.dimxy;
    T* up = uo + g.dimxy;
    for (std::int64_t i = 0; i < g.dimxy; ++i) exa[i] = T(0), iexa[i] = 0;
    for (int it = 0; it < nt; ++it) {
        g.interior(um, uo, up, vel);
        up[src] = up[src] + w[it] * vel[src] * vel[src] * g.dt2;
        g.keys(um, uo, up, vel);
        std::memcpy(frd + static_cast<std::int64_t>(it) * g.nx, up + rec, sizeof(T) * g.nx);
#pragma omp parallel for schedule(static)
        for (std::int64_t i = 0; i < g.dimxy; ++i) {
            const T v3 = vel[i] * vel[i] * vel[i];
            const T vt = cuda_order ? cons / v3 * ((up[i] - T(2) * uo[i]) + um[i])
                                    : cons / v3 * ((um[i] - T(2) * uo[i]) + up[i]);
            if (std::fabs(vt) > std::fabs(exa[i])) {
                exa[i] = vt;
                iexa[i] = static_cast<std::int16_t>(it);
            }
        }
        T* t = um; um = uo; uo = up; up = t;
    }
    return 0;
}

template <typename T>
int exa_backward_impl(T* grad, const T* exa, const std::int16_t* iexa, const T* vel,
                      const T* resid, int order, int dimx, int dimy, int nt, T h, T dt, T ry) {
    if (order != 2 && order != 4 && order != 8) return 1;
    if (nt > 32767) return 4;
    Grid<T> g(order, dimx, dimy, h, dt);
    const int iry = cell_of(ry, h);
    if (iry < 0 || iry + g.ne >= dimy) return 3;
    const std::int64_t rec = static_cast<std::int64_t>(iry + g.ne) * dimx + g.ne;
    std::vector<T> buf(3 * g.dimxy, T(0));
    T* um = buf.data();
    T* uo = um + g.dimxy;
    T* up = uo + g.dimxy;
    for (std::int64_t i = 0; i < g.dimxy; ++i) grad[i] = T(0);
    for (int it = nt - 1; it >= 0; --it) {
        g.interior(um, uo, up, vel);
        const T* rs = resid + static_cast<std::int64_t>(it) * g.nx;
        for (int c = 0; c < g.nx; ++c) {
            const std::int64_t j = rec + c;
            up[j] = up[j] + rs[c] * vel[j] * vel[j] * g.dt2;
        }
        g.keys(um, uo, up, vel);
#pragma omp parallel for schedule(static)
        for (std::int64_t i = 0; i < g.dimxy; ++i)
            if (iexa[i] == it) grad[i] = (-exa[i]) * up[i];
        T* t = um; um = uo; uo = up; up = t;
    }
    return 0;
}

}  // namespace

extern "C" {

int twio_exa_forward_f32(float* frd, float* exa, std::int16_t* iexa, const float* vel,
                         const float* w, int order, int dimx, int dimy, int nt, float h, float dt,
                         float sx, float sy, float ry) {
    return exa_forward_impl<float>(frd, exa, iexa, vel, w, order, dimx, dimy, nt, h, dt, sx, sy, ry);
}

int twio_exa_forward_cuda_order_f32(float* frd, float* exa, std::int16_t* iexa, const float* vel,
                                    const float* w, int order, int dimx, int dimy, int nt, float h,
                                    float dt, float sx, float sy, float ry) {
    return exa_forward_impl<float>(frd, exa, iexa, vel, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                                   true);
}

int twio_exa_backward_f32(float* grad, const float* exa, const std::int16_t* iexa,
                          const float* vel, const float* resid, int order, int dimx, int dimy,
                          int nt, float h, float dt, float ry) {
    return exa_backward_impl<float>(grad, exa, iexa, vel, resid, order, dimx, dimy, nt, h, dt, ry);
}


// Status codes: 0 ok, 1 bad order, 2 source outside the model, 3 receiver row
// outside the grid.
int twio_forward_f32(float* frd, float* virt, const float* vel, const float* w,
                     int order, int dimx, int dimy, int nt, float h, float dt,
                     float sx, float sy, float ry) {
    return forward_impl<float>(frd, virt, vel, w, order, dimx, dimy, nt, h, dt,
                               sx, sy, ry);
}

int twio_forward_f64(double* frd, double* virt, const double* vel,
                     const double* w, int order, int dimx, int dimy, int nt,
                     double h, double dt, double sx, double sy, double ry) {
    return forward_impl<double>(frd, virt, vel, w, order, dimx, dimy, nt, h, dt,
                                sx, sy, ry);
}

int twio_backward_f32(float* grad, const float* virt, const float* vel,
                      const float* resid, int order, int dimx, int dimy, int nt,
                      float h, float dt, float ry, int kahan) {
    return backward_impl<float>(grad, virt, vel, resid, order, dimx, dimy, nt, h,
                                dt, ry, kahan);
}

int twio_backward_f64(double* grad, const double* virt, const double* vel,
                      const double* resid, int order, int dimx, int dimy, int nt,
                      double h, double dt, double ry, int kahan) {
    return backward_impl<double>(grad, virt, vel, resid, order, dimx, dimy, nt,
                                 h, dt, ry, kahan);
}

}  // extern "C"
