// twi_plan.cu -- host side of the C ABI declared in include/twi_b200.h.
//
// A plan owns no device memory: the caller binds a workspace (a PyTorch
// tensor in the Python layer) whose layout is computed here.  Wavefields
// live in "slots" of pitch*dimz floats addressed through one 3-D TMA tensor
// map; which slot holds u^k is decided by the schedule below, so the forward
// pass writes each checkpointed field straight into its checkpoint slot
// (no copies) and the recompute/adjoint passes read them back in place.
//
// Slot map of one shot (SPS slots per shot, global slot 0 is all zeros and
// stands for u^{-1} = u^0 = lambda^{-1} = lambda^{-2} = 0; ROT = 3, or 4 when
// two time steps run per launch so that both outputs avoid both inputs):
//   1 + s*SPS + [0, ROT)                forward/recompute rotation  u^k, k mod ROT
//   1 + s*SPS + ROT + [0, ROT)          adjoint rotation            lambda
//   1 + s*SPS + 2ROT + 2(j-1) + p       checkpoint j >= 1: p=0 -> u^{jK-1}, p=1 -> u^{jK}
// Gradient pass, segment j = nseg-1 .. 0 (K steps each, the last may be
// shorter): recompute u^{jK+1..jK+L} from checkpoint j writing the virtual
// source of each step into a K-slot buffer per shot, then run the L adjoint
// steps backwards reading it.  One extra forward propagation in total.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "twi_b200.h"
#include "twi_kernels.h"
#include "twi_plan_internal.h"

using namespace twi;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
    g_last_error = msg;
    return code;
}

}  // namespace

namespace twi {
// Lets other translation units of the library report through twi_last_error.
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace twi

namespace {

#define TWI_CUDA(expr)                                                                  \
    do {                                                                                \
        cudaError_t e_ = (expr);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return fail(TWI_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define TWI_TRY(expr)                 \
    do {                              \
        int s_ = (expr);              \
        if (s_ != TWI_OK) return s_;  \
    } while (0)

using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

}  // namespace

namespace twi {

// Tensor map over `nslots` slots of [dimz][pitch] floats (x extent dimx, so
// reads past the last column return zeros); nslots == 0 gives a 2-D map.
int make_map(CUtensorMap* tm, const void* base, int dimx, int dimz, long long nslots, int pitch,
             int box_x, int box_z) {
    EncodeTiledFn enc = encode_fn();
    if (!enc) return fail(TWI_ERR_CUDA, "cuTensorMapEncodeTiled entry point unavailable");
    const int rank = nslots > 0 ? 3 : 2;
    cuuint64_t dims[3] = {(cuuint64_t)dimx, (cuuint64_t)dimz, (cuuint64_t)(nslots > 0 ? nslots : 1)};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * dimz * 4};
    cuuint32_t box[3] = {(cuuint32_t)box_x, (cuuint32_t)box_z, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, rank, const_cast<void*>(base), dims,
                     strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return fail(TWI_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return TWI_OK;
}

// Waves of CTAs of a launch of `nctas` CTAs of the one-plan kernel of this
// mode and shape on the current device (a large number when unknown).
double launch_waves(int order, bool exact, StepMode mode, LaunchShape sh, long long nctas) {
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return 1e30;
    const int per_sm = mode == kModeBackward ? backward_resident_ctas(order, exact, sh)
                                             : step_resident_ctas(order, exact, mode, sh);
    return per_sm > 0 ? (double)nctas / ((double)per_sm * sms) : 1e30;
}

// Cell lookup exactly as the reference: FP32 division, truncation toward 0
// (propagator_cpu.cpp:44-48).
int cell_of(float coord, float h) { return static_cast<int>(coord / h); }

int check_order(int order) {
    if (order != 2 && order != 4 && order != 8)
        return fail(TWI_ERR_INVALID, "order must be 2, 4 or 8 (got " + std::to_string(order) + ")");
    return TWI_OK;
}

// Shot/receiver cells in padded coordinates; the shot must be inside the
// model and the receiver row inside the grid (the reference would index out
// of bounds otherwise; its numba path raises for shots outside the model,
// td2d_numba.py:45-49).
int shot_cells(float sx, float sy, float ry, float h, int nx, int nz, int ne, int dimz,
               int* src_r, int* src_c, int* rec_r) {
    const int isx = cell_of(sx, h), isy = cell_of(sy, h), iry = cell_of(ry, h);
    if (!(sx >= 0.f) || !(sy >= 0.f) || isx >= nx || isy >= nz)
        return fail(TWI_ERR_INVALID, "shot position outside the model: isx=" + std::to_string(isx) +
                                         " isy=" + std::to_string(isy));
    if (!(ry >= 0.f) || iry + ne >= dimz)
        return fail(TWI_ERR_INVALID, "receiver row outside the grid: iry=" + std::to_string(iry));
    *src_r = isy + ne;
    *src_c = isx + ne;
    *rec_r = iry + ne;
    return TWI_OK;
}

}  // namespace twi

namespace {

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

struct Slot {
    int base, stride;
};

// Time steps per launch when the problem leaves it open.
constexpr int kDefaultTimeBlock = 1;
// Rows per warp when the problem leaves it open: 4 for the forward-type
// steps, 2 for the adjoint (whose Kahan pairs and virtual-source window halve
// with the rows, so 5 CTAs fit an SM).  An explicit value applies to all.
constexpr int kDefaultAdjointRows = 2;
// Shots per CTA when the problem leaves it open: 4 for the forward-type
// steps, 8 for the adjoint, which reads and writes its group's Kahan pairs
// once per launch, so larger groups halve that traffic.  An explicit value
// applies to all.
constexpr int kDefaultShots = 4;
constexpr int kDefaultAdjointShots = 8;

LaunchShape default_shape(int rows_per_warp) {
    return LaunchShape{rows_per_warp == 8 || rows_per_warp == 2 ? rows_per_warp : 4, 4};
}

}  // namespace

// ---------------------------------------------------------------------------
// plan
// ---------------------------------------------------------------------------

struct twi_plan {
    twi_problem p{};
    int ne = 0, dimx = 0, dimz = 0, pitch = 0;
    long long slot_elems = 0;
    int K = 0, nseg = 0, spc = 1, ngroups = 1, rz = 4, sps = 0;
    int rz_adj = 4;         // rows per warp of single-step adjoint launches
    int spc_adj = 1;        // shots per CTA of adjoint launches (one Kahan pair per group)
    int tb = 1, rot = 3;   // time steps per launch (1 or 2) and rotation slots per role
    bool gradient = true, kahan = true, exa = false;
    bool recon = false;     // boundary saving + reverse reconstruction instead of checkpoints
    bool fused_back = false;   // recon: one fused backward launch per step (else reverse + adjoint)
    int nb = 0;             // boundary (Keys) cells per shot and time level
    long long nslots = 0, nvirt = 0, nacc = 0;
    // workspace regions (byte offsets)
    size_t off_vel = 0, off_wav = 0, off_frd = 0, off_grad = 0, off_coords = 0, off_err = 0,
           off_vpad = 0, off_fields = 0, off_virt = 0, off_acc = 0, off_comp = 0, off_exa = 0,
           off_iexa = 0, off_mpart = 0, off_bnd = 0, total = 0;
    // persistent launches: one launch per run of same-mode steps, reading the
    // steps' arguments from tables in the workspace (uploaded outside any
    // graph capture by sync_table) and two counters regions
    bool persist = false;
    enum { kTabForward = 0, kTabForwardSave = 1, kTabForwardResid = 2, kTabGradient = 3, kTables = 4 };
    size_t off_tab[kTables] = {}, tab_cap[kTables] = {}, off_cnt = 0;
    std::vector<StepArgs> tab_host[kTables];
    // chained launches (StepArgs::chain): one counter per shot group
    bool chained = false;
    size_t off_chain = 0;
    char* ws = nullptr;
    int device = -1;
    CUtensorMap tm_u2{}, tm_u1{}, tm_vel{};
    CUtensorMap ta_u2{}, ta_u1{}, ta_vel{};    // adjoint launches when rz_adj != rz
    CUtensorMap tm2_un{}, tm2_um{}, tm2_v{};   // two-step launches
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t g_fwd[2] = {nullptr, nullptr};
    cudaGraphExec_t g_bwd = nullptr;
    // forward with residual: graph captured for one (observed, misfit) pair
    cudaGraphExec_t g_fwd_res = nullptr;
    const float* res_obs = nullptr;
    double* res_misfit = nullptr;
    bool have_ckpt = false, have_shots = false, have_model = false, need_zero = false;

    int clear_once(cudaStream_t st) {
        if (!need_zero) return TWI_OK;
        TWI_CUDA(cudaMemsetAsync(F(off_fields), 0, (size_t)slot_elems * 4, st));
        TWI_CUDA(cudaMemsetAsync(I(off_err), 0, 4, st));
        TWI_CUDA(cudaMemsetAsync(F(off_vpad), 0, (size_t)slot_elems * 4, st));
        need_zero = false;
        return TWI_OK;
    }

    float* F(size_t off) const { return reinterpret_cast<float*>(ws + off); }
    int* I(size_t off) const { return reinterpret_cast<int*>(ws + off); }

    Slot zero() const { return {0, 0}; }
    Slot urot(int i) const { return {1 + i, sps}; }
    Slot lrot(int i) const { return {1 + rot + i, sps}; }
    Slot ckpt(int j, int part) const { return {1 + 2 * rot + 2 * (j - 1) + part, sps}; }

    // slot of u^k during the forward pass
    Slot fwd_slot(long long k, bool save) const {
        if (k <= 0) return zero();
        if (save && gradient && !exa && !recon) {
            if (k % K == 0 && k / K < nseg) return ckpt((int)(k / K), 1);
            if ((k + 1) % K == 0 && (k + 1) / K < nseg) return ckpt((int)((k + 1) / K), 0);
        }
        return urot((int)(k % rot));
    }
    // slot of u^k while recomputing segment j
    Slot rec_slot(long long k, int j) const {
        const long long c = (long long)j * K;
        if (k <= c) return j == 0 ? zero() : ckpt(j, k == c ? 1 : 0);
        return urot((int)(k % rot));
    }
    Slot lam_slot(long long m) const { return m < 0 ? zero() : lrot((int)(m % rot)); }

    StepArgs base_args() const {
        StepArgs a{};
        a.dimx = dimx;
        a.dimz = dimz;
        a.pitch = pitch;
        a.nx = p.nx;
        a.nz = p.nz;
        a.slot_elems = slot_elems;
        a.fields = F(off_fields);
        a.vel = F(off_vpad);
        a.nshots = p.nshots;
        a.spc = spc;
        const float dt2 = p.dt * p.dt, h2 = p.h * p.h;
        a.dt2 = dt2;
        a.h2 = h2;
        a.dtoh2 = dt2 / h2;
        a.hdt = p.h * p.dt;
        a.cons = static_cast<float>(-2.0 / static_cast<double>(dt2));
        a.src_rc = I(off_coords);
        a.rec_row = I(off_coords) + 2 * p.nshots;
        a.wav = F(off_wav);
        a.wav_stride = p.wavelet_per_shot ? p.nt : 0;
        a.frd_stride = (long long)p.nt * p.nx;
        a.resid_stride = (long long)p.nt * p.nx;
        a.virt_slot_elems = slot_elems;
        a.virt_pitch = pitch;
        a.virt_vec4 = 1;
        a.err = I(off_err);
        return a;
    }

    int launch(StepMode mode, const StepArgs& a, cudaStream_t st, int nsteps = 1) const {
        const bool adj = nsteps == 1 && (mode == kModeAdjoint || mode == kModeBackward) && rz_adj != rz;
        if (mode == kModeBackward) {
            cudaError_t e = adj ? launch_backward(p.order, p.exact != 0, default_shape(rz_adj), ta_u2, ta_u1, ta_vel, a, st)
                                : launch_backward(p.order, p.exact != 0, default_shape(rz), tm_u2, tm_u1, tm_vel, a, st);
            if (e != cudaSuccess)
                return fail(TWI_ERR_CUDA, std::string("backward launch: ") + cudaGetErrorString(e));
            return TWI_OK;
        }
        cudaError_t e = nsteps == 2
            ? launch_step2(p.order, p.exact != 0, mode, default_shape(rz), tm2_un, tm2_um, tm2_v, a, st)
            : adj ? launch_step(p.order, p.exact != 0, mode, default_shape(rz_adj), ta_u2, ta_u1, ta_vel, a, st)
                  : launch_step(p.order, p.exact != 0, mode, default_shape(rz), tm_u2, tm_u1, tm_vel, a, st);
        if (e != cudaSuccess)
            return fail(TWI_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
        return TWI_OK;
    }

    using Step = TwiStep;

    static void set_slots(StepArgs& a, Slot pv, Slot cu, Slot nx, Slot nx2) {
        a.prev_base = pv.base, a.prev_stride = pv.stride;
        a.cur_base = cu.base, a.cur_stride = cu.stride;
        a.next_base = nx.base, a.next_stride = nx.stride;
        a.next2_base = nx2.base, a.next2_stride = nx2.stride;
    }

    static void set_lam_slots(StepArgs& a, Slot pv, Slot cu, Slot nx) {
        a.lprev_base = pv.base, a.lprev_stride = pv.stride;
        a.lcur_base = cu.base, a.lcur_stride = cu.stride;
        a.lnext_base = nx.base, a.lnext_stride = nx.stride;
    }

    // The forward pass as a list of launches: pairs of time steps when the
    // plan runs two per launch (`blocked`), else single steps.
    void forward_steps(bool save, std::vector<Step>& out, bool blocked) const {
        StepArgs a = base_args();
        a.frd = F(off_frd);
        const StepMode mode = save && exa ? kModeExaForward : kModeForward;
        if (exa) {
            a.exa = F(off_exa);
            a.iexa = reinterpret_cast<short*>(ws + off_iexa);
            blocked = false;
        }
        if (recon && save) {   // the Keys cells of every u^k go to the boundary buffer
            a.bnd = F(off_bnd);
            a.bnd_cells = nb;
        }
        for (int it = 0; it < p.nt;) {
            const int n = blocked && it + 1 < p.nt ? 2 : 1;
            a.it = it;
            set_slots(a, fwd_slot(it - 1, save), fwd_slot(it, save), fwd_slot(it + 1, save),
                      n == 2 ? fwd_slot(it + 2, save) : zero());
            out.push_back({mode, a, n});
            it += n;
        }
    }

    // Excitation amplitude: nt adjoint steps assigning -exa * lambda.
    void exa_gradient_steps(std::vector<Step>& out) const {
        StepArgs a = base_args();
        a.resid = F(off_frd);
        a.acc = F(off_acc);
        a.acc_mode = kAccExa;
        a.acc_base = 0;
        a.spc = spc_adj;
        a.exa = F(off_exa);
        a.iexa = reinterpret_cast<short*>(ws + off_iexa);
        for (int it = p.nt - 1; it >= 0; --it) {
            const long long m = (long long)p.nt - 1 - it;
            const Slot pv = lam_slot(m - 2), cu = lam_slot(m - 1), nx_ = lam_slot(m);
            a.it = it;
            a.prev_base = pv.base, a.prev_stride = pv.stride;
            a.cur_base = cu.base, a.cur_stride = cu.stride;
            a.next_base = nx_.base, a.next_stride = nx_.stride;
            out.push_back({kModeAdjoint, a});
        }
    }

    // The gradient pass (without the accumulator reset and the final
    // reduction) as a list of launches: per segment, recompute then adjoint.
    // Boundary saving: backwards from u^{nt}, u^{nt-1} (left by the forward
    // pass), each step first rebuilds u^{it-1} and the virtual source of
    // step it (kModeReverse, pad cells from the boundary buffer), then takes
    // the adjoint step it.  u^0 = u^{-1} = 0 come from the zero slot.
    void recon_gradient_steps(std::vector<Step>& out) const {
        StepArgs a = base_args();
        a.virt_out = F(off_virt);
        a.virt_in = F(off_virt);
        a.virt_stride = 1;
        a.virt_base = 0;
        a.resid = F(off_frd);
        a.acc = F(off_acc);
        a.acc_comp = kahan ? F(off_comp) : nullptr;
        a.acc_mode = kahan ? kAccKahanPerGroup : kAccPlainPerShot;
        a.acc_base = 0;
        a.bnd = F(off_bnd);
        a.bnd_cells = nb;
        auto rslot = [&](long long k) { return k <= 0 ? zero() : urot((int)(k % 3)); };
        if (fused_back) {   // one launch per step; the virtual source stays in registers
            a.spc = spc_adj;
            for (int it = p.nt - 1; it >= 0; --it) {
                const long long m = (long long)p.nt - 1 - it;
                a.it = it;
                set_slots(a, rslot(it + 1), rslot(it), urot((it + 2) % 3), zero());
                set_lam_slots(a, lam_slot(m - 2), lam_slot(m - 1), lam_slot(m));
                out.push_back({kModeBackward, a});
            }
            return;
        }
        for (int it = p.nt - 1; it >= 0; --it) {
            a.it = it;
            set_slots(a, rslot(it + 1), rslot(it), urot((it + 2) % 3), zero());
            a.spc = spc;
            out.push_back({kModeReverse, a});
            const long long m = (long long)p.nt - 1 - it;
            set_slots(a, lam_slot(m - 2), lam_slot(m - 1), lam_slot(m), zero());
            a.spc = spc_adj;
            out.push_back({kModeAdjoint, a});
        }
    }

    void gradient_steps(std::vector<Step>& out, bool blocked) const {
        if (exa) return exa_gradient_steps(out);
        if (recon) return recon_gradient_steps(out);
        StepArgs a = base_args();
        a.virt_out = F(off_virt);
        a.virt_in = F(off_virt);
        a.virt_stride = K;
        a.resid = F(off_frd);   // the resid region aliases the gathers region
        a.acc = F(off_acc);
        a.acc_comp = kahan ? F(off_comp) : nullptr;
        a.acc_mode = kahan ? kAccKahanPerGroup : kAccPlainPerShot;
        a.acc_base = 0;
        for (int j = nseg - 1; j >= 0; --j) {
            const int c0 = j * K;
            const int L = std::min(K, p.nt - c0);
            for (int it = c0; it < c0 + L;) {     // recompute, writing virt
                const int n = blocked && it + 1 < c0 + L ? 2 : 1;
                a.it = it;
                set_slots(a, rec_slot(it - 1, j), rec_slot(it, j), urot((it + 1) % rot),
                          n == 2 ? urot((it + 2) % rot) : zero());
                a.virt_base = it - c0;
                a.frd = nullptr;
                a.spc = spc;
                out.push_back({kModeRecompute, a, n});
                it += n;
            }
            for (int it = c0 + L - 1; it >= c0;) {  // adjoint, reading virt
                const int n = blocked && it - 1 >= c0 ? 2 : 1;
                const long long m = (long long)p.nt - 1 - it;
                a.it = it;
                set_slots(a, lam_slot(m - 2), lam_slot(m - 1), lam_slot(m),
                          n == 2 ? lam_slot(m + 1) : zero());
                a.virt_base = it - c0;
                a.spc = spc_adj;
                out.push_back({kModeAdjoint, a, n});
                it -= n;
            }
        }
    }

    int gradient_prologue(cudaStream_t st) const {
        const size_t acc_bytes = (size_t)nacc * slot_elems * 4;
        if (cudaMemsetAsync(F(off_acc), 0, acc_bytes, st) != cudaSuccess ||
            (kahan && cudaMemsetAsync(F(off_comp), 0, acc_bytes, st) != cudaSuccess))
            return fail(TWI_ERR_CUDA, "memset of gradient accumulators failed");
        return TWI_OK;
    }

    int gradient_epilogue(cudaStream_t st) const {
        cudaError_t e = launch_reduce_grad(F(off_acc), kahan ? F(off_comp) : nullptr, (int)nacc,
                                           slot_elems, pitch, ne, p.nx, p.nz, kahan ? 1 : 0,
                                           F(off_grad), st);
        if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("reduce: ") + cudaGetErrorString(e));
        return TWI_OK;
    }

    // `obs` / `misfit` (both or neither): the gathers region receives the
    // residual modelled - observed and *misfit = 0.5 * sum(residual^2).
    static int forward_table(bool save, const float* obs) {
        return obs ? kTabForwardResid : save ? kTabForwardSave : kTabForward;
    }

    // Bring step table k in line with `steps` (a copy from host memory on
    // `st`, only when the content changed).  Runs outside graph capture.
    int sync_table(int k, const std::vector<Step>& steps, cudaStream_t st) {
        std::vector<StepArgs> v;
        v.reserve(steps.size());
        for (const Step& t : steps) v.push_back(t.a);
        if (v.size() > tab_cap[k]) return fail(TWI_ERR_STATE, "step table too small");
        if (v.size() == tab_host[k].size() &&
            std::memcmp(v.data(), tab_host[k].data(), v.size() * sizeof(StepArgs)) == 0)
            return TWI_OK;
        TWI_CUDA(cudaMemcpyAsync(ws + off_tab[k], v.data(), v.size() * sizeof(StepArgs),
                                 cudaMemcpyHostToDevice, st));
        tab_host[k] = std::move(v);
        return TWI_OK;
    }

    // One persistent launch of `n` steps of one mode whose arguments are the
    // device table entries dev[0..n).
    int launch_persistent(StepMode mode, const StepArgs& a0, const StepArgs* dev, int n,
                          cudaStream_t st) const {
        const bool adj = (mode == kModeAdjoint || mode == kModeBackward) && rz_adj != rz;
        const LaunchShape sh = default_shape(adj ? rz_adj : rz);
        int nbc = 0;
        const int total = mode == kModeBackward ? backward_ctas(p.order, sh.rows_per_warp, a0, &nbc)
                                                : step_ctas(p.order, sh, a0, &nbc);
        const int ngroups = (a0.nshots + a0.spc - 1) / a0.spc;
        if (total <= 0 || ngroups < 1 || total % ngroups != 0)
            return fail(TWI_ERR_INVALID, "persistent launch too large");
        unsigned* cnt = reinterpret_cast<unsigned*>(ws + off_cnt);
        const PersistLaunch L{dev, n, ngroups, total / ngroups, nbc, cnt, cnt + 1, 0};
        TWI_CUDA(cudaMemsetAsync(cnt, 0, (size_t)(1 + ngroups) * sizeof(unsigned), st));
        const CUtensorMap& t2 = adj ? ta_u2 : tm_u2;
        const CUtensorMap& t1 = adj ? ta_u1 : tm_u1;
        const CUtensorMap& tv = adj ? ta_vel : tm_vel;
        cudaError_t e = mode == kModeBackward
                            ? launch_backward_persistent(p.order, p.exact != 0, sh, t2, t1, tv, L, st)
                            : launch_step_persistent(p.order, p.exact != 0, mode, sh, t2, t1, tv, L, st);
        if (e != cudaSuccess)
            return fail(TWI_ERR_CUDA, std::string("persistent launch: ") + cudaGetErrorString(e));
        return TWI_OK;
    }

    // Waves of CTAs of one single-plan launch of `nctas` CTAs on this device.
    double launch_waves(StepMode mode, LaunchShape sh, long long nctas) const {
        return twi::launch_waves(p.order, p.exact != 0, mode, sh, nctas);
    }

    // A step list as launches.  Runs of two or more one-step launches of one
    // mode are chained when the plan chains: the group counters are zeroed,
    // then every launch after the run's first may start while the one before
    // it drains, each CTA waiting for its shot group of the earlier steps.
    int launch_list(const std::vector<Step>& steps, cudaStream_t st) const {
        for (size_t i = 0; i < steps.size();) {
            size_t j = i + 1;
            while (j < steps.size() && steps[i].nsteps == 1 && steps[j].nsteps == 1 &&
                   steps[j].mode == steps[i].mode && steps[j].a.spc == steps[i].a.spc)
                ++j;
            if (!chained || j - i < 2) {
                for (size_t t = i; t < j; ++t) TWI_TRY(launch(steps[t].mode, steps[t].a, st, steps[t].nsteps));
                i = j;
                continue;
            }
            const StepMode mode = steps[i].mode;
            const bool adj = mode == kModeAdjoint || mode == kModeBackward;
            const LaunchShape sh = default_shape(adj ? rz_adj : rz);
            int nbc = 0;
            const int total = mode == kModeBackward ? backward_ctas(p.order, sh.rows_per_warp, steps[i].a, &nbc)
                                                    : step_ctas(p.order, sh, steps[i].a, &nbc);
            const int ngroups = (steps[i].a.nshots + steps[i].a.spc - 1) / steps[i].a.spc;
            if (total <= 0 || ngroups < 1 || ngroups > p.nshots || total % ngroups != 0)
                return fail(TWI_ERR_INVALID, "chained launch too large");
            if (launch_waves(mode, sh, total) > kChainMaxWaves) {   // the tail is too small to pay for it
                for (size_t t = i; t < j; ++t) TWI_TRY(launch(steps[t].mode, steps[t].a, st, steps[t].nsteps));
                i = j;
                continue;
            }
            unsigned* cnt = reinterpret_cast<unsigned*>(ws + off_chain);
            TWI_CUDA(cudaMemsetAsync(cnt, 0, (size_t)ngroups * sizeof(unsigned), st));
            for (size_t t = i; t < j; ++t) {
                StepArgs a = steps[t].a;
                a.chain = cnt;
                a.chain_k = (int)(t - i);
                a.chain_per_group = total / ngroups;
                TWI_TRY(launch(mode, a, st));
            }
            i = j;
        }
        return TWI_OK;
    }

    // The steps of table k, one persistent launch per run of the same mode.
    int launch_table(int k, const std::vector<Step>& steps, cudaStream_t st) const {
        const StepArgs* dev = reinterpret_cast<const StepArgs*>(ws + off_tab[k]);
        for (size_t i = 0; i < steps.size();) {
            size_t j = i + 1;
            while (j < steps.size() && steps[j].mode == steps[i].mode) ++j;
            TWI_TRY(launch_persistent(steps[i].mode, steps[i].a, dev + i, (int)(j - i), st));
            i = j;
        }
        return TWI_OK;
    }

    // The forward / gradient step lists exactly as the enqueue functions
    // build them (for the step tables).
    void forward_list(bool save, const float* obs, std::vector<Step>& steps) const {
        forward_steps(save, steps, tb == 2);
        for (Step& t : steps) t.a.obs = obs;
    }

    int enqueue_forward(bool save, cudaStream_t st, const float* obs = nullptr,
                        double* misfit = nullptr) const {
        if (save && exa) {   // the maxima start from zero
            TWI_CUDA(cudaMemsetAsync(F(off_exa), 0, (size_t)p.nshots * slot_elems * 4, st));
            TWI_CUDA(cudaMemsetAsync(ws + off_iexa, 0, (size_t)p.nshots * slot_elems * 2, st));
        }
        std::vector<Step> steps;
        forward_list(save, obs, steps);
        if (persist) {
            TWI_TRY(launch_table(forward_table(save, obs), steps, st));
        } else {
            TWI_TRY(launch_list(steps, st));
        }
        if (misfit) {
            cudaError_t e = launch_misfit(F(off_frd), (long long)p.nshots * p.nt * p.nx,
                                          reinterpret_cast<double*>(ws + off_mpart), misfit, st);
            if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("misfit: ") + cudaGetErrorString(e));
        }
        return TWI_OK;
    }

    int enqueue_gradient(cudaStream_t st) const {
        TWI_TRY(gradient_prologue(st));
        std::vector<Step> steps;
        gradient_steps(steps, tb == 2);
        if (persist) {
            TWI_TRY(launch_table(kTabGradient, steps, st));
        } else {
            TWI_TRY(launch_list(steps, st));
        }
        return gradient_epilogue(st);
    }

    void drop_graphs() {
        for (auto& g : g_fwd)
            if (g) cudaGraphExecDestroy(g), g = nullptr;
        if (g_bwd) cudaGraphExecDestroy(g_bwd), g_bwd = nullptr;
        if (g_fwd_res) cudaGraphExecDestroy(g_fwd_res), g_fwd_res = nullptr;
    }

    // Run `enqueue` directly, or capture it once into a graph and replay.
    template <typename Fn>
    int run(cudaGraphExec_t* slot, cudaStream_t st, Fn enqueue) {
        if (!p.use_graphs) return enqueue(st);
        if (!*slot) {
            if (!capture_stream)
                TWI_CUDA(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking));
            TWI_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
            int s = enqueue(capture_stream);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(capture_stream, &g);
            if (s != TWI_OK) {
                if (g) cudaGraphDestroy(g);
                return s;
            }
            if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(slot, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        }
        TWI_CUDA(cudaGraphLaunch(*slot, st));
        return TWI_OK;
    }
};

extern "C" {

int twi_version(void) { return 100; }

const char* twi_last_error(void) { return g_last_error.c_str(); }

int twi_plan_create(const twi_problem* prob, twi_plan** out) {
    if (!prob || !out) return fail(TWI_ERR_INVALID, "null argument");
    const twi_problem& p = *prob;
    TWI_TRY(check_order(p.order));
    if (p.nx < 1 || p.nz < 1 || p.nt < 1 || p.nshots < 1)
        return fail(TWI_ERR_INVALID, "nx, nz, nt and nshots must be positive");
    if (!(p.h > 0.f) || !(p.dt > 0.f)) return fail(TWI_ERR_INVALID, "h and dt must be positive");
    if (p.rows_per_warp != 0 && p.rows_per_warp != 2 && p.rows_per_warp != 4 && p.rows_per_warp != 8)
        return fail(TWI_ERR_INVALID, "rows_per_warp must be 0, 2, 4 or 8");
    if (p.rows_per_warp == 2 && p.time_block == 2)
        return fail(TWI_ERR_INVALID, "two time steps per launch need rows_per_warp 4 or 8");
    if (p.ckpt_interval < 0 || p.ckpt_interval == 1)
        return fail(TWI_ERR_INVALID, "ckpt_interval must be 0 (choose) or >= 2");
    if (p.shots_per_cta < 0 || p.shots_per_cta > kMaxShotsPerCta)
        return fail(TWI_ERR_INVALID, "shots_per_cta must be 0 (choose) or 1.." + std::to_string(kMaxShotsPerCta));

    twi_plan* P = new twi_plan();
    P->p = p;
    P->ne = p.order / 2;
    P->dimx = p.nx + p.order;
    P->dimz = p.nz + p.order;
    P->pitch = (P->dimx + kTileX - 1) / kTileX * kTileX;
    P->slot_elems = (long long)P->pitch * P->dimz;
    P->gradient = p.forward_only == 0;
    P->exa = p.exa != 0 && P->gradient;
    if (P->exa && p.nt > 32767) {
        delete P;
        return fail(TWI_ERR_INVALID, "excitation amplitude stores 16-bit step indices: nt <= 32767");
    }
    P->kahan = p.accumulate == 0;
    // excitation amplitude assigns one value per cell and shot: one slot per
    // shot (the adjoint writes acc + s * slot), summed in shot order
    if (P->exa) P->kahan = false;
    P->rz = p.rows_per_warp ? p.rows_per_warp : 4;
    P->rz_adj = p.rows_per_warp ? p.rows_per_warp : kDefaultAdjointRows;
    int K = p.ckpt_interval;
    if (K == 0) K = std::max(2, (int)std::lround(std::sqrt(2.0 * p.nt)));
    K = std::min(K, std::max(2, p.nt));
    P->K = K;
    P->nseg = (p.nt + K - 1) / K;
    int spc = p.shots_per_cta;
    if (spc <= 0) spc = std::min(p.nshots, kDefaultShots);
    P->spc = std::min(spc, p.nshots);
    P->spc_adj = p.shots_per_cta > 0 ? P->spc : std::min(p.nshots, kDefaultAdjointShots);
    P->ngroups = (p.nshots + P->spc_adj - 1) / P->spc_adj;   // Kahan groups of the adjoint
    if (p.time_block < 0 || p.time_block > 2) {
        delete P;
        return fail(TWI_ERR_INVALID, "time_block must be 0 (choose), 1 or 2");
    }
    if (p.reconstruct < 0 || p.reconstruct > 2) {
        delete P;
        return fail(TWI_ERR_INVALID, "reconstruct must be 0, 1 (fused backward) or 2 (reverse and adjoint launches)");
    }
    P->recon = p.reconstruct != 0 && P->gradient && !P->exa;
    P->fused_back = P->recon && p.reconstruct == 1;
    if (P->recon && p.time_block == 2) {
        delete P;
        return fail(TWI_ERR_INVALID, "reverse reconstruction runs one time step per launch");
    }
    if (P->fused_back && P->rz_adj == 8) P->rz_adj = 4;   // the fused kernel has 2- and 4-row tiles
    P->tb = P->exa || P->recon ? 1 : p.time_block == 0 ? kDefaultTimeBlock : p.time_block;
    if (p.persistent < 0 || p.persistent > 1 || (p.persistent == 1 && P->tb == 2)) {
        delete P;
        return fail(TWI_ERR_INVALID, "persistent must be 0 or 1, and persistent launches run one step per work item "
                                     "(time_block 2 is not available with them)");
    }
    P->persist = p.persistent == 1;
    if (p.unchained < 0 || p.unchained > 1) {
        delete P;
        return fail(TWI_ERR_INVALID, "unchained must be 0 or 1");
    }
    P->chained = !P->persist && p.unchained == 0;
    P->rot = P->tb == 2 ? 4 : 3;
    if (P->recon) {   // no checkpoints: one segment, one virtual-source slot per shot
        P->K = p.nt;
        P->nseg = 1;
    }
    P->nb = 2 * P->ne * (P->dimz - 2 * P->ne) + P->ne * P->dimx;
    P->sps = P->gradient ? 2 * P->rot + (P->exa || P->recon ? 0 : 2 * (P->nseg - 1)) : P->rot;
    P->nslots = 1 + (long long)p.nshots * P->sps;
    // the fused backward keeps the virtual source in registers: no slots
    P->nvirt = P->gradient && !P->exa && !P->fused_back ? (long long)p.nshots * (P->recon ? 1 : K) : 0;
    P->nacc = P->gradient ? (P->kahan ? P->ngroups : p.nshots) : 0;

    // workspace layout
    const size_t S = p.nshots, nt = p.nt;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    P->off_vel = take((size_t)p.nx * p.nz * 4);
    P->off_wav = take((p.wavelet_per_shot ? S : 1) * nt * 4);
    P->off_frd = take(S * nt * p.nx * 4);
    P->off_grad = take((size_t)p.nx * p.nz * 4);
    P->off_coords = take(S * 3 * 4);
    P->off_err = take(4);
    P->off_vpad = take((size_t)P->slot_elems * 4);
    P->off_fields = take((size_t)P->nslots * P->slot_elems * 4);
    P->off_virt = take((size_t)P->nvirt * P->slot_elems * 4);
    P->off_acc = take((size_t)P->nacc * P->slot_elems * 4);
    P->off_comp = take(P->kahan && P->gradient ? (size_t)P->nacc * P->slot_elems * 4 : 0);
    P->off_exa = take(P->exa ? (size_t)p.nshots * P->slot_elems * 4 : 0);
    P->off_iexa = take(P->exa ? (size_t)p.nshots * P->slot_elems * 2 : 0);
    P->off_mpart = take(P->gradient ? (size_t)kMisfitBlocks * sizeof(double) : 0);
    P->off_bnd = take(P->recon ? (size_t)(p.nt + 1) * p.nshots * P->nb * 4 : 0);
    if (P->persist) {
        for (int k = 0; k < twi_plan::kTables; ++k) {
            const bool grad_table = k == twi_plan::kTabGradient || k == twi_plan::kTabForwardSave ||
                                    k == twi_plan::kTabForwardResid;
            P->tab_cap[k] = grad_table && !P->gradient ? 0
                          : k == twi_plan::kTabGradient ? (size_t)2 * p.nt : (size_t)p.nt;
            P->off_tab[k] = take(P->tab_cap[k] * sizeof(StepArgs));
        }
        P->off_cnt = take((size_t)(1 + p.nshots) * sizeof(unsigned));
    }
    P->off_chain = take(P->chained ? (size_t)p.nshots * sizeof(unsigned) : 0);
    P->total = off;
    *out = P;
    return TWI_OK;
}

int twi_plan_layout(const twi_plan* P, twi_layout* out) {
    if (!P || !out) return fail(TWI_ERR_INVALID, "null argument");
    out->workspace_bytes = P->total;
    out->vel = P->off_vel;
    out->wavelet = P->off_wav;
    out->gathers = P->off_frd;
    out->resid = P->off_frd;
    out->grad = P->off_grad;
    out->dimx = P->dimx;
    out->dimz = P->dimz;
    out->pitch = P->pitch;
    out->ckpt_interval = P->K;
    out->time_block = P->tb;
    out->nsegments = P->nseg;
    out->shots_per_cta = P->spc;
    out->rows_per_warp = P->rz;
    out->adjoint_rows_per_warp = P->rz_adj;
    out->adjoint_shots_per_cta = P->spc_adj;
    return TWI_OK;
}

int twi_plan_bind(twi_plan* P, void* workspace, size_t bytes) {
    if (!P || !workspace) return fail(TWI_ERR_INVALID, "null argument");
    if (bytes < P->total)
        return fail(TWI_ERR_NOMEM, "workspace too small: need " + std::to_string(P->total) + " bytes");
    if (reinterpret_cast<uintptr_t>(workspace) % 256)
        return fail(TWI_ERR_INVALID, "workspace must be 256-byte aligned");
    P->drop_graphs();
    P->ws = static_cast<char*>(workspace);
    for (auto& t : P->tab_host) t.clear();   // the new workspace holds no step tables yet
    TWI_CUDA(cudaGetDevice(&P->device));
    TWI_CUDA(prepare_step(P->p.order, P->p.exact != 0, default_shape(P->rz)));
    const int HZ = zhalo(P->p.order);
    const int TZ = P->rz * 4;
    TWI_TRY(make_map(&P->tm_u2, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch, kBoxX,
                     TZ + 2 * HZ));
    TWI_TRY(make_map(&P->tm_u1, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch, kTileX,
                     TZ));
    TWI_TRY(make_map(&P->tm_vel, P->F(P->off_vpad), P->dimx, P->dimz, 0, P->pitch, kTileX, TZ));
    if (P->fused_back) TWI_CUDA(prepare_backward(P->p.order, P->p.exact != 0, default_shape(P->rz_adj)));
    if (P->gradient && P->rz_adj != P->rz) {   // the adjoint's own tile height
        TWI_CUDA(prepare_step(P->p.order, P->p.exact != 0, default_shape(P->rz_adj)));
        const int TA = P->rz_adj * 4;
        TWI_TRY(make_map(&P->ta_u2, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch, kBoxX,
                         TA + 2 * HZ));
        TWI_TRY(make_map(&P->ta_u1, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch, kTileX,
                         TA));
        TWI_TRY(make_map(&P->ta_vel, P->F(P->off_vpad), P->dimx, P->dimz, 0, P->pitch, kTileX, TA));
    }
    if (P->tb == 2) {
        TWI_CUDA(prepare_step2(P->p.order, P->p.exact != 0, default_shape(P->rz)));
        const int rn = step2_box_rows(P->p.order, P->rz, 0), ra = step2_box_rows(P->p.order, P->rz, 1);
        TWI_TRY(make_map(&P->tm2_un, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch,
                         kTileX + 8, rn));
        TWI_TRY(make_map(&P->tm2_um, P->F(P->off_fields), P->dimx, P->dimz, P->nslots, P->pitch,
                         kTileX, ra));
        TWI_TRY(make_map(&P->tm2_v, P->F(P->off_vpad), P->dimx, P->dimz, 0, P->pitch, kTileX, ra));
    }
    // the zero slot, error word and velocity padding columns are cleared on
    // the caller's stream by the next set_shots / set_model
    P->need_zero = true;
    P->have_ckpt = false;
    return TWI_OK;
}

int twi_plan_set_shots(twi_plan* P, const float* sx, const float* sy, const float* ry,
                       void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    if (!sx || !sy || !ry) return fail(TWI_ERR_INVALID, "null coordinate array");
    const int S = P->p.nshots;
    std::vector<int> c(3 * S);
    for (int s = 0; s < S; ++s) {
        int r, cc, rr;
        int st = shot_cells(sx[s], sy[s], ry[s], P->p.h, P->p.nx, P->p.nz, P->ne, P->dimz, &r, &cc, &rr);
        if (st != TWI_OK) return fail(st, "shot " + std::to_string(s) + ": " + g_last_error);
        c[2 * s] = r;
        c[2 * s + 1] = cc;
        c[2 * S + s] = rr;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TWI_TRY(P->clear_once(st));
    // through kernel parameters: no copy from pageable memory, no stream sync
    cudaError_t e = launch_store_ints(P->I(P->off_coords), c.data(), (int)c.size(), st);
    if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("shot upload: ") + cudaGetErrorString(e));
    P->have_shots = true;
    P->have_ckpt = false;
    return TWI_OK;
}

int twi_plan_set_model(twi_plan* P, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    TWI_TRY(P->clear_once(static_cast<cudaStream_t>(stream)));
    cudaError_t e = launch_pad_model(P->F(P->off_vel), P->F(P->off_vpad), P->p.nx, P->p.nz, P->ne,
                                     P->dimx, P->dimz, P->pitch, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("pad: ") + cudaGetErrorString(e));
    P->have_model = true;
    P->have_ckpt = false;
    return TWI_OK;
}

int twi_forward(twi_plan* P, int save_checkpoints, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    if (!P->have_shots || !P->have_model)
        return fail(TWI_ERR_STATE, "set shots and model before twi_forward");
    const bool save = save_checkpoints != 0;
    if (save && !P->gradient)
        return fail(TWI_ERR_STATE, "a forward-only plan keeps no checkpoints");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->persist) {
        std::vector<twi_plan::Step> steps;
        P->forward_list(save, nullptr, steps);
        TWI_TRY(P->sync_table(twi_plan::forward_table(save, nullptr), steps, st));
    }
    TWI_TRY(P->run(&P->g_fwd[save ? 1 : 0], st,
                   [&](cudaStream_t s) { return P->enqueue_forward(save, s); }));
    P->have_ckpt = save;
    return TWI_OK;
}

int twi_forward_residual(twi_plan* P, const float* observed, double* misfit, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    if (!P->have_shots || !P->have_model)
        return fail(TWI_ERR_STATE, "set shots and model before twi_forward_residual");
    if (!P->gradient) return fail(TWI_ERR_STATE, "a forward-only plan keeps no checkpoints");
    if (!observed || !misfit) return fail(TWI_ERR_INVALID, "observed and misfit must not be null");
    if (P->g_fwd_res && (P->res_obs != observed || P->res_misfit != misfit)) {
        cudaGraphExecDestroy(P->g_fwd_res);
        P->g_fwd_res = nullptr;
    }
    P->res_obs = observed;
    P->res_misfit = misfit;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->persist) {
        std::vector<twi_plan::Step> steps;
        P->forward_list(true, observed, steps);
        TWI_TRY(P->sync_table(twi_plan::kTabForwardResid, steps, st));
    }
    TWI_TRY(P->run(&P->g_fwd_res, st,
                   [&](cudaStream_t s) { return P->enqueue_forward(true, s, observed, misfit); }));
    P->have_ckpt = true;
    return TWI_OK;
}

int twi_residual(twi_plan* P, const float* observed, double* misfit, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    if (!P->have_ckpt)
        return fail(TWI_ERR_STATE, "twi_residual needs a preceding twi_forward(save_checkpoints=1)");
    if (!observed || !misfit) return fail(TWI_ERR_INVALID, "observed and misfit must not be null");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = (long long)P->p.nshots * P->p.nt * P->p.nx;
    cudaError_t e = launch_residual(P->F(P->off_frd), observed, n, st);
    if (e == cudaSuccess)
        e = launch_misfit(P->F(P->off_frd), n, reinterpret_cast<double*>(P->ws + P->off_mpart), misfit, st);
    if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("residual: ") + cudaGetErrorString(e));
    return TWI_OK;
}

int twi_gradient(twi_plan* P, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    if (!P->have_ckpt)
        return fail(TWI_ERR_STATE, "twi_gradient needs a preceding twi_forward(save_checkpoints=1)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (P->persist) {
        std::vector<twi_plan::Step> steps;
        P->gradient_steps(steps, P->tb == 2);
        TWI_TRY(P->sync_table(twi_plan::kTabGradient, steps, st));
    }
    return P->run(&P->g_bwd, st, [&](cudaStream_t s) { return P->enqueue_gradient(s); });
}

int twi_plan_check(twi_plan* P, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    int err = 0;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    TWI_CUDA(cudaMemcpyAsync(&err, P->I(P->off_err), 4, cudaMemcpyDeviceToHost, st));
    TWI_CUDA(cudaStreamSynchronize(st));
    if (err) {
        cudaMemsetAsync(P->I(P->off_err), 0, 4, st);
        return fail(TWI_ERR_DEVICE, "device error word " + std::to_string(err) +
                                        " (a bounded TMA wait ran out)");
    }
    return TWI_OK;
}

int twi_plan_profile(twi_plan* P, int mode, int repeats, float* ms_per_launch, void* stream) {
    if (!P || !P->ws) return fail(TWI_ERR_STATE, "plan has no workspace");
    const int nsteps = mode >= 10 ? 2 : 1;
    mode = mode >= 10 ? mode - 10 : mode;
    if (!ms_per_launch || repeats < 1 || mode < 0 || (mode > 2 && mode != 5) || (nsteps == 2 && mode == 5))
        return fail(TWI_ERR_INVALID, "mode must be 0, 1, 2, 5 (one step) or 10, 11, 12 (two steps) and repeats >= 1");
    if (mode == 5 && !P->fused_back)
        return fail(TWI_ERR_INVALID, "mode 5 (fused backward) needs a plan with reconstruct = 1");
    if ((mode == 1 || mode == 2) && (P->fused_back || !P->gradient || P->exa))
        return fail(TWI_ERR_INVALID, "modes 1 and 2 need a gradient plan with checkpoints or reconstruct = 2");
    if (nsteps == 2 && P->tb != 2) return fail(TWI_ERR_INVALID, "two-step launches need a plan with time_block 2");
    if (!P->have_shots || !P->have_model) return fail(TWI_ERR_STATE, "set shots and model first");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    StepArgs a = P->base_args();
    const int it = P->p.nt / 2;
    a.it = it;
    StepMode m = static_cast<StepMode>(mode);
    if (m == kModeBackward) {
        const Slot u0 = P->urot(0), u1 = P->urot(1), u2 = P->urot(2);
        const Slot l0 = P->lrot(0), l1 = P->lrot(1), l2 = P->lrot(2);
        twi_plan::set_slots(a, u0, u1, u2, P->zero());
        twi_plan::set_lam_slots(a, l0, l1, l2);
        a.resid = P->F(P->off_frd);
        a.acc = P->F(P->off_acc);
        a.acc_comp = P->kahan ? P->F(P->off_comp) : nullptr;
        a.acc_mode = P->kahan ? kAccKahanPerGroup : kAccPlainPerShot;
        a.bnd = P->F(P->off_bnd);
        a.bnd_cells = P->nb;
        a.spc = P->spc_adj;
    } else if (m == kModeAdjoint) {
        const Slot l0 = P->lrot(0), l1 = P->lrot(1), l2 = P->lrot(2), l3 = P->lrot(P->rot - 1);
        a.prev_base = l0.base, a.cur_base = l1.base, a.next_base = l2.base, a.next2_base = l3.base;
        a.virt_in = P->F(P->off_virt);
        a.resid = P->F(P->off_frd);
        a.acc = P->F(P->off_acc);
        a.acc_comp = P->kahan ? P->F(P->off_comp) : nullptr;
        a.acc_mode = P->kahan ? kAccKahanPerGroup : kAccPlainPerShot;
        a.spc = P->spc_adj;
    } else {
        const Slot u0 = P->urot(0), u1 = P->urot(1), u2 = P->urot(2), u3 = P->urot(P->rot - 1);
        a.prev_base = u0.base, a.cur_base = u1.base, a.next_base = u2.base, a.next2_base = u3.base;
        if (m == kModeRecompute) a.virt_out = P->F(P->off_virt);
        if (m == kModeRecompute && P->recon) {   // its gradient pass rebuilds backwards instead
            m = kModeReverse;
            a.bnd = P->F(P->off_bnd);
            a.bnd_cells = P->nb;
        }
    }
    if (m != kModeBackward) a.prev_stride = a.cur_stride = a.next_stride = a.next2_stride = P->sps;
    a.virt_stride = P->recon ? 1 : P->K;
    a.virt_base = m == kModeAdjoint && !P->recon ? 1 : 0;   // two-step adjoint reads slots 1 and 0
    cudaEvent_t e0, e1;
    TWI_CUDA(cudaEventCreate(&e0));
    TWI_CUDA(cudaEventCreate(&e1));
    int s = TWI_OK;
    if (cudaEventRecord(e0, st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "event record failed");
    for (int r = 0; r < repeats && s == TWI_OK; ++r) s = P->launch(m, a, st, nsteps);
    if (s == TWI_OK && cudaEventRecord(e1, st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "event record failed");
    if (s == TWI_OK && cudaEventSynchronize(e1) != cudaSuccess) s = fail(TWI_ERR_CUDA, "event sync failed");
    float ms = 0.f;
    if (s == TWI_OK && cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) s = fail(TWI_ERR_CUDA, "elapsed failed");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s == TWI_OK) *ms_per_launch = ms / repeats;
    return s;
}

int twi_plan_footprint_bytes(const twi_problem* prob, size_t* bytes) {
    if (!prob || !bytes) return fail(TWI_ERR_INVALID, "null argument");
    twi_plan* P = nullptr;
    TWI_TRY(twi_plan_create(prob, &P));
    *bytes = P->total;
    delete P;
    return TWI_OK;
}

}  // extern "C"

namespace {

// The launch shapes the autotuner tries for `prob`: every combination the
// caller left open (0) of shots per CTA {0, 1, 2, 4, 8} (at most nshots),
// rows per warp {0, 2, 4, 8} and time steps per launch {1, 2} (1 for
// excitation amplitude, reverse reconstruction and 2 rows per warp), each
// timed on a copy of the problem with nt = 8.  0 keeps the per-mode defaults
// (the adjoint's own shots per CTA and rows per warp), which no single value
// reproduces.
std::vector<twi_problem> tune_candidates(const twi_problem& p) {
    std::vector<twi_problem> out;
    for (int spc : {0, 1, 2, 4, 8}) {
        if (p.shots_per_cta ? spc != p.shots_per_cta : spc > std::max(1, p.nshots)) continue;
        for (int rz : {0, 2, 4, 8}) {
            if (p.rows_per_warp && rz != p.rows_per_warp) continue;
            for (int tb : {1, 2}) {
                if ((p.time_block && tb != p.time_block) ||
                    ((p.exa || p.reconstruct || p.persistent || rz == 2) && tb == 2))
                    continue;
                twi_problem q = p;
                q.nt = 8;
                q.ckpt_interval = 2;
                q.use_graphs = 0;
                q.shots_per_cta = spc, q.rows_per_warp = rz, q.time_block = tb;
                out.push_back(q);
            }
        }
    }
    return out;
}

}  // namespace

extern "C" {

int twi_autotune_scratch_bytes(const twi_problem* prob, size_t* bytes) {
    if (!prob || !bytes) return fail(TWI_ERR_INVALID, "null argument");
    size_t most = 0;
    for (const twi_problem& q : tune_candidates(*prob)) {
        size_t b = 0;
        TWI_TRY(twi_plan_footprint_bytes(&q, &b));
        most = std::max(most, b);
    }
    if (most == 0) return fail(TWI_ERR_INVALID, "no launch shape fits the fixed fields of the problem");
    *bytes = most;
    return TWI_OK;
}

int twi_autotune(const twi_problem* prob, void* scratch, size_t scratch_bytes, void* stream,
                 twi_problem* tuned, float* ms_per_step) {
    if (!prob || !scratch || !tuned) return fail(TWI_ERR_INVALID, "null argument");
    const std::vector<twi_problem> cands = tune_candidates(*prob);
    if (cands.empty()) return fail(TWI_ERR_INVALID, "no launch shape fits the fixed fields of the problem");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // shots in the middle of the model, receivers two cells down
    const int S = prob->nshots;
    std::vector<float> sx(S, prob->h * (prob->nx / 2)), sy(S, prob->h * std::min(2, prob->nz - 1));
    const std::vector<float> vel((size_t)prob->nx * prob->nz, 2000.f);   // a uniform model
    float best = -1.f;
    twi_problem best_q{};
    for (const twi_problem& q : cands) {
        twi_plan* P = nullptr;
        TWI_TRY(twi_plan_create(&q, &P));
        int s = twi_plan_bind(P, scratch, scratch_bytes);
        if (s == TWI_OK && cudaMemsetAsync(scratch, 0, P->total, st) != cudaSuccess)
            s = fail(TWI_ERR_CUDA, "scratch clear failed");
        if (s == TWI_OK) s = twi_plan_set_shots(P, sx.data(), sy.data(), sy.data(), stream);
        if (s == TWI_OK && cudaMemcpyAsync(P->F(P->off_vel), vel.data(), vel.size() * 4,
                                           cudaMemcpyHostToDevice, st) != cudaSuccess)
            s = fail(TWI_ERR_CUDA, "model upload failed");
        if (s == TWI_OK) s = twi_plan_set_model(P, stream);
        float total = 0.f;
        // forward, recompute, adjoint; forward and the fused backward for
        // boundary-saving plans; the forward step alone for forward-only and
        // excitation-amplitude plans
        std::vector<int> modes{0};
        if (P->fused_back) modes.push_back(5);
        else if (P->gradient && !P->exa) modes.insert(modes.end(), {1, 2});
        for (size_t mi = 0; mi < modes.size() && s == TWI_OK; ++mi) {
            const int m = modes[mi];
            const int mode = P->tb == 2 ? 10 + m : m;
            float ms = 0.f;
            s = twi_plan_profile(P, mode, 2, &ms, stream);           // warm-up
            if (s == TWI_OK) s = twi_plan_profile(P, mode, 10, &ms, stream);
            total += ms / P->tb;
        }
        twi_plan_destroy(P);
        if (s != TWI_OK) return s;
        if (best < 0.f || total < best) best = total, best_q = q;
    }
    *tuned = *prob;
    tuned->shots_per_cta = best_q.shots_per_cta;
    tuned->rows_per_warp = best_q.rows_per_warp;
    tuned->time_block = best_q.time_block;
    if (ms_per_step) *ms_per_step = best;
    return TWI_OK;
}

int twi_plan_destroy(twi_plan* P) {
    if (!P) return TWI_OK;
    P->drop_graphs();
    if (P->capture_stream) cudaStreamDestroy(P->capture_stream);
    delete P;
    return TWI_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// plan operations used by the request engine (twi_engine.cu)
// ---------------------------------------------------------------------------

void plan_tensor_maps(const twi_plan* P, CUtensorMap out[kMapsPerPlan]) {
    const bool own_adj = P->gradient && P->rz_adj != P->rz;   // ta_* exist
    out[0] = P->tm_u2;
    out[1] = P->tm_u1;
    out[2] = P->tm_vel;
    out[3] = own_adj ? P->ta_u2 : P->tm_u2;
    out[4] = own_adj ? P->ta_u1 : P->tm_u1;
    out[5] = own_adj ? P->ta_vel : P->tm_vel;
}
int plan_adjoint_rows(const twi_plan* P) { return P->rz_adj; }
float* plan_gathers(const twi_plan* P) { return P->F(P->off_frd); }
long long plan_gathers_elems(const twi_plan* P) {
    return (long long)P->p.nshots * P->p.nt * P->p.nx;
}
void plan_steps(const twi_plan* P, int kind, std::vector<TwiStep>& out, size_t* fwd_steps) {
    P->forward_steps(kind == 1, out, false);
    *fwd_steps = out.size();
    if (kind == 1) P->gradient_steps(out, false);
}
int plan_gradient_prologue(const twi_plan* P, cudaStream_t st) { return P->gradient_prologue(st); }
int plan_gradient_epilogue(const twi_plan* P, cudaStream_t st) { return P->gradient_epilogue(st); }
void plan_mark_done(twi_plan* P, int kind) { P->have_ckpt = kind == 1; }
int plan_check_compatible(const twi_plan* P, int kind, int order, bool exact, int rows_per_warp,
                          int back_rows) {
    if (!P->ws) return fail(TWI_ERR_STATE, "bind the plan before submitting it");
    if (kind == 1 && !P->gradient) return fail(TWI_ERR_STATE, "a forward-only plan cannot take a gradient request");
    if (P->exa) return fail(TWI_ERR_INVALID, "excitation-amplitude plans run through twi_forward/twi_gradient only");
    if (P->recon && !P->fused_back)
        return fail(TWI_ERR_INVALID, "plans with separate rebuild and adjoint launches (reconstruct = 2) run "
                                     "through twi_forward/twi_gradient only");
    if (!P->have_shots || !P->have_model) return fail(TWI_ERR_STATE, "set shots and model first");
    if (P->p.order != order || (P->p.exact != 0) != exact ||
        default_shape(P->rz).rows_per_warp != rows_per_warp)
        return fail(TWI_ERR_INVALID, "plan order/arithmetic/rows_per_warp differ from the engine's");
    if (P->fused_back && kind == 1 && P->rz_adj != back_rows)
        return fail(TWI_ERR_INVALID, "plan's backward rows per warp differ from the engine's");
    return TWI_OK;
}

// ---------------------------------------------------------------------------
// batches of plans: one launch per kernel mode and time step for all plans
// ---------------------------------------------------------------------------

struct twi_batch {
    std::vector<twi_plan*> plans;
    int order = 4;
    bool exact = true, use_graphs = true;
    LaunchShape shape{4, 4};
    LaunchShape shape_back{2, 4};   // fused backward launches of boundary-saving plans
    struct Launch {
        StepMode mode;
        size_t job0;   // first job in the phase's table
        int njobs;
        long long nctas;
        bool reset = false;   // first launch of a chain: zero the counters first
        bool pdl = false;     // later launch of a chain
    };
    // chained launches (StepArgs::chain) when every plan chains: plan i's
    // shot groups count in the counters from chain_off[i] on
    bool chained = true;
    size_t off_chain = 0, chain_count = 0;
    std::vector<size_t> chain_off;
    // phases: 0 forward without checkpoints, 1 forward with, 2 gradient
    std::vector<Launch> launches[3];
    size_t njobs[3] = {0, 0, 0};
    size_t off_tmaps = 0, off_jobs[3] = {0, 0, 0}, off_begins[3] = {0, 0, 0}, total = 0;
    char* ws = nullptr;
    bool built[3] = {false, false, false};
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t graphs[3] = {nullptr, nullptr, nullptr};

    void drop_graphs() {
        for (auto& g : graphs)
            if (g) cudaGraphExecDestroy(g), g = nullptr;
    }

    // Step lists of every plan for one phase.
    void steps_of(int phase, std::vector<std::vector<twi_plan::Step>>& per) const {
        per.assign(plans.size(), {});
        for (size_t i = 0; i < plans.size(); ++i) {
            if (phase == 2) plans[i]->gradient_steps(per[i], false);
            else plans[i]->forward_steps(phase == 1, per[i], false);
        }
    }

    static size_t max_steps(const std::vector<std::vector<twi_plan::Step>>& per) {
        size_t m = 0;
        for (const auto& v : per) m = std::max(m, v.size());
        return m;
    }

    // Group the plans' steps tick by tick, one launch per (tick, mode), and
    // upload the job table of the phase.
    int build(int phase) {
        std::vector<std::vector<twi_plan::Step>> per;
        steps_of(phase, per);
        std::vector<MultiJob> jobs;
        jobs.reserve(njobs[phase]);
        launches[phase].clear();
        const size_t T = max_steps(per);
        for (size_t t = 0; t < T; ++t) {
            for (StepMode m : {kModeForward, kModeRecompute, kModeAdjoint, kModeBackward}) {
                Launch L{m, jobs.size(), 0, 0};
                for (size_t i = 0; i < plans.size(); ++i) {
                    if (t >= per[i].size() || per[i][t].mode != m) continue;
                    MultiJob J{};
                    J.a = per[i][t].a;
                    J.plan = (int)i;
                    J.ncta = m == kModeBackward ? backward_ctas(order, shape_back.rows_per_warp, J.a, &J.nbc)
                                                : step_ctas(order, shape, J.a, &J.nbc);
                    if (J.ncta <= 0) return fail(TWI_ERR_INVALID, "batch launch too large");
                    J.cta_begin = (int)L.nctas;
                    L.nctas += J.ncta;
                    ++L.njobs;
                    jobs.push_back(J);
                }
                if (L.njobs) launches[phase].push_back(L);
            }
        }
        if (jobs.size() != njobs[phase]) return fail(TWI_ERR_STATE, "batch job count mismatch");
        if (chained) chain_launches(launches[phase], jobs);
        TWI_CUDA(cudaMemcpy(ws + off_jobs[phase], jobs.data(), jobs.size() * sizeof(MultiJob),
                            cudaMemcpyHostToDevice));
        std::vector<int> begins(jobs.size());
        for (size_t i = 0; i < jobs.size(); ++i) begins[i] = jobs[i].cta_begin;
        TWI_CUDA(cudaMemcpy(ws + off_begins[phase], begins.data(), begins.size() * sizeof(int),
                            cudaMemcpyHostToDevice));
        built[phase] = true;
        return TWI_OK;
    }

    // Runs of two or more consecutive launches of one mode over the same
    // jobs (same plans, shapes and CTA counts) become chains: their jobs'
    // arguments carry the plan's counters, the step's place in the chain and
    // the CTAs per shot group.
    void chain_launches(std::vector<Launch>& Ls, std::vector<MultiJob>& jobs) const {
        auto same = [&](const Launch& x, const Launch& y) {
            if (x.mode != y.mode || x.njobs != y.njobs) return false;
            for (int j = 0; j < x.njobs; ++j) {
                const MultiJob& p = jobs[x.job0 + j];
                const MultiJob& q = jobs[y.job0 + j];
                if (p.plan != q.plan || p.ncta != q.ncta || p.nbc != q.nbc || p.a.spc != q.a.spc) return false;
            }
            return true;
        };
        unsigned* cnt = reinterpret_cast<unsigned*>(ws + off_chain);
        for (size_t i = 0; i < Ls.size();) {
            size_t j = i + 1;
            while (j < Ls.size() && same(Ls[i], Ls[j])) ++j;
            const LaunchShape sh = Ls[i].mode == kModeBackward ? shape_back : shape;
            if (j - i >= 2 && launch_waves(order, exact, Ls[i].mode, sh, Ls[i].nctas) <= kChainMaxWaves) {
                for (size_t t = i; t < j; ++t) {
                    Ls[t].reset = t == i;
                    Ls[t].pdl = t > i;
                    for (int q = 0; q < Ls[t].njobs; ++q) {
                        MultiJob& J = jobs[Ls[t].job0 + q];
                        const int ng = (J.a.nshots + J.a.spc - 1) / J.a.spc;
                        J.a.chain = cnt + chain_off[J.plan];
                        J.a.chain_k = (int)(t - i);
                        J.a.chain_per_group = J.ncta / ng;
                    }
                }
            }
            i = j;
        }
    }

    int enqueue(int phase, cudaStream_t st) const {
        if (phase == 2)
            for (twi_plan* P : plans) TWI_TRY(P->gradient_prologue(st));
        const MultiJob* base = reinterpret_cast<const MultiJob*>(ws + off_jobs[phase]);
        const int* begins = reinterpret_cast<const int*>(ws + off_begins[phase]);
        const CUtensorMap* tm = reinterpret_cast<const CUtensorMap*>(ws + off_tmaps);
        for (const Launch& L : launches[phase]) {
            if (L.reset) TWI_CUDA(cudaMemsetAsync(ws + off_chain, 0, chain_count * sizeof(unsigned), st));
            cudaError_t e = L.mode == kModeBackward
                ? launch_backward_multi(order, exact, shape_back, base + L.job0, begins + L.job0, L.njobs,
                                        L.nctas, tm, st, L.pdl)
                : launch_step_multi(order, exact, L.mode, shape, base + L.job0, begins + L.job0, L.njobs,
                                    L.nctas, tm, st, L.pdl);
            if (e != cudaSuccess)
                return fail(TWI_ERR_CUDA, std::string("batch launch: ") + cudaGetErrorString(e));
        }
        if (phase == 2)
            for (twi_plan* P : plans) TWI_TRY(P->gradient_epilogue(st));
        return TWI_OK;
    }

    int run(int phase, cudaStream_t st) {
        if (!built[phase]) TWI_TRY(build(phase));
        if (!use_graphs) return enqueue(phase, st);
        if (!graphs[phase]) {
            if (!capture_stream)
                TWI_CUDA(cudaStreamCreateWithFlags(&capture_stream, cudaStreamNonBlocking));
            TWI_CUDA(cudaStreamBeginCapture(capture_stream, cudaStreamCaptureModeThreadLocal));
            int s = enqueue(phase, capture_stream);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(capture_stream, &g);
            if (s != TWI_OK) {
                if (g) cudaGraphDestroy(g);
                return s;
            }
            if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("capture: ") + cudaGetErrorString(e));
            e = cudaGraphInstantiate(&graphs[phase], g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("instantiate: ") + cudaGetErrorString(e));
        }
        TWI_CUDA(cudaGraphLaunch(graphs[phase], st));
        return TWI_OK;
    }
};

extern "C" {

int twi_batch_create(twi_plan* const* plans, int nplans, twi_batch** out) {
    if (!plans || !out || nplans < 1) return fail(TWI_ERR_INVALID, "need at least one plan");
    twi_batch* B = new twi_batch();
    for (int i = 0; i < nplans; ++i) {
        twi_plan* P = plans[i];
        if (!P) {
            delete B;
            return fail(TWI_ERR_INVALID, "null plan");
        }
        if (i == 0) {
            B->order = P->p.order;
            B->exact = P->p.exact != 0;
            B->use_graphs = P->p.use_graphs != 0;
            B->shape = default_shape(P->rz);
            B->shape_back = LaunchShape{P->rz_adj, 4};
        }
        if (P->exa || (P->recon && !P->fused_back)) {
            delete B;
            return fail(TWI_ERR_INVALID, "excitation-amplitude plans and plans with separate rebuild and adjoint "
                                         "launches (reconstruct = 2) run through twi_forward/twi_gradient only");
        }
        if (P->p.order != B->order || (P->p.exact != 0) != B->exact ||
                   default_shape(P->rz).rows_per_warp != B->shape.rows_per_warp ||
                   (P->fused_back && P->rz_adj != B->shape_back.rows_per_warp)) {
            delete B;
            return fail(TWI_ERR_INVALID, "plans of a batch must share order, arithmetic and rows_per_warp");
        }
        B->plans.push_back(P);
        B->chained = B->chained && P->chained;
    }
    for (twi_plan* P : B->plans) {
        B->chain_off.push_back(B->chain_count);
        B->chain_count += (size_t)P->p.nshots;   // at least one counter per shot group of any mode
        B->njobs[0] += P->p.nt;
        B->njobs[1] += P->p.nt;
        B->njobs[2] += (P->fused_back ? 1 : 2) * (size_t)P->p.nt;   // fused backward: one job per step
    }
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
    B->off_tmaps = take(B->plans.size() * kMapsPerPlan * sizeof(CUtensorMap));
    for (int ph = 0; ph < 3; ++ph) {
        B->off_jobs[ph] = take(B->njobs[ph] * sizeof(MultiJob));
        B->off_begins[ph] = take(B->njobs[ph] * sizeof(int));
    }
    B->off_chain = take(B->chained ? B->chain_count * sizeof(unsigned) : 0);
    B->total = off;
    *out = B;
    return TWI_OK;
}

int twi_batch_workspace_size(const twi_batch* B, size_t* bytes) {
    if (!B || !bytes) return fail(TWI_ERR_INVALID, "null argument");
    *bytes = B->total;
    return TWI_OK;
}

int twi_batch_bind(twi_batch* B, void* workspace, size_t bytes) {
    if (!B || !workspace) return fail(TWI_ERR_INVALID, "null argument");
    if (bytes < B->total) return fail(TWI_ERR_NOMEM, "batch workspace too small: need " + std::to_string(B->total));
    if (reinterpret_cast<uintptr_t>(workspace) % 256)
        return fail(TWI_ERR_INVALID, "workspace must be 256-byte aligned");
    for (twi_plan* P : B->plans)
        if (!P->ws) return fail(TWI_ERR_STATE, "bind every plan before its batch");
    B->drop_graphs();
    B->ws = static_cast<char*>(workspace);
    std::vector<CUtensorMap> tm(B->plans.size() * kMapsPerPlan);
    for (size_t i = 0; i < B->plans.size(); ++i) plan_tensor_maps(B->plans[i], &tm[i * kMapsPerPlan]);
    TWI_CUDA(cudaMemcpy(B->ws + B->off_tmaps, tm.data(), tm.size() * sizeof(CUtensorMap),
                        cudaMemcpyHostToDevice));
    for (bool& b : B->built) b = false;
    return TWI_OK;
}

int twi_batch_forward(twi_batch* B, int save_checkpoints, void* stream) {
    if (!B || !B->ws) return fail(TWI_ERR_STATE, "batch has no workspace");
    for (twi_plan* P : B->plans)
        if (!P->have_shots || !P->have_model)
            return fail(TWI_ERR_STATE, "set shots and model of every plan before twi_batch_forward");
    const int phase = save_checkpoints ? 1 : 0;
    TWI_TRY(B->run(phase, static_cast<cudaStream_t>(stream)));
    for (twi_plan* P : B->plans) P->have_ckpt = save_checkpoints != 0;
    return TWI_OK;
}

int twi_batch_gradient(twi_batch* B, void* stream) {
    if (!B || !B->ws) return fail(TWI_ERR_STATE, "batch has no workspace");
    for (twi_plan* P : B->plans)
        if (!P->have_ckpt)
            return fail(TWI_ERR_STATE, "twi_batch_gradient needs a preceding twi_batch_forward(save_checkpoints=1)");
    return B->run(2, static_cast<cudaStream_t>(stream));
}

int twi_batch_destroy(twi_batch* B) {
    if (!B) return TWI_OK;
    B->drop_graphs();
    if (B->capture_stream) cudaStreamDestroy(B->capture_stream);
    delete B;
    return TWI_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// reference-shaped entry points (single shot, reference memory layout)
// ---------------------------------------------------------------------------

namespace {

struct RefRun {
    int order, ne, dimx, dimz, nx, nz, nt, pitch;
    long long slot_elems;
    float h, dt;
    char* scratch = nullptr;
    size_t off_vpad = 0, off_fields = 0, off_wav = 0, off_coords = 0, off_err = 0, off_acc = 0,
           off_exa = 0, off_iexa = 0, off_tab = 0, off_cnt = 0, total = 0;
    std::vector<StepArgs> queued;
    StepMode queued_mode = kModeForward;
    CUtensorMap tm_u2{}, tm_u1{}, tm_vel{};
    cudaStream_t st = nullptr;

    float* F(size_t o) const { return reinterpret_cast<float*>(scratch + o); }
    int* I(size_t o) const { return reinterpret_cast<int*>(scratch + o); }

    int setup(int order_, int dimx_, int dimy_, int nt_, float h_, float dt_, bool with_acc,
              cudaStream_t st_, bool with_exa = false) {
        TWI_TRY(check_order(order_));
        order = order_, ne = order_ / 2, dimx = dimx_, dimz = dimy_, nt = nt_, h = h_, dt = dt_;
        nx = dimx - order;
        nz = dimz - order;
        st = st_;
        if (nx < 1 || nz < 1 || nt < 1) return fail(TWI_ERR_INVALID, "dimx, dimy must exceed order and nt >= 1");
        if (!(h > 0.f) || !(dt > 0.f)) return fail(TWI_ERR_INVALID, "h and dt must be positive");
        pitch = (dimx + kTileX - 1) / kTileX * kTileX;
        slot_elems = (long long)pitch * dimz;
        size_t off = 0;
        auto take = [&](size_t b) { size_t o = off; off = align256(off + b); return o; };
        off_vpad = take((size_t)slot_elems * 4);
        off_fields = take((size_t)4 * slot_elems * 4);   // zero slot + 3 rotating
        off_acc = take(with_acc ? (size_t)slot_elems * 4 : 0);
        off_exa = take(with_exa ? (size_t)slot_elems * 4 : 0);
        off_iexa = take(with_exa ? (size_t)slot_elems * 2 : 0);
        off_wav = take((size_t)nt * 4);
        off_coords = take(3 * 4);
        off_err = take(4);
        off_tab = take((size_t)nt * sizeof(StepArgs));   // the pass's steps, one persistent launch
        off_cnt = take(2 * sizeof(unsigned));            // ticket + the one shot's counter
        total = off;
        void* p = nullptr;
        TWI_CUDA(cudaMallocAsync(&p, total, st));
        scratch = static_cast<char*>(p);
        TWI_CUDA(cudaMemsetAsync(scratch, 0, total, st));
        TWI_CUDA(prepare_step(order, true, LaunchShape{4, 4}));
        const int TZ = 16, HZ = zhalo(order);
        TWI_TRY(make_map(&tm_u2, F(off_fields), dimx, dimz, 4, pitch, kBoxX, TZ + 2 * HZ));
        TWI_TRY(make_map(&tm_u1, F(off_fields), dimx, dimz, 4, pitch, kTileX, TZ));
        TWI_TRY(make_map(&tm_vel, F(off_vpad), dimx, dimz, 0, pitch, kTileX, TZ));
        return TWI_OK;
    }

    int load_vel(const float* vel) {
        TWI_CUDA(cudaMemcpy2DAsync(F(off_vpad), (size_t)pitch * 4, vel, (size_t)dimx * 4,
                                   (size_t)dimx * 4, dimz, cudaMemcpyDeviceToDevice, st));
        return TWI_OK;
    }

    StepArgs args() const {
        StepArgs a{};
        a.dimx = dimx, a.dimz = dimz, a.pitch = pitch, a.nx = nx, a.nz = nz;
        a.slot_elems = slot_elems;
        a.fields = F(off_fields);
        a.vel = F(off_vpad);
        a.nshots = 1;
        a.spc = 1;
        const float dt2 = dt * dt, h2 = h * h;
        a.dt2 = dt2, a.h2 = h2, a.dtoh2 = dt2 / h2, a.hdt = h * dt;
        a.cons = static_cast<float>(-2.0 / static_cast<double>(dt2));
        a.src_rc = I(off_coords);
        a.rec_row = I(off_coords) + 2;
        a.wav = F(off_wav);
        a.wav_stride = 0;
        a.frd_stride = (long long)nt * nx;
        a.resid_stride = (long long)nt * nx;
        a.err = I(off_err);
        return a;
    }

    // Steps are queued and run by flush() as ONE persistent launch
    // (twi_persist.cuh): a single shot's step is a few microseconds of work,
    // so nt separate launches would be bound by launch latency.
    int launch(StepMode mode, const StepArgs& a) {
        if (!queued.empty() && queued_mode != mode) TWI_TRY(flush());
        queued_mode = mode;
        queued.push_back(a);
        return TWI_OK;
    }

    int flush() {
        if (queued.empty()) return TWI_OK;
        if (queued.size() > (size_t)nt) return fail(TWI_ERR_STATE, "step table too small");
        StepArgs* tab = reinterpret_cast<StepArgs*>(scratch + off_tab);
        // pageable source: staged before the call returns
        TWI_CUDA(cudaMemcpyAsync(tab, queued.data(), queued.size() * sizeof(StepArgs),
                                 cudaMemcpyHostToDevice, st));
        unsigned* cnt = reinterpret_cast<unsigned*>(scratch + off_cnt);
        TWI_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned), st));
        const LaunchShape sh{4, 4};
        int nbc = 0;
        const int per_step = step_ctas(order, sh, queued[0], &nbc);   // one shot: one group
        if (per_step <= 0) return fail(TWI_ERR_INVALID, "launch too large");
        // two steps' worth of CTAs: the next step's items are claimed while the
        // current one finishes, without a device full of waiting CTAs
        const PersistLaunch L{tab, (int)queued.size(), 1, per_step, nbc, cnt, cnt + 1, 2 * per_step};
        cudaError_t e = launch_step_persistent(order, true, queued_mode, sh, tm_u2, tm_u1, tm_vel, L, st);
        queued.clear();
        if (e != cudaSuccess) return fail(TWI_ERR_CUDA, std::string("step launch: ") + cudaGetErrorString(e));
        return TWI_OK;
    }

    // Leave the last three wavefields in the caller's work arrays the way the
    // reference's loop does (propagator_cpu.cpp:57-78, 129-150: its u3 is the
    // output of each step and the three pointers rotate, so the field written
    // in step c ends up in u3, u1, u2 for c % 3 = 0, 1, 2; arrays no step
    // wrote keep the zeros the reference clears them to).  Step c wrote this
    // run's slot rot_slot(c + 1).  Nothing happens when any pointer is null.
    int mirror_fields(float* u1, float* u2, float* u3) const {
        if (!u1 || !u2 || !u3) return TWI_OK;
        float* buf[3] = {u3, u1, u2};
        const size_t bytes = (size_t)dimx * dimz * 4;
        for (float* b : buf) TWI_CUDA(cudaMemsetAsync(b, 0, bytes, st));
        for (int c = nt - 3 < 0 ? 0 : nt - 3; c < nt; ++c) {
            const long long k = (long long)c + 1;
            const float* src = F(off_fields) + (long long)(1 + (int)(k % 3)) * slot_elems;
            TWI_CUDA(cudaMemcpy2DAsync(buf[c % 3], (size_t)dimx * 4, src, (size_t)pitch * 4,
                                       (size_t)dimx * 4, dimz, cudaMemcpyDeviceToDevice, st));
        }
        return TWI_OK;
    }

    // read the error word, release scratch
    int finish(int status) {
        int err = 0;
        if (scratch) {
            if (status == TWI_OK) {
                if (cudaMemcpyAsync(&err, I(off_err), 4, cudaMemcpyDeviceToHost, st) != cudaSuccess)
                    status = fail(TWI_ERR_CUDA, "error word copy failed");
            }
            cudaFreeAsync(scratch, st);
            scratch = nullptr;
            if (cudaStreamSynchronize(st) != cudaSuccess && status == TWI_OK)
                status = fail(TWI_ERR_CUDA, cudaGetErrorString(cudaGetLastError()));
        }
        if (status == TWI_OK && err)
            status = fail(TWI_ERR_DEVICE, "device error word " + std::to_string(err));
        return status;
    }
};

Slot rot_slot(long long k) { return k <= 0 ? Slot{0, 0} : Slot{1 + (int)(k % 3), 0}; }

int ref_forward(float* frd, float* virt, float* u1, float* u2, float* u3, const float* vel,
                const float* w, int order, int dimx, int dimy, int nt, float h, float dt, float sx,
                float sy, float ry, cudaStream_t st) {
    if (!frd || !vel || !w) return fail(TWI_ERR_INVALID, "null array");
    RefRun R;
    int s = R.setup(order, dimx, dimy, nt, h, dt, false, st);
    if (s == TWI_OK) s = R.load_vel(vel);
    int coords[3];
    if (s == TWI_OK) s = shot_cells(sx, sy, ry, h, R.nx, R.nz, R.ne, R.dimz, &coords[0], &coords[1], &coords[2]);
    if (s == TWI_OK && cudaMemcpyAsync(R.I(R.off_coords), coords, 12, cudaMemcpyHostToDevice, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "coordinate upload failed");
    if (s == TWI_OK && cudaMemcpyAsync(R.F(R.off_wav), w, (size_t)nt * 4, cudaMemcpyDefault, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "wavelet upload failed");
    if (s == TWI_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "sync failed");
    if (s == TWI_OK) {
        StepArgs a = R.args();
        a.frd = frd;
        a.virt_out = virt;
        a.virt_slot_elems = (long long)dimx * dimy;
        a.virt_pitch = dimx;
        a.virt_stride = 0;
        a.virt_vec4 = (dimx % 4 == 0 && reinterpret_cast<uintptr_t>(virt) % 16 == 0) ? 1 : 0;
        for (int it = 0; it < nt && s == TWI_OK; ++it) {
            const Slot pv = rot_slot(it - 1), cu = rot_slot(it), nx_ = rot_slot(it + 1);
            a.it = it;
            a.prev_base = pv.base, a.cur_base = cu.base, a.next_base = nx_.base;
            a.virt_base = it;
            s = R.launch(virt ? kModeRecompute : kModeForward, a);
        }
        if (s == TWI_OK) s = R.flush();
    }
    if (s == TWI_OK) s = R.mirror_fields(u1, u2, u3);
    return R.finish(s);
}

int exa_check(int nt) {
    if (nt > 32767) return fail(TWI_ERR_INVALID, "excitation amplitude stores 16-bit step indices: nt <= 32767");
    return TWI_OK;
}

}  // namespace

extern "C" {

int twi_fdm_exa_forward(float* frd, float* exa, short* iexa, float* u1, float* u2, float* u3,
                        const float* vel, const float* w, int order, int dimx, int dimy, int nt,
                        float h, float dt, float sx, float sy, float ry, void* stream) {
    if (!frd || !exa || !iexa || !vel || !w) return fail(TWI_ERR_INVALID, "null array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RefRun R;
    int s = exa_check(nt);
    if (s == TWI_OK) s = R.setup(order, dimx, dimy, nt, h, dt, false, st, true);
    if (s == TWI_OK) s = R.load_vel(vel);
    int coords[3];
    if (s == TWI_OK) s = shot_cells(sx, sy, ry, h, R.nx, R.nz, R.ne, R.dimz, &coords[0], &coords[1], &coords[2]);
    if (s == TWI_OK && cudaMemcpyAsync(R.I(R.off_coords), coords, 12, cudaMemcpyHostToDevice, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "coordinate upload failed");
    if (s == TWI_OK && cudaMemcpyAsync(R.F(R.off_wav), w, (size_t)nt * 4, cudaMemcpyDefault, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "wavelet upload failed");
    if (s == TWI_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "sync failed");
    if (s == TWI_OK) {
        StepArgs a = R.args();
        a.frd = frd;
        a.exa = R.F(R.off_exa);
        a.iexa = reinterpret_cast<short*>(R.scratch + R.off_iexa);
        for (int it = 0; it < nt && s == TWI_OK; ++it) {
            const Slot pv = rot_slot(it - 1), cu = rot_slot(it), nx_ = rot_slot(it + 1);
            a.it = it;
            a.prev_base = pv.base, a.cur_base = cu.base, a.next_base = nx_.base;
            s = R.launch(kModeExaForward, a);
        }
        if (s == TWI_OK) s = R.flush();
        if (s == TWI_OK &&
            (cudaMemcpy2DAsync(exa, (size_t)dimx * 4, R.F(R.off_exa), (size_t)R.pitch * 4,
                               (size_t)dimx * 4, dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
             cudaMemcpy2DAsync(iexa, (size_t)dimx * 2, R.scratch + R.off_iexa, (size_t)R.pitch * 2,
                               (size_t)dimx * 2, dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess))
            s = fail(TWI_ERR_CUDA, "excitation copy failed");
    }
    if (s == TWI_OK) s = R.mirror_fields(u1, u2, u3);
    return R.finish(s);
}

int twi_fdm_exa_backward(float* grad, const float* exa, const short* iexa, float* u1, float* u2,
                         float* u3, const float* vel, const float* resid, int order, int dimx,
                         int dimy, int nt, float h, float dt, float ry, void* stream) {
    if (!grad || !exa || !iexa || !vel || !resid) return fail(TWI_ERR_INVALID, "null array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RefRun R;
    int s = exa_check(nt);
    if (s == TWI_OK) s = R.setup(order, dimx, dimy, nt, h, dt, true, st, true);
    if (s == TWI_OK) s = R.load_vel(vel);
    int coords[3] = {-1, -1, 0};
    if (s == TWI_OK) {
        const int iry = cell_of(ry, h);
        if (!(ry >= 0.f) || iry + R.ne >= R.dimz)
            s = fail(TWI_ERR_INVALID, "receiver row outside the grid: iry=" + std::to_string(iry));
        coords[2] = iry + R.ne;
    }
    if (s == TWI_OK && cudaMemcpyAsync(R.I(R.off_coords), coords, 12, cudaMemcpyHostToDevice, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "coordinate upload failed");
    if (s == TWI_OK &&
        (cudaMemcpy2DAsync(R.F(R.off_exa), (size_t)R.pitch * 4, exa, (size_t)dimx * 4, (size_t)dimx * 4,
                           dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess ||
         cudaMemcpy2DAsync(R.scratch + R.off_iexa, (size_t)R.pitch * 2, iexa, (size_t)dimx * 2,
                           (size_t)dimx * 2, dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess))
        s = fail(TWI_ERR_CUDA, "excitation copy failed");
    if (s == TWI_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "sync failed");
    if (s == TWI_OK) {
        StepArgs a = R.args();
        a.resid = resid;
        a.acc = R.F(R.off_acc);
        a.acc_mode = kAccExa;
        a.acc_base = 0;
        a.exa = R.F(R.off_exa);
        a.iexa = reinterpret_cast<short*>(R.scratch + R.off_iexa);
        for (int it = nt - 1; it >= 0 && s == TWI_OK; --it) {
            const long long m = (long long)nt - 1 - it;
            const Slot pv = rot_slot(m - 1), cu = rot_slot(m), nx_ = rot_slot(m + 1);
            a.it = it;
            a.prev_base = pv.base, a.cur_base = cu.base, a.next_base = nx_.base;
            s = R.launch(kModeAdjoint, a);
        }
        if (s == TWI_OK) s = R.flush();
        if (s == TWI_OK &&
            cudaMemcpy2DAsync(grad, (size_t)dimx * 4, R.F(R.off_acc), (size_t)R.pitch * 4,
                              (size_t)dimx * 4, dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            s = fail(TWI_ERR_CUDA, "gradient copy failed");
    }
    if (s == TWI_OK) s = R.mirror_fields(u1, u2, u3);
    return R.finish(s);
}

int twi_fdm_forward(float* frd, float* virt, float* u1, float* u2, float* u3, const float* vel,
                    const float* w, int order, int dimx, int dimy, int nt, float h, float dt,
                    float sx, float sy, float ry, void* stream) {
    if (!virt) return fail(TWI_ERR_INVALID, "virt must not be null (use twi_fdm_forward_only)");
    return ref_forward(frd, virt, u1, u2, u3, vel, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                       static_cast<cudaStream_t>(stream));
}

int twi_fdm_forward_only(float* frd, float* u1, float* u2, float* u3, const float* vel,
                         const float* w, int order, int dimx, int dimy, int nt, float h,
                         float dt, float sx, float sy, float ry, void* stream) {
    return ref_forward(frd, nullptr, u1, u2, u3, vel, w, order, dimx, dimy, nt, h, dt, sx, sy, ry,
                       static_cast<cudaStream_t>(stream));
}

int twi_fdm_backward(float* grad, const float* virt, float* u1, float* u2, float* u3,
                     const float* vel, const float* resid, int order, int dimx, int dimy, int nt,
                     float h, float dt, float ry, void* stream) {
    if (!grad || !virt || !vel || !resid) return fail(TWI_ERR_INVALID, "null array");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    RefRun R;
    int s = R.setup(order, dimx, dimy, nt, h, dt, true, st);
    if (s == TWI_OK) s = R.load_vel(vel);
    int coords[3] = {-1, -1, 0};
    if (s == TWI_OK) {
        const int iry = cell_of(ry, h);
        if (!(ry >= 0.f) || iry + R.ne >= R.dimz)
            s = fail(TWI_ERR_INVALID, "receiver row outside the grid: iry=" + std::to_string(iry));
        coords[2] = iry + R.ne;
    }
    if (s == TWI_OK && cudaMemcpyAsync(R.I(R.off_coords), coords, 12, cudaMemcpyHostToDevice, st) != cudaSuccess)
        s = fail(TWI_ERR_CUDA, "coordinate upload failed");
    if (s == TWI_OK && cudaStreamSynchronize(st) != cudaSuccess) s = fail(TWI_ERR_CUDA, "sync failed");
    if (s == TWI_OK) {
        StepArgs a = R.args();
        a.resid = resid;
        a.virt_in = virt;
        a.virt_slot_elems = (long long)dimx * dimy;
        a.virt_pitch = dimx;
        a.virt_stride = 0;
        a.virt_vec4 = (dimx % 4 == 0 && reinterpret_cast<uintptr_t>(virt) % 16 == 0) ? 1 : 0;
        a.acc = R.F(R.off_acc);
        a.acc_mode = kAccPlainPerShot;
        a.acc_base = 0;
        for (int it = nt - 1; it >= 0 && s == TWI_OK; --it) {
            const long long m = (long long)nt - 1 - it;
            const Slot pv = rot_slot(m - 1), cu = rot_slot(m), nx_ = rot_slot(m + 1);
            a.it = it;
            a.prev_base = pv.base, a.cur_base = cu.base, a.next_base = nx_.base;
            a.virt_base = it;
            s = R.launch(kModeAdjoint, a);
        }
        if (s == TWI_OK) s = R.flush();
        if (s == TWI_OK &&
            cudaMemcpy2DAsync(grad, (size_t)dimx * 4, R.F(R.off_acc), (size_t)R.pitch * 4,
                              (size_t)dimx * 4, dimy, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
            s = fail(TWI_ERR_CUDA, "gradient copy failed");
    }
    if (s == TWI_OK) s = R.mirror_fields(u1, u2, u3);
    return R.finish(s);
}

}  // extern "C"
