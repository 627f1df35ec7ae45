// twi_kernels.h -- launch-level interface between the host planner
// (twi_plan.cu) and the time-step kernels (twi_step.cu).
#pragma once

#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

namespace twi {

// What one launch of the step kernel does for each shot it owns.
enum StepMode : int {
    kModeForward = 0,     // u^{n+1}; point source; optional receiver gather
    kModeRecompute = 1,   // u^{n+1}; point source; virtual source written out
    kModeAdjoint = 2,     // lambda step; adjoint source on the receiver row;
                          // gradient term accumulated
    kModeExaForward = 3,  // forward step; the virtual source of largest
                          // magnitude and its step index kept per cell
    kModeReverse = 4,     // u^{n-1} from u^n and u^{n+1} (the forward step run
                          // backwards, source removed); pad cells restored
                          // from the boundary buffer; virtual source written
    kModeBackward = 5,    // kModeReverse and kModeAdjoint of the same step in
                          // one pass (twi_backward.cu): the virtual source
                          // stays in registers
};

// Gradient accumulator layout used by kModeAdjoint.
enum AccMode : int {
    kAccNone = 0,
    kAccPlainPerShot = 1,   // acc[shot] += term  (reference summation order)
    kAccKahanPerGroup = 2,  // Kahan pair (acc, comp)[group] over steps and shots
    kAccExa = 3,            // acc[shot] = -exa * lambda at the step stored in iexa
};

// Geometry: the padded grid has dimz rows of dimx cells stored with a row
// pitch of `pitch` floats (a multiple of 128); ne = order/2 pad cells on
// every side; nx, nz are the model dimensions.  Wavefields live in "slots"
// of pitch*dimz floats; slot(shot) = base + shot*stride.
struct StepArgs {
    int dimx, dimz, pitch, nx, nz;
    long long slot_elems;
    float* fields;
    const float* vel;           // padded velocity [dimz][pitch] (boundary cells)
    int prev_base, prev_stride;
    int cur_base, cur_stride;
    int next_base, next_stride;
    int next2_base, next2_stride;   // second output of a two-step launch (twi_step2.cu)
    int nshots;   // shots in this launch (grid.z * spc covers them)
    int spc;      // shots per CTA
    int it;       // time index of this step
    float dtoh2, dt2, h2, hdt, cons;
    // point source (modes 0, 1): src_rc[2*s] = padded row, [2*s+1] = column
    const int* src_rc;
    const float* wav;
    long long wav_stride;       // wav[s*wav_stride + it]
    // receivers: padded row per shot
    const int* rec_row;
    float* frd;                 // gathers (mode 0, may be null)
    long long frd_stride;       // frd[s*frd_stride + it*nx + ix]
    const float* obs;           // observed gathers, same layout as frd: when set,
                                // frd receives the residual modelled - observed
    // adjoint source (mode 2)
    const float* resid;
    long long resid_stride;     // resid[s*resid_stride + it*nx + ix]
    // virtual source out (mode 1) / in (mode 2): element (slot, r, c) at
    // virt[(slot)*virt_slot_elems + r*virt_pitch + c]
    float* virt_out;
    const float* virt_in;
    long long virt_slot_elems;
    int virt_pitch;
    int virt_base, virt_stride;
    int virt_vec4;              // 1 when float4 access is aligned
    // gradient accumulators (mode 2), same pitch/slot size as the fields
    float* acc;
    float* acc_comp;
    // excitation amplitude (modes 3 and kAccExa): per shot, same pitch/slot size
    float* exa;
    short* iexa;
    // boundary saving: Keys cells of u^k, bnd[(k*nshots + s)*bnd_cells + idx]
    // (idx in the boundary CTAs' cell order); written by kModeForward when
    // set, read by kModeReverse
    float* bnd;
    int bnd_cells;
    int acc_mode;
    int acc_base;               // slot of group 0 / shot 0
    int* err;                   // device error word (bit 0: TMA wait timeout)
    // kModeBackward: the adjoint field's slots (prev/cur/next above hold
    // u^{it+1}, u^it and the rebuilt u^{it-1})
    int lprev_base, lprev_stride;
    int lcur_base, lcur_stride;
    int lnext_base, lnext_stride;
    // Chained launches (one launch per step, each free to start its CTAs
    // while the previous one drains): chain[g] counts the finished CTAs of
    // shot group g over the chain's launches.  A CTA of group g of the
    // chain's launch k waits until chain[g] >= k * chain_per_group and adds
    // one when it is done; chained launches order their CTAs group by group.
    // Null: stream order alone.
    unsigned* chain;
    int chain_k, chain_per_group;
};

// A persistent launch (twi_persist.cuh): `nsteps` consecutive time steps of
// one plan pass in one launch, steps[s] holding the arguments of step s
// (device memory).  Each step has `ngroups` shot groups of `per_group` CTAs
// (`nbc` boundary CTAs, then the interior tiles).  ticket and count[ngroups]
// must be zero when the launch starts.
struct PersistLaunch {
    const StepArgs* steps;
    int nsteps, ngroups, per_group, nbc;
    unsigned* ticket;
    unsigned* count;
    int max_ctas;   // 0: as many CTAs as fit the device; else at most this many
};

// The part of a time step's arguments that changes from step to step.
struct StepDyn {
    int it;
    int prev_base, prev_stride;
    int cur_base, cur_stride;
    int next_base, next_stride;
    int virt_base;
    int lprev_base, lprev_stride;   // kModeBackward: the adjoint field's slots
    int lcur_base, lcur_stride;
    int lnext_base, lnext_stride;
};

__host__ __device__ inline StepDyn dyn_of(const StepArgs& a) {
    return StepDyn{a.it, a.prev_base, a.prev_stride, a.cur_base, a.cur_stride,
                   a.next_base, a.next_stride, a.virt_base,
                   a.lprev_base, a.lprev_stride, a.lcur_base, a.lcur_stride,
                   a.lnext_base, a.lnext_stride};
}

// The per-step part of `d` written into `a`.
__host__ __device__ inline void apply_dyn(StepArgs& a, const StepDyn& d) {
    a.it = d.it;
    a.prev_base = d.prev_base, a.prev_stride = d.prev_stride;
    a.cur_base = d.cur_base, a.cur_stride = d.cur_stride;
    a.next_base = d.next_base, a.next_stride = d.next_stride;
    a.virt_base = d.virt_base;
    a.lprev_base = d.lprev_base, a.lprev_stride = d.lprev_stride;
    a.lcur_base = d.lcur_base, a.lcur_stride = d.lcur_stride;
    a.lnext_base = d.lnext_base, a.lnext_stride = d.lnext_stride;
}

// Tensor maps per plan in the device tables of batches and the engine: the
// plan's u^n box, u^{n-1} box and velocity box at its main tile height, then
// the same three at the tile height of its adjoint-type launches.
constexpr int kMapsPerPlan = 6;

// One job of a multi-plan launch (device memory, 64-byte aligned).
struct alignas(64) MultiJob {
    StepArgs a;
    int cta_begin;   // first CTA of this job in the launch
    int plan;        // index of the plan's tensor maps (kMapsPerPlan per plan)
    int nbc;         // boundary CTAs per shot group
    int ncta;        // CTAs of this job
};

// An engine launch, passed as a kernel parameter: per job its CTA offset,
// the device-resident template of its request and kernel mode (the static
// arguments) and the per-step integers.
constexpr int kEngineMaxJobs = 64;
struct EngineLaunch {
    int njobs;
    int cta_begin[kEngineMaxJobs];
    const MultiJob* tmpl[kEngineMaxJobs];
    StepDyn dyn[kEngineMaxJobs];
};

struct LaunchShape {
    int rows_per_warp;   // 4 or 8
    int warps;           // warps per CTA, stacked along z
};

// Launches one time step.  tm_u2 is a tensor map over the field slots with a
// (136, TZ + order) box (4-column / ne-row halo), tm_u1 the same slots with a
// (128, TZ) box and tm_vel the padded velocity with a (128, TZ) box, where
// TZ = 4 * rows_per_warp.
cudaError_t launch_step(int order, bool exact, StepMode mode, LaunchShape shape,
                        const CUtensorMap& tm_u2, const CUtensorMap& tm_u1,
                        const CUtensorMap& tm_vel, const StepArgs& a, cudaStream_t stream);

// CTAs a single-plan launch of `a` uses, and its boundary CTAs per shot group.
int step_ctas(int order, LaunchShape shape, const StepArgs& a, int* nbc);

// CTAs of the single-plan kernel resident per SM on the current device (0 on
// error); with the SM count this gives a launch's number of waves.
int step_resident_ctas(int order, bool exact, StepMode mode, LaunchShape shape);
int backward_resident_ctas(int order, bool exact, LaunchShape shape);

// Chained launches pay a fixed cost per CTA (the counter poll before its first
// copies, the release after its last store) and win back about half a wave
// of tail per launch, so runs are chained only while one launch is at most
// this many waves of CTAs.
constexpr double kChainMaxWaves = 8.0;

// One launch covering several jobs (tensor maps in device memory);
// begins[i] = jobs[i].cta_begin, ascending.  `chained`: a later launch of a
// chain (the jobs' arguments carry its counters), free to start while the
// stream's previous launch drains.
cudaError_t launch_step_multi(int order, bool exact, StepMode mode, LaunchShape shape,
                              const MultiJob* jobs, const int* begins, int njobs, long long nctas,
                              const CUtensorMap* tmaps, cudaStream_t stream, bool chained = false);

// One engine launch (job entries in device memory, index in parameters).
cudaError_t launch_step_engine(int order, bool exact, StepMode mode, LaunchShape shape,
                               const EngineLaunch& L, long long nctas, const CUtensorMap* tmaps,
                               cudaStream_t stream);

// Set kernel attributes for all modes of (order, exact, shape) on the current
// device.  Must run before a stream capture that launches them.
cudaError_t prepare_step(int order, bool exact, LaunchShape shape);

// Tile geometry shared by host and device.
constexpr int kTileX = 128;                    // columns per CTA (32 lanes x float4)
constexpr int kHaloX = 4;                      // x halo, keeps TMA x origins 16-byte aligned
constexpr int kBoxX = kTileX + 2 * kHaloX;     // 136 columns per staged row
__host__ __device__ constexpr int zhalo(int order) { return order / 2; }
// Boundary (Keys) cells are computed by dedicated CTAs, one thread per cell
// and this many cells per thread, ahead of the interior tiles in the grid.
constexpr int kBoundaryCellsPerThread = 4;
constexpr int kThreads = 128;
// Largest shot group of one CTA (its shots' source and receiver cells are
// staged in shared memory by the fused backward kernel).
constexpr int kMaxShotsPerCta = 32;

// Two-step launches (twi_step2.cu): output tiles of kTile2X columns.  tm_un
// is a tensor map over the field slots with a (136, 4*rows_per_warp + 2*order)
// box, tm_um the same slots with a (128, 4*rows_per_warp + order) box and
// tm_v the padded velocity with that box (step2_box_rows gives the rows:
// which = 0 for tm_un, 1 for the others).  Modes 0-2; step A is time a.it,
// step B a.it + 1 (a.it - 1 for the adjoint).
constexpr int kTile2X = 120;
long long step2_ctas(int order, int rows_per_warp, const StepArgs& a);
int step2_box_rows(int order, int rows_per_warp, int which);
cudaError_t launch_step2(int order, bool exact, StepMode mode, LaunchShape shape,
                         const CUtensorMap& tm_un, const CUtensorMap& tm_um, const CUtensorMap& tm_v,
                         const StepArgs& a, cudaStream_t stream);
cudaError_t prepare_step2(int order, bool exact, LaunchShape shape);

// Fused backward step of boundary-saving plans (twi_backward.cu): rebuild
// u^{it-1} (kModeReverse), step lambda (kModeAdjoint) and accumulate the
// gradient with the virtual source held in registers.  Same tensor maps as
// launch_step (tm_c: (136, TZ + order) box, tm_p and tm_vel: (128, TZ));
// rows_per_warp 2 or 4.
int backward_ctas(int order, int rows_per_warp, const StepArgs& a, int* nbc);
cudaError_t launch_backward(int order, bool exact, LaunchShape shape, const CUtensorMap& tm_c,
                            const CUtensorMap& tm_p, const CUtensorMap& tm_vel, const StepArgs& a,
                            cudaStream_t stream);
cudaError_t prepare_backward(int order, bool exact, LaunchShape shape);

// Persistent launches (twi_persist.cuh): every step of P in one launch; the
// CTAs of one step are those a one-step launch of P.steps[0] would use
// (step_ctas / backward_ctas give nbc and the total).
cudaError_t launch_step_persistent(int order, bool exact, StepMode mode, LaunchShape shape,
                                   const CUtensorMap& tm_u2, const CUtensorMap& tm_u1,
                                   const CUtensorMap& tm_vel, const PersistLaunch& P,
                                   cudaStream_t stream);
cudaError_t launch_backward_persistent(int order, bool exact, LaunchShape shape, const CUtensorMap& tm_c,
                                       const CUtensorMap& tm_p, const CUtensorMap& tm_vel,
                                       const PersistLaunch& P, cudaStream_t stream);
// Fused backward steps of several plans in one launch (job table in device
// memory) and engine launches of it; each job reads its plan's adjoint-height
// tensor maps.
cudaError_t launch_backward_multi(int order, bool exact, LaunchShape shape, const MultiJob* jobs,
                                  const int* begins, int njobs, long long nctas,
                                  const CUtensorMap* tmaps, cudaStream_t stream, bool chained = false);
cudaError_t launch_backward_engine(int order, bool exact, LaunchShape shape, const EngineLaunch& L,
                                   long long nctas, const CUtensorMap* tmaps, cudaStream_t stream);

// Store n host integers into device memory through kernel parameters
// (chunks of 2048), ordered on `stream` without a host synchronisation.
cudaError_t launch_store_ints(int* dst, const int* src, int n, cudaStream_t stream);

// (nx, nz) z-fastest user model -> padded [dimz][pitch] x-fastest,
// edge-replicated by ne cells (TimeOperator.py:55-58); columns >= dimx are 0.
cudaError_t launch_pad_model(const float* vel_user, float* vpad, int nx, int nz, int ne,
                             int dimx, int dimz, int pitch, cudaStream_t stream);

// Combine gradient accumulators and write the (nx, nz) z-fastest result:
// plain mode sums slots 0..nacc-1 in order; Kahan mode adds every slot's
// (sum, -comp) pair with compensation.
// misfit = 0.5 * sum(r[i]^2) over n samples, FP64, in a fixed order (the
// same bits on every call); `partial` holds kMisfitBlocks doubles of scratch.
constexpr int kMisfitBlocks = 592;
cudaError_t launch_misfit(const float* r, long long n, double* partial, double* misfit,
                          cudaStream_t stream);
// frd[i] = frd[i] - obs[i] for n samples (one FP32 subtraction each).
cudaError_t launch_residual(float* frd, const float* obs, long long n, cudaStream_t stream);

cudaError_t launch_reduce_grad(const float* acc, const float* acc_comp, int nacc,
                               long long slot_elems, int pitch, int ne, int nx, int nz,
                               int kahan, float* grad_user, cudaStream_t stream);

}  // namespace twi
