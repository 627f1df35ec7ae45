// twi_plan_internal.h -- plan operations shared between translation units of
// the library (not part of the C ABI).
#pragma once

#include <string>
#include <vector>

#include "twi_b200.h"
#include "twi_kernels.h"

namespace twi {

// One launch of one plan: the kernel mode, its arguments and the time steps
// it advances (1, or 2 for the two-step kernel; the engine and batches use
// single steps only).
struct TwiStep {
    StepMode mode;
    StepArgs a;
    int nsteps = 1;
};

// Shared by the plan and the allocation-free entry point (twi_plan.cu); each
// reports its failure through twi_last_error.
// Tensor map over `nslots` slots of [dimz][pitch] floats (x extent dimx);
// nslots == 0 gives a 2-D map.
int make_map(CUtensorMap* tm, const void* base, int dimx, int dimz, long long nslots, int pitch,
             int box_x, int box_z);
// order must be 2, 4 or 8.
int check_order(int order);
// The reference's cell lookup (int)(coord/h) in FP32 (propagator_cpu.cpp:44-48).
int cell_of(float coord, float h);
// Padded source row/column and receiver row of one shot; the shot must lie
// inside the model and the receiver row inside the grid.
int shot_cells(float sx, float sy, float ry, float h, int nx, int nz, int ne, int dimz, int* src_r,
               int* src_c, int* rec_r);
void set_last_error(const std::string& msg);
// Waves of CTAs of a one-plan launch of `nctas` CTAs of this mode and shape
// on the current device (huge when the device cannot be queried).
double launch_waves(int order, bool exact, StepMode mode, LaunchShape sh, long long nctas);

}  // namespace twi

// Tensor maps of a bound plan (kMapsPerPlan): u^n box, u^{n-1} box, velocity
// box at the main tile height, then the same at the adjoint-type launches'
// height; and that height in rows per warp.
void plan_tensor_maps(const twi_plan* P, CUtensorMap out[twi::kMapsPerPlan]);
int plan_adjoint_rows(const twi_plan* P);
// Rows per warp of fused backward launches for an engine or plan created with
// `rows_per_warp` (0 = choose): 2 unless 4 is asked for explicitly.
inline int backward_rows(int rows_per_warp) {
    return rows_per_warp == 4 || rows_per_warp == 8 ? 4 : 2;
}
// The gathers / residual region and its element count.
float* plan_gathers(const twi_plan* P);
long long plan_gathers_elems(const twi_plan* P);
// All steps of a request: forward (with checkpoints when kind == 1), then
// for kind == 1 the gradient steps; *fwd_steps = number of forward steps.
void plan_steps(const twi_plan* P, int kind, std::vector<twi::TwiStep>& out, size_t* fwd_steps);
int plan_gradient_prologue(const twi_plan* P, cudaStream_t st);
int plan_gradient_epilogue(const twi_plan* P, cudaStream_t st);
void plan_mark_done(twi_plan* P, int kind);
// rows_per_warp: the engine's tile height; back_rows: its fused backward's.
int plan_check_compatible(const twi_plan* P, int kind, int order, bool exact, int rows_per_warp,
                          int back_rows);
