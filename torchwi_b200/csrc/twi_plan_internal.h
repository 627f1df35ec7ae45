// twi_plan_internal.h -- plan operations shared between translation units of
// the library (not part of the C ABI).
#pragma once

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

}  // namespace twi

// Tensor maps of a bound plan: u^n box, u^{n-1} box, velocity box.
void plan_tensor_maps(const twi_plan* P, CUtensorMap out[3]);
// The gathers / residual region and its element count.
float* plan_gathers(const twi_plan* P);
long long plan_gathers_elems(const twi_plan* P);
// All steps of a request: forward (with checkpoints when kind == 1), then
// for kind == 1 the gradient steps; *fwd_steps = number of forward steps.
void plan_steps(const twi_plan* P, int kind, std::vector<twi::TwiStep>& out, size_t* fwd_steps);
int plan_gradient_prologue(const twi_plan* P, cudaStream_t st);
int plan_gradient_epilogue(const twi_plan* P, cudaStream_t st);
void plan_mark_done(twi_plan* P, int kind);
int plan_check_compatible(const twi_plan* P, int kind, int order, bool exact, int rows_per_warp);
