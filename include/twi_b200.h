/* twi_b200.h -- C ABI of the B200 time-domain 2D acoustic propagator.
 *
 * Plain C types only: device pointers are `void*`/`float*` into memory the
 * caller owns (PyTorch tensors in the Python layer), streams are
 * `cudaStream_t` passed as `void*` (NULL = legacy default stream).  Every
 * function returns an int status; on failure twi_last_error() returns a
 * message for the calling thread.
 *
 * Two levels:
 *   1. Reference-shaped entry points (twi_fdm_*) with the argument lists of
 *      TorchWI's native propagator functions, for code that binds those
 *      directly.
 *   2. The plan API: batched shots, checkpointed adjoint, Kahan-summed
 *      gradient, CUDA-graph time loops.  This is what torchwi_b200.Time2d
 *      uses.
 */
#ifndef TWI_B200_H
#define TWI_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    TWI_OK = 0,
    TWI_ERR_INVALID = 1, /* bad argument (order, sizes, shot/receiver position, ...) */
    TWI_ERR_CUDA = 2,    /* a CUDA runtime call failed */
    TWI_ERR_STATE = 3,   /* call out of sequence (e.g. gradient before forward) */
    TWI_ERR_DEVICE = 4,  /* a kernel raised the device error word (bounded wait ran out) */
    TWI_ERR_NOMEM = 5    /* workspace too small */
};

/* Library version (major*10000 + minor*100 + patch). */
int twi_version(void);

/* Message describing the last failure on this thread ("" if none). */
const char* twi_last_error(void);

/* ------------------------------------------------------------------------
 * 1. Reference-shaped entry points
 *
 * Layout as in the reference: vel, u1, u2, u3 and grad are [dimy][dimx]
 * (x fastest) with dimx = nx + order, dimy = ny + order; frd and resid are
 * [nt][nx]; virt is [nt][dimy][dimx].  All array pointers are device
 * pointers except `w`, which may be host or device memory (the reference
 * keeps it on the host).  Semantics are those of the reference's CPU
 * propagator (unpadded grid, Keys on left/right/bottom, free top), computed
 * on the GPU with bit-identical FP32 results.  u1/u2/u3 ([dimy][dimx]
 * device arrays, as the reference's work arrays) receive on return the last
 * three wavefields, arranged as the reference's rotating pointers leave
 * them; passing NULL for any of them skips that.  Scratch is taken with
 * cudaMallocAsync on `stream` and released before return.
 * ------------------------------------------------------------------------ */

/* Replaces c_fdm_forward / cuda_fdm_forward
 * (torchwi/propagator/td2d/propagator_cpu.h:2-18,
 *  torchwi/propagator/td2d/propagator_cuda.h:2-18; bound from Python in
 *  wrapper_cuda.cpp:45-79). */
int twi_fdm_forward(float* frd, float* virt, float* u1, float* u2, float* u3,
                    const float* vel, const float* w, int order, int dimx, int dimy,
                    int nt, float h, float dt, float sx, float sy, float ry,
                    void* stream);

/* Replaces c_fdm_backward / cuda_fdm_backward
 * (propagator_cpu.h:20-34, propagator_cuda.h:21-35; wrapper_cuda.cpp:81-113).
 * `grad` ([dimy][dimx]) is overwritten, not accumulated. */
int twi_fdm_backward(float* grad, const float* virt, float* u1, float* u2, float* u3,
                     const float* vel, const float* resid, int order, int dimx,
                     int dimy, int nt, float h, float dt, float ry, void* stream);

/* Replaces c_fdm_forward_only / cuda_fdm_forward_only
 * (propagator_cpu.h:37-53, propagator_cuda.h:38-53;
 *  wrapper_forward_cuda.cpp:30-61). */
int twi_fdm_forward_only(float* frd, float* u1, float* u2, float* u3, const float* vel,
                         const float* w, int order, int dimx, int dimy, int nt, float h,
                         float dt, float sx, float sy, float ry, void* stream);

/* Forward modelling of one shot that allocates no device memory, for
 * callers that cannot call cudaMalloc (code running inside another
 * framework's memory pool or a fixed arena, hosts that forbid allocation
 * after start-up, callers that must avoid an allocation's implicit
 * synchronisation).  No counterpart in the reference.
 *
 * Same inputs and output as twi_fdm_forward_only, without the unused
 * u1/u2/u3; `vel` and `frd` are device pointers, `w` host or device.  The
 * scratch is a file-scope device array of 32 MiB reserved on every GPU that
 * loads the library: grids need
 *   5 * roundup(dimx,128) * dimy * 4 + nt * 4 bytes (+ < 2 KiB)
 * to fit, larger ones are rejected with TWI_ERR_INVALID.  Every call looks
 * up the scratch address on the current device (cudaGetSymbolAddress)
 * before any work, so the address stays valid across device resets.  All
 * calls share the scratch: calls whose work overlaps on the GPU race, so
 * issue them on one stream or synchronise between them.  Synchronises
 * `stream` before returning. */
int twi_fdm_forward_only_noalloc(float* frd, const float* vel, const float* w, int order,
                                 int dimx, int dimy, int nt, float h, float dt, float sx,
                                 float sy, float ry, void* stream);

/* Excitation-amplitude variants, replacing the reference's td2d_exa_cuda
 * module functions (torchwi/propagator/td2d/propagator_exa_cuda.h:2-38,
 * wrapper_exa_cuda.cpp:9-83).  exa is [dimy][dimx] float, iexa [dimy][dimx]
 * int16 (the step of the largest-magnitude virtual source); nt <= 32767. */
int twi_fdm_exa_forward(float* frd, float* exa, short* iexa, float* u1, float* u2, float* u3,
                        const float* vel, const float* w, int order, int dimx, int dimy, int nt,
                        float h, float dt, float sx, float sy, float ry, void* stream);
int twi_fdm_exa_backward(float* grad, const float* exa, const short* iexa, float* u1, float* u2,
                         float* u3, const float* vel, const float* resid, int order, int dimx,
                         int dimy, int nt, float h, float dt, float ry, void* stream);

/* ------------------------------------------------------------------------
 * 2. Plan API
 *
 * Replaces the per-shot Time2d work buffers and the Python-side loop over
 * shots (torchwi/operator/TimeOperator.py:18-82, TimeFunction.py:108-148,
 * examples/time/inv_torch.py:128-137): one plan holds one model, `nshots`
 * shots and a workspace the caller allocates.
 * ------------------------------------------------------------------------ */

typedef struct twi_problem {
    int order;            /* 2, 4 or 8 (spatial accuracy) */
    int nx, nz;           /* model cells (unpadded) */
    int nt;               /* time steps */
    float h, dt;          /* grid spacing [m], time step [s] */
    int nshots;           /* shots advanced together */
    int ckpt_interval;    /* steps between wavefield checkpoints; 0 = choose */
    int exact;            /* 1: reference arithmetic (bit-identical to TorchWI's CPU
                             propagator); 0: fast FP32 with FMA */
    int accumulate;       /* 0: Kahan-compensated FP32 over steps and shots;
                             1: plain FP32 per shot, summed in shot order (the
                             reference's order: bit-identical gradients) */
    int shots_per_cta;    /* shots sharing one velocity tile in a CTA, 1..32; 0 = choose
                             (4, and 8 for adjoint launches) */
    int rows_per_warp;    /* 2, 4 or 8 (2: not with time_block 2); 0 = choose
                             (4, and 2 for one-step adjoint launches) */
    int use_graphs;       /* 1: capture the time loops into CUDA graphs */
    int wavelet_per_shot; /* 1: wavelet region is [nshots][nt]; 0: one [nt] */
    int forward_only;     /* 1: no checkpoint, virtual-source or gradient memory;
                             twi_gradient and save_checkpoints are refused */
    int exa;              /* 1: excitation-amplitude gradient (no checkpoints): the
                             forward pass keeps the largest virtual source per cell
                             and its step (16-bit, nt <= 32767); plan-level calls only */
    int time_block;       /* time steps per launch of twi_forward / twi_gradient: 1, 2
                             (the fields are read once per two steps), 0 = choose;
                             excitation-amplitude plans always use 1 */
    int reconstruct;      /* 1: boundary saving instead of checkpoints -- the forward
                             pass keeps the Keys cells of every time level, the
                             gradient pass rebuilds the wavefield backwards from the
                             last two levels; (nt+1) * nshots * boundary cells floats
                             instead of the checkpoint and virtual-source slots.
                             Each backward step is one fused launch: rebuild, virtual
                             source (in registers), adjoint step and gradient term.
                             2: the same with the rebuild and the adjoint step as two
                             launches per step and the virtual source passed through
                             one slot per shot.  Gradients agree with the reference
                             within its FP32 tolerance, not bit for bit (1 and 2 give
                             the same bits).  One step per launch; plan-level calls
                             only */
    int persistent;       /* 1: every pass (or checkpoint segment) of twi_forward and
                             twi_gradient is one persistent launch: CTAs take
                             (step, shot group, tile) work items in step order and
                             wait, with bounded waits, for the group's previous
                             step; 0: one launch per time step.  The same bits
                             either way; not with time_block 2 */
    int unchained;        /* 0: a run of one-step launches of one kind (a pass, or
                             a checkpoint segment's recompute or adjoint phase) is
                             chained: each launch may start its CTAs while the one
                             before it drains, and a CTA waits (bounded) only for
                             its shot group of the earlier steps; 1: every launch
                             waits for the previous one in stream order.  The same
                             bits either way; not with persistent launches */
} twi_problem;

/* Byte offsets of the caller-visible regions inside the workspace. */
typedef struct twi_layout {
    size_t workspace_bytes; /* total size to allocate (256-byte aligned base) */
    size_t vel;             /* in : model (nx, nz), z fastest, float */
    size_t wavelet;         /* in : [nshots or 1][nt] float */
    size_t gathers;         /* out: [nshots][nt][nx] float (twi_forward) */
    size_t resid;           /* in : [nshots][nt][nx] float adjoint source (twi_gradient) */
    size_t grad;            /* out: (nx, nz) float, z fastest (twi_gradient) */
    int dimx, dimz, pitch;  /* padded grid and its row pitch (floats) */
    int ckpt_interval, nsegments, shots_per_cta, rows_per_warp;
    int time_block;         /* time steps per launch chosen for this plan */
    int adjoint_rows_per_warp; /* rows per warp of one-step adjoint launches */
    int adjoint_shots_per_cta; /* shots per CTA (one Kahan group) of adjoint launches */
} twi_layout;

typedef struct twi_plan twi_plan;

/* Validate `prob` and size the workspace; no device memory is touched. */
int twi_plan_create(const twi_problem* prob, twi_plan** plan);
int twi_plan_layout(const twi_plan* plan, twi_layout* out);
/* Attach a device workspace of at least layout.workspace_bytes bytes on the
 * current device; drops captured graphs. */
int twi_plan_bind(twi_plan* plan, void* workspace, size_t bytes);
/* Shot and receiver positions in metres (host arrays of nshots floats);
 * cells are (int)(coord/h) in FP32 as in propagator_cpu.cpp:44-48.  Shots
 * must lie inside the model, receiver rows inside the grid. */
int twi_plan_set_shots(twi_plan* plan, const float* sx, const float* sy, const float* ry,
                       void* stream);
/* Pad the model from the `vel` region into the internal grid. */
int twi_plan_set_model(twi_plan* plan, void* stream);
/* Forward pass for all shots: gathers -> `gathers`.  With save_checkpoints
 * the wavefield pairs needed by twi_gradient are kept. */
int twi_forward(twi_plan* plan, int save_checkpoints, void* stream);
/* Forward pass with checkpoints that writes the L2 residual instead of the
 * gathers: resid[s][it][ix] = modelled - observed[s][it][ix] (one FP32
 * subtraction, the same bits as the reference driver's `frd - true`), and
 * *misfit = 0.5 * sum(resid^2) accumulated in FP64 in a fixed order
 * (examples/time/inv_torch.py:133-136, where torch forms the residual and
 * misfit after the gathers come back).  `observed` is a device array
 * laid out like `gathers`; `misfit` is one device double.  Follow with
 * twi_gradient. */
int twi_forward_residual(twi_plan* plan, const float* observed, double* misfit, void* stream);
/* The residual and misfit of twi_forward_residual, formed after a
 * twi_forward(plan, 1, stream) from the gathers it left: resid = gathers -
 * observed in place (the same bits) and *misfit as there.  Lets a caller
 * bring `observed` to the device while the forward pass runs (no
 * counterpart in the reference, whose driver forms the residual with torch,
 * examples/time/inv_torch.py:133-136).  Follow with twi_gradient. */
int twi_residual(twi_plan* plan, const float* observed, double* misfit, void* stream);
/* Adjoint pass for all shots from the `resid` region: recomputes the
 * forward field segment by segment from the checkpoints and writes the
 * shot-summed velocity gradient to `grad`. */
int twi_gradient(twi_plan* plan, void* stream);
/* Synchronise `stream` and report a raised device error word. */
int twi_plan_check(twi_plan* plan, void* stream);
/* Measurement hook (no counterpart in the reference): launch `repeats`
 * steady-state time steps of one kernel mode (0 forward, 1 recompute with
 * virtual-source output -- the reverse reconstruction for plans with
 * `reconstruct` --, 2 adjoint with gradient accumulation, 5 the fused
 * backward step of plans with reconstruct = 1; 10, 11, 12 the
 * two-step launches of modes 0-2 for plans with time_block 2) for all
 * shots and return the mean device time per launch in *ms_per_launch (CUDA
 * events on `stream`).  Overwrites rotating wavefield slots and the gradient
 * accumulators, never the checkpoints; call after twi_forward. */
int twi_plan_profile(twi_plan* plan, int mode, int repeats, float* ms_per_launch, void* stream);
int twi_plan_destroy(twi_plan* plan);
/* Diagnostics (no counterpart in the reference).  Every wait in the kernels
 * is bounded in time; when one runs out the kernel raises the device error
 * word (TWI_ERR_DEVICE from twi_plan_check), waits for its own copies in
 * flight and returns, leaving the context usable.  This launches a kernel
 * whose wait can never complete (nothing arrives at its barrier) with a
 * limit of `limit_us` microseconds and returns TWI_OK when the wait ran out
 * and was reported as designed; *elapsed_ms gets the kernel's duration. */
int twi_check_wait_timeout(int limit_us, float* elapsed_ms, void* stream);
/* The same for the counter wait of chained and persistent launches (a CTA
 * waiting until its shot group of the earlier steps is done): with
 * preset_error = 0 the counter never reaches its target and the wait must run
 * out after `limit_us` and raise the error word; with preset_error = 1 the
 * word already holds another CTA's error and the wait must leave at once.
 * TWI_OK when the wait ended as designed; *elapsed_ms gets the kernel's
 * duration. */
int twi_check_counter_wait(int limit_us, int preset_error, float* elapsed_ms, void* stream);
/* Workspace bytes a plan of `prob` needs (host only; admission control). */
int twi_plan_footprint_bytes(const twi_problem* prob, size_t* bytes);

/* Launch-shape autotuning (the reference has none: its CUDA path uses fixed
 * 16x16 blocks, td2d_cuda.cu).  Times every launch shape that the fields of
 * `prob` left at 0 allow -- shots per CTA 0/1/2/4/8 (at most nshots), rows
 * per warp 0/2/4/8, one or two time steps per launch (one for excitation
 * amplitude, reverse reconstruction and 2 rows per warp; 0 = the per-mode
 * defaults, which give the adjoint its own shape and which no single value
 * reproduces) -- on the current device, on a copy of the problem with nt = 8 in the
 * caller's `scratch` (twi_autotune_scratch_bytes, any contents), and writes
 * *prob with the fastest shape into `tuned` and, if not NULL, its device
 * milliseconds per time step of a gradient (forward + recompute + adjoint;
 * forward only for forward-only plans).  Synchronises `stream`. */
int twi_autotune_scratch_bytes(const twi_problem* prob, size_t* bytes);
int twi_autotune(const twi_problem* prob, void* scratch, size_t scratch_bytes, void* stream,
                 twi_problem* tuned, float* ms_per_step);

/* ------------------------------------------------------------------------
 * 3. Batches of plans
 *
 * Several bound plans -- any grid sizes, shot counts and nt, sharing order,
 * arithmetic and rows_per_warp -- advanced together: every time step is one
 * launch per kernel mode covering all plans that still have work (plans
 * with fewer steps drop out).  Results equal running each plan on its own,
 * bit for bit.  Replaces the reference's one-shot-per-process Horovod loop
 * for many models (examples/time/inv_torch.py:128-137).  No counterpart in
 * the reference's native code.
 * ------------------------------------------------------------------------ */

typedef struct twi_batch twi_batch;

/* Host only: checks the plans and sizes the batch's device workspace (job
 * tables and tensor maps). */
int twi_batch_create(twi_plan* const* plans, int nplans, twi_batch** batch);
int twi_batch_workspace_size(const twi_batch* batch, size_t* bytes);
/* Every plan must be bound first; rebinding a plan requires rebinding the
 * batch. */
int twi_batch_bind(twi_batch* batch, void* workspace, size_t bytes);
/* twi_forward / twi_gradient of every plan, interleaved step by step. */
int twi_batch_forward(twi_batch* batch, int save_checkpoints, void* stream);
int twi_batch_gradient(twi_batch* batch, void* stream);
int twi_batch_destroy(twi_batch* batch);

/* ------------------------------------------------------------------------
 * 4. Request engine (continuous batching)
 *
 * Requests are bound plans with shots, model and wavelet set: kind 0 =
 * forward modelling (gathers), kind 1 = gradient (forward with checkpoints,
 * residual gathers - observed, checkpointed adjoint; the observed gathers
 * [nshots][nt][nx] are a device pointer, NULL meaning zero data).  Each tick advances every
 * in-flight request by one time step, one launch per kernel mode for all of
 * them; requests join and leave between ticks.  A request's result equals
 * running its plan alone, bit for bit.  No counterpart in the reference.
 * ------------------------------------------------------------------------ */

typedef struct twi_engine twi_engine;

/* max_requests: requests in flight at once (further ones wait). */
int twi_engine_create(int order, int exact, int rows_per_warp, int max_requests,
                      twi_engine** engine);
int twi_engine_workspace_size(const twi_engine* engine, size_t* bytes);
/* Device workspace for job tables and tensor maps; also allocates the pinned
 * host staging ring on first bind. */
int twi_engine_bind(twi_engine* engine, void* workspace, size_t bytes);
/* Queue a request; `tag` identifies it in twi_engine_run's report.  The plan
 * and the observed buffer must stay alive until the request is reported. */
int twi_engine_submit(twi_engine* engine, twi_plan* plan, int kind, const float* observed,
                      long long tag);
/* Enqueue up to `ticks` ticks on `stream` (returns early once a request
 * finished) and report up to max_done finished tags.  A reported request's
 * outputs are complete once `stream` reaches this point. */
int twi_engine_run(twi_engine* engine, int ticks, void* stream, long long* done_tags,
                   int max_done, int* ndone);
/* Requests in flight on the device, and submitted or finished but not yet
 * reported. */
int twi_engine_pending(const twi_engine* engine, int* in_flight, int* waiting);
int twi_engine_destroy(twi_engine* engine);

#ifdef __cplusplus
}
#endif

#endif /* TWI_B200_H */
