"""Python owner of a C-ABI plan: one velocity model, a batch of shots and a
device workspace allocated through PyTorch's caching allocator.

The workspace holds the model, wavelet, gathers/residual and gradient
regions (exposed here as tensor views) plus the internal wavefield slots,
checkpoints and gradient accumulators.  All work is enqueued on the current
PyTorch stream.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _capi
from ._capi import Layout, Problem, check


@dataclass
class PlanOptions:
    """Tuning and numerics switches of a plan.

    exact:       reproduce the reference CPU propagator's arithmetic bit for
                 bit (FP32 storage, FP64 where its C++ promotes); False uses
                 plain FP32 with FMA.
    accumulate:  "kahan" (compensated FP32 over time steps and shots) or
                 "plain" (per-shot FP32 sums added in shot order, the
                 reference's own order -> bit-identical gradients).
    ckpt_interval: steps between saved wavefield pairs (0 = sqrt(2 nt)).
    shots_per_cta, rows_per_warp: launch shape (0 = default).
    use_graphs:  capture the time loops into CUDA graphs.
    forward_only: size the plan for forward modelling only (no checkpoint,
                 virtual-source or gradient memory).
    exa:         excitation-amplitude gradient (the reference's exa=True mode):
                 no checkpoints; the forward pass keeps the largest virtual
                 source per cell and its step, the adjoint assigns
                 -exa*lambda at that step.  nt <= 32767.
    time_block:  time steps per kernel launch in forward and gradient passes
                 (1 or 2; 0 = the library's choice).  Two steps read the
                 wavefields once per two steps; results are identical.
    reconstruct: boundary saving instead of checkpoints: the forward pass keeps
                 the absorbing-boundary cells of every step and the gradient
                 pass rebuilds the wavefield backwards in time (much less
                 memory; gradients within FP32 tolerance of the reference,
                 not bit-identical).  Each backward step is one fused launch
                 (rebuild, virtual source, adjoint step, gradient term).
    split_backward: with reconstruct, run the rebuild and the adjoint step
                 as two launches per step with the virtual source passed
                 through memory (the same bits; kept for comparison).
    persistent:  run each pass (each checkpoint segment's recompute and
                 adjoint phase) as ONE persistent launch instead of one
                 launch per time step (the same bits).
    chained:     let each one-step launch of a pass start while the previous
                 one drains, its CTAs waiting only for their shot group of
                 the previous step (the same bits; False: plain stream order).
    """

    exact: bool = True
    accumulate: str = "kahan"
    ckpt_interval: int = 0
    shots_per_cta: int = 0
    rows_per_warp: int = 0
    use_graphs: bool = True
    forward_only: bool = False
    exa: bool = False
    time_block: int = 0
    reconstruct: bool = False
    split_backward: bool = False
    persistent: bool = False
    chained: bool = True


def _stream_handle() -> ctypes.c_void_p:
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def footprint_bytes(nx, nz, nt, nshots, order=4, wavelet_per_shot=False,
                    options: PlanOptions | None = None) -> int:
    """Workspace bytes a plan of this size needs (for HBM admission)."""
    o = options or PlanOptions()
    prob = _problem(nx, nz, nt, 10.0, 1e-3, nshots, order, wavelet_per_shot, o)
    n = ctypes.c_size_t()
    check(_capi.lib().twi_plan_footprint_bytes(ctypes.byref(prob), ctypes.byref(n)))
    return int(n.value)


_TUNED: dict = {}


def autotune(nx, nz, nshots, order=4, h=10.0, dt=1e-3, options: PlanOptions | None = None,
             device=None) -> tuple[PlanOptions, float]:
    """Fastest launch shape (shots per CTA, rows per warp, time steps per
    launch) for plans of this grid and shot count on `device`, timed by the
    library on a short copy of the problem; fields already set (non-zero) in
    `options` stay fixed.  Returns (options with the shape filled in, device
    milliseconds per time step of a gradient).  Results are cached per
    problem and device."""
    o = options or PlanOptions()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    key = (dev.index, nx, nz, nshots, order, o.exact, o.accumulate, o.forward_only, o.exa,
           o.shots_per_cta, o.rows_per_warp, o.time_block, o.reconstruct, o.split_backward,
           o.persistent, o.chained)
    if key in _TUNED:
        return _TUNED[key]
    import dataclasses
    prob = _problem(nx, nz, 8, h, dt, nshots, order, False, o)
    L = _capi.lib()
    n = ctypes.c_size_t()
    check(L.twi_autotune_scratch_bytes(ctypes.byref(prob), ctypes.byref(n)))
    with torch.cuda.device(dev):
        scratch = torch.empty(int(n.value), dtype=torch.uint8, device=dev)
        tuned = Problem()
        ms = ctypes.c_float()
        check(L.twi_autotune(ctypes.byref(prob), ctypes.c_void_p(scratch.data_ptr()), n,
                             _stream_handle(), ctypes.byref(tuned), ctypes.byref(ms)))
    res = (dataclasses.replace(o, shots_per_cta=int(tuned.shots_per_cta),
                               rows_per_warp=int(tuned.rows_per_warp),
                               time_block=int(tuned.time_block)), float(ms.value))
    _TUNED[key] = res
    return res


def shot_blocks(shots: slice, nx, nz, nt, order=4, options: PlanOptions | None = None,
                budget: int | None = None, device=None) -> list[slice]:
    """Split `shots` into contiguous blocks whose plans each fit `budget`
    bytes (default: 80 % of the device's free memory), halving the block size
    until one fits; a single shot always makes a block."""
    if budget is None:
        free, _ = torch.cuda.mem_get_info(device)
        budget = int(free * 0.8)
    n = shots.stop - shots.start
    per = max(n, 1)
    while per > 1 and footprint_bytes(nx, nz, nt, per, order, options=options) > budget:
        per = (per + 1) // 2
    return [slice(a, min(a + per, shots.stop)) for a in range(shots.start, shots.stop, per)]


def _problem(nx, nz, nt, h, dt, nshots, order, wavelet_per_shot, o: PlanOptions) -> Problem:
    if o.accumulate not in ("kahan", "plain"):
        raise ValueError("accumulate must be 'kahan' or 'plain'")
    return Problem(order=int(order), nx=int(nx), nz=int(nz), nt=int(nt), h=float(h), dt=float(dt),
                   nshots=int(nshots), ckpt_interval=int(o.ckpt_interval), exact=int(bool(o.exact)),
                   accumulate=0 if o.accumulate == "kahan" else 1,
                   shots_per_cta=int(o.shots_per_cta), rows_per_warp=int(o.rows_per_warp),
                   use_graphs=int(bool(o.use_graphs)), wavelet_per_shot=int(bool(wavelet_per_shot)),
                   forward_only=int(bool(o.forward_only)), exa=int(bool(o.exa)),
                   time_block=int(o.time_block),
                   reconstruct=(2 if o.split_backward else 1) if o.reconstruct else 0,
                   persistent=int(bool(o.persistent)), unchained=int(not o.chained))


class ShotPlan:
    """A batch of `nshots` shots over one (nx, nz) model."""

    def __init__(self, nx, nz, h, dt, nt, order=4, nshots=1, wavelet_per_shot=False,
                 options: PlanOptions | None = None, device=None):
        if not torch.cuda.is_available():
            raise _capi.TwiError(_capi.TWI_ERR_CUDA, "torchwi_b200 needs a CUDA device")
        self.options = options or PlanOptions()
        self.nx, self.nz, self.nt, self.order = int(nx), int(nz), int(nt), int(order)
        self.h, self.dt, self.nshots = float(h), float(dt), int(nshots)
        self.wavelet_per_shot = bool(wavelet_per_shot)
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        if self.device.index is None:   # "cuda" means the current device
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._lib = _capi.lib()
        prob = _problem(nx, nz, nt, h, dt, nshots, order, wavelet_per_shot, self.options)
        self._h = ctypes.c_void_p()
        check(self._lib.twi_plan_create(ctypes.byref(prob), ctypes.byref(self._h)))
        self.layout = Layout()
        check(self._lib.twi_plan_layout(self._h, ctypes.byref(self.layout)))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(int(self.layout.workspace_bytes), dtype=torch.uint8,
                                         device=self.device)
            check(self._lib.twi_plan_bind(self._h, ctypes.c_void_p(self.workspace.data_ptr()),
                                          ctypes.c_size_t(self.workspace.numel())))
        lay = self.layout
        S, nt_ = self.nshots, self.nt
        self.vel = self._view(lay.vel, (self.nx, self.nz))
        self.wavelet = self._view(lay.wavelet, (S if self.wavelet_per_shot else 1, nt_))
        self.gathers = self._view(lay.gathers, (S, nt_, self.nx))
        self.resid = self._view(lay.resid, (S, nt_, self.nx))
        self.grad = self._view(lay.grad, (self.nx, self.nz))
        self._have_ckpt = False

    def _view(self, offset, shape):
        n = int(np.prod(shape))
        return self.workspace[offset:offset + 4 * n].view(torch.float32).view(*shape)

    # -- inputs -----------------------------------------------------------------
    def set_shots(self, sx, sy, ry):
        """Shot and receiver positions in metres, one entry per shot."""
        def arr(a):
            a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
            a = np.ascontiguousarray(np.broadcast_to(a.astype(np.float32).reshape(-1),
                                                     (self.nshots,)))
            return a
        self._sx, self._sy, self._ry = arr(sx), arr(sy), arr(ry)
        f = ctypes.POINTER(ctypes.c_float)
        with torch.cuda.device(self.device):
            check(self._lib.twi_plan_set_shots(
                self._h, self._sx.ctypes.data_as(f), self._sy.ctypes.data_as(f),
                self._ry.ctypes.data_as(f), _stream_handle()))
        self._have_ckpt = False

    def set_model(self, vel: torch.Tensor):
        """Velocity (nx, nz), z fastest (the reference's user layout)."""
        if tuple(vel.shape) != (self.nx, self.nz):
            raise ValueError(f"velocity must have shape {(self.nx, self.nz)}, got {tuple(vel.shape)}")
        with torch.cuda.device(self.device):
            self.vel.copy_(vel.detach().to(self.device, torch.float32, non_blocking=True))
            check(self._lib.twi_plan_set_model(self._h, _stream_handle()))
        self._have_ckpt = False

    def set_wavelet(self, w):
        w = w if isinstance(w, torch.Tensor) else torch.as_tensor(np.asarray(w))
        w = w.detach().to(self.device, torch.float32, non_blocking=True)
        self.wavelet.copy_(w.reshape(self.wavelet.shape) if w.numel() == self.wavelet.numel()
                           else w.reshape(1, -1).expand_as(self.wavelet))

    # -- passes -----------------------------------------------------------------
    def forward(self, save_checkpoints=True) -> torch.Tensor:
        """Run all shots; returns the gathers view [nshots, nt, nx]."""
        with torch.cuda.device(self.device):
            check(self._lib.twi_forward(self._h, int(bool(save_checkpoints)), _stream_handle()))
        self._have_ckpt = bool(save_checkpoints)
        return self.gathers

    def forward_residual(self, observed: torch.Tensor, misfit: torch.Tensor | None = None) -> torch.Tensor:
        """Forward pass with checkpoints that leaves the residual
        modelled - observed in the resid region (observed [nshots, nt, nx],
        float32, on this plan's device) and returns the misfit
        0.5*sum(residual^2) as a 0-d float64 device tensor (written into
        `misfit` when given).  Follow with gradient(None)."""
        if observed.device != self.device or observed.dtype != torch.float32 or not observed.is_contiguous():
            raise _capi.TwiInvalid(_capi.TWI_ERR_INVALID,
                                   "observed must be a contiguous float32 tensor on the plan's device")
        if observed.numel() != self.gathers.numel():
            raise _capi.TwiInvalid(_capi.TWI_ERR_INVALID, f"observed must hold {tuple(self.gathers.shape)} samples")
        if misfit is None:
            misfit = torch.empty((), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(self._lib.twi_forward_residual(self._h, ctypes.c_void_p(observed.data_ptr()),
                                                 ctypes.c_void_p(misfit.data_ptr()), _stream_handle()))
        self._have_ckpt = True
        self._keep_obs = observed   # the captured graph reads it
        return misfit

    def residual(self, observed: torch.Tensor, misfit: torch.Tensor | None = None) -> torch.Tensor:
        """After forward(save_checkpoints=True): turn the gathers into the
        residual modelled - observed in place and return the misfit
        0.5*sum(residual^2) (0-d float64 on the device), the same bits as
        forward_residual.  `observed` only has to be on the device when the
        forward pass ends, so its upload can overlap the pass.  Follow with
        gradient(None)."""
        if observed.device != self.device or observed.dtype != torch.float32 or not observed.is_contiguous():
            raise _capi.TwiInvalid(_capi.TWI_ERR_INVALID,
                                   "observed must be a contiguous float32 tensor on the plan's device")
        if observed.numel() != self.gathers.numel():
            raise _capi.TwiInvalid(_capi.TWI_ERR_INVALID, f"observed must hold {tuple(self.gathers.shape)} samples")
        if misfit is None:
            misfit = torch.empty((), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            check(self._lib.twi_residual(self._h, ctypes.c_void_p(observed.data_ptr()),
                                         ctypes.c_void_p(misfit.data_ptr()), _stream_handle()))
        return misfit

    def gradient(self, resid: torch.Tensor | None = None) -> torch.Tensor:
        """Adjoint pass from `resid` [nshots, nt, nx] (already in the resid
        region when None); returns the (nx, nz) gradient view."""
        with torch.cuda.device(self.device):
            if resid is not None:
                self.resid.copy_(resid.detach().to(self.device, torch.float32).reshape(self.resid.shape))
            check(self._lib.twi_gradient(self._h, _stream_handle()))
        return self.grad

    def profile_step(self, mode: int, repeats: int = 20) -> float:
        """Mean device milliseconds per TIME STEP of one kernel mode (0
        forward, 1 recompute, 2 adjoint, 5 the fused backward step of a
        boundary-saving plan) as this plan launches it: a two-step launch's
        time is halved."""
        if self.layout.time_block == 2:
            return self.profile(10 + mode, repeats) / 2
        return self.profile(mode, repeats)

    def profile(self, mode: int, repeats: int = 20) -> float:
        """Mean device milliseconds per launch of one kernel mode (0 forward,
        1 recompute, 2 adjoint, 5 fused backward; 10, 11, 12 the two-step
        launches of a plan with time_block 2) at steady state, all shots."""
        ms = ctypes.c_float()
        with torch.cuda.device(self.device):
            check(self._lib.twi_plan_profile(self._h, int(mode), int(repeats), ctypes.byref(ms),
                                             _stream_handle()))
        return float(ms.value)

    def check(self):
        """Synchronise and raise if a kernel set the device error word."""
        with torch.cuda.device(self.device):
            check(self._lib.twi_plan_check(self._h, _stream_handle()))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                # a caller that knows the plan's work has finished (an event
                # after its last use) spares the device-wide wait
                done = getattr(self, "_done", None)
                if done is not None:
                    done.synchronize()
                else:
                    torch.cuda.synchronize(self.device)
            except Exception:
                pass
            self._lib.twi_plan_destroy(h)
            self._h = None


class PlanBatch:
    """Several ShotPlans (any grid sizes, shot counts and nt; same order,
    arithmetic and rows_per_warp) advanced together: each time step is one
    launch per kernel mode covering every plan.  Results equal running each
    plan on its own, bit for bit.  Set each plan's wavelet, shots and model
    as usual; outputs land in each plan's own regions (gathers, grad)."""

    def __init__(self, plans: list[ShotPlan]):
        if not plans:
            raise ValueError("PlanBatch needs at least one plan")
        self.plans = list(plans)
        self.device = plans[0].device
        self._lib = _capi.lib()
        arr = (ctypes.c_void_p * len(plans))(*[p._h for p in plans])
        self._h = ctypes.c_void_p()
        check(self._lib.twi_batch_create(arr, len(plans), ctypes.byref(self._h)))
        n = ctypes.c_size_t()
        check(self._lib.twi_batch_workspace_size(self._h, ctypes.byref(n)))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(max(int(n.value), 256), dtype=torch.uint8, device=self.device)
            check(self._lib.twi_batch_bind(self._h, ctypes.c_void_p(self.workspace.data_ptr()),
                                           ctypes.c_size_t(self.workspace.numel())))

    def forward(self, save_checkpoints=True):
        with torch.cuda.device(self.device):
            check(self._lib.twi_batch_forward(self._h, int(bool(save_checkpoints)), _stream_handle()))
        for p in self.plans:
            p._have_ckpt = bool(save_checkpoints)
        return [p.gathers for p in self.plans]

    def gradient(self):
        with torch.cuda.device(self.device):
            check(self._lib.twi_batch_gradient(self._h, _stream_handle()))
        return [p.grad for p in self.plans]

    def check(self):
        for p in self.plans:
            p.check()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize(self.device)
            except Exception:
                pass
            self._lib.twi_batch_destroy(h)
            self._h = None
