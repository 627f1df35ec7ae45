"""Time-domain 2D acoustic operator modules (mirror of
torchwi/operator/TimeOperator.py:18-82).

Same constructor and call signatures as the reference:

    model = Time2d(nx, ny, h, w, dt, order, device, prop='ext', exa=False)
    frd = model(vel, sx, sy, ry)          # vel (nx, ny) z fastest -> (nt, nx)
    loss(frd).backward()                   # vel.grad (nx, ny)

Differences, all deliberate:
  * the grid is never padded to multiples of 16 (the reference's CUDA path
    does, TimeOperator.py:36-38, which moves the absorbing boundary); the
    result equals the reference's CPU propagator bit for bit in `exact` mode;
  * the virtual-source history (nt*dimxy floats, TimeOperator.py:82) is not
    stored: the adjoint recomputes the forward field from checkpoints;
  * the returned gathers are a fresh tensor, not a view of a module buffer,
    and backward after another forward recomputes what it needs;
  * device must be CUDA: there is no CPU fallback.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import torch

from ..plan import PlanOptions, ShotPlan
from . import TimeFunction


def _scalar(x) -> float:
    return float(x.item() if isinstance(x, torch.Tensor) else x)


class Time2dForward(torch.nn.Module):
    """Forward modelling only (no gradient)."""

    forward_only = True

    def __init__(self, nx, ny, h, w, dt, order, device, options: PlanOptions | None = None):
        super().__init__()
        self.device = TimeFunction._check_device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.h = float(h)
        self.w = torch.as_tensor(w).detach().to("cpu", torch.float32)
        self.nt = int(self.w.numel())
        self.dt = float(dt)
        self.order = int(order)
        self.ne = self.order // 2
        self.nx_org, self.ny_org = int(nx), int(ny)
        self.nx, self.ny = self.nx_org, self.ny_org
        self.dimx, self.dimy = self.nx + self.order, self.ny + self.order
        self.dimxy = self.dimx * self.dimy
        self.options = options or PlanOptions()
        self._plan: ShotPlan | None = None
        self._token = 0
        self._exa = None
        self.time_modeling = TimeFunction.get_operator(self.device, forward_only=True)

    def _plan_or_new(self) -> ShotPlan:
        if self._plan is None:
            opts = self.options
            if self.forward_only:
                opts = dataclasses.replace(opts, forward_only=True)
            self._plan = ShotPlan(self.nx, self.ny, self.h, self.dt, self.nt, self.order, nshots=1,
                                  options=opts, device=self.device)
            self._plan.set_wavelet(self.w)
        return self._plan

    def _prepare(self, vel, sx, sy, ry) -> ShotPlan:
        plan = self._plan_or_new()
        plan.set_model(vel)
        plan.set_shots(np.float32(_scalar(sx)), np.float32(_scalar(sy)), np.float32(_scalar(ry)))
        self._token += 1
        return plan

    def forward(self, vel, sx, sy, ry):
        return self.time_modeling(vel, (sx, sy, ry, self))


class Time2d(Time2dForward):
    """Forward modelling with the adjoint velocity gradient."""

    forward_only = False

    def __init__(self, nx, ny, h, w, dt, order, device, prop="ext", exa=False,
                 options: PlanOptions | None = None):
        if exa:   # excitation-amplitude gradient (TimeFunction.py:62-104)
            options = dataclasses.replace(options or PlanOptions(), exa=True)
        super().__init__(nx, ny, h, w, dt, order, device, options)
        self.exa = bool(exa)
        self.time_modeling = TimeFunction.get_operator(self.device, prop, exa)


class Time2dBatch(torch.nn.Module):
    """All shots of a survey in one plan: forward (nshots, nt, nx) gathers,
    backward accumulates the shot-summed gradient into vel.grad.

        model = Time2dBatch(nx, nz, h, w, dt, order, nshots, device)
        frd = model(vel, sx, sy, ry)       # sx, sy, ry: (nshots,) metres
        loss = 0.5 * ((frd - obs) ** 2).sum(); loss.backward()

    `w` is (nt,) shared by all shots or (nshots, nt)."""

    def __init__(self, nx, nz, h, w, dt, order, nshots, device="cuda",
                 options: PlanOptions | None = None):
        super().__init__()
        w = torch.as_tensor(w).detach().to(torch.float32)
        dev = TimeFunction._check_device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.nt = int(w.shape[-1])
        self.nx, self.nz, self.nshots = int(nx), int(nz), int(nshots)
        self.plan = ShotPlan(nx, nz, h, dt, self.nt, order, nshots=nshots,
                             wavelet_per_shot=(w.dim() == 2), options=options, device=dev)
        self.plan.set_wavelet(w)
        self._token = 0

    def forward(self, vel, sx, sy, ry):
        return _BatchOperator.apply(vel, (sx, sy, ry, self))


class _BatchOperator(torch.autograd.Function):
    @staticmethod
    def forward(ctx, vel, args):
        sx, sy, ry, m = args
        m.plan.set_model(vel)
        m.plan.set_shots(sx, sy, ry)
        m._token += 1
        frd = m.plan.forward(save_checkpoints=True).clone()
        ctx.m, ctx.coords, ctx.token = m, (sx, sy, ry), m._token
        ctx.save_for_backward(vel.detach())
        return frd

    @staticmethod
    def backward(ctx, grad_output):
        (vel,) = ctx.saved_tensors
        m = ctx.m
        if m._token != ctx.token:
            m.plan.set_model(vel)
            m.plan.set_shots(*ctx.coords)
            m.plan.forward(save_checkpoints=True)
        return m.plan.gradient(grad_output).clone(), None


class Time2dModels(torch.nn.Module):
    """Several velocity models of different grid sizes, each with its own
    shots (and its own nt), advanced together: every time step of all of
    them is one launch per kernel mode (a PlanBatch).  Backward gives each
    model its shot-summed gradient.

        m = Time2dModels([(nx0, nz0), (nx1, nz1)], h, [w0, w1], dt, order, [S0, S1], device)
        frd0, frd1 = m([vel0, vel1], [(sx0, sy0, ry0), (sx1, sy1, ry1)])
        (loss(frd0) + loss(frd1)).backward()       # vel0.grad, vel1.grad

    `w` is one wavelet for all models or a list (each (nt,) or (S_i, nt));
    `h`, `dt` and `order` are shared.  Results equal running each model
    alone (Time2dBatch), bit for bit."""

    def __init__(self, shapes, h, w, dt, order, nshots, device="cuda",
                 options: PlanOptions | None = None):
        super().__init__()
        from ..plan import PlanBatch
        dev = TimeFunction._check_device(device)
        if dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        shapes = [(int(a), int(b)) for a, b in shapes]
        nshots = [int(n) for n in nshots]
        if len(nshots) != len(shapes):
            raise ValueError("one shot count per model")
        ws = list(w) if isinstance(w, (list, tuple)) else [w] * len(shapes)
        if len(ws) != len(shapes):
            raise ValueError("one wavelet per model (or one for all)")
        self.plans = []
        for (nx, nz), ns, wi in zip(shapes, nshots, ws):
            wi = torch.as_tensor(wi).detach().to(torch.float32)
            p = ShotPlan(nx, nz, h, dt, int(wi.shape[-1]), order, nshots=ns,
                         wavelet_per_shot=(wi.dim() == 2), options=options, device=dev)
            p.set_wavelet(wi)
            self.plans.append(p)
        self.batch = PlanBatch(self.plans)
        self._token = 0

    def forward(self, vels, coords):
        if len(vels) != len(self.plans) or len(coords) != len(self.plans):
            raise ValueError("one velocity model and one (sx, sy, ry) per model")
        return _ModelsOperator.apply(self, tuple(tuple(c) for c in coords), *vels)


class _ModelsOperator(torch.autograd.Function):
    @staticmethod
    def forward(ctx, m, coords, *vels):
        m._token += 1
        for p, v, c in zip(m.plans, vels, coords):
            p.set_model(v)
            p.set_shots(*c)
        frds = m.batch.forward(save_checkpoints=True)
        ctx.m, ctx.coords, ctx.token = m, coords, m._token
        ctx.save_for_backward(*[v.detach() for v in vels])
        return tuple(f.clone() for f in frds)

    @staticmethod
    def backward(ctx, *grad_outputs):
        vels = ctx.saved_tensors
        m = ctx.m
        if m._token != ctx.token:   # another forward reused the plans since
            for p, v, c in zip(m.plans, vels, ctx.coords):
                p.set_model(v)
                p.set_shots(*c)
            m.batch.forward(save_checkpoints=True)
        for p, g in zip(m.plans, grad_outputs):
            if g is None:
                p.resid.zero_()
            else:
                p.resid.copy_(g.detach().to(p.device, torch.float32).reshape(p.resid.shape))
        grads = m.batch.gradient()
        return (None, None) + tuple(g.clone() for g in grads)
