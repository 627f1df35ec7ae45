"""Full-waveform inversion driver over the batched operator.

Mirror of the reference's inversion example and parameter classes
(examples/time/inv_torch.py:15-151, torchwi/parameter/Param.py:3-64), with the
per-shot loop replaced by one batched plan per rank:

* the model is a `VelocityParameter`, `SlothParameter` or `SlownessParameter`
  (same interface as the reference's: `forward()` clips the parameter to
  [vmin, vmax] in place and returns the velocity);
* every epoch runs ONE forward pass over all of this rank's shots that writes
  the residual modelled - observed straight into the plan's residual region
  and reduces the misfit 0.5*sum(r^2) on the device (`twi_forward_residual`),
  then one checkpointed adjoint pass for the shot-summed gradient;
* ranks own contiguous blocks of shots and combine gradient and misfit with
  one all-reduce per epoch (`dist.ShardedGradient`); the reference does the
  same with Horovod (inv_torch.py:52-55, 139-141);
* the gradient is normalised by the infinity norm of the first epoch's
  gradient (`grad_norm='first'`, inv_torch.py:57-64) and the optimizer is
  Adam, Nesterov, momentum or plain gradient descent as in inv_torch.py:45-55.

Observed gathers stay resident on the device for the whole inversion, so an
epoch moves nothing between host and device except the misfit (8 bytes).
"""

from __future__ import annotations

from typing import Callable

import torch

from .dist import ShardedGradient, shard_shots
from .plan import PlanOptions, ShotPlan, shot_blocks


# ----------------------------------------------------------------------------
# model parameterisations (torchwi/parameter/Param.py:3-64)
# ----------------------------------------------------------------------------

class BaseParameter(torch.nn.Module):
    """A trainable model parameter `par` that maps to velocity.

    `vmin` / `vmax` (velocity bounds) are used only when both are given and
    non-zero, as in the reference; the parameter bounds are the images of the
    velocity bounds, ordered."""

    def __init__(self, vel, vmin=None, vmax=None):
        super().__init__()
        self.vmin, self.vmax = vmin, vmax
        self.par = torch.nn.Parameter(self.vel_to_par(vel))
        if vmin and vmax:
            a, b = self.vel_to_par(vmin), self.vel_to_par(vmax)
            self.pmin, self.pmax = min(a, b), max(a, b)

    def vel_to_par(self, vel):
        return vel

    def par_to_vel(self, par):
        return par

    def gradient(self):
        return self.par.grad

    def gradient_times(self, multiplier):
        self.par.grad *= multiplier

    def grad_norm(self):
        return self.par.grad.norm(float("inf"))

    def normalize_gradient(self, gnorm0):
        self.par.grad /= gnorm0

    def vel(self):
        return self.par_to_vel(self.par)

    def pclip(self):
        if self.vmin and self.vmax:
            with torch.no_grad():
                self.par[:] = torch.clamp(self.par, self.pmin, self.pmax)

    def forward(self):
        self.pclip()
        return self.vel()

    def report(self):
        return f"Parameter: {type(self).__name__}"


class VelocityParameter(BaseParameter):
    """par = v."""


class SlothParameter(BaseParameter):
    """par = 1/v^2."""

    def vel_to_par(self, vel):
        return 1.0 / vel ** 2

    def par_to_vel(self, par):
        return torch.sqrt(1.0 / par)


class SlownessParameter(BaseParameter):
    """par = 1/v."""

    def vel_to_par(self, vel):
        return 1.0 / vel

    def par_to_vel(self, par):
        return 1.0 / par


PARAMETERS = {"velocity": VelocityParameter, "sloth": SlothParameter, "slowness": SlownessParameter}


def make_optimizer(params, name: str = "adam", lr: float = 0.02, momentum: float = 0.9):
    """The optimizer choices of inv_torch.py:45-55 (adam | nag | momentum | gd)."""
    if name == "adam":
        return torch.optim.Adam(params, lr=lr)
    if name == "nag":
        return torch.optim.SGD(params, lr=lr, momentum=momentum, nesterov=True)
    if name == "momentum":
        return torch.optim.SGD(params, lr=lr, momentum=momentum)
    if name == "gd":
        return torch.optim.SGD(params, lr=lr)
    raise ValueError(f"unknown optimizer {name!r} (adam | nag | momentum | gd)")


# ----------------------------------------------------------------------------
# per-rank misfit + gradient over the batched plan
# ----------------------------------------------------------------------------

def plan_residual_local_fn(nx, nz, h, dt, w, order, sx, sy, ry, observed: torch.Tensor,
                           options: PlanOptions | None = None, device=None,
                           hbm_budget: int | None = None, observed_first: int = 0) -> Callable:
    """`local_fn(vel, shots) -> (misfit, gradient)` for `ShardedGradient`:
    the shots of the block run through batched plans (as many shots per plan
    as fit `hbm_budget`, default 80 % of free device memory), the residual
    and misfit formed on the device by the forward pass.  `observed` holds the
    gathers [n, nt, nx] of shots observed_first .. observed_first+n-1 on
    `device` (all shots, or just this rank's block)."""
    opts = options or PlanOptions()
    dev = torch.device(device) if device is not None else observed.device
    nt = int(w.numel()) if isinstance(w, torch.Tensor) else len(w)
    plans: dict[tuple[int, int], list[tuple[slice, ShotPlan]]] = {}

    def chunks(shots: slice) -> list[tuple[slice, ShotPlan]]:
        key = (shots.start, shots.stop)
        if key in plans:
            return plans[key]
        out = []
        for sl in shot_blocks(shots, nx, nz, nt, order, opts, hbm_budget, dev):
            p = ShotPlan(nx, nz, h, dt, nt, order, nshots=sl.stop - sl.start, options=opts, device=dev)
            p.set_wavelet(torch.as_tensor(w))
            p.set_shots(sx[sl], sy[sl], ry[sl])
            out.append((sl, p))
        plans[key] = out
        return out

    def fn(vel, shots: slice):
        grad = None
        misfit = torch.zeros((), dtype=torch.float64, device=dev)
        for sl, p in chunks(shots):
            p.set_model(vel)
            misfit += p.forward_residual(observed[sl.start - observed_first:sl.stop - observed_first])
            g = p.gradient(None)
            grad = g.clone() if grad is None else grad.add_(g)
        return misfit, grad

    return fn


class Inversion:
    """Gradient-based FWI of one velocity model from the shots of a survey.

    `local_fn(vel, shots) -> (misfit, gradient)` computes one rank's share; it
    defaults to `plan_residual_local_fn` on the device of `vel_init` (pass
    `observed` then).  With torch.distributed initialised, shots are split
    across ranks and every epoch does one all-reduce of [gradient, misfit]."""

    def __init__(self, vel_init: torch.Tensor, nshots: int, *, local_fn: Callable | None = None,
                 h=None, dt=None, w=None, order=4, sx=None, sy=None, ry=None, observed=None,
                 vmin=None, vmax=None, parameter: str = "velocity", optimizer: str = "adam",
                 lr: float = 0.02, momentum: float = 0.9, grad_norm: str = "first",
                 options: PlanOptions | None = None, group=None, hbm_budget: int | None = None,
                 observed_first: int = 0):
        if grad_norm not in ("first", "none"):
            raise ValueError("grad_norm must be 'first' or 'none'")
        nx, nz = vel_init.shape
        if local_fn is None:
            if observed is None or w is None or h is None or dt is None:
                raise ValueError("the plan-backed driver needs h, dt, w, sx, sy, ry and observed")
            local_fn = plan_residual_local_fn(nx, nz, h, dt, w, order, sx, sy, ry, observed,
                                              options=options, device=vel_init.device,
                                              hbm_budget=hbm_budget, observed_first=observed_first)
        self.model = PARAMETERS[parameter](vel_init.detach().clone(), vmin, vmax)
        self.optimizer = make_optimizer(self.model.parameters(), optimizer, lr, momentum)
        self.gradient_fn = ShardedGradient(local_fn, nshots, group=group)
        self.grad_norm = grad_norm
        self.gnorm0 = None
        self.history: list[float] = []

    def velocity(self) -> torch.Tensor:
        with torch.no_grad():
            return self.model.vel().detach().clone()

    def epoch(self) -> float:
        """One iteration: misfit and gradient over all shots, normalisation,
        optimizer step.  Returns the misfit of the model before the step."""
        self.optimizer.zero_grad()
        vel = self.model()
        misfit, grad = self.gradient_fn(vel.detach())
        vel.backward(grad.to(vel.dtype))     # chain rule to the parameter
        if self.grad_norm == "first":
            if self.gnorm0 is None:
                self.gnorm0 = self.model.gradient().norm(float("inf"))
            self.model.normalize_gradient(self.gnorm0)
        self.optimizer.step()
        loss = float(misfit)
        self.history.append(loss)
        return loss

    def run(self, epochs: int, callback: Callable | None = None) -> list[float]:
        for e in range(epochs):
            loss = self.epoch()
            if callback is not None:
                callback(e, loss, self)
        return self.history


__all__ = ["BaseParameter", "VelocityParameter", "SlothParameter", "SlownessParameter",
           "PARAMETERS", "make_optimizer", "plan_residual_local_fn", "Inversion", "shard_shots"]
