"""autograd Functions of the time-domain operator (mirror of
torchwi/operator/TimeFunction.py:32-148).

`get_operator(device, prop, exa, forward_only)` returns the `apply` of a
torch.autograd.Function with the reference's calling convention
``op(vel, (sx, sy, ry, m))`` where `m` is the owning Time2d module.  The
work runs on the GPU through the C-ABI plan of `m` (checkpointed adjoint,
no stored virtual-source history); there is no CPU path.
"""

from __future__ import annotations

import torch

from .._capi import TwiError, TWI_ERR_INVALID


def _check_device(device):
    dev = torch.device(device)
    if dev.type != "cuda":
        raise NotImplementedError(
            "torchwi_b200 runs on CUDA devices only; use the reference package for device='cpu'")
    return dev


def get_operator(device, prop="ext", exa=False, forward_only=False):
    """Mirror of TimeFunction.get_operator (TimeFunction.py:32-148)."""
    _check_device(device)
    if prop not in ("ext", "numba"):
        raise NotImplementedError("Check prop=[ext|numba]")

    if forward_only:

        class TimeForwardOperator(torch.autograd.Function):
            @staticmethod
            def forward(ctx, vel, args):
                sx, sy, ry, m = args
                plan = m._prepare(vel, sx, sy, ry)
                return plan.forward(save_checkpoints=False)[0].clone()

            @staticmethod
            def backward(ctx, grad_output):
                return None, None

        return TimeForwardOperator.apply

    class TimeOperator(torch.autograd.Function):
        @staticmethod
        def forward(ctx, vel, args):
            sx, sy, ry, m = args
            plan = m._prepare(vel, sx, sy, ry)
            frd = plan.forward(save_checkpoints=True)[0].clone()
            ctx.m = m
            ctx.save_for_backward(vel.detach())
            ctx.coords = (sx, sy, ry)
            ctx.token = m._token
            return frd

        @staticmethod
        def backward(ctx, grad_output):
            (vel,) = ctx.saved_tensors
            m = ctx.m
            if m._token != ctx.token:
                # another forward reused the plan since: rebuild the checkpoints
                plan = m._prepare(vel, *ctx.coords)
                plan.forward(save_checkpoints=True)
            grad = m._plan.gradient(grad_output.reshape(1, m.nt, m.nx))
            return grad.clone(), None

    return TimeOperator.apply


__all__ = ["get_operator", "TwiError", "TWI_ERR_INVALID"]
