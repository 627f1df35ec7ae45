"""Shot-parallel gradients over several GPUs (one process per GPU).

Replaces the reference's Horovod data parallelism (one shot per rank,
gradient all-reduce with op=Sum, examples/time/inv_torch.py:52-55,61,139):
the shots of a survey are split into contiguous blocks, each rank runs its
block through its own batched plan, and the shot-summed gradient and the
misfit are combined with ONE all-reduce (sum) per gradient.  Shots are
independent, so there is no other exchange.
"""

from __future__ import annotations

from typing import Callable

import torch
import torch.distributed as dist


def shard_shots(nshots: int, world: int | None = None, rank: int | None = None) -> slice:
    """Contiguous block of shots owned by `rank` (sizes differ by at most 1)."""
    if world is None:
        world = dist.get_world_size() if dist.is_initialized() else 1
    if rank is None:
        rank = dist.get_rank() if dist.is_initialized() else 0
    base, extra = divmod(nshots, world)
    start = rank * base + min(rank, extra)
    return slice(start, start + base + (1 if rank < extra else 0))


class ShardedGradient:
    """Callable ``(vel) -> (misfit, gradient)`` summed over all shots of all
    ranks.  ``local_fn(vel, shots: slice) -> (misfit, gradient)`` computes the
    contribution of this rank's shots (misfit a 0-d tensor, gradient (nx, nz)
    on the rank's device); ranks without shots contribute zeros but still take
    part in the collective, so every rank issues the same collectives in the
    same order."""

    def __init__(self, local_fn: Callable, nshots: int, group=None):
        self.local_fn = local_fn
        self.nshots = nshots
        self.group = group

    def __call__(self, vel: torch.Tensor):
        world = dist.get_world_size(self.group) if dist.is_initialized() else 1
        rank = dist.get_rank(self.group) if dist.is_initialized() else 0
        mine = shard_shots(self.nshots, world, rank)
        if mine.stop > mine.start:
            misfit, grad = self.local_fn(vel, mine)
            misfit = misfit.reshape(()).to(grad.dtype)
        else:
            grad = torch.zeros_like(vel, dtype=torch.float32)
            misfit = torch.zeros((), dtype=torch.float32, device=grad.device)
        if world > 1:
            packed = torch.cat([grad.reshape(-1), misfit.reshape(1)])
            dist.all_reduce(packed, op=dist.ReduceOp.SUM, group=self.group)
            grad = packed[:-1].reshape(grad.shape)
            misfit = packed[-1]
        return misfit, grad


def plan_local_fn(make_plan: Callable[[slice], object], observed: torch.Tensor):
    """local_fn for ShardedGradient backed by a batched ShotPlan per shard.
    ``make_plan(shots)`` returns a ShotPlan whose shots are set; ``observed``
    holds the gathers of all shots [nshots, nt, nx] on the rank's device."""
    cache = {}

    def fn(vel, shots: slice):
        key = (shots.start, shots.stop)
        if key not in cache:
            cache[key] = make_plan(shots)
        plan = cache[key]
        plan.set_model(vel)
        misfit = plan.forward_residual(observed[shots])   # residual + misfit on the device
        return misfit, plan.gradient(None).clone()

    return fn
