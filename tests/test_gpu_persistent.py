"""Persistent launches (PlanOptions(persistent=True)): each pass of a plan --
the forward pass, each checkpoint segment's recompute and adjoint phases,
the fused backward pass -- runs as one launch whose CTAs take (step, shot
group, tile) work items in step order and wait, with bounded waits, for the
group's previous step.  Same kernels per item, so every result must be
bit-identical to one launch per time step."""
import numpy as np
import pytest
import torch

from golden_io import bits_equal
from torchwi_b200 import PlanOptions, ShotPlan, synthetic

pytestmark = pytest.mark.gpu


def _run(s, **kw):
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, s.order, nshots=s.nshots, options=PlanOptions(**kw))
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel).cuda())
    obs = p.forward(save_checkpoints=False).clone() if not kw.get("forward_only") else None
    if kw.get("forward_only"):
        out = [p.forward(save_checkpoints=False).clone()]
        p.check()
        return out
    p.set_model(torch.from_numpy(s.vel_start).cuda())
    frd = p.forward(save_checkpoints=True).clone()
    m = p.forward_residual(obs)
    resid = p.resid.clone()
    g = p.gradient(None).clone()
    # a second gradient through the same (now captured) graphs
    p.forward_residual(obs)
    g2 = p.gradient(None).clone()
    p.check()
    return [obs, frd, resid, m.reshape(1), g, g2]


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("mode", [dict(), dict(accumulate="plain", ckpt_interval=7),
                                  dict(reconstruct=True), dict(reconstruct=True, split_backward=True),
                                  dict(exa=True), dict(forward_only=True)])
def test_persistent_equals_one_launch_per_step(order, mode):
    s = synthetic.small_case(nx=97, nz=41, nt=150, order=order, nshots=11, seed=order + 3)
    a = _run(s, **mode)
    b = _run(s, persistent=True, **mode)
    for x, y in zip(a, b):
        assert bits_equal(x.cpu().numpy(), y.cpu().numpy())
    assert all(np.isfinite(x.cpu().numpy()).all() for x in b)


@pytest.mark.parametrize("graphs", [True, False])
def test_persistent_config2_shape(graphs):
    # the benchmark's launch shapes (64 shots, 1000 x 300) on a short run
    s = synthetic.config2(nshots=64, nt=60)
    a = _run(s, reconstruct=True, use_graphs=graphs)
    b = _run(s, reconstruct=True, persistent=True, use_graphs=graphs)
    for x, y in zip(a, b):
        assert bits_equal(x.cpu().numpy(), y.cpu().numpy())
