"""Chained launches (PlanOptions(chained=True), the default): within a run of
one-step launches of one kind, each launch may start its CTAs while the one
before it drains, and a CTA waits, bounded, only until its shot group of
the earlier steps is done.  The kernels and their arithmetic are unchanged,
so every result must equal plain stream order (chained=False) bit for bit."""
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
    if kw.get("forward_only"):
        out = [p.forward(save_checkpoints=False).clone()]
        p.check()
        return out
    obs = p.forward(save_checkpoints=False).clone()
    p.set_model(torch.from_numpy(s.vel_start).cuda())
    frd = p.forward(save_checkpoints=True).clone()
    m = p.forward_residual(obs)
    resid = p.resid.clone()
    g = p.gradient(None).clone()
    # the same passes again through the captured graphs
    p.forward_residual(obs)
    g2 = p.gradient(None).clone()
    p.check()
    return [obs, frd, resid, m.reshape(1), g, g2]


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("mode", [dict(), dict(accumulate="plain", ckpt_interval=7),
                                  dict(reconstruct=True), dict(reconstruct=True, split_backward=True),
                                  dict(exa=True), dict(forward_only=True), dict(time_block=2),
                                  dict(shots_per_cta=1, rows_per_warp=2)])
def test_chained_equals_stream_order(order, mode):
    s = synthetic.small_case(nx=97, nz=41, nt=150, order=order, nshots=11, seed=order + 5)
    a = _run(s, chained=False, **mode)
    b = _run(s, chained=True, **mode)
    for x, y in zip(a, b):
        assert bits_equal(x.cpu().numpy(), y.cpu().numpy())
    assert all(np.isfinite(x.cpu().numpy()).all() for x in b)


@pytest.mark.parametrize("graphs", [True, False])
@pytest.mark.parametrize("recon", [True, False])
def test_chained_config2_shape(graphs, recon):
    # the benchmark's launch shapes (64 shots, 1000 x 300) on a short run
    s = synthetic.config2(nshots=64, nt=60)
    a = _run(s, reconstruct=recon, use_graphs=graphs, chained=False)
    b = _run(s, reconstruct=recon, use_graphs=graphs, chained=True)
    for x, y in zip(a, b):
        assert bits_equal(x.cpu().numpy(), y.cpu().numpy())

