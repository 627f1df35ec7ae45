"""Batches of plans with different grids, shot counts and nt: one launch per
kernel mode and time step for all of them, results bit-identical to running
each plan alone (same kernels, same per-plan shot grouping)."""
import numpy as np
import pytest
import torch

from golden_io import bits_equal
from torchwi_b200 import PlanBatch, PlanOptions, ShotPlan, synthetic

pytestmark = pytest.mark.gpu

CASES = [dict(nx=70, nz=33, nt=120, nshots=3, seed=1),
         dict(nx=150, nz=45, nt=90, nshots=5, seed=2),
         dict(nx=41, nz=24, nt=150, nshots=2, seed=3)]


def _plan(s, opts):
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=s.nshots, options=opts)
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel_start))
    return p


@pytest.mark.parametrize("accumulate,graphs,rz,recon,chained",
                         [("plain", True, 0, False, True), ("plain", False, 0, False, True),
                          ("kahan", True, 0, False, True), ("kahan", False, 0, False, True),
                          ("kahan", True, 2, False, True), ("plain", True, 0, True, True),
                          ("kahan", True, 0, True, True), ("kahan", False, 4, True, True),
                          ("kahan", True, 0, True, False), ("plain", True, 0, False, False)])
def test_batch_equals_plans_alone(accumulate, graphs, rz, recon, chained):
    """recon: boundary-saving plans, whose backward steps are fused launches
    (one multi-plan launch of the fused backward kernel per step).  chained:
    runs of like launches start while the previous one drains (the default);
    the plans alone run in stream order either way."""
    surveys = [synthetic.small_case(order=4, **c) for c in CASES]
    opts = PlanOptions(accumulate=accumulate, ckpt_interval=11, use_graphs=graphs, rows_per_warp=rz,
                       reconstruct=recon, chained=False)
    bopts = PlanOptions(accumulate=accumulate, ckpt_interval=11, use_graphs=graphs, rows_per_warp=rz,
                        reconstruct=recon, chained=chained)
    alone = []
    for s in surveys:
        p = _plan(s, opts)
        frd = p.forward(save_checkpoints=True).clone()
        g = p.gradient(0.25 * frd).clone()
        alone.append((frd.cpu().numpy(), g.cpu().numpy()))
    plans = [_plan(s, bopts) for s in surveys]
    batch = PlanBatch(plans)
    for rep in range(2):   # a second call replays the captured graphs
        gathers = [g.clone() for g in batch.forward(save_checkpoints=True)]
        for p, g in zip(plans, gathers):
            p.resid.copy_(0.25 * g)
        grads = [g.clone() for g in batch.gradient()]
        batch.check()
        for k in range(len(surveys)):
            assert bits_equal(gathers[k].cpu().numpy(), alone[k][0]), (rep, k)
            assert bits_equal(grads[k].cpu().numpy(), alone[k][1]), (rep, k)


@pytest.mark.parametrize("recon", [False, True])
def test_batch_order8_equals_plans_alone(recon):
    """Order 8 through the multi-plan kernels, which read their step arguments
    from shared memory (the widest register window of the three orders)."""
    cases = [dict(nx=70, nz=33, nt=90, nshots=3, seed=4), dict(nx=101, nz=45, nt=70, nshots=5, seed=5)]
    surveys = [synthetic.small_case(order=8, **c) for c in cases]

    def plan8(s, opts):
        p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 8, nshots=s.nshots, options=opts)
        p.set_wavelet(torch.from_numpy(s.w))
        p.set_shots(s.sx, s.sy, s.ry)
        p.set_model(torch.from_numpy(s.vel_start))
        return p

    opts = PlanOptions(ckpt_interval=11, reconstruct=recon, chained=False)
    alone = []
    for s in surveys:
        p = plan8(s, opts)
        frd = p.forward(save_checkpoints=True).clone()
        alone.append((frd.cpu().numpy(), p.gradient(0.25 * frd).clone().cpu().numpy()))
    plans = [plan8(s, PlanOptions(ckpt_interval=11, reconstruct=recon)) for s in surveys]
    batch = PlanBatch(plans)
    gathers = [g.clone() for g in batch.forward(save_checkpoints=True)]
    for p, g in zip(plans, gathers):
        p.resid.copy_(0.25 * g)
    grads = [g.clone() for g in batch.gradient()]
    batch.check()
    for k in range(len(surveys)):
        assert np.isfinite(grads[k].cpu().numpy()).all()
        assert bits_equal(gathers[k].cpu().numpy(), alone[k][0]), k
        assert bits_equal(grads[k].cpu().numpy(), alone[k][1]), k
