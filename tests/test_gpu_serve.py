"""Serving loop on the GPU: requests of different grids, shot counts, nt and
kinds share the device tick by tick; each result equals the same request run
alone (bit for bit: same kernels, same per-request shot grouping), including
when the HBM budget forces shot chunking or sequential admission."""
import numpy as np
import pytest
import torch

from golden_io import bits_equal, rel_l2
from torchwi_b200 import PlanOptions, ShotPlan, synthetic
from torchwi_b200.serve import Request, Server, plain_service_times

pytestmark = pytest.mark.gpu

OPTS = PlanOptions(accumulate="plain", ckpt_interval=13)


def _pool():
    a = synthetic.small_case(nx=90, nz=40, nt=10, seed=1)
    b = synthetic.small_case(nx=150, nz=55, nt=10, seed=2)
    return {"a": torch.from_numpy(a.vel_start).cuda(), "b": torch.from_numpy(b.vel_start).cuda()}


def _requests(models, with_obs):
    rng = np.random.default_rng(3)
    out = []
    specs = [("gradient", "a", 5, 140), ("forward", "b", 3, 90), ("gradient", "b", 7, 60),
             ("forward", "a", 2, 200), ("gradient", "a", 1, 110)]
    for kind, m, ns, nt in specs:
        nx, nz = models[m].shape
        ix = ((np.arange(ns) + 0.5) * nx / ns).astype(np.int64)
        sx = ix * 10.0
        sy = np.full(ns, 20.0)
        w = synthetic.ricker(15.0, 1e-3, nt).astype(np.float32)
        obs = None
        if kind == "gradient" and with_obs:
            obs = torch.from_numpy(rng.standard_normal((ns, nt, nx)).astype(np.float32)).cuda() * 1e-3
        out.append(Request(kind=kind, model=m, sx=sx, sy=sy, ry=sy.copy(), w=w, observed=obs))
    return out


def _alone(models, r, opts=OPTS):
    nx, nz = models[r.model].shape
    o = PlanOptions(**{**opts.__dict__, "forward_only": r.kind == "forward"})
    p = ShotPlan(nx, nz, 10.0, 1e-3, r.nt, 4, nshots=r.nshots, options=o)
    p.set_wavelet(torch.from_numpy(r.w))
    p.set_shots(r.sx, r.sy, r.ry)
    p.set_model(models[r.model])
    g = p.forward(save_checkpoints=r.kind == "gradient")
    if r.kind == "forward":
        return g.clone()
    if r.observed is not None:
        g.sub_(r.observed)
    return p.gradient(None).clone()


def _serve(models, reqs, budget=None, ticks=17):
    srv = Server(models, h=10.0, dt=1e-3, options=OPTS, hbm_budget=budget, max_requests=8)
    for r in reqs:
        srv.submit(r)
    while srv.busy():
        srv.poll(ticks)
    return srv


@pytest.mark.parametrize("with_obs", [False, True])
def test_mix_equals_alone(with_obs):
    models = _pool()
    reqs = _requests(models, with_obs)
    _serve(models, reqs)
    for r in reqs:
        assert r.result is not None and r.done_at is not None
        assert bits_equal(r.result.cpu().numpy(), _alone(models, r).cpu().numpy()), (r.kind, r.model)


@pytest.mark.parametrize("with_obs", [False, True])
def test_request_joining_mid_flight_equals_alone(with_obs):
    """Requests submitted while others are already on the device join the
    next ticks (continuous batching) and still give the bits they give
    alone."""
    models = _pool()
    reqs = _requests(models, with_obs)
    srv = Server(models, h=10.0, dt=1e-3, options=OPTS, max_requests=8)
    first, late = reqs[:2], reqs[2:]
    for r in first:
        srv.submit(r)
    assert srv.poll(5) == []            # both admitted, 5 of their >= 90 steps done
    assert srv.engine.pending()[0] == 2
    for r in late:
        srv.submit(r)
        srv.poll(3)                      # admitted beside the ones in flight
        in_flight, _ = srv.engine.pending()
        assert in_flight >= 2, "a late request ran alone"
    while srv.busy():
        srv.poll(17)
    for r in reqs:
        assert r.result is not None
        assert bits_equal(r.result.cpu().numpy(), _alone(models, r).cpu().numpy()), (r.kind, r.model)


def test_boundary_saving_requests_mix_equals_alone():
    """Gradient requests of boundary-saving plans (fused backward steps: one
    engine launch of the fused kernel per tick for all of them) next to
    forward requests, some joining mid-flight, give the bits they give
    alone."""
    opts = PlanOptions(accumulate="plain", reconstruct=True)
    models = _pool()
    reqs = _requests(models, True)
    srv = Server(models, h=10.0, dt=1e-3, options=opts, max_requests=8)
    for r in reqs[:3]:
        srv.submit(r)
    srv.poll(7)
    for r in reqs[3:]:
        srv.submit(r)
    while srv.busy():
        srv.poll(13)
    for r in reqs:
        assert bits_equal(r.result.cpu().numpy(), _alone(models, r, opts).cpu().numpy()), (r.kind, r.model)


def test_memory_limited_admission_and_chunking():
    models = _pool()
    reqs = _requests(models, True)
    from torchwi_b200 import footprint_bytes
    # room for one shot of the largest request at a time: requests run in
    # chunks, one chunk in flight
    big = max(footprint_bytes(*models[r.model].shape, r.nt, 1, 4,
                              options=PlanOptions(**{**OPTS.__dict__, "forward_only": r.kind == "forward"}))
              for r in reqs)
    _serve(models, reqs, budget=int(big * 1.5))
    for r in reqs:
        ref = _alone(models, r).cpu().numpy()
        if r.kind == "forward":
            assert bits_equal(r.result.cpu().numpy(), ref)
        else:   # chunk sums are added in a different association
            assert rel_l2(r.result.cpu().numpy(), ref) <= 1e-6


def test_plain_service_times_runs():
    models = _pool()
    reqs = _requests(models, False)[:2]
    t = plain_service_times(models, reqs, 10.0, 1e-3, options=OPTS)
    assert len(t) == 2 and all(x > 0 for x in t)
