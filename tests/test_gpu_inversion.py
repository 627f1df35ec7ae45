"""Device-side residual + misfit (twi_forward_residual) and the inversion
driver over the batched plan, against the explicit per-shot form that the
reference's inversion example runs (examples/time/inv_torch.py:123-151)."""
import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal
from torchwi_b200 import PlanOptions, ShotPlan, Time2d, synthetic
from torchwi_b200.inversion import Inversion, VelocityParameter, make_optimizer

pytestmark = pytest.mark.gpu


def _survey(nshots=6, seed=21):
    s = synthetic.small_case(nx=70, nz=33, nt=140, order=4, nshots=nshots, seed=seed)
    obs = np.stack([O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k])
                    for k in range(nshots)])
    return s, obs


def _plan(s, **kw):
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=s.nshots, options=PlanOptions(**kw))
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel_start).cuda())
    return p


@pytest.mark.parametrize("graphs", [True, False])
def test_forward_residual_equals_explicit_residual(graphs):
    s, obs = _survey()
    obs_d = torch.from_numpy(obs).cuda()
    p = _plan(s, accumulate="plain", use_graphs=graphs)
    frd = p.forward(save_checkpoints=True).clone()
    r_ref = frd - obs_d
    g_ref = p.gradient(r_ref).clone()

    m = p.forward_residual(obs_d)
    assert bits_equal(p.resid.cpu().numpy(), r_ref.cpu().numpy())
    g = p.gradient(None).clone()
    p.check()
    assert bits_equal(g.cpu().numpy(), g_ref.cpu().numpy())
    r64 = r_ref.cpu().numpy().astype(np.float64)
    want = 0.5 * float(np.sum(r64 * r64))
    assert abs(m.item() - want) <= 1e-12 * want

    # same inputs -> the same bits; another observed tensor -> its own misfit
    m2 = p.forward_residual(obs_d)
    assert m2.item() == m.item()
    obs_b = (0.5 * obs_d).contiguous()
    m3 = p.forward_residual(obs_b)
    r_b = (frd - obs_b).cpu().numpy().astype(np.float64)
    want_b = 0.5 * float(np.sum(r_b * r_b))
    assert abs(m3.item() - want_b) <= 1e-12 * want_b


def test_forward_residual_rejects_bad_observed():
    from torchwi_b200 import TwiInvalid
    s, obs = _survey(nshots=2)
    p = _plan(s)
    with pytest.raises(TwiInvalid):
        p.forward_residual(torch.from_numpy(obs))                      # host tensor
    with pytest.raises(TwiInvalid):
        p.forward_residual(torch.from_numpy(obs[:1]).cuda())           # wrong size


def _reference_loop(s, obs, epochs, lr, vmin, vmax):
    """The reference's per-shot epoch (inv_torch.py:123-151): Time2d per shot,
    autograd accumulation over shots, first-gradient normalisation, Adam."""
    model = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda",
                   options=PlanOptions(accumulate="plain"))
    velgen = VelocityParameter(torch.from_numpy(s.vel_start).cuda(), vmin, vmax)
    opt = make_optimizer(velgen.parameters(), "adam", lr)
    gnorm0, losses = None, []
    for _ in range(epochs):
        total = torch.tensor(0.0)
        opt.zero_grad()
        for k in range(s.nshots):
            sx, sy, ry = (torch.tensor(a[k]) for a in (s.sx, s.sy, s.ry))
            frd = model(velgen(), sx, sy, ry)
            loss = 0.5 * torch.sum((frd - torch.from_numpy(obs[k]).cuda()) ** 2)
            loss.backward()
            total.add_(loss.item())
        if gnorm0 is None:
            gnorm0 = velgen.gradient().norm(float("inf"))
        velgen.normalize_gradient(gnorm0)
        opt.step()
        losses.append(total.item())
    with torch.no_grad():
        return velgen.vel().detach().clone(), losses


def test_inversion_matches_per_shot_reference_loop():
    s, obs = _survey()
    lr, vmin, vmax = 20.0, 1400.0, 3000.0
    inv = Inversion(torch.from_numpy(s.vel_start).cuda(), s.nshots, h=s.h, dt=s.dt,
                    w=torch.from_numpy(s.w), order=4, sx=s.sx, sy=s.sy, ry=s.ry,
                    observed=torch.from_numpy(obs).cuda(), vmin=vmin, vmax=vmax, lr=lr,
                    options=PlanOptions(accumulate="plain"))
    hist = inv.run(3)
    v_ref, l_ref = _reference_loop(s, obs, 3, lr, vmin, vmax)
    assert bits_equal(inv.velocity().cpu().numpy(), v_ref.cpu().numpy())
    np.testing.assert_allclose(hist, l_ref, rtol=1e-5)


def test_inversion_reduces_misfit_in_chunks():
    """Kahan accumulation, shots split over several plans by a small HBM
    budget: the misfit goes down over a few epochs."""
    s, obs = _survey(nshots=8, seed=5)
    inv = Inversion(torch.from_numpy(s.vel_start).cuda(), s.nshots, h=s.h, dt=s.dt,
                    w=torch.from_numpy(s.w), order=4, sx=s.sx, sy=s.sy, ry=s.ry,
                    observed=torch.from_numpy(obs).cuda(), vmin=1400.0, vmax=3000.0, lr=10.0,
                    hbm_budget=6 * 2 ** 20)
    hist = inv.run(6)
    assert hist[-1] < 0.7 * hist[0], hist


@pytest.mark.parametrize("reconstruct", [False, True])
def test_residual_after_forward_equals_forward_residual(reconstruct):
    """twi_residual (residual + misfit formed after a saving forward pass, so
    the observed gathers can be uploaded during the pass) gives the bits of
    the fused twi_forward_residual: residual, misfit and gradient."""
    s = synthetic.small_case(nx=90, nz=40, nt=160, order=4, nshots=5, seed=31)
    dev = torch.device("cuda")
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=s.nshots,
                 options=PlanOptions(reconstruct=reconstruct), device=dev)
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel).to(dev))
    obs = p.forward(save_checkpoints=False).clone()
    out = []
    for fused in (True, False):
        p.set_model(torch.from_numpy(s.vel_start).to(dev))
        if fused:
            m = p.forward_residual(obs)
        else:
            p.forward(save_checkpoints=True)
            m = p.residual(obs)
        r = p.resid.clone()
        g = p.gradient(None).clone()
        p.check()
        out.append((m.item(), r.cpu().numpy(), g.cpu().numpy()))
    assert out[0][0] == out[1][0] and out[0][0] > 0
    assert np.array_equal(out[0][1].view(np.int32), out[1][1].view(np.int32))
    assert np.array_equal(out[0][2].view(np.int32), out[1][2].view(np.int32))
