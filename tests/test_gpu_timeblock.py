"""Two time steps per launch (twi_step2.cu, PlanOptions(time_block=2)):
gathers, virtual sources and plain gradients bit-identical to the CPU
checker, on grids whose tiles end inside the bottom pad, with odd nt and
odd checkpoint segments (single-step launches finish them)."""
import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal, load_json, rel_l2, sha
from torchwi_b200 import PlanOptions, ShotPlan, Time2d, synthetic

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def _oracle_shots(s, vel, resid_fn=None):
    out = []
    for k in range(s.nshots):
        if resid_fn is None:
            out.append(O.shot_gather(vel, s.w, s.h, s.dt, s.order, s.sx[k], s.sy[k], s.ry[k]))
        else:
            out.append(O.shot_gradient(vel, s.w, s.h, s.dt, s.order, s.sx[k], s.sy[k], s.ry[k],
                                       lambda f, k=k: resid_fn(k, f)))
    return out


def _plan(s, **kw):
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, s.order, nshots=s.nshots, options=PlanOptions(**kw))
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    return p


# nz chosen so that a tile's first row lies in the bottom pad (dimz = 16k + 1)
@pytest.mark.parametrize("order,nx,nz,nt", [(2, 67, 15, 121), (4, 130, 13, 120), (8, 37, 9, 91),
                                            (4, 250, 44, 100), (2, 121, 30, 80)])
@pytest.mark.parametrize("rz", [4, 8])
def test_two_step_gathers_bitexact(order, nx, nz, nt, rz):
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=3, seed=nx + nz)
    p = _plan(s, time_block=2, rows_per_warp=rz, accumulate="plain")
    assert p.layout.time_block == 2
    p.set_model(torch.from_numpy(s.vel).cuda())
    frd = p.forward(save_checkpoints=False).clone()
    p.check()
    ref = _oracle_shots(s, s.vel)
    for k in range(s.nshots):
        assert bits_equal(frd[k].cpu().numpy(), ref[k]), k


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("K", [2, 7, 0])
def test_two_step_gradient_plain_bitexact(order, K):
    s = synthetic.small_case(nx=70, nz=31, nt=121, order=order, nshots=3, seed=11)
    obs = _oracle_shots(s, s.vel)
    res = _oracle_shots(s, s.vel_start, resid_fn=lambda k, f: (f - obs[k]).astype(np.float32))
    g_ref = res[0][1]
    for k in range(1, s.nshots):
        g_ref = (g_ref + res[k][1]).astype(np.float32)
    p = _plan(s, accumulate="plain", ckpt_interval=K, time_block=2)
    p.set_model(torch.from_numpy(s.vel_start).cuda())
    frd = p.forward(save_checkpoints=True).clone()
    for k in range(s.nshots):
        assert bits_equal(frd[k].cpu().numpy(), res[k][0])
    g = p.gradient(frd - torch.from_numpy(np.stack(obs)).cuda()).cpu().numpy()
    p.check()
    assert bits_equal(g, g_ref)


@pytest.mark.parametrize("spc", [1, 3])
def test_two_step_kahan_and_residual(spc):
    """Kahan sums in a different order than single steps: within the
    gradient tolerance of the reference; the fused residual is bit-identical."""
    s = synthetic.small_case(nx=90, nz=40, nt=150, order=4, nshots=5, seed=12)
    obs = torch.from_numpy(np.stack(_oracle_shots(s, s.vel))).cuda()
    g = {}
    for tb in (1, 2):
        p = _plan(s, time_block=tb, shots_per_cta=spc)
        p.set_model(torch.from_numpy(s.vel_start).cuda())
        m = p.forward_residual(obs).item()
        r = p.resid.clone()
        g[tb] = (m, r, p.gradient(None).clone())
        p.check()
    assert g[1][0] == g[2][0]
    assert torch.equal(g[1][1], g[2][1])
    assert rel_l2(g[2][2].cpu().numpy(), g[1][2].cpu().numpy()) <= 1e-6


def test_two_step_profile_and_layout():
    s = synthetic.small_case(nx=64, nz=32, nt=40, order=4, nshots=2)
    p = _plan(s, time_block=2)
    p.set_model(torch.from_numpy(s.vel).cuda())
    for mode in (0, 1, 2):
        assert p.profile(10 + mode, repeats=2) > 0
        assert p.profile_step(mode, repeats=2) > 0
    p.check()
    q = _plan(s, time_block=1)
    q.set_model(torch.from_numpy(s.vel).cuda())
    from torchwi_b200 import TwiInvalid
    with pytest.raises(TwiInvalid):
        q.profile(10)


def test_two_step_config2_shot_full_size():
    rec = load_json("config2_shot.json")
    s = synthetic.config2(nshots=64, nt=4000)
    k = rec["shot"]
    sx, sy, ry = (torch.tensor(a[k]) for a in (s.sx, s.sy, s.ry))
    model = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda",
                   options=PlanOptions(accumulate="plain", time_block=2))
    with torch.no_grad():
        obs = model(torch.from_numpy(s.vel).cuda(), sx, sy, ry)
    assert sha(obs.cpu().numpy()) == rec["obs_sha256"]
    par = torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda())
    frd = model(par, sx, sy, ry)
    assert sha(frd.detach().cpu().numpy()) == rec["frd_sha256"]
    (0.5 * torch.sum((frd - obs) ** 2)).backward()
    assert sha(par.grad.cpu().numpy()) == rec["grad_sha256"]
    model_k = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda",
                     options=PlanOptions(time_block=2))
    par_k = torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda())
    frd_k = model_k(par_k, sx, sy, ry)
    (0.5 * torch.sum((frd_k - obs) ** 2)).backward()
    assert rel_l2(par_k.grad.cpu().numpy(), par.grad.cpu().numpy()) <= GRAD_TOL


def test_autotune_picks_a_shape_with_identical_results():
    from torchwi_b200 import autotune
    s = synthetic.small_case(nx=100, nz=40, nt=60, order=4, nshots=6, seed=3)
    opts, ms = autotune(s.nx, s.nz, s.nshots, 4, s.h, s.dt, PlanOptions(accumulate="plain"))
    assert ms > 0
    # 0: the per-mode defaults won
    assert opts.shots_per_cta in (0, 1, 2, 4) and opts.rows_per_warp in (0, 2, 4, 8)
    assert opts.time_block in (1, 2)
    assert autotune(s.nx, s.nz, s.nshots, 4, s.h, s.dt, PlanOptions(accumulate="plain")) == (opts, ms)
    fixed, _ = autotune(s.nx, s.nz, s.nshots, 4, s.h, s.dt, PlanOptions(accumulate="plain", rows_per_warp=8))
    assert fixed.rows_per_warp == 8
    out = []
    for o in (PlanOptions(accumulate="plain"), opts):
        p = _plan(s, **{k: getattr(o, k) for k in ("accumulate", "shots_per_cta", "rows_per_warp", "time_block")})
        p.set_model(torch.from_numpy(s.vel).cuda())
        out.append(p.forward(save_checkpoints=False).clone())
        p.check()
    assert torch.equal(out[0], out[1])
