"""Boundary saving with reverse reconstruction (PlanOptions(reconstruct=True)):
the forward pass is unchanged (gathers bit-identical to the CPU checker);
the gradient rebuilds the wavefield backwards in time in FP32, so it is held
to the gradient tolerance of the reference, 1e-4 relative L2."""
import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal, load_json, rel_l2, sha
from torchwi_b200 import PlanBatch, PlanOptions, ShotPlan, Time2d, TwiInvalid, synthetic

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-4


def _plan(s, **kw):
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, s.order, nshots=s.nshots, options=PlanOptions(**kw))
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    return p


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("accumulate", ["plain", "kahan"])
def test_reconstructed_gradient_within_tolerance(order, accumulate):
    s = synthetic.small_case(nx=80, nz=40, nt=400, order=order, nshots=3, seed=17)
    obs = [O.shot_gather(s.vel, s.w, s.h, s.dt, order, s.sx[k], s.sy[k], s.ry[k]) for k in range(3)]
    res = [O.shot_gradient(s.vel_start, s.w, s.h, s.dt, order, s.sx[k], s.sy[k], s.ry[k],
                           lambda f, k=k: (f - obs[k]).astype(np.float32)) for k in range(3)]
    g_ref = res[0][1]
    for k in (1, 2):
        g_ref = (g_ref + res[k][1]).astype(np.float32)
    p = _plan(s, accumulate=accumulate, reconstruct=True)
    p.set_model(torch.from_numpy(s.vel_start).cuda())
    m = p.forward_residual(torch.from_numpy(np.stack(obs)).cuda())
    for k in range(3):   # the forward pass is the checkpointed plan's, residual included
        assert bits_equal(p.resid[k].cpu().numpy(), (res[k][0] - obs[k]).astype(np.float32))
    assert m.item() > 0
    g = p.gradient(None).cpu().numpy()
    p.check()
    err = rel_l2(g, g_ref)
    print(f"order {order} {accumulate}: reconstructed gradient rel L2 = {err:.2e}")
    assert err <= GRAD_TOL


def test_reconstructed_config2_shot_full_size():
    rec = load_json("config2_shot.json")
    s = synthetic.config2(nshots=64, nt=4000)
    k = rec["shot"]
    sx, sy, ry = (torch.tensor(a[k]) for a in (s.sx, s.sy, s.ry))
    ref = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda",
                 options=PlanOptions(accumulate="plain"))
    with torch.no_grad():
        obs = ref(torch.from_numpy(s.vel).cuda(), sx, sy, ry)
    par = torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda())
    (0.5 * torch.sum((ref(par, sx, sy, ry) - obs) ** 2)).backward()
    assert sha(par.grad.cpu().numpy()) == rec["grad_sha256"]
    model = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda",
                   options=PlanOptions(reconstruct=True))
    par_r = torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda())
    frd = model(par_r, sx, sy, ry)
    assert sha(frd.detach().cpu().numpy()) == rec["frd_sha256"]
    (0.5 * torch.sum((frd - obs) ** 2)).backward()
    err = rel_l2(par_r.grad.cpu().numpy(), par.grad.cpu().numpy())
    print(f"config2 shot (nt=4000): reconstructed gradient rel L2 = {err:.2e}")
    assert err <= GRAD_TOL


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("accumulate", ["plain", "kahan"])
@pytest.mark.parametrize("shape", [(80, 40, 300, 3, 0), (37, 23, 200, 11, 4), (130, 41, 120, 9, 2)])
def test_fused_backward_equals_split_launches(order, accumulate, shape):
    """One fused launch per backward step (the virtual source in registers)
    gives the same bits as the rebuild and adjoint launches with the virtual
    source passed through memory."""
    nx, nz, nt, nshots, rz = shape
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=nshots, seed=nx + nshots)
    grads = []
    for split in (False, True):
        p = _plan(s, accumulate=accumulate, reconstruct=True, split_backward=split, rows_per_warp=rz)
        p.set_model(torch.from_numpy(s.vel_start).cuda())
        f = p.forward(save_checkpoints=True)
        grads.append(p.gradient(0.5 * f).cpu().numpy())
        p.check()
    assert bits_equal(grads[0], grads[1])
    assert np.abs(grads[0]).max() > 0


def test_split_backward_plans_stay_out_of_batches():
    # fused boundary-saving plans batch (tests/test_gpu_batch.py); the form with
    # separate rebuild and adjoint launches runs through its own plan only
    s = synthetic.small_case(nx=40, nz=20, nt=50, nshots=2)
    p = _plan(s, reconstruct=True, split_backward=True)
    p.set_model(torch.from_numpy(s.vel).cuda())
    with pytest.raises(TwiInvalid):
        PlanBatch([p])
    PlanBatch([_plan(s, reconstruct=True)])
