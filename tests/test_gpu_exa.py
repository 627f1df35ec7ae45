"""Excitation-amplitude gradient (the reference's exa=True path,
propagator_exa_cuda.cu) against the CPU restatement: gathers, the stored
amplitudes and 16-bit step indices, and the gradient, bit for bit."""
import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal
from torchwi_b200 import Time2d, synthetic
from torchwi_b200.propagator import td2d_exa_b200

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("order", [2, 4, 8])
@pytest.mark.parametrize("shape", [(40, 24, 150), (37, 23, 130)])
def test_native_exa_bitexact(order, shape):
    nx, nz, nt = shape
    s = synthetic.small_case(nx=nx, nz=nz, nt=nt, order=order, nshots=1, seed=nx + 2 * order)
    dimx, dimy = nx + order, nz + order
    vpad = O.pad_model(s.vel, order)
    args = (order, dimx, dimy, nt, s.h, s.dt, s.sx[0], s.sy[0], s.ry[0])
    f_or, e_or, i_or = O.twio_exa_forward(vpad, s.w, *args)
    dev = torch.device("cuda")
    frd = torch.zeros(nt * nx, device=dev)
    exa = torch.zeros(dimx * dimy, device=dev)
    iexa = torch.zeros(dimx * dimy, dtype=torch.int16, device=dev)
    u = [torch.zeros(dimx * dimy, device=dev) for _ in range(3)]
    vp = torch.from_numpy(vpad).to(dev)
    td2d_exa_b200.forward(frd, exa, iexa, *u, vp, torch.from_numpy(s.w), *args)
    assert bits_equal(frd.cpu().numpy().reshape(nt, nx), f_or)
    assert bits_equal(exa.cpu().numpy(), e_or)
    assert np.array_equal(iexa.cpu().numpy(), i_or)
    resid = (0.4 * f_or - 0.01).astype(np.float32)
    g_or = O.twio_exa_backward(e_or, i_or, vpad, resid, order, dimx, dimy, nt, s.h, s.dt, s.ry[0])
    g = td2d_exa_b200.backward(exa, iexa, *u, vp, torch.from_numpy(resid).to(dev).reshape(-1),
                               order, dimx, dimy, nt, s.h, s.dt, s.ry[0])
    assert bits_equal(g.cpu().numpy(), g_or)


def test_time2d_exa_gradient_over_shots():
    s = synthetic.small_case(nx=60, nz=30, nt=160, order=4, nshots=3, seed=9)
    model = Time2d(s.nx, s.nz, s.h, torch.from_numpy(s.w), s.dt, 4, "cuda", exa=True)
    obs = [O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k]) for k in range(3)]
    par = torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda())
    g_ref = None
    ne, dimx, dimy = 2, s.nx + 4, s.nz + 4
    vpad = O.pad_model(s.vel_start, 4)
    for k in range(3):
        sx, sy, ry = (torch.tensor(a[k]) for a in (s.sx, s.sy, s.ry))
        frd = model(par, sx, sy, ry)
        (0.5 * torch.sum((frd - torch.from_numpy(obs[k]).cuda()) ** 2)).backward()
        f, e, i = O.twio_exa_forward(vpad, s.w, 4, dimx, dimy, s.nt, s.h, s.dt, s.sx[k], s.sy[k], s.ry[k])
        assert bits_equal(frd.detach().cpu().numpy(), f)
        g = O.twio_exa_backward(e, i, vpad, (f - obs[k]).astype(np.float32), 4, dimx, dimy, s.nt,
                                s.h, s.dt, s.ry[k])
        g = g.reshape(dimy, dimx)[ne:ne + s.nz, ne:ne + s.nx].T
        g_ref = g.copy() if g_ref is None else (g_ref + g).astype(np.float32)
    assert bits_equal(par.grad.cpu().numpy(), g_ref)


def test_exa_rejects_long_nt():
    from torchwi_b200 import PlanOptions, ShotPlan, TwiInvalid
    with pytest.raises(TwiInvalid):
        ShotPlan(20, 10, 10.0, 1e-3, 40000, 4, nshots=1, options=PlanOptions(exa=True))


@pytest.mark.parametrize("spc", [1, 4])
def test_plan_exa_many_shots(spc):
    """Eight shots in one plan, several per CTA: one excitation slot and one
    gradient slot per shot, the per-shot gradients summed in shot order."""
    from torchwi_b200 import PlanOptions, ShotPlan
    s = synthetic.small_case(nx=70, nz=33, nt=140, order=4, nshots=8, seed=13)
    ne, dimx, dimy = 2, s.nx + 4, s.nz + 4
    vpad = O.pad_model(s.vel_start, 4)
    obs = [O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k]) for k in range(8)]
    p = ShotPlan(s.nx, s.nz, s.h, s.dt, s.nt, 4, nshots=8,
                 options=PlanOptions(exa=True, shots_per_cta=spc))
    p.set_wavelet(torch.from_numpy(s.w))
    p.set_shots(s.sx, s.sy, s.ry)
    p.set_model(torch.from_numpy(s.vel_start))
    frd = p.forward(save_checkpoints=True).clone()
    g_ref = None
    for k in range(8):
        f, e, i = O.twio_exa_forward(vpad, s.w, 4, dimx, dimy, s.nt, s.h, s.dt, s.sx[k], s.sy[k], s.ry[k])
        assert bits_equal(frd[k].cpu().numpy(), f), k
        g = O.twio_exa_backward(e, i, vpad, (f - obs[k]).astype(np.float32), 4, dimx, dimy, s.nt,
                                s.h, s.dt, s.ry[k])
        g = g.reshape(dimy, dimx)[ne:ne + s.nz, ne:ne + s.nx].T
        g_ref = g.copy() if g_ref is None else (g_ref + g).astype(np.float32)
    g = p.gradient(frd - torch.from_numpy(np.stack(obs)).cuda()).cpu().numpy()
    p.check()
    assert bits_equal(g, g_ref)
