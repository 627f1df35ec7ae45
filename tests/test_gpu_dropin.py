"""Route 1 of the drop-in: the reference's own, unmodified operator code
(torchwi.Time2d / Time2dForward and TimeFunction, installed from the
reference into baseline/_ref together with its CPU extensions) running on
the drop-in CUDA modules.  The native modules torchwi.propagator.td2d_cuda
and td2d_forward_cuda are replaced by torchwi_b200.propagator.td2d_b200 and
td2d_forward_b200, exactly as a maintainer would register them; the
reference's Time2d(device='cuda') then runs forward modelling and autograd
backward on the B200 kernels.  Its results must equal the reference's own
Time2d(device='cpu') bit for bit -- on grids whose nx and nz are multiples of
16, where the reference's CUDA path pads nothing (TimeOperator.py:36-38).
On other grids that path hands the backward an (nt, nx) residual with the
padded nx (TimeFunction.py:128-141, propagator_cuda.cu:142); the drop-in
module refuses it with a RuntimeError instead of reading past the array.

Skips when baseline/_ref holds no reference install."""
import os
import sys

import numpy as np
import pytest
import torch

from golden_io import bits_equal
from torchwi_b200 import synthetic

pytestmark = pytest.mark.gpu

REF = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref")


@pytest.fixture(scope="module")
def torchwi_ref():
    if not os.path.isdir(os.path.join(REF, "torchwi")):
        pytest.skip("the reference is not installed in baseline/_ref")
    if REF not in sys.path:
        sys.path.append(REF)
    import torchwi
    import torchwi.propagator as P

    from torchwi_b200.propagator import td2d_b200, td2d_forward_b200

    if not os.path.abspath(torchwi.__file__).startswith(REF):
        pytest.skip(f"another torchwi is importable first: {torchwi.__file__}")
    # the registration a maintainer adds (route 1)
    P.td2d_cuda = td2d_b200
    P.td2d_forward_cuda = td2d_forward_b200
    sys.modules["torchwi.propagator.td2d_cuda"] = td2d_b200
    sys.modules["torchwi.propagator.td2d_forward_cuda"] = td2d_forward_b200
    return torchwi


def _run(torchwi, s, device, shots):
    """Observed gathers (true model, Time2dForward), then gathers and the
    shot-summed gradient of 0.5*sum((frd-obs)^2) on the starting model
    through the reference's autograd Function, shot by shot as its
    inversion loop does (examples/time/inv_torch.py:128-137)."""
    w = torch.from_numpy(s.w)
    fwd = torchwi.Time2dForward(s.nx, s.nz, s.h, w, s.dt, s.order, device)
    model = torchwi.Time2d(s.nx, s.nz, s.h, w, s.dt, s.order, device)
    vel = torch.from_numpy(s.vel).to(device)
    par = torch.nn.Parameter(torch.from_numpy(s.vel_start).to(device))
    obs, frd = [], []
    for k in shots:
        xyz = [torch.tensor(a[k]) for a in (s.sx, s.sy, s.ry)]
        with torch.no_grad():
            o = fwd(vel, *xyz).clone()
        f = model(par, *xyz)
        (0.5 * torch.sum((f - o) ** 2)).backward()
        obs.append(o.cpu().numpy())
        frd.append(f.detach().clone().cpu().numpy())   # the reference reuses its frd buffer
    return np.stack(obs), np.stack(frd), par.grad.cpu().numpy()


@pytest.mark.parametrize("order", [2, 4, 8])
def test_reference_operator_on_dropin_modules(torchwi_ref, order):
    s = synthetic.small_case(nx=96, nz=48, nt=260, order=order, nshots=3, seed=60 + order)
    shots = list(range(s.nshots))
    obs_c, frd_c, g_c = _run(torchwi_ref, s, "cpu", shots)
    obs_g, frd_g, g_g = _run(torchwi_ref, s, "cuda", shots)
    assert bits_equal(obs_g, obs_c)
    assert bits_equal(frd_g, frd_c)
    assert bits_equal(g_g, g_c)
    assert np.abs(g_c).max() > 0


def test_padded_grid_residual_is_refused(torchwi_ref):
    # nx = 90: the reference's CUDA path pads to 96 and passes the backward an
    # (nt, 90) residual that its kernels would index as (nt, 96)
    s = synthetic.small_case(nx=90, nz=48, nt=120, order=4, nshots=1, seed=5)
    with pytest.raises(RuntimeError, match="resid holds"):
        _run(torchwi_ref, s, "cuda", [0])
