"""The reference's example programs as batched calls, from RSF inputs to
gather files and back: modelled gathers equal the CPU checker's bit for bit,
and an inversion read from those files equals one fed in memory."""
import os

import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal
from torchwi_b200 import PlanOptions, synthetic
from torchwi_b200.inversion import Inversion
from torchwi_b200.io import load_gathers, rsf
from torchwi_b200.workflows import forward_modeling, invert_from_files

pytestmark = pytest.mark.gpu


def _write_survey(d, s, vel, name):
    rsf.tofile(os.path.join(d, name), vel, n1=s.nz, n2=s.nx, d1=s.h, d2=s.h)
    rsf.tofile(os.path.join(d, "wav.rsf"), s.w, n1=s.nt, d1=s.dt)
    sxy = np.stack([s.sx, s.sy], 1).astype(np.float32)
    rsf.tofile(os.path.join(d, "shot.rsf"), sxy, n1=2, n2=s.nshots)


@pytest.mark.parametrize("budget", [None, int(0.3 * 2 ** 20)])   # the second: blocks of 2, 2, 1 shots
def test_forward_modeling_writes_reference_gathers(tmp_path, budget):
    s = synthetic.small_case(nx=64, nz=30, nt=130, order=8, nshots=5, seed=31)
    d = str(tmp_path)
    _write_survey(d, s, s.vel, "vel.rsf")
    out = os.path.join(d, "forward")
    done = forward_modeling(os.path.join(d, "vel.rsf"), os.path.join(d, "wav.rsf"),
                            os.path.join(d, "shot.rsf"), out, order=8, hbm_budget=budget)
    assert done == list(range(5))
    for k in range(5):
        got = np.fromfile(os.path.join(out, "seismo.%04d" % k), dtype=np.float32).reshape(s.nt, s.nx)
        want = O.shot_gather(s.vel, s.w, s.h, s.dt, 8, s.sx[k], s.sy[k], s.sy[k])
        assert bits_equal(got, want), k
    g = load_gathers(os.path.join(out, "seismo.%04d"), range(5), s.nt, s.nx, device="cuda")
    assert g.is_cuda and g.shape == (5, s.nt, s.nx)


def test_inversion_from_files_equals_in_memory(tmp_path):
    s = synthetic.small_case(nx=48, nz=26, nt=120, order=4, nshots=4, seed=32)
    d = str(tmp_path)
    _write_survey(d, s, s.vel, "true.rsf")
    rsf.tofile(os.path.join(d, "vinit.rsf"), s.vel_start, n1=s.nz, n2=s.nx, d1=s.h, d2=s.h)
    out = os.path.join(d, "forward")
    forward_modeling(os.path.join(d, "true.rsf"), os.path.join(d, "wav.rsf"),
                     os.path.join(d, "shot.rsf"), out, order=4)
    kw = dict(vmin=1400.0, vmax=3200.0, lr=15.0, options=PlanOptions(accumulate="plain"))
    inv = invert_from_files(os.path.join(d, "vinit.rsf"), os.path.join(d, "wav.rsf"),
                            os.path.join(d, "shot.rsf"), os.path.join(out, "seismo.%04d"), 2,
                            order=4, **kw)
    obs = np.stack([O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.sy[k])
                    for k in range(4)])
    ref = Inversion(torch.from_numpy(s.vel_start).cuda(), 4, h=s.h, dt=s.dt,
                    w=torch.from_numpy(s.w), order=4, sx=s.sx, sy=s.sy, ry=s.sy,
                    observed=torch.from_numpy(obs).cuda(), **kw)
    ref.run(2)
    assert bits_equal(inv.velocity().cpu().numpy(), ref.velocity().cpu().numpy())
    assert inv.history == ref.history
