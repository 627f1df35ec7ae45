"""Time2dModels: several velocity models of different grid sizes, shot
counts and nt in one autograd operator over a PlanBatch; gathers and
gradients bit-identical to the CPU checker, model by model."""
import numpy as np
import pytest
import torch

import oracle as O
from golden_io import bits_equal
from torchwi_b200 import PlanOptions, Time2dModels, synthetic

pytestmark = pytest.mark.gpu


def test_models_of_different_sizes_in_one_batch():
    cases = [synthetic.small_case(nx=60, nz=30, nt=120, nshots=2, seed=1),
             synthetic.small_case(nx=90, nz=41, nt=100, nshots=3, seed=2),
             synthetic.small_case(nx=45, nz=25, nt=130, nshots=1, seed=3)]
    h, dt = cases[0].h, cases[0].dt
    m = Time2dModels([(s.nx, s.nz) for s in cases], h, [torch.from_numpy(s.w) for s in cases], dt, 4,
                     [s.nshots for s in cases], "cuda", options=PlanOptions(accumulate="plain"))
    obs = [np.stack([O.shot_gather(s.vel, s.w, h, dt, 4, s.sx[k], s.sy[k], s.ry[k])
                     for k in range(s.nshots)]) for s in cases]
    pars = [torch.nn.Parameter(torch.from_numpy(s.vel_start).cuda()) for s in cases]
    coords = [tuple(torch.from_numpy(a) for a in (s.sx, s.sy, s.ry)) for s in cases]
    frds = m(pars, coords)
    # the third model's gathers stay out of the loss: its gradient is zero
    loss = sum(0.5 * torch.sum((f - torch.from_numpy(o).cuda()) ** 2) for f, o in zip(frds[:2], obs[:2]))
    loss.backward()
    for i, s in enumerate(cases):
        res = [O.shot_gradient(s.vel_start, s.w, h, dt, 4, s.sx[k], s.sy[k], s.ry[k],
                               lambda f, k=k: (f - obs[i][k]).astype(np.float32)) for k in range(s.nshots)]
        for k in range(s.nshots):
            assert bits_equal(frds[i][k].detach().cpu().numpy(), res[k][0]), (i, k)
        if i < 2:
            g = res[0][1]
            for k in range(1, s.nshots):
                g = (g + res[k][1]).astype(np.float32)
            assert bits_equal(pars[i].grad.cpu().numpy(), g), i
        else:
            assert not pars[i].grad.any()
