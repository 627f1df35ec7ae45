"""Inversion driver host logic on CPU: parameterisations, optimizer choices,
the epoch update, and two gloo ranks against one process.  The per-rank
misfit and gradient come from the CPU checker, standing in for the plans."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from torchwi_b200.inversion import (Inversion, SlothParameter, SlownessParameter,
                                    VelocityParameter, make_optimizer)


def test_velocity_parameter_clips_in_place():
    v = torch.tensor([[1000.0, 2000.0], [3500.0, 2500.0]])
    p = VelocityParameter(v, 1500.0, 3000.0)
    out = p()
    assert torch.equal(out, torch.tensor([[1500.0, 2000.0], [3000.0, 2500.0]]))
    assert torch.equal(p.par.data, out.detach())        # clipped in place


def test_bounds_need_both_limits():
    v = torch.tensor([1000.0, 4000.0])
    assert torch.equal(VelocityParameter(v, None, 3000.0)().detach(), v)
    assert torch.equal(VelocityParameter(v, 0.0, 3000.0)().detach(), v)


@pytest.mark.parametrize("cls", [SlothParameter, SlownessParameter])
def test_inverse_parameterisations_round_trip_and_order_bounds(cls):
    v = torch.tensor([1200.0, 2000.0, 5000.0], dtype=torch.float64)
    p = cls(v, 1500.0, 4500.0)
    assert p.pmin < p.pmax
    out = p().detach()
    np.testing.assert_allclose(out.numpy(), [1500.0, 2000.0, 4500.0], rtol=1e-12)


def test_optimizer_choices():
    w = [torch.nn.Parameter(torch.zeros(3))]
    assert isinstance(make_optimizer(w, "adam", 0.1), torch.optim.Adam)
    nag = make_optimizer(w, "nag", 0.1, 0.8)
    assert nag.defaults["nesterov"] and nag.defaults["momentum"] == 0.8
    assert make_optimizer(w, "momentum", 0.1).defaults["momentum"] == 0.9
    assert make_optimizer(w, "gd", 0.1).defaults["momentum"] == 0
    with pytest.raises(ValueError):
        make_optimizer(w, "lbfgs")


def _oracle_local_fn(s, obs):
    import oracle as O

    def fn(vel, shots):
        g_tot, misfit = None, 0.0
        for k in range(shots.start, shots.stop):
            f, g = O.shot_gradient(vel.numpy(), s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k],
                                   lambda f, k=k: (f - obs[k]).astype(np.float32))
            misfit += 0.5 * float(np.sum((f.astype(np.float64) - obs[k]) ** 2))
            g_tot = g if g_tot is None else g_tot + g
        return torch.tensor(misfit, dtype=torch.float64), torch.from_numpy(g_tot)

    return fn


def _survey():
    import oracle as O
    from torchwi_b200 import synthetic

    s = synthetic.small_case(nx=36, nz=20, nt=100, order=4, nshots=3, seed=12)
    obs = [O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k]) for k in range(3)]
    return s, obs


def _run(epochs, group=None):
    s, obs = _survey()
    inv = Inversion(torch.from_numpy(s.vel_start), s.nshots, local_fn=_oracle_local_fn(s, obs),
                    vmin=1400.0, vmax=3000.0, optimizer="gd", lr=15.0, group=group)
    hist = inv.run(epochs)
    return inv.velocity().numpy(), np.array(hist)


def test_epoch_is_normalised_gradient_descent():
    s, obs = _survey()
    fn = _oracle_local_fn(s, obs)
    misfit, g = fn(torch.from_numpy(s.vel_start), slice(0, 3))
    v1, hist = _run(1)
    want = np.clip(s.vel_start, 1400.0, 3000.0) - 15.0 * g.numpy() / np.abs(g.numpy()).max()
    np.testing.assert_allclose(v1, want, rtol=1e-6)
    assert hist[0] == pytest.approx(misfit.item(), rel=1e-6)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        v, hist = _run(2)
        if rank == 0:
            np.save(out, np.concatenate([v.ravel(), hist]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_two_ranks_match_one_process(tmp_path):
    out = str(tmp_path / "v.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    v, hist = _run(2)
    want = np.concatenate([v.ravel(), hist])
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-4)
