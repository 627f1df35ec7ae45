"""Multi-process shot sharding + gradient all-reduce (world size 2, gloo,
CPU).  The per-rank gradient comes from the CPU checker, so this exercises
the host-side logic that bench.py runs over NCCL on GPUs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from torchwi_b200.dist import ShardedGradient, shard_shots


def test_shard_shots_covers_everything_once():
    for n in (1, 2, 5, 64, 257):
        for world in (1, 2, 3, 8):
            seen = []
            for r in range(world):
                s = shard_shots(n, world, r)
                seen.extend(range(s.start, s.stop))
            assert seen == list(range(n))


def _oracle_local_fn(survey, obs):
    import oracle as O

    def fn(vel, shots):
        g_tot, misfit = None, 0.0
        for k in range(shots.start, shots.stop):
            f, g = O.shot_gradient(vel.numpy(), survey.w, survey.h, survey.dt, 4, survey.sx[k],
                                   survey.sy[k], survey.ry[k],
                                   lambda f, k=k: (f - obs[k]).astype(np.float32))
            misfit += 0.5 * float(np.sum((f - obs[k]) ** 2, dtype=np.float64))
            g_tot = g if g_tot is None else g_tot + g
        return torch.tensor(misfit, dtype=torch.float32), torch.from_numpy(g_tot)

    return fn


def _survey():
    from torchwi_b200 import synthetic
    import oracle as O

    s = synthetic.small_case(nx=40, nz=24, nt=120, order=4, nshots=5, seed=8)
    obs = [O.shot_gather(s.vel, s.w, s.h, s.dt, 4, s.sx[k], s.sy[k], s.ry[k]) for k in range(5)]
    return s, obs


def _worker(rank, world, port, nshots, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s, obs = _survey()
        sg = ShardedGradient(_oracle_local_fn(s, obs), nshots)
        misfit, grad = sg(torch.from_numpy(s.vel_start))
        if rank == 0:
            np.save(out, np.concatenate([grad.numpy().ravel(), [misfit.item()]]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


@pytest.mark.parametrize("nshots", [5, 1])
def test_two_ranks_match_single_process(tmp_path, nshots):
    out = str(tmp_path / "g.npy")
    mp.start_processes(_worker, args=(2, _free_port(), nshots, out), nprocs=2, join=True,
                       start_method="spawn")
    got = np.load(out)
    s, obs = _survey()
    misfit, grad = ShardedGradient(_oracle_local_fn(s, obs), nshots)(torch.from_numpy(s.vel_start))
    want = np.concatenate([grad.numpy().ravel(), [misfit.item()]])
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-6 * np.abs(want).max())
