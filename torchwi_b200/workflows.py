"""The reference's two time-domain example programs as batched library calls.

* `forward_modeling` -- examples/time/forward_modeling.py:20-52: read the
  model, wavelet and shot table (RSF), model every shot, write one raw
  float32 gather file per shot (`outdir/seismo.%04d`, shape (nt, nx)).
  Here each rank takes a contiguous block of shots and runs it through
  forward-only plans (as many shots per plan as fit the device), and the
  gathers are written in parallel.
* `invert_from_files` -- examples/time/inv_torch.py:15-151: the same inputs
  plus the observed gather files; the rank's gathers are loaded into HBM once
  and the `Inversion` driver runs the epochs.

Receivers sit at the source depth (`ry = sy`), as in both examples.
"""

from __future__ import annotations

import dataclasses
import os

import numpy as np
import torch

from .dist import shard_shots
from .inversion import Inversion
from .io import load_gathers, read_survey, save_gathers
from .plan import PlanOptions, ShotPlan, shot_blocks


def forward_modeling(fvel: str, fwav: str, fshot: str, outdir: str, order: int = 4,
                     device=None, options: PlanOptions | None = None, pattern: str = "seismo.%04d",
                     hbm_budget: int | None = None) -> list[int]:
    """Model this rank's shots and write their gathers; returns the shot
    indices written."""
    s = read_survey(fvel, fwav, fshot)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    opts = dataclasses.replace(options or PlanOptions(), forward_only=True)
    mine = shard_shots(s.nshot)
    os.makedirs(outdir, exist_ok=True)
    vel = torch.from_numpy(np.ascontiguousarray(s.vel)).to(dev)
    w = torch.from_numpy(np.ascontiguousarray(s.w))
    done = []
    for sl in shot_blocks(mine, s.nx, s.ny, s.nt, order, opts, hbm_budget, dev):
        p = ShotPlan(s.nx, s.ny, s.h, s.dt, s.nt, order, nshots=sl.stop - sl.start, options=opts,
                     device=dev)
        p.set_wavelet(w)
        p.set_shots(s.sx[sl], s.sy[sl], s.sy[sl])
        p.set_model(vel)
        frd = p.forward(save_checkpoints=False)
        idx = list(range(sl.start, sl.stop))
        save_gathers(frd, os.path.join(outdir, pattern), idx)
        done += idx
        del p
    return done


def invert_from_files(fvel: str, fwav: str, fshot: str, ftrue: str, epochs: int, order: int = 4,
                      device=None, callback=None, **kwargs) -> Inversion:
    """Run `epochs` of FWI from the reference example's inputs; keyword
    arguments go to `Inversion` (vmin, vmax, optimizer, lr, momentum,
    grad_norm, parameter, options, hbm_budget).  Returns the driver (its
    `history` holds the misfit per epoch, `velocity()` the model)."""
    s = read_survey(fvel, fwav, fshot)
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    mine = shard_shots(s.nshot)
    # only this rank's gathers go to the device
    observed = load_gathers(ftrue, range(mine.start, mine.stop), s.nt, s.nx, device=dev)
    inv = Inversion(torch.from_numpy(np.ascontiguousarray(s.vel)).to(dev), s.nshot, h=s.h, dt=s.dt,
                    w=torch.from_numpy(np.ascontiguousarray(s.w)), order=order, sx=s.sx, sy=s.sy,
                    ry=s.sy, observed=observed, observed_first=mine.start, **kwargs)
    inv.run(epochs, callback)
    return inv


__all__ = ["forward_modeling", "invert_from_files"]
