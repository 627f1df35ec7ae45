"""Golden hashes at the larger grids and shot counts, written by running the
REFERENCE operator (TorchWI's ``Time2d`` / ``Time2dForward`` with
device='cpu' and its CPU extension built from the reference sources, as
make_golden.py does).  Needs the reference tree ($REFROOT, else a checkout
named ``reference`` beside this repository), about 45 GB of host memory and
several minutes.

    python tests/golden/make_golden_large.py

large.json holds, per case, the SHA-256 of the FP32 bytes of every
observed gather (true model), every gather on the starting model and the
shot-summed gradient of 0.5*sum((frd-obs)^2), accumulated shot by shot as
the reference's inversion loop does, plus norms:
  grid_4000x1200 -- one shot, nt=2000 (row pitch 4096 on the GPU);
  grid_2000x600  -- one shot, nt=4500 (more than 4000 steps);
  survey_256     -- 256 shots on a 1000x300 model of the config-2 class,
                    dt=0.8 ms, nt=500 (checkpoint intervals of 50 steps give
                    10 segments).

The reference's full propagator cannot run the two single-shot grids: it
stores the virtual-source history at virt[it*dimxy + i] with 32-bit int
arithmetic (propagator_cpu.cpp:70) and faults once nt*dimxy reaches 2^31
(here 9.6e9 and 5.4e9 samples).  For those cases the gathers come from the
reference's forward-only operator (Time2dForward, no history), and the
gradient from the oracle's restatement of the same propagator, which
indexes in 64 bits and equals the reference bit for bit wherever the
reference runs (tests/test_oracle.py); its gathers are checked against the
reference's here.  Each record names the source of its gradient.
"""

from __future__ import annotations

import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import make_golden as G  # noqa: E402


def _record(s, obs, frd, losses, grad, seconds):
    l2 = lambda a: float(np.linalg.norm(np.asarray(a, dtype=np.float64)))  # noqa: E731
    return {"name": s.name, "nx": s.nx, "nz": s.nz, "nt": s.nt, "order": s.order,
            "h": s.h, "dt": s.dt, "nshots": s.nshots,
            "obs_sha256": [G._sha(o) for o in obs], "frd_sha256": [G._sha(f) for f in frd],
            "grad_sha256": G._sha(grad), "obs_l2": [l2(o) for o in obs], "frd_l2": [l2(f) for f in frd],
            "grad_l2": l2(grad), "loss": [float(x) for x in losses], "seconds": seconds}


def _forward_only_and_oracle_gradient(torchwi, s):
    """Gathers from the reference's forward-only operator; the gradient of
    0.5*sum((frd-obs)^2) (adjoint source frd - obs, as autograd forms it)
    from the oracle's 64-bit-indexed restatement, one shot."""
    import oracle as O

    w = torch.from_numpy(s.w)
    model = torchwi.Time2dForward(s.nx, s.nz, s.h, w, s.dt, s.order, "cpu")
    xyz = [torch.tensor(a[0]) for a in (s.sx, s.sy, s.ry)]
    with torch.no_grad():
        obs = model(torch.from_numpy(s.vel), *xyz).clone().numpy()
        frd = model(torch.from_numpy(s.vel_start), *xyz).clone().numpy()
    frd_o, grad = O.shot_gradient(s.vel_start, s.w, s.h, s.dt, s.order, s.sx[0], s.sy[0], s.ry[0],
                                  lambda f: (f - obs).astype(np.float32))
    assert np.array_equal(frd_o.view(np.int32), frd.view(np.int32)), "oracle gathers differ from the reference's"
    loss = 0.5 * float(np.sum((frd.astype(np.float64) - obs) ** 2))
    return obs[None], frd[None], np.asarray([loss]), grad


def main():
    sys.path.insert(0, G.REPO)
    from torchwi_b200 import synthetic

    torch.set_num_threads(os.cpu_count() or 1)
    G._require_reference()
    torchwi = G._load_reference()
    # name -> (survey, gradient source)
    cases = {
        "grid_4000x1200": (lambda: synthetic.layered_case(4000, 1200, 2000, nshots=1, seed=41), "oracle"),
        "grid_2000x600": (lambda: synthetic.layered_case(2000, 600, 4500, nshots=1, seed=42), "oracle"),
        "survey_256": (lambda: synthetic.layered_case(1000, 300, 500, nshots=256, seed=43, dt=0.8e-3),
                       "reference"),
    }
    out = {}
    for name, (make, source) in cases.items():
        s = make()
        t0 = time.time()
        if source == "reference":
            obs, frd, losses, grad = G._run_gradient(torchwi, s, s.vel, s.vel_start, list(range(s.nshots)))
        else:
            obs, frd, losses, grad = _forward_only_and_oracle_gradient(torchwi, s)
        out[name] = _record(s, obs, frd, losses, grad, time.time() - t0)
        out[name]["gathers_source"] = "reference"
        out[name]["gradient_source"] = source
        print(name, "done", round(out[name]["seconds"], 1), "s", flush=True)
        del obs, frd, grad
    with open(os.path.join(HERE, "large.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
