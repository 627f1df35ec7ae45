"""Generate the golden fixtures in this directory by running the REFERENCE
(TorchWI's own ``Time2d(device='cpu')`` operator and its CPU extension built
from the reference sources).  Needs the reference tree ($REFROOT, else a
checkout named ``reference`` beside this repository) and a C++ compiler; it
is NOT run by the tests -- the tests only read the fixtures it wrote.

    python tests/golden/make_golden.py

Fixtures:
  small_o{2,4,8}.npz, small_odd_o4.npz -- full arrays for small cases:
      model, start model, wavelet, coordinates, observed gathers (true model),
      gathers on the start model, per-shot misfit and the shot-summed
      gradient of 0.5*sum((frd-obs)^2), exactly as autograd accumulates it.
  config1.json -- SHA-256 of every config-1 shot gather (float32 bytes) plus
      norms, and config1_shot0_decimated.npy (every 4th sample).
  config2_shot.json -- SHA-256 + norms of one config-2 shot: observed gather,
      start-model gather and its gradient (full 1000x300, nt=4000).
"""

from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFROOT = os.environ.get("REFROOT") or os.path.join(os.path.dirname(REPO), "reference")


def _require_reference():
    if not os.path.isdir(os.path.join(REFROOT, "torchwi")):
        raise SystemExit(f"reference tree not found at {REFROOT}: set REFROOT to the TorchWI checkout")


def _load_reference():
    """Import the reference package and register its CPU extensions (built
    from its unmodified sources with torch's extension builder)."""
    from torch.utils.cpp_extension import load

    if os.path.exists("/usr/bin/g++"):
        os.environ["CXX"] = "/usr/bin/g++"  # /opt/gcc lacks libgomp.spec
    src = os.path.join(REFROOT, "torchwi", "propagator", "td2d")
    build = "/tmp/twi_golden_ext"
    os.makedirs(build, exist_ok=True)
    cpu = load("td2d_cpu", [os.path.join(src, f) for f in
                            ("td2d_cpu.cpp", "propagator_cpu.cpp", "wrapper_cpu.cpp")],
               extra_cflags=["-O2", "-fopenmp"], extra_ldflags=["-fopenmp"],
               build_directory=build, verbose=False)
    build2 = build + "_fwd"
    os.makedirs(build2, exist_ok=True)
    fwd = load("td2d_forward_cpu", [os.path.join(src, f) for f in
                                    ("td2d_cpu.cpp", "propagator_forward_cpu.cpp",
                                     "wrapper_forward_cpu.cpp")],
               extra_cflags=["-O2", "-fopenmp"], extra_ldflags=["-fopenmp"],
               build_directory=build2, verbose=False)
    sys.path.insert(0, REFROOT)
    import torchwi.propagator as P

    P.td2d_cpu = cpu
    P.td2d_forward_cpu = fwd
    sys.modules["torchwi.propagator.td2d_cpu"] = cpu
    sys.modules["torchwi.propagator.td2d_forward_cpu"] = fwd
    import torchwi

    return torchwi


def _sha(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float32).tobytes()).hexdigest()


def _run_gradient(torchwi, s, vel_obs, vel_start, shots):
    """Observed gathers on vel_obs, then misfit + gradient on vel_start,
    accumulated over `shots` exactly as the reference inversion loop does
    (examples/time/inv_torch.py:128-137)."""
    w = torch.from_numpy(s.w.astype(np.float32))
    model = torchwi.Time2d(s.nx, s.nz, s.h, w, s.dt, s.order, "cpu")
    obs, frd, losses = [], [], []
    with torch.no_grad():
        for k in shots:
            o = model(torch.from_numpy(vel_obs), torch.tensor(s.sx[k]),
                      torch.tensor(s.sy[k]), torch.tensor(s.ry[k]))
            obs.append(o.clone().numpy())
    par = torch.nn.Parameter(torch.from_numpy(vel_start.copy()))
    for j, k in enumerate(shots):
        f = model(par, torch.tensor(s.sx[k]), torch.tensor(s.sy[k]), torch.tensor(s.ry[k]))
        frd.append(f.detach().clone().numpy())
        loss = 0.5 * torch.sum((f - torch.from_numpy(obs[j])) ** 2)
        loss.backward()
        losses.append(float(loss.item()))
    return np.stack(obs), np.stack(frd), np.asarray(losses), par.grad.numpy().copy()


def main():
    sys.path.insert(0, REPO)
    from torchwi_b200 import synthetic

    torch.set_num_threads(os.cpu_count() or 1)
    _require_reference()
    torchwi = _load_reference()

    # -- small full-array fixtures ------------------------------------------------
    cases = [("small_o2", dict(nx=40, nz=24, nt=200, order=2)),
             ("small_o4", dict(nx=40, nz=24, nt=200, order=4)),
             ("small_o8", dict(nx=40, nz=24, nt=200, order=8)),
             ("small_odd_o4", dict(nx=37, nz=23, nt=180, order=4, nshots=3))]
    for name, kw in cases:
        s = synthetic.small_case(**kw)
        obs, frd, losses, grad = _run_gradient(torchwi, s, s.vel, s.vel_start,
                                               list(range(s.nshots)))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), vel=s.vel,
                            vel_start=s.vel_start, w=s.w, sx=s.sx, sy=s.sy, ry=s.ry,
                            h=s.h, dt=s.dt, order=s.order, obs=obs, frd=frd,
                            losses=losses, grad=grad)
        print(name, "done", obs.shape, grad.shape)

    # -- config 1: all shot gathers, by hash ------------------------------------------
    s = synthetic.config1()
    w = torch.from_numpy(s.w)
    model = torchwi.Time2dForward(s.nx, s.nz, s.h, w, s.dt, s.order, "cpu")
    rec = {"name": s.name, "nx": s.nx, "nz": s.nz, "nt": s.nt, "order": s.order,
           "rec_crop": list(s.rec_crop), "shots": []}
    t0 = time.time()
    with torch.no_grad():
        for k in range(s.nshots):
            g = model(torch.from_numpy(s.vel), torch.tensor(s.sx[k]),
                      torch.tensor(s.sy[k]), torch.tensor(s.ry[k])).clone().numpy()
            rec["shots"].append({"sx": float(s.sx[k]), "sha256": _sha(g),
                                 "l2": float(np.linalg.norm(g.astype(np.float64))),
                                 "absmax": float(np.abs(g).max())})
            if k == 0:
                np.save(os.path.join(HERE, "config1_shot0_decimated.npy"), g[::4, ::2])
    rec["seconds"] = time.time() - t0
    with open(os.path.join(HERE, "config1.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print("config1 done", rec["seconds"])

    # -- config 2: one shot at full size, by hash ------------------------------------
    s = synthetic.config2(nshots=64, nt=4000)
    k = 31
    t0 = time.time()
    obs, frd, losses, grad = _run_gradient(torchwi, s, s.vel, s.vel_start, [k])
    rec = {"name": s.name, "shot": k, "sx": float(s.sx[k]), "nx": s.nx, "nz": s.nz,
           "nt": s.nt, "order": s.order,
           "obs_sha256": _sha(obs[0]), "frd_sha256": _sha(frd[0]), "grad_sha256": _sha(grad),
           "obs_l2": float(np.linalg.norm(obs[0].astype(np.float64))),
           "frd_l2": float(np.linalg.norm(frd[0].astype(np.float64))),
           "grad_l2": float(np.linalg.norm(grad.astype(np.float64))),
           "loss": float(losses[0]), "seconds": time.time() - t0}
    with open(os.path.join(HERE, "config2_shot.json"), "w") as f:
        json.dump(rec, f, indent=1)
    print("config2 done", rec["seconds"])


if __name__ == "__main__":
    main()
