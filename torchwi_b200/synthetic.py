"""Seeded synthetic workloads with the shapes of the published benchmark
configurations (the reference ships no data: its Marmousi inputs are not
distributed, so these stand in for them).

Every generator returns plain numpy arrays in the reference's user layout:
velocity ``(nx, nz)`` with z fastest, wavelet ``(nt,)`` FP32, and shot /
receiver coordinates in metres (``sx, sy, ry``), exact multiples of ``h`` so
the reference's float-division cell lookup lands on the intended cell.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .source.wavelets import ricker


@dataclass
class Survey:
    name: str
    vel: np.ndarray                 # (nx, nz) float32, z fastest
    h: float
    dt: float
    w: np.ndarray                   # (nt,) float32
    sx: np.ndarray                  # (S,) metres
    sy: np.ndarray                  # (S,) metres
    ry: np.ndarray                  # (S,) metres
    order: int = 4
    vel_start: np.ndarray | None = None   # smoothed starting model (gradient configs)
    rec_crop: tuple[int, int] | None = None  # receiver columns reported
    meta: dict = field(default_factory=dict)

    @property
    def nx(self) -> int:
        return self.vel.shape[0]

    @property
    def nz(self) -> int:
        return self.vel.shape[1]

    @property
    def nt(self) -> int:
        return self.w.shape[0]

    @property
    def nshots(self) -> int:
        return self.sx.shape[0]


def _extend(vel: np.ndarray, n: int) -> np.ndarray:
    """Edge-replicated extension by n cells on left, right and bottom (the
    top stays the free surface)."""
    return np.pad(vel, ((n, n), (0, n)), mode="edge")


def config1(nshots: int = 10) -> Survey:
    """Plain forward modelling: 200x100 cells, h=10 m, linear 1500->3000 m/s
    plus a seeded +-200 m/s Gaussian anomaly (sigma 15 cells), 20-cell
    absorbing extension on the sides and bottom, Ricker 10 Hz, dt=1 ms,
    nt=1000, 10 shots at z=2 cells, receivers on every surface column."""
    nx, nz, h, ext = 200, 100, 10.0, 20
    rng = np.random.default_rng(0)
    ix = np.arange(nx, dtype=np.float64)[:, None]
    iz = np.arange(nz, dtype=np.float64)[None, :]
    v = 1500.0 + 1500.0 * iz / (nz - 1) + 0.0 * ix
    sign = rng.choice([-1.0, 1.0])
    cx = rng.uniform(0.3, 0.7) * nx
    cz = rng.uniform(0.3, 0.7) * nz
    v = v + sign * 200.0 * np.exp(-((ix - cx) ** 2 + (iz - cz) ** 2) / (2 * 15.0 ** 2))
    vel = _extend(v, ext).astype(np.float32)
    shots_ix = np.arange(10, nx, nx // nshots)[:nshots] + ext
    sx = shots_ix.astype(np.float64) * h
    sy = np.full(nshots, 2 * h)
    return Survey("config1", vel, h, 1.0e-3, ricker(10.0, 1.0e-3, 1000).astype(np.float32),
                  sx, sy, sy.copy(), order=4, rec_crop=(ext, ext + nx),
                  meta={"anomaly_sign": float(sign), "ext": ext})


def _layered(nx: int, nz: int, rng: np.random.Generator, depths=None) -> np.ndarray:
    x = np.arange(nx, dtype=np.float64)

    def undulation():
        u = np.zeros(nx)
        for _ in range(3):
            amp = rng.uniform(1.0, 3.0)
            lam = rng.uniform(100.0, 500.0)
            ph = rng.uniform(0.0, 2 * np.pi)
            u += amp * np.sin(2 * np.pi * x / lam + ph)
        return np.clip(u, -5.0, 5.0)

    d1, d2 = depths if depths is not None else (nz / 3.0, 2.0 * nz / 3.0)
    z1 = d1 + undulation()
    z2 = d2 + undulation()
    iz = np.arange(nz, dtype=np.float64)[None, :]
    v = np.where(iz < z1[:, None], 1800.0, np.where(iz < z2[:, None], 2500.0, 3200.0))
    return v


def config2(nshots: int = 64, nt: int = 4000, seed: int = 1) -> Survey:
    """Plain forward + adjoint gradient: 3-layer 1800/2500/3200 m/s model on
    1000x300 cells (interfaces near z=100 and 200 with seeded undulations of
    at most 5 cells), starting model = Gaussian smoothing (sigma 10 cells),
    64 surface shots, 1000 receivers, Ricker 8 Hz, dt=0.8 ms, nt=4000."""
    from scipy.ndimage import gaussian_filter

    nx, nz, h, dt = 1000, 300, 10.0, 0.8e-3
    rng = np.random.default_rng(seed)
    true = _layered(nx, nz, rng)
    start = gaussian_filter(true, 10.0)
    shots_ix = ((np.arange(nshots) + 0.5) * nx / nshots).astype(np.int64)
    sx = shots_ix.astype(np.float64) * h
    sy = np.full(nshots, 2 * h)
    return Survey(f"config2_{nshots}x{nt}", true.astype(np.float32), h, dt,
                  ricker(8.0, dt, nt).astype(np.float32), sx, sy, sy.copy(), order=4,
                  vel_start=start.astype(np.float32))


def layered_case(nx: int, nz: int, nt: int, nshots: int = 1, seed: int = 11, h: float = 10.0,
                 dt: float = 1.0e-3) -> Survey:
    """Parity workload on any grid (e.g. 2000x600, 4000x1200): the config-2
    model class -- three layers 1800/2500/3200 m/s with seeded undulating
    interfaces, here at 100 and 200 cells depth whatever nz is, so that
    reflections return within a few thousand steps -- plus a +-5 %
    near-surface perturbation along the whole line (period 150 cells, centred
    20 cells down), so that even the direct and diving waves of every shot
    differ between the true model and the starting model (the true model
    smoothed with sigma 10 cells).  Ricker 8 Hz, surface shots spread
    evenly."""
    from scipy.ndimage import gaussian_filter

    true = _layered(nx, nz, np.random.default_rng(seed), depths=(min(100.0, nz / 3.0),
                                                                  min(200.0, 2.0 * nz / 3.0)))
    ix = np.arange(nx, dtype=np.float64)[:, None]
    iz = np.arange(nz, dtype=np.float64)[None, :]
    true = true * (1.0 + 0.05 * np.sin(2 * np.pi * ix / 150.0) * np.exp(-(iz - 20.0) ** 2 / (2 * 8.0 ** 2)))
    shots_ix = ((np.arange(nshots) + 0.5) * nx / nshots).astype(np.int64)
    sx = shots_ix.astype(np.float64) * h
    sy = np.full(nshots, 2 * h)
    return Survey(f"layered_{nx}x{nz}x{nt}", true.astype(np.float32), h, dt,
                  ricker(8.0, dt, nt).astype(np.float32), sx, sy, sy.copy(), order=4,
                  vel_start=gaussian_filter(true, 10.0).astype(np.float32))


def config3(nshots: int = 256, nt: int = 6000) -> Survey:
    """Batched shots with checkpointing: the config-2 model class with 256
    shots and nt=6000."""
    s = config2(nshots=nshots, nt=nt)
    s.name = f"config3_{nshots}x{nt}"
    return s


def config4(nmodels: int = 32, seed: int = 4) -> list[Survey]:
    """Uneven batch: seeded models with nx~U{200..2000}, nz~U{100..600},
    h=10 m, smooth 1500-4500 m/s background plus 1-5 elliptical inclusions,
    8-64 shots each, nt~U{2000..6000}, dt=1 ms (CFL 0.45 at 4500 m/s),
    Ricker 8 Hz."""
    rng = np.random.default_rng(seed)
    out = []
    h, dt = 10.0, 1.0e-3
    for m in range(nmodels):
        nx = int(rng.integers(200, 2001))
        nz = int(rng.integers(100, 601))
        nt = int(rng.integers(2000, 6001))
        ns = int(rng.integers(8, 65))
        ix = np.arange(nx, dtype=np.float64)[:, None]
        iz = np.arange(nz, dtype=np.float64)[None, :]
        vtop = rng.uniform(1500.0, 2200.0)
        vbot = rng.uniform(3000.0, 4000.0)
        v = vtop + (vbot - vtop) * iz / (nz - 1) + 0.0 * ix
        for _ in range(int(rng.integers(1, 6))):
            cx, cz = rng.uniform(0, nx), rng.uniform(0, nz)
            ax, az = rng.uniform(10, nx / 4), rng.uniform(5, nz / 4)
            dv = rng.uniform(-400.0, 400.0)
            inside = ((ix - cx) / ax) ** 2 + ((iz - cz) / az) ** 2 <= 1.0
            v = np.where(inside, v + dv, v)
        v = np.clip(v, 1500.0, 4500.0)
        shots_ix = ((np.arange(ns) + 0.5) * nx / ns).astype(np.int64)
        sx = shots_ix.astype(np.float64) * h
        sy = np.full(ns, 2 * h)
        from scipy.ndimage import gaussian_filter
        out.append(Survey(f"config4_m{m}", v.astype(np.float32), h, dt,
                          ricker(8.0, dt, nt).astype(np.float32), sx, sy, sy.copy(),
                          order=4,
                          vel_start=gaussian_filter(v, 8.0).astype(np.float32)))
    return out


def small_case(nx=48, nz=32, nt=300, nshots=2, order=4, seed=7, h=10.0, dt=1.0e-3,
               freq=15.0) -> Survey:
    """Small seeded case for fast parity checks: linear background plus noise
    anomaly, shots spread across the surface."""
    rng = np.random.default_rng(seed)
    iz = np.arange(nz, dtype=np.float64)[None, :]
    v = 1500.0 + 1000.0 * iz / max(nz - 1, 1) + 0.0 * np.arange(nx)[:, None]
    v = v + 80.0 * rng.standard_normal((nx, nz))
    shots_ix = ((np.arange(nshots) + 0.5) * nx / nshots).astype(np.int64)
    sx = shots_ix.astype(np.float64) * h
    sy = np.full(nshots, 2 * h)
    from scipy.ndimage import gaussian_filter
    return Survey(f"small_{nx}x{nz}x{nt}_o{order}", v.astype(np.float32), h, dt,
                  ricker(freq, dt, nt).astype(np.float32), sx, sy, sy.copy(), order=order,
                  vel_start=gaussian_filter(v, 3.0).astype(np.float32))


SERVE_GRIDS = ((500, 200), (1000, 300), (2000, 600), (4000, 1200))


def config5(rate: float, nreq: int = 24, seed: int = 5, max_shots: int = 128,
            nt_range=(2000, 8000), grids=SERVE_GRIDS, h: float = 10.0, dt: float = 1.0e-3):
    """Serving stream: Poisson arrivals at `rate` req/s (seeded), forward or
    gradient requests (50/50) on a resident pool of one layered model per grid
    size {500x200, 1000x300, 2000x600, 4000x1200}, 1..max_shots surface shots,
    nt uniform in nt_range, Ricker 8 Hz, h = 10 m, dt = 1 ms (CFL 0.32).
    Returns (models {name: (nx, nz) float32}, requests [dict])."""
    rng = np.random.default_rng(seed)
    models = {}
    for nx, nz in grids:
        m = _layered(nx, nz, np.random.default_rng(seed * 1000 + nx))
        models[f"layered_{nx}x{nz}"] = m.astype(np.float32)
    names = list(models)
    t = 0.0
    reqs = []
    for i in range(nreq):
        t += rng.exponential(1.0 / rate)
        g = int(rng.integers(len(grids)))
        nx, nz = grids[g]
        ns = int(rng.integers(1, max_shots + 1))
        nt = int(rng.integers(nt_range[0], nt_range[1] + 1))
        kind = "forward" if rng.random() < 0.5 else "gradient"
        ix = ((np.arange(ns) + 0.5) * nx / ns).astype(np.int64)
        sx = ix.astype(np.float64) * h
        sy = np.full(ns, 2 * h)
        reqs.append(dict(kind=kind, model=names[g], sx=sx, sy=sy, ry=sy.copy(),
                         w=ricker(8.0, dt, nt).astype(np.float32), arrival=t))
    return models, reqs
