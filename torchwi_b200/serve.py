"""Serving loop: forward-modelling and gradient requests of different grid
sizes, continuously batched on one GPU.

* Models stay resident on the device (a pool keyed by model id).
* Requests are admitted in arrival order while the sum of their plan
  footprints fits the HBM budget; a request larger than the whole budget is
  split into shot chunks that each fit (gathers are concatenated, gradients
  summed).
* In-flight requests advance together: every tick is one launch per kernel
  mode covering all of them (the C engine in twi_engine.cu); requests join
  and leave between ticks, so a small request does not wait for a large one
  to finish.
* A request's result equals running it alone (same kernels, same inputs).

Latency is measured on the host clock from a request's arrival to the moment
its outputs are complete on the device (stream synchronised).
"""

from __future__ import annotations

import ctypes
import dataclasses
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _capi
from ._capi import check
from .plan import PlanOptions, ShotPlan, _stream_handle, footprint_bytes


class Engine:
    """Thin owner of a C request engine (continuous batching)."""

    def __init__(self, order=4, exact=True, rows_per_warp=0, max_requests=64, device=None):
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self._lib = _capi.lib()
        self._h = ctypes.c_void_p()
        check(self._lib.twi_engine_create(int(order), int(bool(exact)), int(rows_per_warp),
                                          int(max_requests), ctypes.byref(self._h)))
        n = ctypes.c_size_t()
        check(self._lib.twi_engine_workspace_size(self._h, ctypes.byref(n)))
        with torch.cuda.device(self.device):
            self.workspace = torch.empty(int(n.value), dtype=torch.uint8, device=self.device)
            check(self._lib.twi_engine_bind(self._h, ctypes.c_void_p(self.workspace.data_ptr()),
                                            ctypes.c_size_t(self.workspace.numel())))
        self._buf = (ctypes.c_longlong * 256)()

    def submit(self, plan: ShotPlan, kind: str, observed: torch.Tensor | None, tag: int):
        k = {"forward": 0, "gradient": 1}[kind]
        ptr = ctypes.c_void_p(observed.data_ptr()) if observed is not None else None
        check(self._lib.twi_engine_submit(self._h, plan._h, k, ptr, ctypes.c_longlong(tag)))

    def run(self, ticks=64) -> list[int]:
        n = ctypes.c_int()
        with torch.cuda.device(self.device):
            check(self._lib.twi_engine_run(self._h, int(ticks), _stream_handle(), self._buf,
                                           len(self._buf), ctypes.byref(n)))
        return [int(self._buf[i]) for i in range(n.value)]

    def pending(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        check(self._lib.twi_engine_pending(self._h, ctypes.byref(a), ctypes.byref(b)))
        return a.value, b.value

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                torch.cuda.synchronize(self.device)
            except Exception:
                pass
            self._lib.twi_engine_destroy(h)
            self._h = None


@dataclass
class Request:
    """One forward ('forward') or gradient ('gradient') request on a resident
    model.  observed: gathers [nshots, nt, nx] on the device for a gradient
    (None = zero data).  arrival: seconds after the stream starts."""

    kind: str
    model: str
    sx: np.ndarray
    sy: np.ndarray
    ry: np.ndarray
    w: np.ndarray
    observed: torch.Tensor | None = None
    arrival: float = 0.0
    tag: int = -1
    # filled by the server
    result: torch.Tensor | None = None
    done_at: float | None = None

    @property
    def nshots(self):
        return len(self.sx)

    @property
    def nt(self):
        return len(self.w)


@dataclass
class _Chunk:
    req: Request
    shots: slice
    plan: ShotPlan | None = None
    footprint: int = 0
    cells: int = 0          # cell updates per time step (shots x nx x nz)
    work: float = 0.0       # cell updates of the whole chunk (3 passes for a gradient)


def chunk_shots(nshots: int, footprint_of, budget: int) -> list[slice]:
    """Split shots into the fewest equal-size chunks whose footprint fits."""
    if footprint_of(nshots) <= budget:
        return [slice(0, nshots)]
    lo, hi = 1, nshots
    if footprint_of(1) > budget:
        raise MemoryError("a single shot of this request exceeds the HBM budget")
    while lo < hi:   # largest chunk that fits
        mid = (lo + hi + 1) // 2
        if footprint_of(mid) <= budget:
            lo = mid
        else:
            hi = mid - 1
    nchunks = -(-nshots // lo)
    size = -(-nshots // nchunks)
    return [slice(i, min(i + size, nshots)) for i in range(0, nshots, size)]


class Server:
    """Continuous-batching server over a resident model pool.

    Admission (policy="fifo", the default): waiting chunks are admitted in
    arrival order while (a) their plan footprints fit the HBM budget and (b)
    the cell updates per time step of everything in flight stay below
    `saturation_cells` -- roughly what fills the GPU; besides, any waiting
    chunk of at most `backfill_cells` cell updates per step is admitted at
    once (if it fits the budget) and runs alongside whatever is in flight,
    so a small request does not wait behind a large one and a large one
    keeps its place in line.  policy="sjf" takes the shortest waiting chunk
    first instead (lower median latency, a longer tail for early large
    requests).  There is always at least one request in flight."""

    def __init__(self, models: dict, h: float, dt: float, order=4, hbm_budget: int | None = None,
                 options: PlanOptions | None = None, max_requests=64, device=None,
                 saturation_cells: int = 8_000_000, backfill_cells: int = 2_000_000,
                 policy: str = "fifo"):
        if policy not in ("fifo", "sjf"):
            raise ValueError("policy must be 'fifo' or 'sjf'")
        self.policy = policy
        self.backfill_cells = int(backfill_cells)
        self.device = torch.device(device) if device is not None else torch.device(
            "cuda", torch.cuda.current_device())
        self.models = {k: v.to(self.device, torch.float32) for k, v in models.items()}
        self.h, self.dt, self.order = float(h), float(dt), int(order)
        self.options = options or PlanOptions()
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(free * 0.8)
        self.budget = int(hbm_budget)
        self.engine = Engine(order, self.options.exact, self.options.rows_per_warp, max_requests,
                             self.device)
        self.queue: list[_Chunk] = []
        self.inflight: dict[int, _Chunk] = {}
        self.used = 0
        self.saturation_cells = int(saturation_cells)
        self.active_cells = 0
        self._parts: dict[int, list] = {}
        self._next = 0
        self.finished: list[Request] = []
        # reported by the engine, results being copied out: (event, chunk, result)
        self._completing: list = []

    def _options(self, req: Request) -> PlanOptions:
        return dataclasses.replace(self.options, forward_only=req.kind == "forward")

    def _footprint(self, req: Request, nshots: int) -> int:
        nx, nz = self.models[req.model].shape
        return footprint_bytes(nx, nz, req.nt, nshots, self.order, options=self._options(req))

    def submit(self, req: Request):
        req.tag = self._next
        self._next += 1
        parts = chunk_shots(req.nshots, lambda n: self._footprint(req, n), self.budget)
        self._parts[req.tag] = [None] * len(parts)
        nx, nz = self.models[req.model].shape
        for s in parts:
            n = s.stop - s.start
            cells = n * nx * nz
            self.queue.append(_Chunk(req, s, footprint=self._footprint(req, n), cells=cells,
                                     work=cells * req.nt * (3.0 if req.kind == "gradient" else 1.0)))

    def _next_chunk(self):
        """The next chunk to admit, or None.  The queue is kept in arrival
        order (chunks of one request stay together)."""
        fits = lambda ch: self.used + ch.footprint <= self.budget  # noqa: E731
        if self.policy == "sjf":
            order = sorted(range(len(self.queue)), key=lambda i: self.queue[i].work)
            for i in order:
                ch = self.queue[i]
                if fits(ch) and not (self.inflight and self.active_cells + ch.cells > self.saturation_cells):
                    return self.queue.pop(i)
            return None
        if self.queue:   # the head of the line, when the GPU has room for it
            ch = self.queue[0]
            if fits(ch) and not (self.inflight and self.active_cells + ch.cells > self.saturation_cells):
                return self.queue.pop(0)
        for i, ch in enumerate(self.queue):   # small chunks run alongside
            if ch.cells <= self.backfill_cells and fits(ch):
                return self.queue.pop(i)
        return None

    def _admit(self):
        while self.queue:
            ch = self._next_chunk()
            if ch is None:
                break
            r = ch.req
            nx, nz = self.models[r.model].shape
            p = ShotPlan(nx, nz, self.h, self.dt, r.nt, self.order, nshots=ch.shots.stop - ch.shots.start,
                         options=self._options(r), device=self.device)
            p.set_wavelet(torch.from_numpy(np.asarray(r.w, np.float32)))
            p.set_shots(r.sx[ch.shots], r.sy[ch.shots], r.ry[ch.shots])
            p.set_model(self.models[r.model])
            ch.plan = p
            key = self._next
            self._next += 1
            obs = r.observed[ch.shots] if r.observed is not None else None
            if obs is not None and not obs.is_contiguous():
                obs = obs.contiguous()
            ch.obs = obs
            self.engine.submit(p, r.kind, obs, key)
            self.inflight[key] = ch
            self.used += ch.footprint
            self.active_cells += ch.cells

    def poll(self, ticks=64) -> list[Request]:
        """Admit what fits, advance the device, return requests that completed.

        The stream is never drained: when the engine reports a request, its
        result is copied out on the stream and an event marks the copy; the
        request completes (and its plan and memory are released) once that
        event has passed, while the other requests keep the GPU busy."""
        self._admit()
        if self.inflight:
            done_keys = self.engine.run(ticks)
            stream = torch.cuda.current_stream(self.device)
            for key in done_keys:
                ch = self.inflight.pop(key)
                res = (ch.plan.gathers if ch.req.kind == "forward" else ch.plan.grad).clone()
                ev = torch.cuda.Event()
                ev.record(stream)
                self._completing.append((ev, ch, res))
        elif self._completing:   # nothing left to advance: wait for the oldest copy
            self._completing[0][0].synchronize()
        return self._retire()

    def _retire(self) -> list[Request]:
        now = time.perf_counter()
        out, keep = [], []
        for ev, ch, res in self._completing:
            if not ev.query():
                keep.append((ev, ch, res))
                continue
            r = ch.req
            parts = self._parts[r.tag]
            idx = next(i for i, p in enumerate(parts) if p is None)
            parts[idx] = (ch.shots.start, res)
            self.used -= ch.footprint
            self.active_cells -= ch.cells
            ch.plan._done = ev   # its work has finished: no device-wide wait on release
            ch.plan = None
            if all(p is not None for p in parts):
                parts.sort(key=lambda t: t[0])
                if r.kind == "forward":
                    r.result = torch.cat([t[1] for t in parts], dim=0)
                else:
                    g = parts[0][1]
                    for t in parts[1:]:
                        g = g + t[1]
                    r.result = g
                r.done_at = now
                del self._parts[r.tag]
                self.finished.append(r)
                out.append(r)
        self._completing = keep
        return out

    def busy(self) -> bool:
        return bool(self.queue or self.inflight or self._completing)


def run_stream(server: Server, requests: list[Request], ticks=64) -> dict:
    """Replay `requests` (sorted by arrival, seconds) in real time through the
    server; returns throughput and latency percentiles."""
    t0 = time.perf_counter()
    pending = sorted(requests, key=lambda r: r.arrival)
    i = 0
    while i < len(pending) or server.busy():
        now = time.perf_counter() - t0
        while i < len(pending) and pending[i].arrival <= now:
            server.submit(pending[i])
            i += 1
        if server.busy():
            server.poll(ticks)
        elif i < len(pending):
            time.sleep(min(0.002, max(0.0, pending[i].arrival - now)))
    t_end = time.perf_counter() - t0
    lat = np.array([r.done_at - t0 - r.arrival for r in requests])
    return {"requests": len(requests), "seconds": t_end,
            "throughput_req_s": len(requests) / t_end,
            "p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean())}


def plain_service_times(models: dict, requests: list[Request], h, dt, order=4,
                        options: PlanOptions | None = None, device=None) -> list[float]:
    """The plain per-request form: each request alone, one after the other,
    one plan per request (no batching); returns service seconds."""
    out = []
    for r in requests:
        vel = models[r.model]
        nx, nz = vel.shape
        torch.cuda.synchronize()
        t = time.perf_counter()
        o = dataclasses.replace(options or PlanOptions(), forward_only=r.kind == "forward")
        p = ShotPlan(nx, nz, h, dt, r.nt, order, nshots=r.nshots, options=o, device=device)
        p.set_wavelet(torch.from_numpy(np.asarray(r.w, np.float32)))
        p.set_shots(r.sx, r.sy, r.ry)
        p.set_model(vel)
        g = p.forward(save_checkpoints=r.kind == "gradient")
        if r.kind == "gradient":
            if r.observed is not None:
                g.sub_(r.observed)
            p.gradient(None)
        torch.cuda.synchronize()
        out.append(time.perf_counter() - t)
        del p
    return out


def fifo_latencies(arrivals, services):
    """Latencies of a single FIFO server with the given service times."""
    t, lat = 0.0, []
    for a, s in zip(arrivals, services):
        t = max(t, a) + s
        lat.append(t - a)
    return np.array(lat)
