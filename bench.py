"""Benchmark: batched, checkpointed FWI gradient on one B200 per rank.

Workload (one "step" = one full gradient of the survey): 64 surface shots on
the 1000 x 300 three-layer model (h = 10 m, Ricker 8 Hz, dt = 0.8 ms,
nt = 4000, order 4): forward modelling that keeps the absorbing-boundary
cells of every step, L2 residual and misfit, then the backward pass that
rebuilds the forward field in reverse time and takes the adjoint step in
the same fused launch, Kahan-summed gradient (--checkpoints: checkpoints
and a recompute pass instead).  Synthetic data (seeded model generator,
observed gathers modelled on the true model).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl {b200,reference}]

Under torchrun each rank runs its own 64 shots of a 64*N-shot survey
(weak scaling) and the shot-summed gradient and misfit are all-reduced with
NCCL.  Rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

NX, NZ, NT, NSHOTS = 1000, 300, 4000, 64
# Minimal DRAM bytes per cell-update of each kernel mode as this design runs
# it (forward; recompute + virtual-source write; adjoint + virtual-source
# read + gradient read/write; fused backward: u^it, u^{it+1}, lambda^it,
# lambda^{it+1}, v read, u^{it-1}, lambda^{it-1} written, gradient read/write)
ALG_BYTES = {0: 16, 1: 20, 2: 28, 5: 36}
# The same for the reference algorithm's steps, whatever the implementation:
# 16 B per forward-type step (u^{n-1}, u^n, v read, u^{n+1} written), 24 B per
# adjoint step (the same plus the gradient read and write); a backward time
# step recomputes the forward field and takes an adjoint step: 40 B
REF_ALG_BYTES = {0: 16, 1: 16, 2: 24, 5: 40}
MODE_NAMES = {0: "forward step", 1: "recompute step (+virtual source)", 2: "adjoint step (+gradient)",
              5: "fused backward step (reverse reconstruction + adjoint + gradient)"}
TRAFFIC_SHOTS = 64                      # shots per launch of the captures in profiles/traffic.json


def _launches_per_gradient(nt, K, time_block, backward="checkpoints", persistent=False):
    """Kernel launches of one gradient: model padding, the forward steps, the
    two misfit passes, the backward steps (per checkpoint segment its
    recompute and adjoint steps; with boundary saving one fused launch per
    step, or a rebuild and an adjoint launch), the gradient reduction.
    Two-step launches cover pairs of steps; an odd remainder runs alone.
    Persistent launches cover each run of steps of one kernel mode: the
    forward pass, each segment's recompute and adjoint phases, the fused
    backward pass."""
    if persistent:
        segs = (nt + K - 1) // K
        back = 1 if backward == "fused" else 2 * nt if backward == "split" else 2 * segs
        return 1 + 1 + 2 + back + 1
    per = (lambda n: (n + 1) // 2) if time_block == 2 else (lambda n: n)
    if backward == "fused":
        back = nt
    elif backward == "split":
        back = 2 * nt
    else:
        back = 2 * sum(per(min(K, nt - j * K)) for j in range((nt + K - 1) // K))
    return 1 + per(nt) + 2 + back + 1


def _peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
               "-lms", "200"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except Exception:
                self.proc.kill()
        return False

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                rows.append((float(parts[0]), float(parts[1]), parts[4:8]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v == "Active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------
# reference CPU implementation (the reference's own propagator, compiled from
# its sources into oracle/_ref) -- the CPU baseline and the reference arm
# ----------------------------------------------------------------------------

def cpu_reference_shot_gradient(survey, k):
    """One shot-gradient with the reference's compiled CPU propagator."""
    import oracle as O

    obs = O.shot_gather(survey.vel, survey.w, survey.h, survey.dt, 4, survey.sx[k], survey.sy[k],
                        survey.ry[k], backend="ref")
    t0 = time.perf_counter()
    O.shot_gradient(survey.vel_start, survey.w, survey.h, survey.dt, 4, survey.sx[k], survey.sy[k],
                    survey.ry[k], lambda f: (f - obs).astype(np.float32), backend="ref")
    return time.perf_counter() - t0


ONE_THREAD_NT = 400


def cpu_one_thread_seconds():
    """Seconds of one config-2 shot-gradient with nt=ONE_THREAD_NT on one
    thread (run in a child process with OMP_NUM_THREADS=1)."""
    from torchwi_b200 import synthetic
    short = synthetic.config2(nshots=64, nt=ONE_THREAD_NT)
    return cpu_reference_shot_gradient(short, 31)


def cpu_baseline(survey, nsample=1):
    import oracle as O

    kind = "reference" if O.have_ref() else "port"
    if kind == "port":
        return None
    cores = os.cpu_count() or 1
    secs = [cpu_reference_shot_gradient(survey, 31 + i) for i in range(nsample)]
    out = {"value": nsample / sum(secs), "unit": "shot-gradients/s", "cores": cores, "kind": kind,
           "sample": f"{nsample} shot-gradient(s) of the 1000x300 nt=4000 survey "
                     f"(forward + adjoint, reference CPU propagator, OMP_NUM_THREADS={cores})"}
    try:   # the same on one thread, on a shorter run scaled by nt
        env = dict(os.environ, OMP_NUM_THREADS="1")
        code = f"import sys; sys.path.insert(0, {REPO!r}); import bench; print(bench.cpu_one_thread_seconds())"
        r = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, timeout=600)
        t1 = float(r.stdout.strip().splitlines()[-1]) * (survey.nt / ONE_THREAD_NT)
        out["one_thread"] = {"value": 1.0 / t1, "unit": "shot-gradients/s", "cores": 1,
                             "sample": f"one shot-gradient with nt={ONE_THREAD_NT}, time scaled "
                                       f"linearly to nt={survey.nt}"}
    except Exception as e:   # reported, not fatal
        out["one_thread"] = {"unavailable": str(e)[:200]}
    return out


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from torchwi_b200 import synthetic
    import oracle as O

    survey = synthetic.config2(nshots=NSHOTS, nt=NT)
    cores = os.cpu_count() or 1
    if not O.have_ref():
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU propagator (oracle/_ref) not built"}))
        return
    for i in range(args.warmup):
        cpu_reference_shot_gradient(survey, i % NSHOTS)
    secs = [cpu_reference_shot_gradient(survey, i % NSHOTS) for i in range(args.steps)]
    value = len(secs) / sum(secs)
    line = {
        "impl": "reference", "metric": "shot-gradients/s", "value": value, "unit": "shot-gradients/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(secs) / len(secs), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "config2 FWI gradient, 1000x300 cells, nt=4000, order 4; "
                               "one shot per step (bounded sample of the 64-shot survey)",
                   "parallelism": f"cpu openmp x{cores}"},
        "cpu_baseline": {"value": value, "unit": "shot-gradients/s", "cores": cores,
                         "kind": "reference",
                         "sample": "one shot-gradient per step, reference CPU propagator"},
        "e2e": {"value": value, "unit": "shot-gradients/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------
# B200 arm
# ----------------------------------------------------------------------------

def run_b200(args):
    import torch
    import torch.distributed as dist

    from torchwi_b200 import PlanOptions, ShotPlan, synthetic

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=dev)

    survey = synthetic.config2(nshots=NSHOTS * world, nt=NT)
    mine = slice(rank * NSHOTS, (rank + 1) * NSHOTS)
    sx, sy, ry = survey.sx[mine], survey.sy[mine], survey.ry[mine]
    opts = PlanOptions(exact=not args.fast, accumulate="kahan", ckpt_interval=args.ckpt,
                       shots_per_cta=args.spc, rows_per_warp=args.rz, use_graphs=True,
                       time_block=args.time_block, reconstruct=args.reconstruct,
                       split_backward=args.split_backward, persistent=args.persistent,
                       chained=not args.unchained)
    fused = args.reconstruct and not args.split_backward
    tuned_ms = None
    if args.autotune:   # outside the timed region
        from torchwi_b200 import autotune
        opts, tuned_ms = autotune(NX, NZ, NSHOTS, 4, survey.h, survey.dt, opts, dev)
    plan = ShotPlan(NX, NZ, survey.h, survey.dt, NT, 4, nshots=NSHOTS, options=opts, device=dev)
    plan.set_wavelet(torch.from_numpy(survey.w))
    plan.set_shots(sx, sy, ry)

    # observed data: modelled on the true model (outside the timed region)
    plan.set_model(torch.from_numpy(survey.vel).to(dev))
    obs = plan.forward(save_checkpoints=False).clone()
    vel0 = torch.from_numpy(survey.vel_start).to(dev)

    misfit_buf = torch.empty((), dtype=torch.float64, device=dev)

    # events around the forward and the backward pass of every timed step
    # (on the launching stream, inside the timed region)
    marks = []

    def fwi_step(vel, obs_d, mark=False):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if mark else None
        if ev:
            ev[0].record()
        plan.set_model(vel)
        # forward with checkpoints; the receiver writes store modelled - observed
        # in the resid region and a fixed-order FP64 reduction gives the misfit
        loss = plan.forward_residual(obs_d, misfit_buf)
        if ev:
            ev[1].record()
        g = plan.gradient(None)
        if ev:
            ev[2].record()
            marks.append(ev)
        if world > 1:
            dist.all_reduce(g)
            dist.all_reduce(loss)
        return loss, g

    for _ in range(args.warmup):
        fwi_step(vel0, obs)
    plan.check()

    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        pass

    def timed(fn, steps):
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = e0.elapsed_time(e1)
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    with ClockSampler(uuid) as clk:
        ms = timed(lambda: fwi_step(vel0, obs, mark=True), args.steps)
    plan.check()
    clocks = clk.summary()
    ms_step = ms / args.steps
    total_shots = NSHOTS * world
    value = total_shots / (ms_step / 1e3)
    gcell = 2.0 * total_shots * NX * NZ * NT / (ms_step / 1e3) / 1e9

    # end to end: host inputs (pinned), H2D copies and D2H of the result in the region
    vel_h = torch.from_numpy(survey.vel_start).pin_memory()
    obs_h = obs.cpu().pin_memory()
    g_h = torch.empty((NX, NZ), dtype=torch.float32).pin_memory()
    loss_h = torch.empty((), dtype=torch.float64).pin_memory()
    vel_buf = torch.empty_like(vel0)
    obs_buf = torch.empty_like(obs)

    # The 1 GB of observed gathers goes up on a copy stream while the forward
    # pass runs (the residual is formed after the pass, twi_residual); the
    # next step's upload waits until this step's gradient pass is done with it.
    copy_stream = torch.cuda.Stream(device=dev)
    obs_ready = torch.cuda.Event()

    def e2e_step():
        cur = torch.cuda.current_stream(dev)
        copy_stream.wait_stream(cur)
        with torch.cuda.stream(copy_stream):
            obs_buf.copy_(obs_h, non_blocking=True)
            obs_ready.record(copy_stream)
        vel_buf.copy_(vel_h, non_blocking=True)
        plan.set_model(vel_buf)
        plan.forward(save_checkpoints=True)
        cur.wait_event(obs_ready)
        loss = plan.residual(obs_buf, misfit_buf)
        g = plan.gradient(None)
        if world > 1:
            dist.all_reduce(g)
            dist.all_reduce(loss)
        g_h.copy_(g, non_blocking=True)
        loss_h.copy_(loss, non_blocking=True)

    e2e_step()
    ms_e2e = timed(e2e_step, max(1, args.steps // 2)) / max(1, args.steps // 2)
    h2d = vel_h.numel() * 4 + obs_h.numel() * 4
    d2h = g_h.numel() * 4 + 8

    # Roofline of the dominant pass, from the events inside the timed region:
    # the backward pass is nt launches of the fused backward kernel (or nt
    # recompute + nt adjoint launches with checkpoints), so its time / nt is
    # the kernel's average launch duration, graph gaps included.
    fwd_ms = sum(e[0].elapsed_time(e[1]) for e in marks) / len(marks)
    bwd_ms = sum(e[1].elapsed_time(e[2]) for e in marks) / len(marks)
    cells = NSHOTS * NX * NZ
    peak, peak_kind = _peak_hbm()
    back_modes = (5,) if fused else (1, 2)
    names = dict(MODE_NAMES)
    if args.reconstruct:   # a reconstruction plan's second pass rebuilds the field backwards
        names[1] = "reverse reconstruction step (+virtual source)"
    bwd_name = names[5] if fused else f"{names[1]} + {names[2]}"
    per_step = {"forward": fwd_ms / NT, "backward": bwd_ms / NT}
    dom = "backward" if bwd_ms >= fwd_ms else "forward"
    dom_modes = back_modes if dom == "backward" else (0,)
    ref_bytes = sum(REF_ALG_BYTES[m] for m in dom_modes)
    own_bytes = sum(ALG_BYTES[m] for m in dom_modes)
    achieved = ref_bytes * cells / (per_step[dom] / 1e3) / 1e9
    achieved_own = own_bytes * cells / (per_step[dom] / 1e3) / 1e9
    # the same kernels launched alone, back to back (after the timed region)
    iso_modes = (0,) + back_modes
    ms_launch = {m: plan.profile_step(m, repeats=args.profile_reps) for m in iso_modes}
    # DRAM bytes per launch from one ncu capture of each mode at 64 shots on
    # this grid at the shipped launch shape; a launch's traffic grows with the
    # shots it processes, so other shot counts scale it by NSHOTS / 64
    traffic = None
    traffic_source = (f"ncu dram__bytes_read+write per launch at {TRAFFIC_SHOTS} shots, scaled by "
                      f"{NSHOTS}/{TRAFFIC_SHOTS}, summed over the pass's kernels per time step")
    tpath = os.path.join(REPO, "profiles", "traffic.json")
    if os.path.exists(tpath):
        try:
            with open(tpath) as f:
                tj = json.load(f)
            parts = [tj.get(str(m)) for m in dom_modes]
            if all(t is not None for t in parts):
                traffic = sum(parts) * NSHOTS / TRAFFIC_SHOTS
            # the launch shape the capture ran with, against this run's
            for m in dom_modes:
                cap = tj.get("_shape", {}).get(str(m))
                adj = m in (2, 5)
                now = [plan.layout.adjoint_rows_per_warp if adj else plan.layout.rows_per_warp,
                       plan.layout.adjoint_shots_per_cta if adj else plan.layout.shots_per_cta]
                if cap is not None and list(cap) != now:
                    traffic_source += f"; mode {m} captured at (rows per warp, shots per CTA) {cap}, this run {now}"
        except Exception:
            traffic = None

    # the plain form: one shot per launch sequence, no graphs, no batching
    plain = None
    if args.plain_shots > 0 and rank == 0:
        popts = PlanOptions(exact=not args.fast, accumulate="kahan", ckpt_interval=args.ckpt,
                            shots_per_cta=1, use_graphs=False, reconstruct=args.reconstruct,
                            split_backward=args.split_backward)
        p1 = ShotPlan(NX, NZ, survey.h, survey.dt, NT, 4, nshots=1, options=popts, device=dev)
        p1.set_wavelet(torch.from_numpy(survey.w))

        def plain_run(nsh):
            acc = torch.zeros((NX, NZ), device=dev)
            for k in range(nsh):
                p1.set_shots(sx[k:k + 1], sy[k:k + 1], ry[k:k + 1])
                p1.set_model(vel0)
                f = p1.forward(True)
                f.sub_(obs[k:k + 1])
                acc += p1.gradient(None)
            return acc

        plain_run(1)
        ms_plain = timed(lambda: plain_run(args.plain_shots), 1) if world == 1 else None
        if ms_plain:
            plain = {"value": args.plain_shots / (ms_plain / 1e3), "unit": "shot-gradients/s",
                     "shots_timed": args.plain_shots}
        del p1

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(survey, nsample=1)

    if world > 1:
        dist.barrier()
    if rank == 0:
        launches = args.steps * _launches_per_gradient(
            NT, plan.layout.ckpt_interval, plan.layout.time_block,
            "fused" if fused else "split" if args.reconstruct else "checkpoints", args.persistent)
        line = {
            "metric": "shot-gradients/s", "value": value, "unit": "shot-gradients/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded 3-layer model, observed gathers modelled on the true model)",
            "config": {"workload": f"{args.workload}: batched FWI gradient "
                                   f"({'checkpoints' if args.checkpoints else 'boundary saving'}), "
                                   f"{NSHOTS} shots/GPU, 1000x300 cells, nt={NT}, order 4, "
                                   "Keys ABC, Kahan gradient",
                       "global_batch": total_shots, "parallelism": f"shots sharded over {world} GPU(s)",
                       "arith": "fast-fp32" if args.fast else "reference-exact",
                       "ckpt_interval": plan.layout.ckpt_interval,
                       "shots_per_cta": plan.layout.shots_per_cta,
                       "rows_per_warp": plan.layout.rows_per_warp,
                       "adjoint_rows_per_warp": plan.layout.adjoint_rows_per_warp,
                       "adjoint_shots_per_cta": plan.layout.adjoint_shots_per_cta,
                       "time_block": plan.layout.time_block,
                       "launches": "one persistent launch per pass" if args.persistent
                                   else "one launch per time step (CUDA graph)" + (
                                       "" if args.unchained else ", chained: each launch starts "
                                       "while the previous one drains"),
                       "autotuned": bool(args.autotune),
                       "adjoint_wavefield": ("boundary saving, reverse reconstruction, "
                                             + ("rebuild and adjoint launches" if args.split_backward
                                                else "fused backward launch")) if args.reconstruct
                                            else f"checkpoints every {plan.layout.ckpt_interval} steps",
                       "l2": "inputs larger than L2 (workspace %.1f GB)" % (plan.workspace.numel() / 1e9)},
            "gcell_per_s": gcell,
            "clocks": clocks,
            "e2e": {"value": total_shots / (ms_e2e / 1e3), "unit": "shot-gradients/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "how": "public ShotPlan API from pinned host buffers: the model and the observed "
                           "gathers copied up every step (the gathers on a copy stream, overlapping the "
                           "forward pass), residual + misfit after the pass, gradient and misfit copied back"},
            "gpu_launches": launches,
            "roofline": {"bound": "hbm", "kernel": bwd_name if dom == "backward" else names[0],
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                         "alg_bytes_per_cell": ref_bytes,
                         "alg_bytes_basis": "reference algorithm: 16 B per forward-type step, 24 B per "
                                            "adjoint step, per cell-update; one launch = "
                                            f"{cells} cell-updates",
                         "own_alg_bytes_per_cell": own_bytes,
                         "frac_own_bytes": achieved_own / peak,
                         "traffic": traffic, "traffic_source": traffic_source,
                         "ms_per_time_step": {"forward pass": per_step["forward"],
                                              "backward pass": per_step["backward"],
                                              "source": "CUDA events around each pass of every timed step"},
                         "isolated_launch_ms": {names[m]: v for m, v in ms_launch.items()},
                         "whole_gradient_frac": 56.0 * cells * NT / (ms_step / 1e3) / 1e9 / peak},
            "plain_form": plain,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_config4(args):
    """Uneven batch: 32 seeded models (200x100 .. 2000x600 cells, 8-64 shots,
    nt 2000-6000).  Models are packed into waves whose plan footprints fit the
    free HBM; each wave is one PlanBatch (one launch per kernel mode and time
    step for all its models).  Timed: forward with checkpoints, residual,
    gradient, for every wave."""
    import torch

    from torchwi_b200 import PlanBatch, PlanOptions, ShotPlan, footprint_bytes, synthetic

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    models = synthetic.config4()
    if args.models:
        models = models[:args.models]
    opts = PlanOptions(exact=not args.fast, accumulate="kahan", reconstruct=not args.checkpoints,
                       chained=not args.unchained)
    free, _ = torch.cuda.mem_get_info(dev)
    budget = int(free * 0.80)
    fps = [footprint_bytes(m.nx, m.nz, m.nt, m.nshots, 4, options=opts) for m in models]
    obs_bytes = [4 * m.nshots * m.nt * m.nx for m in models]
    order = sorted(range(len(models)), key=lambda i: -fps[i])
    waves, cur, used = [], [], 0
    for i in order:
        need = fps[i] + obs_bytes[i]
        if cur and used + need > budget:
            waves.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += need
    if cur:
        waves.append(cur)
    total_ms, shots, cells = 0.0, 0, 0
    per_wave = []
    for w in waves:
        plans = []
        for i in w:
            m = models[i]
            p = ShotPlan(m.nx, m.nz, m.h, m.dt, m.nt, 4, nshots=m.nshots, options=opts, device=dev)
            p.set_wavelet(torch.from_numpy(m.w))
            p.set_shots(m.sx, m.sy, m.ry)
            p.set_model(torch.from_numpy(m.vel).to(dev))
            plans.append(p)
        batch = PlanBatch(plans)
        obs = [g.clone() for g in batch.forward(save_checkpoints=False)]
        starts = [torch.from_numpy(models[i].vel_start).to(dev) for i in w]

        def step():
            for p, v in zip(plans, starts):
                p.set_model(v)
            gathers = batch.forward(save_checkpoints=True)
            for g, o in zip(gathers, obs):
                g.sub_(o)
            return batch.gradient()

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
        batch.check()
        ms = e0.elapsed_time(e1) / args.steps
        total_ms += ms
        wshots = sum(models[i].nshots for i in w)
        wcells = sum(2 * models[i].nshots * models[i].nx * models[i].nz * models[i].nt for i in w)
        shots += wshots
        cells += wcells
        per_wave.append({"models": len(w), "shots": wshots, "ms": ms,
                         "footprint_gb": sum(fps[i] for i in w) / 1e9})
        del batch, plans, obs, starts
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "config4 uneven batch", "metric": "shot-gradients/s",
                      "adjoint_wavefield": "checkpoints" if args.checkpoints else "boundary saving, fused backward",
                      "launches": "stream order" if args.unchained
                                  else "chained where one launch is at most 8 waves of CTAs",
                      "value": shots / (total_ms / 1e3), "unit": "shot-gradients/s",
                      "gcell_per_s": cells / (total_ms / 1e3) / 1e9, "models": len(models),
                      "shots": shots, "ms_total": total_ms, "waves": per_wave,
                      "arith": "fast-fp32" if args.fast else "reference-exact",
                      "hbm_budget_gb": budget / 1e9}), flush=True)


def run_serve(args):
    """Serving stream (config 5): Poisson arrivals of forward and gradient
    requests on a resident pool of four grid sizes, replayed in real time
    through the continuous-batching server; the same trace through the plain
    per-request form (each request alone, FIFO) gives the comparison.
    Observed gathers are zero (the residual is the modelled data): the work is
    identical to real data.  The sample size is bounded by --requests,
    --max-shots and --nt-max (defaults: 12 requests per rate, the config-5
    ranges of 1-128 shots and nt 2000-8000)."""
    import torch

    from torchwi_b200 import PlanOptions, synthetic
    from torchwi_b200.serve import Request, Server, fifo_latencies, plain_service_times, run_stream

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    opts = PlanOptions(exact=not args.fast, accumulate="kahan", reconstruct=not args.checkpoints)
    out = []
    for rate in args.rates:
        models_np, reqs_np = synthetic.config5(rate, nreq=args.requests, max_shots=args.max_shots,
                                               nt_range=(args.nt_min, args.nt_max))
        models = {k: torch.from_numpy(v).to(dev) for k, v in models_np.items()}
        mk = lambda: [Request(**r) for r in reqs_np]
        # warm the kernels once with the first request
        srv = Server(models, h=10.0, dt=1e-3, options=opts, max_requests=64, device=dev)
        warm = mk()[:1]
        srv.submit(warm[0])
        while srv.busy():
            srv.poll(64)
        srv = Server(models, h=10.0, dt=1e-3, options=opts, max_requests=64, device=dev,
                     policy=args.policy)
        reqs = mk()
        stats = run_stream(srv, reqs, ticks=args.ticks)
        svc = plain_service_times(models, mk(), 10.0, 1e-3, options=opts, device=dev)
        lat = fifo_latencies([r["arrival"] for r in reqs_np], svc)
        shots = sum(len(r["sx"]) for r in reqs_np)
        makespan = float(np.max(lat + np.array([r["arrival"] for r in reqs_np])))
        out.append({"rate_req_s": rate, **stats,
                    "shots_per_s": shots / stats["seconds"],
                    "plain": {"throughput_req_s": len(reqs) / makespan,
                              "p50_s": float(np.percentile(lat, 50)),
                              "p99_s": float(np.percentile(lat, 99)),
                              "service_s_total": float(sum(svc))}})
        del srv
        torch.cuda.empty_cache()
    print(json.dumps({"workload": "config5 serving stream", "requests_per_rate": args.requests,
                      "policy": args.policy,
                      "adjoint_wavefield": "checkpoints" if args.checkpoints else "boundary saving, fused backward",
                      "max_shots": args.max_shots, "nt_range": [args.nt_min, args.nt_max],
                      "grids": [list(g) for g in synthetic.SERVE_GRIDS],
                      "arith": "fast-fp32" if args.fast else "reference-exact",
                      "points": out}), flush=True)


def main():
    global NSHOTS, NT
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--fast", action="store_true", help="fast FP32 arithmetic instead of exact")
    ap.add_argument("--ckpt", type=int, default=0)
    ap.add_argument("--spc", type=int, default=0)
    ap.add_argument("--rz", type=int, default=0)
    ap.add_argument("--time-block", type=int, default=0, help="time steps per launch (0 = plan default)")
    ap.add_argument("--autotune", action="store_true", help="time the launch shapes first and use the fastest")
    ap.add_argument("--checkpoints", action="store_true",
                    help="checkpoints every --ckpt steps and a recompute pass instead of the default "
                         "boundary saving with reverse reconstruction")
    ap.add_argument("--persistent", action="store_true",
                    help="one persistent launch per pass instead of one launch per time step")
    ap.add_argument("--unchained", action="store_true",
                    help="every launch waits for the previous one in stream order (no chained launches)")
    ap.add_argument("--split-backward", action="store_true",
                    help="boundary saving: rebuild and adjoint as two launches per step instead of "
                         "the fused backward launch")
    ap.add_argument("--plain-shots", type=int, default=4)
    ap.add_argument("--profile-reps", type=int, default=20)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shots", type=int, default=NSHOTS, help="shots per GPU")
    ap.add_argument("--nt", type=int, default=NT, help="time steps")
    ap.add_argument("--rates", type=float, nargs="+", default=[5.0, 200.0])
    ap.add_argument("--requests", type=int, default=12)
    ap.add_argument("--max-shots", type=int, default=128)
    ap.add_argument("--nt-min", type=int, default=2000)
    ap.add_argument("--nt-max", type=int, default=8000)
    ap.add_argument("--ticks", type=int, default=64)
    ap.add_argument("--policy", default="fifo", choices=["fifo", "sjf"],
                    help="serve: admission order (arrival order with small requests backfilled, "
                         "or shortest first)")
    ap.add_argument("--workload", default="config2", choices=["config2", "config3", "config4", "serve"],
                    help="config2: the 64-shot gradient (default, the contract line); "
                         "config3: 256 shots, nt=6000 (with --checkpoints: a checkpoint every 50 steps); "
                         "config4: 32 uneven models in HBM-sized waves")
    ap.add_argument("--models", type=int, default=0, help="config4: first N models only")
    args = ap.parse_args()
    args.reconstruct = not args.checkpoints
    if args.workload == "config3":
        NSHOTS, NT = 256, 6000
        args.ckpt = args.ckpt or 50
    else:
        NSHOTS, NT = args.shots, args.nt
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "config4":
        run_config4(args)
    elif args.workload == "serve":
        run_serve(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
