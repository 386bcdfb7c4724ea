"""Benchmark of the B200 room solver.

Default workload (N=1): the large thermal room, 10x8x3 m on a 320x256x96
MAC grid (7.86 M cells), two facing 3 m/s fans, Boussinesq buoyancy, heated
floor / cooled ceiling patches, four seeded boxes, dt = 0.005 s, pressure to
1e-8.  A step is one projection time step of that room; inputs are larger
than L2 (u, v, w, p, T alone are 315 MB), so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload large_thermal|lbm_room|basic_room|batch256|serving_c5|lbm_c4]
                    [--precision mixed|fp64|fp32|fp16] [--graph 1|0]

The default is the mixed-precision path (FP32 increments and FP32 multigrid
preconditioner, FP64 state and outer CG), each step replayed from a CUDA
graph; --precision fp64 runs the reference's method (plain FP64 CG).

Under torchrun every rank runs its own replica of the room on its GPU (rooms
are independent: weak scaling, no collective on the data path); the time is
the max over ranks.  The reference arm times the reference's own CPU solver
(oracle/_ref, compiled from the reference sources) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ff-room_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "cell-steps/s & room-solves/s, mixed-prec batched vs plain FP64 on B200; p50/p99"
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0

# Algorithmic bytes per cell (FP64 fields, 2-byte stencil code, 1-byte
# masks/codes): each array a kernel must read or write, counted once.
CG_INIT_B = 50.0       # read u*,v*,w* + code, write r, d, x
CG_ITER_B = 74.0       # phase A (r, d_old, x, code -> d, Ad, x) + phase B (r, Ad -> r)
CG_FINAL_B = 24.0      # x += alpha d
# Multigrid-preconditioned CG, split form (the bench path), per fine cell:
# the level-0 arrays each pass reads or writes, counted once per pass
# (level 1 and below, 24 MB and less for the large room, count nothing).
# Per iteration (two red-black sweeps per level visit): residual update 34
# (r read and written, q, code; r32 and z written), pre-smoothing black,
# red, black 3 x 14 (z, r32, code read, z written; the colours share DRAM
# sectors), restriction 11 (z, r32, code; the level-1 rhs), post-smoothing
# black 14.5 (the same plus the level-1 correction), red and black 2 x 14,
# red + r.z 22 (z, r32, code, r; z written), direction + operator 46 (z,
# d_old, x, code; d, q, x written).  Once per solve: the warm-start
# extrapolation 40, the set-up 68 (predicted faces, code, the previous
# pressure; r, two directions, r32, z written) and the final x update 24.
# The smoothing passes find z, r32 and the codes (78 MB for the large room)
# in L2: measured DRAM traffic is 83.2 B per cell and iteration
# (profiles/traffic.json), so this model counts bytes the L2 serves.
PCG_ITER_B = 197.5
PCG_ONCE_B = 132.0
# LBM step kernel per lattice cell: read and write 19 populations, the
# flag byte, the cell velocity (FP64 with FP64 populations, else FP32) and
# p (FP64); boundary cells also read a 4-byte blocked-direction mask.
LBM_STEP_B = {"fp64": 2 * 19 * 8 + 1 + 3 * 8 + 8, "fp32": 2 * 19 * 4 + 1 + 3 * 4 + 8,
              "fp16": 2 * 19 * 2 + 1 + 3 * 4 + 8}


def measured_peak():
    try:
        with open(PEAKS) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region.  The
    sampler polls every 200 ms; entering waits (up to 3 s) for its first
    sample and leaving for one taken after the region ended, so a region
    shorter than the polling period is still bracketed by two samples."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.stamps = []
        self.proc = None
        self.t_enter = self.t_exit = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t_end = time.perf_counter() + 3.0
            while not self.rows and time.perf_counter() < t_end and self.proc.poll() is None:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        self.t_enter = time.perf_counter()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.stamps.append(time.perf_counter())
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        self.t_exit = time.perf_counter()
        if self.proc:
            t_end = self.t_exit + 1.0
            while (not self.stamps or self.stamps[-1] < self.t_exit) and time.perf_counter() < t_end \
                    and self.proc.poll() is None:
                time.sleep(0.005)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for i, n in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower() == "active":
                    reasons.add(n)
        inside = sum(1 for t in self.stamps if self.t_enter is not None and self.t_exit is not None
                     and self.t_enter <= t <= self.t_exit)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows), "samples_inside_region": inside,
                "sampling": "every 200 ms, plus one sample just before and one just after the region"}


def load_traffic(key: str, sub: str = None):
    """A measured DRAM-traffic figure (bytes per cell, per cell-iteration)
    from the committed ncu summary profiles/traffic.json, or None."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            v = json.load(fh).get(key)
        return v.get(sub) if (sub is not None and isinstance(v, dict)) else v
    except Exception:
        return None


def scaled_traffic(per_unit, units):
    return None if per_unit is None else per_unit * units


def solve_traffic(mg: bool, cells: int, iters: float):
    """DRAM bytes of one pressure solve from the measured per-cell figures:
    per iteration, plus once per solve (set-up, warm start, final update)
    for the multigrid solve."""
    if not mg:
        return scaled_traffic(load_traffic("cg_bytes_per_cell_iter"), cells * iters)
    it = load_traffic("pcg_split_bytes_per_cell_iter")
    once = load_traffic("pcg_split_bytes_per_cell_once") or 0.0
    return None if it is None else cells * (once + it * iters)


# ------------------------------------------------------------- workloads

def make_workload(name: str, precision: str, grid=None):
    from ffrb import workloads
    from ffrb.params import params_from_scene
    from ffrb.scene import build_room
    if name == "large_thermal":
        cfg, params = workloads.large_thermal(**({"grid": grid} if grid else {}))
        if precision == "fp64":
            params = params.with_(precision="fp64", poisson="cg")
        return "fluid", cfg, build_room(cfg), params
    if name == "basic_room":
        cfg = workloads.basic_room()
        return "fluid", cfg, build_room(cfg), params_from_scene(cfg)
    if name == "lbm_room":
        cfg, tau, dt = workloads.lbm_room(**({"grid": grid} if grid else {}))
        return "lbm", cfg, build_room(cfg), {"tau": tau, "dt": dt, "storage": "fp64" if precision == "fp64"
                                            else ("fp16" if precision == "fp16" else "fp32")}
    raise SystemExit(f"unknown workload {name}")


# ---------------------------------------------------------- our arm

def run_ours(args, rank: int, world: int, dist, with_e2e: bool = True):
    import torch
    from ffrb import capi
    kind, cfg, room, params = make_workload(args.workload, args.precision, args.grid)
    dev = torch.cuda.current_device()
    cells = room.n_cells
    if kind == "fluid":
        h = capi.FluidHandle(room, params)
        h.set_split(args.split)
        if not args.warm_start and getattr(params, "poisson", "") == "mgpcg":
            h.set_warm_start(False)
        if args.graph:
            h.use_graph(True)
    else:
        h = capi.LbmHandle(room, params["tau"], args.steps + args.warmup, 0.0, params["dt"], params["storage"])
    h.advance(args.warmup)
    h.synchronize()
    stream = torch.cuda.ExternalStream(h.stream())
    if not (kind == "fluid" and args.graph):
        h.profile(True)
    l0 = capi.launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(dev) as clk:
        ev0.record(stream)
        recs = h.advance(args.steps)
        ev1.record(stream)
        torch.cuda.synchronize()
    launches = capi.launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    prof = h.profile_read()
    h.profile(False)
    from ffrb.replicas import max_over_ranks
    ms = max_over_ranks(ms, dist, device="cuda")
    steps_done = len(recs)
    value = world * cells * steps_done / (ms / 1e3)
    peak, peak_kind = measured_peak()
    if kind == "fluid":
        iters = [r["cg_iterations"] for r in recs]
        mg = params.poisson == "mgpcg"
        if mg:
            bytes_cg = sum(cells * (PCG_ONCE_B + PCG_ITER_B * it) for it in iters)
            split = args.split == 1 or (args.graph and args.split != 0)
            kname = ("multigrid-preconditioned CG, one kernel per pass (k_sp_*)" +
                     (" in a CUDA graph" if args.graph else ", host-paced") if split
                     else "k_pcg (persistent multigrid-preconditioned CG)")
        else:
            bytes_cg = sum(cells * (CG_INIT_B + CG_ITER_B * it + CG_FINAL_B) for it in iters)
            kname = "k_cg (persistent pressure CG)"
        if args.graph:
            # events cannot bracket kernels inside a replayed step graph: time
            # the pressure solve of the last step again from its own graph
            ms_solve, it_solve = h.time_pressure(3)
            bytes_one = cells * ((PCG_ONCE_B + PCG_ITER_B * it_solve) if mg else
                                 (CG_INIT_B + CG_ITER_B * it_solve + CG_FINAL_B))
            achieved = bytes_one / (ms_solve / 1e3) / 1e9
            launches_cg = 1
            bytes_cg = bytes_one
            prof = {"pressure_estimate": (ms_solve * steps_done, steps_done)}
        else:
            t_cg = prof["pressure"][0] / 1e3
            achieved = bytes_cg / t_cg / 1e9
            launches_cg = max(1, prof["pressure"][1])
        roof = {"bound": "hbm", "kernel": kname, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                # measured DRAM bytes per cell and iteration (ncu, full-size
                # room) times the cells and iterations of one launch
                "traffic": solve_traffic(mg, cells, it_solve if args.graph else float(np.mean(iters))),
                "algorithmic_bytes_per_launch": bytes_cg / launches_cg,
                "share_of_step": round(prof.get("pressure", prof.get("pressure_estimate"))[0] / ms, 4),
                "groups_ms": {g: round(v[0], 3) for g, v in prof.items()}}
        if roof["traffic"]:
            # the same launch measured by the DRAM bytes ncu counted for it
            t_launch = (ms_solve / 1e3) if args.graph else (prof["pressure"][0] / 1e3 / launches_cg)
            roof["frac_by_traffic"] = round(roof["traffic"] / t_launch / 1e9 / peak, 4)
        if args.graph:
            roof["timing"] = "pressure solve of the last step re-run 3x from its own CUDA graph"
        extra = {"cg_iterations_mean": float(np.mean(iters)), "velocity_change_last": recs[-1]["velocity_change"]}
    else:
        b = LBM_STEP_B[params["storage"]] * cells * steps_done
        t_k = prof["stream_collide"][0] / 1e3
        achieved = b / t_k / 1e9
        roof = {"bound": "hbm", "kernel": "k_lbm_step (fused pull-stream/collide)", "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": scaled_traffic(load_traffic("lbm_step_bytes_per_cell", params["storage"]), cells),
                "algorithmic_bytes_per_launch": b / max(1, steps_done),
                "share_of_step": round(prof["stream_collide"][0] / ms, 4),
                "groups_ms": {g: round(v[0], 3) for g, v in prof.items()}}
        extra = {"storage": params["storage"]}
    h.close()
    e2e = run_e2e(args, kind, room, params) if (rank == 0 and with_e2e) else None
    return {"value": value, "ms": ms, "steps": steps_done, "launches": launches, "roofline": roof,
            "clocks": clk.summary(), "extra": extra, "e2e": e2e, "cells": cells, "kind": kind}


def run_plain_fp64(args):
    """The reference's method on this GPU, on the same room: plain FP64 CG
    from a zero pressure (FFR_PREC_FP64, FFR_POISSON_CG), 2 timed steps
    after 1 warm-up step from rest, each step replayed from a CUDA graph.
    The like-for-like comparison beside the headline value, which adds the
    mixed-precision multigrid method.  A failure here is reported in the
    block and leaves the rest of the line intact."""
    import copy
    a = copy.copy(args)
    a.precision, a.steps, a.warmup = "fp64", 2, 1
    try:
        r = run_ours(a, 0, 1, None, with_e2e=False)
    except Exception as e:  # noqa: BLE001 - reported, not raised
        return {"error": f"{type(e).__name__}: {e}"}
    return {"value": r["value"], "unit": "cell-steps/s", "steps": r["steps"], "warmup": 1,
            "ms_per_step": r["ms"] / max(1, r["steps"]), "cg_iterations_mean": r["extra"]["cg_iterations_mean"],
            "method": "plain FP64 CG from a zero pressure (the reference's method) on this GPU, same room, "
                      "steps 2-3 from rest",
            "roofline": r["roofline"], "gpu_launches": r["launches"], "clocks": r["clocks"]}


def run_e2e(args, kind, room, params):
    """The same metric through the public C ABI from host buffers: upload the
    room and the initial fields, run the steps, read every field back."""
    from ffrb import capi
    n = room.n_cells
    shapes = room.shapes()
    init = {k: np.zeros(int(np.prod(shapes[k]))) for k in ("u", "v", "w", "p")}
    h2d = sum(a.nbytes for a in init.values()) + n + 3 * 8 * (room.nx + room.ny + room.nz)
    t0 = time.perf_counter()
    if kind == "fluid":
        h = capi.FluidHandle(room, params, init)
        h.set_split(args.split)
        if not args.warm_start and getattr(params, "poisson", "") == "mgpcg":
            h.set_warm_start(False)
        if args.graph:
            h.use_graph(True)
        recs = h.advance(args.steps)
        out = {k: h.get(k) for k in "uvwpT"}
    else:
        h = capi.LbmHandle(room, params["tau"], args.steps, 0.0, params["dt"], params["storage"], init)
        recs = h.advance(args.steps)
        out = {k: h.get(k) for k in "uvwp"}
    h.close()
    t = time.perf_counter() - t0
    d2h = sum(a.nbytes for a in out.values()) + 48 * len(recs)
    steps = len(recs)
    return {"value": n * steps / t, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d / steps,
            "d2h_bytes_per_step": d2h / steps, "wall_s": t,
            "includes": "room upload + solver setup + steps + all fields read back"}


# ------------------------------------------------- CPU reference timing

def host_threads() -> int:
    """Threads the reference's OpenMP loops run on: OMP_NUM_THREADS when it
    is set, else every core this process may run on (its affinity mask)."""
    try:
        n = int(os.environ.get("OMP_NUM_THREADS", "").split(",")[0])
        if n > 0:
            return n
    except ValueError:
        pass
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_reference(kind, room, params, nsteps=20, budget_s=15.0, single_thread=True):
    """The reference solver (oracle/_ref driver) on a bounded sample of the
    workload: the first steps of the room from rest, stopping at the first
    step that starts after `budget_s` seconds of stepping; the value is the
    cells divided by the median wall time of one step() call.  With
    single_thread, a one-thread estimate is added beside it."""
    import oracle as orc
    threads = host_threads()
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    cells = room.n_cells
    if not orc.ref_available():
        return None
    drv = orc.RefDriver()
    if kind == "lbm":
        _, recs = drv.lbm_run(room, params["tau"], params["dt"], 0.0, 2)
        t = statistics.median(r.seconds for r in recs)
        return {"value": cells / t, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
                "sample": f"{len(recs)} LBM steps of the {room.nx}x{room.ny}x{room.nz} lattice, median step() "
                          "time (the reference LBM has no OpenMP)",
                "steps_timed": len(recs), "seconds_stepping": round(sum(r.seconds for r in recs), 2)}
    # the reference has one pressure method: plain FP64 CG, to the same
    # tolerance and iteration cap
    p = params.with_(precision="fp64", poisson="cg")
    _, _, recs = drv.fluid_run(room, p, nsteps, use_openmp=True, time_budget=budget_s)
    t = statistics.median(r.seconds for r in recs)
    its = [r.cg_iterations for r in recs]
    out = {"value": cells / t, "unit": "cell-steps/s", "cores": threads, "kind": "reference",
           "sample": (f"first {len(recs)} steps of the {room.nx}x{room.ny}x{room.nz} room from rest through the "
                      f"reference FluidSolver (OpenMP, {threads} threads; plain FP64 CG to tol "
                      f"{params.poisson_tol:g}, {min(its)}-{max(its)} iterations per step); value = cells / "
                      f"median step() wall time ({t * 1e3:.1f} ms)"),
           "steps_timed": len(recs), "seconds_stepping": round(sum(r.seconds for r in recs), 2),
           "cg_iterations": its}
    if single_thread:
        out["single_thread"] = cpu_reference_single_thread(drv, room, p, float(np.median(its)))
    return out


def cpu_reference_single_thread(drv, room, p, cg_its: float, m: int = 40):
    """The reference solver on one host thread (use_openmp off), estimated
    from two capped first steps: one step with the CG capped at m iterations
    and one capped at 2m give the time per CG iteration and the rest of the
    step; the estimate is that rest plus cg_its iterations (the iteration
    count the multi-threaded sample needed).  A full single-thread step of a
    large room takes about a minute, so it is not run whole."""
    _, _, r1 = drv.fluid_run(room, p.with_(poisson_max_iter=m), 1, use_openmp=False)
    _, _, r2 = drv.fluid_run(room, p.with_(poisson_max_iter=2 * m), 1, use_openmp=False)
    t_it = max(0.0, (r2[0].seconds - r1[0].seconds) / m)
    t_rest = max(0.0, r1[0].seconds - m * t_it)
    t_step = t_rest + cg_its * t_it
    return {"value": room.n_cells / t_step, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
            "sample": (f"first step from rest with the CG capped at {m} and {2 * m} iterations "
                       f"({r1[0].seconds:.2f} s, {r2[0].seconds:.2f} s): {t_it * 1e3:.2f} ms per CG iteration, "
                       f"{t_rest:.2f} s for the rest of the step, extrapolated to {cg_its:.0f} iterations "
                       f"= {t_step:.1f} s per step (an extrapolation, not a timed full step)")}


def reference_arm(args):
    """bench.py --impl reference: the reference's CPU solver, rank 0 only."""
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    kind, cfg, room, params = make_workload(args.workload, args.precision, args.grid)
    import oracle as orc
    if not orc.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref was not built (reference sources absent at build time)"}))
        return
    # one run of up to warmup + steps reference steps, bounded in time so the
    # whole arm ends within a few minutes; the reference steps from rest
    # with no separate warm-up, and every step it took is a timed sample
    cb = cpu_reference(kind, room, params, nsteps=max(1, args.warmup + args.steps),
                       budget_s=float(args.ref_budget), single_thread=False)
    v = cb["value"]
    nsteps = cb.get("steps_timed", args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "cell-steps/s", "n_gpus": world,
            "steps": nsteps, "warmup": 0, "steps_requested": args.steps, "warmup_requested": args.warmup,
            "ms_per_step": room.n_cells / v * 1e3, "value_is": "cells / median wall time of one step()",
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config_of(args, room, kind, params, reference=True),
            "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def config_of(args, room, kind, params, reference=False):
    """The workload keys (identical for both arms) and the method that ran:
    for the reference arm, the reference's own method (FP64 fields, plain
    CG from a zero pressure, OpenMP on the host cores)."""
    c = {"workload": args.workload, "grid": [room.nx, room.ny, room.nz], "cells": room.n_cells,
         "l2": "inputs larger than L2 (no flush)" if room.n_cells * 8 * 5 > 126e6 else "L2 flush not applied",
         "parallelism": "host cores (OpenMP)" if reference else f"replicas x{args.gpus}"}
    if kind == "fluid":
        c.update({"precision": params.precision, "poisson": params.poisson, "poisson_tol": params.poisson_tol,
                  "dt": params.dt, "advection": params.advection, "thermal": params.thermal,
                  "buoyancy": params.buoyancy,
                  "pressure_start": ("extrapolated previous pressures" if args.warm_start and params.poisson == "mgpcg"
                                     else "zero")})
        if reference:
            c.update({"precision": "fp64", "poisson": "cg", "pressure_start": "zero",
                      "method": "reference FluidSolver (unpreconditioned FP64 CG)"})
    else:
        c.update(params)
        if reference:
            c.update({"storage": "fp64", "method": "reference LBMSolver (FP64, one thread)"})
    return c


# ------------------------------------------------ serving / batched rooms

def serving_requests(kind: str, n: int, max_cells: int, max_steps: int):
    """A bounded sample of the serving stream (Poisson arrivals at 200/s,
    log-uniform sizes; seed 11) or of the 256 uneven rooms (seed 7, all at
    t = 0): the first n requests with at most max_cells cells, each capped at
    max_steps steps."""
    from ffrb import workloads
    from ffrb.params import params_from_scene
    from ffrb.serve import requests_from_configs
    from ffrb.scene import build_room
    if kind == "serving":
        stream = workloads.serving_stream()
        pick = [rq for rq in stream if np.prod(rq.cfg.room.grid) <= max_cells][:n]
        return requests_from_configs([rq.cfg for rq in pick], [rq.params for rq in pick],
                                     [rq.t_arrival - pick[0].t_arrival for rq in pick], max_steps)
    rooms = [c for c in workloads.batch_rooms() if np.prod(c.room.grid) <= max_cells][:n]
    return requests_from_configs(rooms, [params_from_scene(c) for c in rooms], [0.0] * len(rooms), max_steps)


def run_serving(kind: str, n: int, max_cells: int, max_steps: int, batched: bool = True, chunk: int = 10,
                warm_start: bool = True):
    """The serving sample through the continuous-batching server: batched
    (every active room in one launch per stage, rooms joining and leaving
    between chunks) or one stream per room with tuned schedules."""
    import torch
    from ffrb.serve import Request, Server, Tuner, report, serial_solve
    reqs = serving_requests(kind, n, max_cells, max_steps)
    tuner = Tuner()   # default schedules: one 16-block cluster per room up to 1 M cells
    free, total = torch.cuda.mem_get_info()
    srv = Server(mem_budget=int(free * 0.6), max_active=64, tuner=tuner, batched=batched, chunk=chunk,
                 warm_start=warm_start)
    # untimed warm-up of both arms on a few short requests (module loading,
    # memory-pool growth, pinned-buffer cache)
    warm = [Request(r.rid, 0.0, r.room, r.params, 2) for r in reqs[:4]]
    srv.run(warm, realtime=False)
    serial_solve(warm[:1], {"precision": "fp64", "poisson": "cg", "use_multigrid": False})
    l0 = __import__("ffrb.capi", fromlist=["x"]).launch_count()
    with ClockSampler(torch.cuda.current_device()) as clk:
        out = srv.run(reqs, realtime=(kind == "serving"))
    launches = __import__("ffrb.capi", fromlist=["x"]).launch_count() - l0
    rep = report(out)
    base = serial_solve(reqs, {"precision": "fp64", "poisson": "cg", "use_multigrid": False})
    rb = report(base, makespan=max(o.t_done for o in base))
    rep["serial_fp64_room_solves_per_s"] = rb["room_solves_per_s"]
    rep["serial_fp64_cell_steps_per_s"] = rb["cell_steps_per_s"]
    rep["speedup_vs_serial_fp64"] = rep["room_solves_per_s"] / rb["room_solves_per_s"]
    rep["sample"] = (f"{len(reqs)} requests with <= {max_cells} cells, cap {max_steps} steps"
                     + (", Poisson arrivals in real time" if kind == "serving" else ", all at t = 0"))
    rep["schedules"] = (f"batched, chunks of {chunk} steps" if batched else
                        "one stream per room; default schedules (16-block cluster up to 1 M cells, "
                        "else split solve on the whole GPU), CUDA-graph steps")
    rep["gpu_launches"] = launches
    rep["clocks"] = clk.summary()
    return rep


# ------------------------------------- C3: 256 uneven rooms in one batch

def _serial_fp64_estimate(reqs, sample: int = 8, steps: int = 20):
    """Serial plain FP64 GPU solve time of `reqs` (each to its own step
    count), estimated from a stratified sample: `sample` rooms spread over
    the size range each run `steps` steps from rest with the reference's
    method (FP64, unpreconditioned CG); every request is charged the
    per-cell-step time of the sampled room nearest in size, times its cells
    and steps.  Returns (seconds, description)."""
    from ffrb import capi
    order = sorted(range(len(reqs)), key=lambda i: reqs[i].room.n_cells)
    pick = [order[int(round(k * (len(order) - 1) / max(1, sample - 1)))] for k in range(sample)]
    rates = []
    for i in pick:
        rq = reqs[i]
        p = rq.params.with_(precision="fp64", poisson="cg", use_multigrid=False)
        h = capi.FluidHandle(rq.room, p)
        h.advance(1)
        h.synchronize()
        t0 = time.perf_counter()
        h.advance(steps)
        h.synchronize()
        dt = time.perf_counter() - t0
        h.close()
        rates.append((rq.room.n_cells, rq.room.n_cells * steps / dt))
    total = 0.0
    for rq, st in ((r, getattr(r, "steps_done", r.max_steps)) for r in reqs):
        rate = min(rates, key=lambda cr: abs(np.log(cr[0] / rq.room.n_cells)))[1]
        total += rq.room.n_cells * st / rate
    desc = (f"plain FP64 CG on the GPU, one room at a time: {sample} rooms spread over the size range each timed "
            f"for {steps} steps after one untimed step; every request charged the per-cell-step time of the "
            f"sampled room nearest in size times its cells and steps (an extrapolation)")
    return total, desc


def run_batch256(steps: int = 500, engines=("batched", "streams")):
    """The 256 uneven rooms (seed 7, dims U{32..128} per axis, 500 steps,
    mixed precision) advanced as one batch: every stage one launch for all
    rooms, each step one CUDA-graph replay with the multigrid solve in a
    WHILE node; beside it the same rooms on one stream per room."""
    import torch
    from ffrb import capi, workloads
    from ffrb.params import params_from_scene
    from ffrb.serve import Server, requests_from_configs
    cfgs = workloads.batch_rooms(steps=steps)
    reqs = requests_from_configs(cfgs, [params_from_scene(c) for c in cfgs], [0.0] * len(cfgs), steps)
    cells = sum(r.room.n_cells for r in reqs)
    free, _ = torch.cuda.mem_get_info()
    out = {"rooms": len(reqs), "cells": cells, "steps_per_room": steps,
           "sample": "all 256 rooms of the seed-7 batch, 500 steps each, all at t = 0 (no convergence stop)"}
    # untimed warm-up: a few small rooms through both engines
    small = sorted(reqs, key=lambda r: r.room.n_cells)[:4]
    from ffrb.serve import Request
    warm = [Request(r.rid, 0.0, r.room, r.params, 2) for r in small]
    for eng in engines:
        Server(mem_budget=int(free * 0.5), max_active=len(reqs), batched=(eng == "batched"), chunk=2).run(
            warm, realtime=False)
    from ffrb.tune import TUNED_TABLE, load_tuned
    tuner = load_tuned()
    out["schedules"] = ("streams engine: the tuned per-size-class table (ffrb/tuned_b200.json)"
                        if os.path.exists(TUNED_TABLE) else "streams engine: default schedules")
    for eng in engines:
        l0 = capi.launch_count()
        srv = Server(mem_budget=int(free * 0.6), max_active=len(reqs), batched=(eng == "batched"), chunk=50,
                     tuner=tuner)
        with ClockSampler(torch.cuda.current_device()) as clk:
            t0 = time.perf_counter()
            res = srv.run(reqs, realtime=False)
            span = time.perf_counter() - t0
        done_steps = sum(o.steps for o in res)
        by_cells = {o.rid: o for o in res}
        out[eng] = {"room_solves_per_s": len(res) / span, "makespan_s": span,
                    "cell_steps_per_s": sum(by_cells[r.rid].steps * r.room.n_cells for r in reqs) / span,
                    "steps_done": done_steps, "gpu_launches": capi.launch_count() - l0,
                    "clocks": clk.summary()}
    for r in reqs:
        r.steps_done = steps
    t_serial, desc = _serial_fp64_estimate(reqs)
    out["serial_fp64_room_solves_per_s"] = len(reqs) / t_serial
    out["serial_fp64_estimate"] = desc
    for eng in engines:
        out[eng]["speedup_vs_serial_fp64"] = out[eng]["room_solves_per_s"] * t_serial / len(reqs)
    return out


# ------------------------------------------------ C4: the LBM lattice

LBM_STABLE_TAU = 0.6


def run_lbm_c4(steps: int = 200, warmup: int = 10):
    """The 384x320x128 D3Q19 lattice (fan inlet at lattice speed 0.05, six
    boxes) with FP64, FP32 and FP16 population storage: lattice cell-steps/s
    over `steps` steps (CUDA events on the solver's stream) and the step
    kernel against the HBM roofline.  The configuration's tau = 0.52 drives
    this lattice to NaN within 250 steps (in FP64, whose arithmetic matches
    the reference's bit for bit; 0.55 within 500), so the timing runs at
    tau = 0.6, which stays finite over 10000 steps; the work per step does
    not depend on tau."""
    import torch
    from ffrb import capi, workloads
    from ffrb.scene import build_room
    cfg, tau_cfg, dt = workloads.lbm_room()
    tau = LBM_STABLE_TAU
    room = build_room(cfg)
    peak, peak_kind = measured_peak()
    out = {"grid": [room.nx, room.ny, room.nz], "cells": room.n_cells, "tau": tau, "tau_configured": tau_cfg,
           "steps": steps,
           "note": "tau 0.52 diverges to NaN within 250 steps on this lattice (FP64, the reference's arithmetic); "
                   "timed at tau 0.6 (finite over 10000 steps)"}
    for storage in ("fp64", "fp32", "fp16"):
        h = capi.LbmHandle(room, tau, steps + warmup, 0.0, dt, storage)
        h.advance(warmup)
        h.synchronize()
        stream = torch.cuda.ExternalStream(h.stream())
        h.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        recs = h.advance(steps)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        prof = h.profile_read()
        h.close()
        t_k = prof["stream_collide"][0] / 1e3
        b = LBM_STEP_B[storage] * room.n_cells * len(recs)
        out[storage] = {"lattice_cell_steps_per_s": room.n_cells * len(recs) / (ms / 1e3),
                        "ms_per_step": ms / len(recs),
                        "step_kernel_GBps": round(b / t_k / 1e9, 1),
                        "step_kernel_frac": round(b / t_k / 1e9 / peak, 4),
                        "step_kernel_share": round(prof["stream_collide"][0] / ms, 4),
                        "algorithmic_bytes_per_cell": LBM_STEP_B[storage],
                        "traffic_bytes_per_cell": load_traffic("lbm_step_bytes_per_cell", storage)}
    out["peak_GBps"] = peak
    out["peak_source"] = peak_kind
    return out


# ------------------------------------------------ C5: the serving stream

def run_serving_c5(n: int = 96, max_steps: int = 200, tol: float = 1e-4, max_cells: int = None,
                   engines=("streams",)):
    """A time-bounded prefix of the serving stream (seed 11, Poisson
    arrivals at 200/s, log-uniform sizes up to 256x256x96): the first n
    requests, arriving in real time, each solved in mixed precision until
    max|du|/dt < tol or max_steps, through the continuous-batching server."""
    import torch
    from ffrb import capi, workloads
    from ffrb.serve import Request, Server, report, requests_from_configs
    stream = workloads.serving_stream()
    pick = [rq for rq in stream if max_cells is None or np.prod(rq.cfg.room.grid) <= max_cells][:n]
    reqs = requests_from_configs([rq.cfg for rq in pick],
                                 [rq.params.with_(convergence_tol=tol) for rq in pick],
                                 [rq.t_arrival - pick[0].t_arrival for rq in pick], max_steps)
    free, _ = torch.cuda.mem_get_info()
    warm = [Request(r.rid, 0.0, r.room, r.params, 2) for r in sorted(reqs, key=lambda r: r.room.n_cells)[:4]]
    out = {"requests": len(reqs), "cells_max": max(r.room.n_cells for r in reqs),
           "cells_min": min(r.room.n_cells for r in reqs), "stop_rule": f"max|du|/dt < {tol:g} or {max_steps} steps",
           "sample": (f"the first {len(reqs)} requests of the seed-11 stream"
                      + (f" with <= {max_cells} cells" if max_cells else " (full size mix)")
                      + f", arriving in real time over {reqs[-1].t_arrival:.2f} s")}
    results = {}
    from ffrb.tune import TUNED_TABLE, load_tuned
    tuner = load_tuned()
    out["schedules"] = ("streams engine: the tuned per-size-class table (ffrb/tuned_b200.json)"
                        if os.path.exists(TUNED_TABLE) else "streams engine: default schedules")
    for eng in engines:
        srv = Server(mem_budget=int(free * 0.6), max_active=64, batched=(eng == "batched"), chunk=10,
                     tuner=tuner)
        srv.run(warm, realtime=False)
        l0 = capi.launch_count()
        with ClockSampler(torch.cuda.current_device()) as clk:
            res = srv.run(reqs, realtime=True)
        rep = report(res)
        conv = [o for o in res if o.converged]
        rep["p50_time_to_converged_s"] = float(np.percentile([o.latency for o in conv], 50)) if conv else None
        rep["p99_time_to_converged_s"] = float(np.percentile([o.latency for o in conv], 99)) if conv else None
        rep["median_final_velocity_change"] = float(np.median([o.velocity_change for o in res]))
        rep["gpu_launches"] = capi.launch_count() - l0
        rep["clocks"] = clk.summary()
        results[eng] = (rep, res)
        out[eng] = rep
    # the serial baseline solves the same requests to the same step counts
    steps_of = {o.rid: o.steps for o in results[engines[0]][1]}
    for r in reqs:
        r.steps_done = steps_of[r.rid]
    t_serial, desc = _serial_fp64_estimate(reqs)
    out["serial_fp64_room_solves_per_s"] = len(reqs) / t_serial
    out["serial_fp64_estimate"] = desc
    for eng in engines:
        out[eng]["speedup_vs_serial_fp64"] = out[eng]["room_solves_per_s"] * t_serial / len(reqs)
    return out


def serving_arm(args):
    import torch
    torch.cuda.set_device(0)
    rep = run_serving(args.workload, args.requests, args.max_cells, args.max_steps, bool(args.batched), args.chunk,
                      bool(args.warm_start))
    line = {"metric": METRIC, "value": rep["room_solves_per_s"], "unit": "room-solves/s", "n_gpus": 1,
            "steps": args.max_steps, "warmup": 0, "ms_per_step": None, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32/f64", "data": "synthetic",
            "config": {"workload": args.workload, "requests": rep["requests"], "max_cells": args.max_cells,
                       "max_steps": args.max_steps, "precision": "mixed", "poisson": "mgpcg",
                       "pressure_start": "extrapolated previous pressures" if args.warm_start else "zero"},
            "serving": rep, "gpu_launches": rep["gpu_launches"], "clocks": rep["clocks"]}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large_thermal")
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--ref-budget", type=float, default=90.0,
                    help="--impl reference: seconds of reference stepping after which the sample stops")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=lambda s: tuple(int(x) for x in s.split(",")), default=None,
                    help="override the grid (profiling runs on a smaller case)")
    ap.add_argument("--requests", type=int, default=48, help="serving/batch sample size")
    ap.add_argument("--max-cells", type=int, default=600_000, help="serving/batch: largest room in the sample")
    ap.add_argument("--max-steps", type=int, default=40, help="serving/batch: step cap per room")
    ap.add_argument("--no-serving", action="store_true",
                    help="default run: skip the plain FP64 comparison and the serving, batch and lattice samples")
    ap.add_argument("--tol", type=float, default=1e-4, help="serving_c5: the stop rule's max|du|/dt")
    ap.add_argument("--batched", type=int, default=0,
                    help="serving/batch: 1 = one launch per stage for all active rooms, 0 = one stream per room")
    ap.add_argument("--chunk", type=int, default=10, help="serving/batch: steps between membership changes")
    ap.add_argument("--graph", type=int, default=1,
                    help="replay each step as a CUDA graph (the multigrid solve then runs one kernel per pass)")
    ap.add_argument("--warm-start", type=int, default=1, choices=[0, 1],
                    help="multigrid solve from the extrapolated previous pressures (1) or from zero (0)")
    ap.add_argument("--split", type=int, default=-1, choices=[-1, 0, 1],
                    help="multigrid schedule: 1 one kernel per pass (host-paced outside graphs), "
                         "0 one persistent kernel, -1 split in graphs only")
    args = ap.parse_args()
    if args.impl == "reference":
        reference_arm(args)
        return
    if args.workload in ("serving", "batch"):
        serving_arm(args)
        return
    if args.workload in ("batch256", "serving_c5", "lbm_c4"):
        import torch
        torch.cuda.set_device(0)
        if args.workload == "batch256":
            rep = run_batch256(args.max_steps if args.max_steps != 40 else 500)
            value, unit = rep["batched"]["room_solves_per_s"], "room-solves/s"
        elif args.workload == "serving_c5":
            rep = run_serving_c5(args.requests, args.max_steps, args.tol)
            value, unit = rep["streams"]["room_solves_per_s"], "room-solves/s"
        else:
            rep = run_lbm_c4(args.steps)
            value, unit = rep["fp32"]["lattice_cell_steps_per_s"], "lattice-cell-steps/s"
        print(json.dumps({"metric": METRIC, "value": value, "unit": unit, "n_gpus": 1, "dtype": "f32/f64",
                          "data": "synthetic", "higher_is_better": True, "config": {"workload": args.workload},
                          args.workload: rep}))
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as td
        torch.cuda.set_device(local)
        td.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = td
    else:
        torch.cuda.set_device(0)
    res = run_ours(args, rank, world, dist)
    if rank == 0:
        kind, cfg, room, params = make_workload(args.workload, args.precision, args.grid)
        cb = None
        if not args.no_cpu_baseline:
            cb = cpu_reference(kind, room, params)
        dtype = {"fp64": "f64", "mixed": "f32/f64", "fp32": "f32", "fp16": "f16/f32"}.get(args.precision, args.precision)
        extra_blocks = {}
        if not args.no_serving and args.workload == "large_thermal" and world == 1:
            # the other benchmark configurations, each a bounded sample
            if kind == "fluid" and args.precision != "fp64":
                pf = run_plain_fp64(args)
                if "value" in pf:
                    pf["headline_over_plain_fp64"] = res["value"] / pf["value"]
                extra_blocks["plain_fp64_same_room"] = pf
            extra_blocks["serving"] = run_serving_c5(96, 200, 1e-4)
            extra_blocks["serving_reference_tol"] = run_serving_c5(48, 2000, 1.0, max_cells=600_000,
                                                                   engines=("streams",))
            extra_blocks["batch256"] = run_batch256()
            extra_blocks["lbm_c4"] = run_lbm_c4()
        line = {"metric": METRIC, "value": res["value"], "unit": "cell-steps/s", "n_gpus": world,
                "steps": res["steps"], "warmup": args.warmup, "ms_per_step": res["ms"] / max(1, res["steps"]),
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
                "data": "synthetic", "config": config_of(args, room, kind, params),
                "roofline": res["roofline"], "cpu_baseline": cb, "e2e": res["e2e"],
                "gpu_launches": res["launches"], "clocks": res["clocks"], "detail": res["extra"]}
        line.update(extra_blocks)
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
