"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a container that has the reference sources, after
``make -C oracle REF=<reference checkout>`` has built oracle/_ref:

    python tests/golden/make_golden.py --ref <reference checkout>

For every case the reference's own Python ``Scene`` builds the masks on the
reference's compiled ``_ffroom_core`` (oracle/_ref), the reference
``FluidSolver`` / ``LBMSolver`` runs N steps through its public API with a
per-step callback, and the fields, the StepResult history and the cell
types are stored.  The C driver (oracle/_ref/libffr_refdriver.so, the same
reference sources) adds the CG iteration count of every step and is checked
to agree with the module bit for bit.  Cases with a fixed-temperature patch
(not expressible through the reference Scene) come from the driver alone,
which applies the patch after each step as a per-step callback would.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "ff-room_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from ffrb import workloads  # noqa: E402
from ffrb.params import FluidParams, params_from_scene  # noqa: E402
from ffrb.scene import (FanConfig, ObstacleConfig, OpeningConfig, RoomConfig, SceneConfig,  # noqa: E402
                        SolverConfig, build_room)


def cases():
    """(name, SceneConfig, nsteps, extra) — extra may carry FluidParams."""
    out = []
    out.append(("c1_upwind_10", workloads.basic_room("upwind"), 10, {}))
    out.append(("c1_quick_10", workloads.basic_room("quick"), 10, {}))
    out.append(("c1_laxw_10", workloads.basic_room("lax_wendroff"), 10, {}))
    out.append(("c1_upwind_500", workloads.basic_room("upwind"), 500, {}))
    two = SceneConfig.load_yaml(os.path.join(REF, "examples", "two_fans.yaml"))
    out.append(("two_fans_10", two, 10, {}))
    cool = SceneConfig.load_yaml(os.path.join(REF, "examples", "summer_cooling.yaml"))
    out.append(("summer_cooling_10", cool, 10, {}))
    cool_q = SceneConfig.load_yaml(os.path.join(REF, "examples", "summer_cooling.yaml"))
    cool_q.solver.advection = "quick"
    out.append(("summer_cooling_quick_10", cool_q, 10, {}))
    # odd dims, a fan on the west wall inside an obstacle, QUICK
    edge = SceneConfig(room=RoomConfig(size=(2.6, 1.8, 1.4), grid=(13, 9, 7)),
                       fans=[FanConfig(position=(0.05, 0.9, 0.7), direction=(0.0, 0.0), velocity=2.0, radius=0.25)],
                       obstacles=[ObstacleConfig(bbox_min=(0.0, 0.6, 0.4), bbox_max=(0.4, 1.2, 1.0)),
                                  ObstacleConfig(bbox_min=(1.2, 0.0, 0.0), bbox_max=(1.8, 0.8, 0.6))],
                       solver=SolverConfig(dt=0.01, poisson_tol=1e-8, advection="quick"))
    out.append(("edge_odd_quick_10", edge, 10, {}))
    # oblique fan (3 velocity components), no obstacle, stretched grid
    obl = SceneConfig(room=RoomConfig(size=(4.0, 3.0, 2.5), grid=(16, 12, 10), stretch=1.05),
                      fans=[FanConfig(position=(0.4, 1.5, 1.0), direction=(30.0, 20.0), velocity=1.5, radius=0.3)],
                      solver=SolverConfig(dt=0.005, poisson_tol=1e-8))
    out.append(("oblique_stretch_10", obl, 10, {}))
    # fan blowing up: outflow on the ceiling
    up = SceneConfig(room=RoomConfig(size=(3.0, 3.0, 3.0), grid=(12, 12, 12)),
                     fans=[FanConfig(position=(1.5, 1.5, 0.2), direction=(0.0, 90.0), velocity=2.0, radius=0.3)],
                     obstacles=[ObstacleConfig(bbox_min=(0.2, 0.2, 0.0), bbox_max=(0.9, 0.9, 1.5))],
                     solver=SolverConfig(dt=0.01, poisson_tol=1e-8, advection="lax_wendroff"))
    out.append(("updraft_laxw_10", up, 10, {}))
    # openings on two walls + a fan, QUICK, with buoyancy
    vent = SceneConfig(room=RoomConfig(size=(4.0, 3.0, 2.5), grid=(16, 12, 10)),
                       fans=[FanConfig(position=(2.0, 2.6, 0.9), direction=(270.0, 0.0), velocity=2.0, radius=0.2)],
                       openings=[OpeningConfig(wall="north", center=(2.0, 1.2), size=(0.8, 1.0), T_outside=18.0),
                                 OpeningConfig(wall="west", center=(1.5, 1.0), size=(0.6, 1.6))],
                       solver=SolverConfig(dt=0.02, poisson_tol=1e-8, T_initial=28.0, T_outside=24.0,
                                           buoyancy=True, advection="quick"))
    out.append(("vent_quick_10", vent, 10, {}))
    # heat patches (extension), small version of the large thermal room
    cfg, prm = workloads.large_thermal(grid=(40, 32, 12))
    prm = prm.with_(precision="fp64", poisson="cg", poisson_tol=1e-8, poisson_max_iter=5000)
    out.append(("thermal_small_10", cfg, 10, {"params": prm, "driver_only": True}))
    # the large thermal room scaled down to 80x64x24 (same room, fans, boxes,
    # heat patches, dt and pressure tolerance 1e-8) over its full 2000 steps;
    # generated with the reference's OpenMP loops on (its parallel
    # reductions), the same method
    cfg, prm = workloads.large_thermal(grid=(80, 64, 24))
    prm = prm.with_(precision="fp64", poisson="cg", poisson_tol=1e-8, poisson_max_iter=20000, use_openmp=True)
    out.append(("thermal_80x64x24_2000", cfg, 2000, {"params": prm, "driver_only": True}))
    # LBM
    out.append(("lbm_basic_10", SceneConfig.load_yaml(os.path.join(REF, "examples", "basic_room.yaml")), 10,
                {"lbm": (0.8, 0.01, 1.0)}))
    lcfg, tau, dt = workloads.lbm_room(grid=(24, 20, 12), seed=4)
    out.append(("lbm_small_20", lcfg, 20, {"lbm": (0.6, dt, 1e-4)}))
    lv = SceneConfig(room=RoomConfig(size=(3.0, 2.0, 2.0), grid=(15, 10, 10)),
                     fans=[FanConfig(position=(1.5, 1.8, 1.0), direction=(270.0, 0.0), velocity=2.0, radius=0.3)],
                     obstacles=[ObstacleConfig(bbox_min=(0.5, 0.5, 0.0), bbox_max=(1.0, 1.0, 1.0))],
                     openings=[OpeningConfig(wall="south", center=(1.5, 1.0), size=(1.0, 1.0)),
                               OpeningConfig(wall="east", center=(1.0, 1.0), size=(0.8, 0.8))],
                     solver=SolverConfig(dt=0.01))
    out.append(("lbm_openings_10", lv, 10, {"lbm": (0.6, 0.01, 1e-4)}))
    return out


def ref_config(cfg: SceneConfig):
    d = cfg.to_dict()
    d.pop("heat_patches", None)
    d["solver"].pop("precision", None)
    return RefSceneConfig.from_dict(d)


def run_case(name, cfg, nsteps, extra, core, drv, Oracle):
    room = build_room(cfg)
    meta = {"name": name, "config": cfg.to_dict(), "nsteps": nsteps}
    rec = {}
    if "lbm" in extra:
        tau, dt, tol = extra["lbm"]
        rs = RefScene(ref_config(cfg))
        ct = rs.grid.cell_type_shaped().reshape(-1)
        assert np.array_equal(ct, room.cell_type), f"{name}: mask mismatch"
        solver = core.LBMSolver(rs.grid, rs.bm, tau, nsteps, tol, dt)
        hist = []
        for _ in range(nsteps):
            hist.append(solver.step())
        fields = {k: np.array(getattr(rs.grid, k + "_shaped")()).reshape(-1) for k in "uvwp"}
        fd, recs = drv.lbm_run(room, tau, dt, tol, nsteps)
        for k in "uvwp":
            assert np.array_equal(fd[k], fields[k]), f"{name}: driver/module differ in {k}"
        meta["lbm"] = {"tau": tau, "dt": dt, "tol": tol}
        rec["cg_iterations"] = np.zeros(nsteps, np.int32)
    elif extra.get("driver_only"):
        prm = extra["params"]
        fields, ct, recs = drv.fluid_run(room, prm, nsteps)
        assert np.array_equal(ct, room.cell_type)
        hist = recs
        meta["params"] = prm.__dict__
        rec["cg_iterations"] = np.array([r.cg_iterations for r in recs], np.int32)
    else:
        rcfg = ref_config(cfg)
        rs = RefScene(rcfg)
        ct = rs.grid.cell_type_shaped().reshape(-1)
        assert np.array_equal(ct, room.cell_type), f"{name}: mask mismatch"
        # SolverBridge.run's parameter mapping (solver_bridge.py:108-127)
        sc = rcfg.solver
        params = core.FluidSolverParams()
        params.rho, params.nu, params.dt = sc.rho, sc.nu, sc.dt
        params.max_steps, params.convergence_tol = sc.max_steps, sc.convergence_tol
        params.poisson.max_iter, params.poisson.tol = sc.poisson_max_iter, sc.poisson_tol
        params.thermal = bool(rcfg.openings) or sc.buoyancy or (sc.T_target is not None)
        params.T_initial = sc.T_initial
        params.T_target = sc.T_target if sc.T_target is not None else 1e30
        params.buoyancy, params.k_thermal, params.cp = sc.buoyancy, sc.k_thermal, sc.cp
        params.beta = 1.0 / (sc.T_initial + 273.15)
        ref_bridge._apply_solver_flags(sc, params, core)
        solver = core.FluidSolver(rs.grid, rs.bm, params)
        hist = []
        for _ in range(nsteps):
            hist.append(solver.step())
        fields = {k: np.array(getattr(rs.grid, k + "_shaped")()).reshape(-1) for k in "uvwpT"}
        prm = params_from_scene(cfg)
        fd, _, recs = drv.fluid_run(room, prm, nsteps)
        for k in "uvwpT":
            assert np.array_equal(fd[k], fields[k]), f"{name}: driver/module differ in {k}"
        for h, r in zip(hist, recs):
            assert h.velocity_change == r.velocity_change and h.pressure_residual == r.pressure_residual
        meta["params"] = prm.__dict__
        rec["cg_iterations"] = np.array([r.cg_iterations for r in recs], np.int32)
    for k in ("step", "velocity_change", "pressure_residual", "divergence_max", "converged", "T_mean"):
        rec[k] = np.array([getattr(h, k) for h in hist])
    if "lbm" not in extra and not extra.get("driver_only"):
        pass
    arrays = {"cell_type": room.cell_type}
    arrays.update({"f_" + k: v for k, v in fields.items()})
    arrays.update({"h_" + k: v for k, v in rec.items()})
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    # the restated oracle must agree before the fixture is accepted
    return path


SWEEP_CAP = 80


def sweep_placements():
    """Two fan positions near the window × the two directions the scene's
    notes compare, plus a slow fan that should not reach the target."""
    from ffrb.sweep import Placement, placement_grid
    pls = placement_grid([(3.0, 3.8, 0.9), (1.0, 3.8, 0.9)], [(270.0, 0.0), (90.0, 0.0)])
    pls.append(Placement("slow", 0, (3.0, 3.8, 0.9), (270.0, 0.0), 0.5))
    return pls


def cooling_sweep(drv):
    """tests/golden/cooling_sweep.json: time to cool of summer_cooling.yaml
    per fan placement, from the reference's own SolverBridge.run (which
    stops on FluidSolver's T_target test).  The target is chosen from the
    reference's uncapped temperature histories (the C driver) so that no
    step's T_mean lies within reach of mixed-precision rounding of it, with
    some placements reaching it inside the cap and at least one not."""
    from ffrb.sweep import variant
    base = SceneConfig.load_yaml(os.path.join(REF, "examples", "summer_cooling.yaml"))
    pls = sweep_placements()
    hist = []
    for pl in pls:
        cfg = variant(base, pl)
        cfg.solver.T_target = None
        _, _, recs = drv.fluid_run(build_room(cfg), params_from_scene(cfg), SWEEP_CAP)
        hist.append(np.array([r.T_mean for r in recs]))
    best = None
    for tgt in np.round(np.arange(31.950, 31.995, 0.0005), 4):
        reached = [bool(np.any(h <= tgt)) for h in hist]
        if sum(reached) < 3 or all(reached):
            continue
        margin = min(float(np.min(np.abs(h - tgt))) for h in hist)
        if best is None or margin > best[1]:
            best = (float(tgt), margin)
    tgt, margin = best
    out = {"base": base.to_dict(), "T_target": tgt, "cap": SWEEP_CAP, "margin": margin, "placements": []}
    for pl, h in zip(pls, hist):
        cfg = variant(base, pl, tgt, SWEEP_CAP)
        seen = []
        res = ref_bridge.SolverBridge(ref_config(cfg)).run(
            progress_callback=lambda s, vc, dm, tm: seen.append(tm), print_interval=0)
        k = res.steps
        assert np.array_equal(np.array(seen), h[:k]), f"{pl.label}: bridge and driver histories differ"
        out["placements"].append({"label": pl.label, "fan": pl.fan, "position": list(pl.position),
                                  "direction": list(pl.direction), "velocity": pl.velocity,
                                  "steps": int(k), "reached": bool(res.converged),
                                  "T_mean": [float(x) for x in seen]})
    with open(os.path.join(HERE, "cooling_sweep.json"), "w") as fh:
        json.dump(out, fh, indent=1)


def bridge_traces(core):
    """tests/golden/bridge_*.json/.npz: every call the reference's own
    SolverBridge.run / run_animated make into `_ffroom_core`, recorded on the
    reference's compiled module (tests/bridge_trace.py), for the GPU test
    that replays them on this repository's drop-in module.  A progress
    callback reads each step's (step, vel_change, div_max, T_mean), as the
    documented callback does."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from bridge_trace import Recorder

    def progress(step, vc, dm, tm):
        pass

    def basic():
        return RefSceneConfig.load_yaml(os.path.join(REF, "examples", "basic_room.yaml"))

    def cooling():
        c = RefSceneConfig.load_yaml(os.path.join(REF, "examples", "summer_cooling.yaml"))
        c.solver.max_steps = 120          # a bounded prefix of its 5000 steps
        return c

    def basic_lbm():
        c = basic()
        c.solver.method = "lbm"
        return c

    jobs = [("bridge_basic_room_run", basic, "run"), ("bridge_basic_room_animated", basic, "animated"),
            ("bridge_summer_cooling_run", cooling, "run"), ("bridge_basic_room_lbm_run", basic_lbm, "run")]
    for name, make, how in jobs:
        rec = Recorder(core)
        sys.modules["_ffroom_core"] = rec
        try:
            bridge = ref_bridge.SolverBridge(make())
            if how == "run":
                res = bridge.run(progress_callback=progress, print_interval=0)
            else:
                res, snaps = bridge.run_animated(save_every=100, progress_callback=progress, print_interval=0)
        finally:
            sys.modules["_ffroom_core"] = core
        rec.save(os.path.join(HERE, name + ".json"), os.path.join(HERE, name + ".npz"))
        print(name, "ops", len(rec.ops), "arrays", len(rec.arrays), "steps", res.steps, "converged", res.converged)


def mask_hashes():
    """sha256 of the masks of the synthetic workloads, built by the
    reference Scene, so that CPU tests can pin the restated scene builder
    without the reference present."""
    out = {}
    cfg, _ = workloads.large_thermal()
    out["large_thermal"] = cfg
    lcfg, _, _ = workloads.lbm_room()
    out["lbm_room"] = lcfg
    for i, c in enumerate(workloads.batch_rooms()[:16]):
        out[f"batch{i}"] = c
    for i, rq in enumerate(workloads.serving_stream()[:16]):
        out[f"serve{i}"] = rq.cfg
    hashes = {}
    for name, c in out.items():
        rs = RefScene(ref_config(c))
        ct = np.ascontiguousarray(rs.grid.cell_type_shaped().reshape(-1))
        mine = build_room(c).cell_type
        assert np.array_equal(ct, mine), f"mask mismatch for {name}"
        hashes[name] = {"sha256": hashlib.sha256(ct.tobytes()).hexdigest(),
                        "counts": np.bincount(ct, minlength=4).tolist(), "grid": list(c.room.grid)}
    with open(os.path.join(HERE, "mask_hashes.json"), "w") as fh:
        json.dump(hashes, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", required=True, help="the reference checkout (its python/ and examples/)")
    ap.add_argument("--only", default="", help="comma-separated case names (also cooling_sweep, mask_hashes)")
    args = ap.parse_args()
    REF = args.ref
    sys.path.insert(0, os.path.join(ROOT, "oracle", "_ref"))
    sys.path.insert(0, os.path.join(REF, "python"))
    import _ffroom_core as core  # the reference module built by oracle/Makefile
    assert not hasattr(core, "__backend__"), "picked up the B200 module instead of the reference"
    from ff_room.config import SceneConfig as RefSceneConfig  # noqa: E402
    from ff_room.scene import Scene as RefScene  # noqa: E402
    import ff_room.solver_bridge as ref_bridge  # noqa: E402
    from oracle import Oracle, RefDriver  # noqa: E402
    drv = RefDriver()
    only = set(args.only.split(",")) if args.only else None
    for name, cfg, n, extra in cases():
        if only is not None and name not in only:
            continue
        print("case", name, flush=True)
        run_case(name, cfg, n, extra, core, drv, Oracle)
    if only is None or "cooling_sweep" in only:
        cooling_sweep(drv)
    if only is None or "mask_hashes" in only:
        mask_hashes()
    if only is None or "bridge_traces" in only:
        bridge_traces(core)
    print("done")
