"""Fan-placement sweeps for "time to cool".

ff-room's cooling scenes (examples/summer_cooling.yaml) stop a run when the
mean room temperature reaches ``solver.T_target`` (FluidSolver.cpp:538-547:
with T_target below T_initial the run converges on the first step whose
T_mean <= T_target).  Comparing fan positions and directions means running
one such scene per placement; here every placement is one request to the
continuous-batching server, so all placements advance together (one launch
per stage for the whole set) and each leaves the batch on its own
convergence step.

The time to cool of a placement is ``steps * dt`` seconds of simulated time
when it reached the target within the step cap, else ``None``.
"""
from __future__ import annotations

import copy
from dataclasses import dataclass
from typing import Iterable, List, Optional, Sequence, Tuple

from .params import params_from_scene
from .scene import SceneConfig, build_room
from .serve import Request, Server, estimate_bytes


@dataclass
class Placement:
    """One fan setting of a sweep: the index of the fan in the base scene and
    the position / direction / velocity it gets (None keeps the base's)."""
    label: str
    fan: int = 0
    position: Optional[Tuple[float, float, float]] = None
    direction: Optional[Tuple[float, float]] = None
    velocity: Optional[float] = None


@dataclass
class SweepResult:
    label: str
    steps: int
    reached: bool
    time_to_target_s: Optional[float]
    T_mean: float
    latency_s: float


def placement_grid(positions: Iterable[Tuple[float, float, float]], directions: Iterable[Tuple[float, float]],
                   fan: int = 0) -> List[Placement]:
    """Every position with every direction, labelled ``p<i>_d<j>``."""
    dirs = list(directions)
    return [Placement(f"p{i}_d{j}", fan, tuple(p), tuple(d)) for i, p in enumerate(positions)
            for j, d in enumerate(dirs)]


def variant(base: SceneConfig, pl: Placement, T_target: Optional[float] = None,
            max_steps: Optional[int] = None) -> SceneConfig:
    """The base scene with one fan moved / turned (a deep copy)."""
    cfg = copy.deepcopy(base)
    f = cfg.fans[pl.fan]
    if pl.position is not None:
        f.position = tuple(pl.position)
    if pl.direction is not None:
        f.direction = tuple(pl.direction)
    if pl.velocity is not None:
        f.velocity = float(pl.velocity)
    if T_target is not None:
        cfg.solver.T_target = float(T_target)
    if max_steps is not None:
        cfg.solver.max_steps = int(max_steps)
    cfg.metadata = dict(cfg.metadata or {}, placement=pl.label)
    return cfg


def requests(base: SceneConfig, placements: Sequence[Placement], T_target: Optional[float] = None,
             max_steps: Optional[int] = None, precision: str = "mixed", poisson: str = "mgpcg") -> List[Request]:
    """One server request per placement, all arriving at t=0.  A scene
    without a temperature target (solver.T_target unset and none given)
    is rejected: it would run on the velocity test instead."""
    out = []
    for i, pl in enumerate(placements):
        cfg = variant(base, pl, T_target, max_steps)
        if cfg.solver.T_target is None:
            raise ValueError("a cooling sweep needs solver.T_target")
        p = params_from_scene(cfg).with_(precision=precision, poisson=poisson)
        out.append(Request(i, 0.0, build_room(cfg), p, int(cfg.solver.max_steps)))
    return out


def cooling_sweep(base: SceneConfig, placements: Sequence[Placement], T_target: Optional[float] = None,
                  max_steps: Optional[int] = None, server: Optional[Server] = None, precision: str = "mixed",
                  poisson: str = "mgpcg") -> List[SweepResult]:
    """Runs every placement to its target (or the step cap) on the server
    (by default a batched one holding every placement at once; the plain CG
    solver has no batched form, so poisson="cg" runs one stream per room)
    and returns the results fastest first (placements that never reached
    the target last, in input order)."""
    reqs = requests(base, placements, T_target, max_steps, precision, poisson)
    if server is None:
        need = sum(estimate_bytes(r.room, r.params) for r in reqs)
        server = Server(mem_budget=need, max_active=len(reqs), batched=(poisson == "mgpcg"))
    outs = {o.rid: o for o in server.run(reqs, realtime=False)}
    res = []
    for r, pl in zip(reqs, placements):
        o = outs[r.rid]
        res.append(SweepResult(pl.label, o.steps, o.converged, o.steps * r.params.dt if o.converged else None,
                               o.T_mean, o.latency))
    order = sorted(range(len(res)), key=lambda i: (not res[i].reached, res[i].steps if res[i].reached else 0, i))
    return [res[i] for i in order]
