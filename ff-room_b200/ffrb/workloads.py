"""Synthetic room workloads (seeded), shaped like the benchmark configurations.

Every builder returns ``SceneConfig`` objects (plus solver parameters where
the configuration fixes them), built only from numpy's ``default_rng`` with
the seeds recorded here, so the oracle and the GPU see identical rooms.

* ``basic_room``     5x4x2.5 m on 25x20x12, one fan, one box (the ff-room
                     example scene, examples/basic_room.yaml).
* ``large_thermal``  10x8x3 m on 320x256x96, two facing fans, Boussinesq
                     buoyancy, heated floor / cooled ceiling patches, four
                     random boxes (seed 2).
* ``batch_rooms``    256 uneven rooms, dims U{32..128}, 1-3 fans, 0-5 boxes
                     (seed 7).
* ``lbm_room``       384x320x128 lattice, fan inlet at lattice speed 0.05,
                     six random boxes (seed 4).
* ``serving_stream`` Poisson arrivals at 200/s for 60 s, log-uniform cell
                     counts from 24^3 to 256x256x96 (seed 11).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional, Tuple

import numpy as np

from .params import FluidParams
from .scene import (FanConfig, HeatPatchConfig, ObstacleConfig, RoomConfig, SceneConfig,
                    SolverConfig)

KELVIN = 273.15


def basic_room(advection: str = "upwind", steps: int = 500, tol: float = 1e-4) -> SceneConfig:
    """The ff-room example scene with the benchmark's tolerances."""
    return SceneConfig(
        room=RoomConfig(size=(5.0, 4.0, 2.5), grid=(25, 20, 12)),
        fans=[FanConfig(position=(0.5, 2.0, 1.2), direction=(0.0, 0.0), velocity=3.0, radius=0.15)],
        obstacles=[ObstacleConfig(bbox_min=(2.0, 0.5, 0.0), bbox_max=(3.0, 1.8, 0.9))],
        solver=SolverConfig(dt=0.01, max_steps=steps, convergence_tol=tol, rho=1.2, nu=1.5e-5,
                            poisson_max_iter=1000, poisson_tol=1e-6, advection=advection),
        metadata={"name": "basic_room"},
    )


def _random_boxes(rng, n: int, size: Tuple[float, float, float], side: Tuple[float, float],
                  on_floor: bool = True) -> List[ObstacleConfig]:
    out = []
    for b in range(n):
        sx, sy, sz = rng.uniform(side[0], side[1], 3)
        x0 = rng.uniform(0.0, max(1e-9, size[0] - sx))
        y0 = rng.uniform(0.0, max(1e-9, size[1] - sy))
        z0 = 0.0 if on_floor else rng.uniform(0.0, max(1e-9, size[2] - sz))
        sz = min(sz, size[2] * 0.8)
        out.append(ObstacleConfig(bbox_min=(float(x0), float(y0), float(z0)),
                                  bbox_max=(float(x0 + sx), float(y0 + sy), float(z0 + sz)),
                                  name=f"box{b}"))
    return out


def large_thermal(grid=(320, 256, 96), seed: int = 2) -> Tuple[SceneConfig, FluidParams]:
    """Single large room with thermal buoyancy.

    beta = 3.4e-3 1/K and kappa = 2.1e-5 m^2/s are set directly
    (k_thermal = kappa * rho * cp); T0 = 300 K, floor patch 305 K over
    x in [3, 7] m, y in [2, 6] m, ceiling patch 298 K over the same extent.
    dt = 0.005 s, multigrid-preconditioned CG to 1e-8.
    """
    rng = np.random.default_rng(seed)
    size = (10.0, 8.0, 3.0)
    cfg = SceneConfig(
        room=RoomConfig(size=size, grid=tuple(grid)),
        fans=[FanConfig(position=(0.5, 4.0, 1.2), direction=(0.0, 0.0), velocity=3.0, radius=0.2, name="west"),
              FanConfig(position=(9.5, 4.0, 1.2), direction=(180.0, 0.0), velocity=3.0, radius=0.2, name="east")],
        obstacles=_random_boxes(rng, 4, size, (0.3, 1.5)),
        heat_patches=[HeatPatchConfig("floor", (3.0, 7.0), (2.0, 6.0), 305.0 - KELVIN),
                      HeatPatchConfig("ceiling", (3.0, 7.0), (2.0, 6.0), 298.0 - KELVIN)],
        solver=SolverConfig(dt=0.005, max_steps=2000, convergence_tol=1e-4, poisson_max_iter=20000,
                            poisson_tol=1e-8, buoyancy=True, T_initial=300.0 - KELVIN,
                            poisson_method="multigrid", precision="mixed"),
        metadata={"name": "large_thermal", "seed": seed},
    )
    rho, cp = 1.2, 1005.0
    params = FluidParams(rho=rho, nu=1.5e-5, dt=0.005, max_steps=2000, convergence_tol=1e-4,
                         poisson_max_iter=20000, poisson_tol=1e-8, advection=0, thermal=True,
                         T_initial=300.0 - KELVIN, T_target=1e30, buoyancy=True, g_accel=9.81,
                         beta=3.4e-3, k_thermal=2.1e-5 * rho * cp, cp=cp,
                         precision="mixed", poisson="mgpcg")
    return cfg, params


def _wall_fan(rng, size, name: str) -> FanConfig:
    """A fan one cell-layer in from a random wall, blowing into the room
    along the wall normal."""
    wall = int(rng.integers(0, 4))          # west, east, south, north
    speed = float(rng.uniform(1.0, 5.0))
    rad = float(rng.uniform(0.1, 0.3))
    z = float(rng.uniform(0.3, 0.8) * size[2])
    inset = 0.05
    if wall == 0:
        pos, az = (inset * size[0], float(rng.uniform(0.2, 0.8) * size[1]), z), 0.0
    elif wall == 1:
        pos, az = ((1 - inset) * size[0], float(rng.uniform(0.2, 0.8) * size[1]), z), 180.0
    elif wall == 2:
        pos, az = (float(rng.uniform(0.2, 0.8) * size[0]), inset * size[1], z), 90.0
    else:
        pos, az = (float(rng.uniform(0.2, 0.8) * size[0]), (1 - inset) * size[1], z), 270.0
    return FanConfig(position=pos, direction=(az, 0.0), velocity=speed, radius=rad, name=name)


def room_dt(cfg: SceneConfig, cfl: float = 0.5) -> float:
    """dt = cfl * min(h) / max fan speed (the batched rooms' CFL rule)."""
    h = min(s / n for s, n in zip(cfg.room.size, cfg.room.grid))
    umax = max([f.velocity for f in cfg.fans] or [1.0])
    return cfl * h / umax


def batch_rooms(n_rooms: int = 256, seed: int = 7, dims=(32, 128), steps: int = 500) -> List[SceneConfig]:
    rng = np.random.default_rng(seed)
    rooms = []
    for r in range(n_rooms):
        grid = tuple(int(g) for g in rng.integers(dims[0], dims[1] + 1, 3))
        size = tuple(float(s) for s in rng.uniform(3.0, 12.0, 3))
        fans = [_wall_fan(rng, size, f"fan{f}") for f in range(int(rng.integers(1, 4)))]
        obs = _random_boxes(rng, int(rng.integers(0, 6)), size, (0.3, 1.5))
        cfg = SceneConfig(room=RoomConfig(size=size, grid=grid), fans=fans, obstacles=obs,
                          solver=SolverConfig(max_steps=steps, convergence_tol=1e-4, poisson_tol=1e-6,
                                              poisson_max_iter=2000, precision="mixed",
                                              poisson_method="multigrid"),
                          metadata={"name": f"batch{r}", "seed": seed})
        cfg.solver.dt = room_dt(cfg)
        rooms.append(cfg)
    return rooms


def lbm_room(grid=(384, 320, 128), seed: int = 4, u_lat: float = 0.05) -> Tuple[SceneConfig, float, float]:
    """D3Q19 room: 12x10x4 m at h = 0.03125 m; a 3 m/s fan inlet at lattice
    speed u_lat fixes dt = u_lat * h / 3.  Returns (cfg, tau, dt)."""
    rng = np.random.default_rng(seed)
    h = 12.0 / grid[0]
    size = (grid[0] * h, grid[1] * h, grid[2] * h)
    speed = 3.0
    dt = u_lat * h / speed
    cfg = SceneConfig(
        room=RoomConfig(size=size, grid=tuple(grid)),
        fans=[FanConfig(position=(0.5, size[1] / 2, size[2] * 0.4), direction=(0.0, 0.0), velocity=speed,
                        radius=0.3, name="inlet")],
        obstacles=_random_boxes(rng, 6, size, (0.3, 1.5)),
        solver=SolverConfig(method="lbm", tau=0.52, dt=dt, max_steps=10000, convergence_tol=1e-4),
        metadata={"name": "lbm_room", "seed": seed},
    )
    return cfg, 0.52, dt


@dataclass
class Request:
    t_arrival: float
    cfg: SceneConfig
    params: FluidParams


def serving_stream(rate: float = 200.0, duration: float = 60.0, seed: int = 11,
                   cells=(24 ** 3, 256 * 256 * 96), max_steps: int = 500) -> List[Request]:
    """Poisson arrivals; total cell count log-uniform; the room shape takes
    its aspect from random sizes (x, y in [3, 12] m, z in [2.4, 4] m) and
    h = cbrt(volume / cells)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= duration:
            break
        n = float(np.exp(rng.uniform(math.log(cells[0]), math.log(cells[1]))))
        size = (float(rng.uniform(3.0, 12.0)), float(rng.uniform(3.0, 12.0)), float(rng.uniform(2.4, 4.0)))
        h = (size[0] * size[1] * size[2] / n) ** (1.0 / 3.0)
        grid = tuple(max(8, int(round(s / h))) for s in size)
        fans = [_wall_fan(rng, size, f"fan{f}") for f in range(int(rng.integers(1, 4)))]
        obs = _random_boxes(rng, int(rng.integers(0, 6)), size, (0.3, 1.5))
        heated = bool(rng.random() < 0.5)
        cfg = SceneConfig(room=RoomConfig(size=size, grid=grid), fans=fans, obstacles=obs,
                          solver=SolverConfig(max_steps=max_steps, convergence_tol=1e-4, poisson_tol=1e-6,
                                              poisson_max_iter=2000, buoyancy=heated,
                                              precision="mixed", poisson_method="multigrid"),
                          metadata={"name": f"req{len(out)}", "seed": seed})
        if heated:
            cfg.heat_patches = [HeatPatchConfig("floor", (0.3 * size[0], 0.7 * size[0]),
                                                (0.3 * size[1], 0.7 * size[1]), cfg.solver.T_initial + 5.0)]
        cfg.solver.dt = room_dt(cfg)
        from .params import params_from_scene
        out.append(Request(t, cfg, params_from_scene(cfg)))
    return out
