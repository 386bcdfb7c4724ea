"""Scene description → room masks and boundary lists.

Host-side mirror of the caller of the solver boundary:
  * ``SceneConfig`` and friends restate ff-room's configuration dataclasses
    (python/ff_room/config.py:14-204) so that the same YAML files load here;
  * ``build_room`` restates ``Scene._build`` (python/ff_room/scene.py:72-231)
    and the mask writers of ``BoundaryManager`` (cpp/src/core/
    BoundaryManager.cpp:6-44,132-135) in numpy, producing a ``RoomSpec``;
  * ``build_on_core`` replays the same construction through any module that
    exposes the ``_ffroom_core`` class surface (this package's GPU module or
    the reference's), exactly as ``Scene._build`` does.

The cell mapping (``int(x / L * N)``), the fan patch (one cell thick on the
dominant axis, transverse ``int((c ± r) / L * N)`` clamped), the fan velocity
(the unsnapped unit vector times the speed), the auto-outflow wall and the
marking order (obstacles, fans, openings, auto-outflow) follow the reference
so that masks are bit-identical.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, asdict, is_dataclass
from typing import List, Optional, Sequence, Tuple

import numpy as np

FLUID, SOLID, INFLOW, OUTFLOW = 0, 1, 2, 3


# --------------------------------------------------------------- config

@dataclass
class RoomConfig:
    """Room box and grid (config.py:14-21)."""
    size: Tuple[float, float, float] = (5.0, 4.0, 2.5)
    grid: Tuple[int, int, int] = (25, 20, 12)
    stretch: float = 1.0


@dataclass
class FanConfig:
    """Fan as a square inflow patch (config.py:24-59)."""
    position: Tuple[float, float, float] = (0.5, 2.0, 1.0)
    direction: Tuple[float, float] = (0.0, 0.0)
    velocity: float = 3.0
    radius: float = 0.15
    name: str = "fan0"

    def direction_vector(self) -> Tuple[float, float, float]:
        az = math.radians(self.direction[0])
        el = math.radians(self.direction[1])
        return (math.cos(el) * math.cos(az), math.cos(el) * math.sin(az), math.sin(el))

    def snapped_axis(self) -> int:
        vec = self.direction_vector()
        return int(max(range(3), key=lambda a: abs(vec[a])))

    def snapped_sign(self) -> float:
        vec = self.direction_vector()
        return 1.0 if vec[self.snapped_axis()] >= 0 else -1.0


@dataclass
class ObstacleConfig:
    """Axis-aligned solid box (config.py:62-67)."""
    bbox_min: Tuple[float, float, float] = (2.0, 1.5, 0.0)
    bbox_max: Tuple[float, float, float] = (2.5, 2.5, 0.8)
    name: str = "obstacle0"


@dataclass
class OpeningConfig:
    """Window or door (config.py:70-89)."""
    wall: str = "east"
    center: Tuple[float, float] = (2.0, 1.2)
    size: Tuple[float, float] = (0.8, 1.0)
    T_outside: Optional[float] = None
    name: str = "opening0"


@dataclass
class HeatPatchConfig:
    """Fixed-temperature patch on the floor or ceiling layer.

    Not part of ff-room: it realises the heated floor / cooled ceiling of the
    large thermal room workload.  The patch covers the cells of the k=0
    (floor) or k=Nz-1 (ceiling) layer inside ``[x0,x1]x[y0,y1]`` metres and
    holds them at ``T`` (°C) after every step.
    """
    wall: str = "floor"
    x_range: Tuple[float, float] = (0.0, 1.0)
    y_range: Tuple[float, float] = (0.0, 1.0)
    T: float = 20.0


@dataclass
class SolverConfig:
    """Solver options (config.py:92-142) plus ``precision``."""
    dt: float = 0.01
    max_steps: int = 1000
    convergence_tol: float = 1.0
    rho: float = 1.2
    nu: float = 1.5e-5
    poisson_max_iter: int = 1000
    poisson_tol: float = 1e-6
    method: str = "projection"
    tau: float = 0.8
    advection: str = "upwind"
    parallel: bool = False
    poisson_method: str = "cg"
    T_initial: float = 20.0
    T_outside: float = 20.0
    T_target: Optional[float] = None
    buoyancy: bool = False
    k_thermal: float = 0.026
    cp: float = 1005.0
    precision: str = "fp64"


def _tup(v):
    return tuple(v) if isinstance(v, list) else v


@dataclass
class SceneConfig:
    """Complete scene (config.py:145-204), YAML/JSON compatible."""
    room: RoomConfig = field(default_factory=RoomConfig)
    fans: List[FanConfig] = field(default_factory=list)
    obstacles: List[ObstacleConfig] = field(default_factory=list)
    openings: List[OpeningConfig] = field(default_factory=list)
    solver: SolverConfig = field(default_factory=SolverConfig)
    metadata: dict = field(default_factory=dict)
    heat_patches: List[HeatPatchConfig] = field(default_factory=list)

    def to_dict(self) -> dict:
        def cvt(o):
            if is_dataclass(o):
                return {k: cvt(v) for k, v in asdict(o).items()}
            if isinstance(o, (list, tuple)):
                return [cvt(x) for x in o]
            return o
        return cvt(self)

    def to_reference_dict(self) -> dict:
        """The dict ff-room's own SceneConfig.from_dict accepts
        (config.py:172-186): the reference's keys only, with this build's
        extensions kept where its from_dict skips them — the storage
        precision as a top-level ``precision`` (only when not fp64) and
        ``heat_patches`` (only when there are any).  For a scene the
        reference can express, this is exactly the reference's to_dict."""
        d = self.to_dict()
        prec = d["solver"].pop("precision")
        hp = d.pop("heat_patches")
        if hp:
            d["heat_patches"] = hp
        if prec != "fp64":
            d["precision"] = prec
        return d

    @classmethod
    def from_dict(cls, d: dict) -> "SceneConfig":
        solver = SolverConfig(**(d.get("solver", {}) or {}))
        if "precision" in d:
            solver.precision = d["precision"]
        return cls(
            room=RoomConfig(**{k: _tup(v) for k, v in d.get("room", {}).items()}),
            fans=[FanConfig(**{k: _tup(v) for k, v in f.items()}) for f in d.get("fans", []) or []],
            obstacles=[ObstacleConfig(**{k: _tup(v) for k, v in o.items()})
                       for o in d.get("obstacles", []) or []],
            openings=[OpeningConfig(**{k: _tup(v) for k, v in o.items()})
                      for o in d.get("openings", []) or []],
            solver=solver,
            metadata=d.get("metadata", {}) or {},
            heat_patches=[HeatPatchConfig(**{k: _tup(v) for k, v in h.items()})
                          for h in d.get("heat_patches", []) or []],
        )

    @classmethod
    def load_yaml(cls, path: str) -> "SceneConfig":
        import yaml
        with open(path) as fh:
            return cls.from_dict(yaml.safe_load(fh))


# ----------------------------------------------------------------- room

@dataclass
class Fan:
    box: Tuple[int, int, int, int, int, int]
    vel: Tuple[float, float, float]


@dataclass
class Patch:
    """A BoundaryManager outflow entry; ``T_outside`` set for openings."""
    axis: int
    side: int
    a_min: int
    a_max: int
    b_min: int
    b_max: int
    T_outside: Optional[float] = None

    @property
    def is_opening(self) -> bool:
        return self.T_outside is not None


@dataclass
class HeatPatch:
    box: Tuple[int, int, int, int, int, int]
    T: float


@dataclass
class RoomSpec:
    """Everything the solver needs about one room, in reference units."""
    nx: int
    ny: int
    nz: int
    lx: float
    ly: float
    lz: float
    xs: np.ndarray
    ys: np.ndarray
    zs: np.ndarray
    dxv: np.ndarray
    dyv: np.ndarray
    dzv: np.ndarray
    stretched: bool
    cell_type: np.ndarray          # uint8, (nx, ny, nz) flattened k-fastest
    solids: List[Tuple[int, ...]] = field(default_factory=list)
    fans: List[Fan] = field(default_factory=list)
    outflows: List[Patch] = field(default_factory=list)   # insertion order, openings included
    heats: List[HeatPatch] = field(default_factory=list)

    @property
    def n_cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def dx(self) -> float:
        return self.lx / self.nx

    @property
    def openings(self) -> List[Patch]:
        return [p for p in self.outflows if p.is_opening]

    def shapes(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        return {"u": (nx + 1, ny, nz), "v": (nx, ny + 1, nz), "w": (nx, ny, nz + 1),
                "p": (nx, ny, nz), "T": (nx, ny, nz)}


def stretched_faces(n: int, length: float, ratio: float) -> list:
    """Geometric wall-refined face coordinates (scene.py:34-59)."""
    if abs(ratio - 1.0) < 1e-6:
        return [i * length / n for i in range(n + 1)]
    half = n // 2
    first = (length / 2.0) * (ratio - 1.0) / (ratio ** half - 1.0)
    faces = [0.0]
    for i in range(half):
        faces.append(faces[-1] + first * ratio ** i)
    widths = [faces[i + 1] - faces[i] for i in range(half)]
    for wdt in reversed(widths):
        faces.append(faces[-1] + wdt)
    if n % 2 == 1:
        faces.insert(half + 1, (faces[half] + faces[half + 1]) / 2.0)
    scale = length / faces[-1]
    return [x * scale for x in faces]


def empty_room(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float,
               stretch: float = 1.0) -> RoomSpec:
    """Grid ctor (Grid.cpp:6-37) plus optional set_face_coords (Grid.cpp:39-47)."""
    if nx <= 0 or ny <= 0 or nz <= 0:
        raise ValueError("Grid dimensions must be positive")
    dx, dy, dz = lx / nx, ly / ny, lz / nz
    if stretch > 1.0 + 1e-6:
        xs = np.array(stretched_faces(nx, lx, stretch))
        ys = np.array(stretched_faces(ny, ly, stretch))
        zs = np.array(stretched_faces(nz, lz, stretch))
        dxv, dyv, dzv = np.diff(xs), np.diff(ys), np.diff(zs)
        stretched = True
    else:
        xs = np.array([i * dx for i in range(nx + 1)])
        ys = np.array([j * dy for j in range(ny + 1)])
        zs = np.array([k * dz for k in range(nz + 1)])
        dxv, dyv, dzv = np.full(nx, dx), np.full(ny, dy), np.full(nz, dz)
        stretched = False
    return RoomSpec(nx, ny, nz, lx, ly, lz, xs, ys, zs, dxv, dyv, dzv, stretched,
                    np.zeros(nx * ny * nz, dtype=np.uint8))


def _mark_box(room: RoomSpec, box, value: int) -> None:
    ct = room.cell_type.reshape(room.nx, room.ny, room.nz)
    i0, i1, j0, j1, k0, k1 = box
    i0, j0, k0 = max(0, i0), max(0, j0), max(0, k0)
    i1, j1, k1 = min(room.nx - 1, i1), min(room.ny - 1, j1), min(room.nz - 1, k1)
    if i0 <= i1 and j0 <= j1 and k0 <= k1:
        ct[i0:i1 + 1, j0:j1 + 1, k0:k1 + 1] = value


def add_solid_box(room: RoomSpec, box) -> None:
    """BoundaryManager::add_solid_box (BoundaryManager.cpp:6-14)."""
    room.solids.append(tuple(int(b) for b in box))
    _mark_box(room, box, SOLID)


def add_fan(room: RoomSpec, fan: Fan) -> None:
    """BoundaryManager::add_fan (BoundaryManager.cpp:16-22)."""
    room.fans.append(fan)
    _mark_box(room, fan.box, INFLOW)


def add_outflow(room: RoomSpec, patch: Patch) -> None:
    """BoundaryManager::add_outflow / add_opening (BoundaryManager.cpp:24-44,
    132-135).  The patch is not clamped by the reference; an out-of-range
    patch is rejected here instead of writing out of bounds."""
    nx, ny, nz = room.nx, room.ny, room.nz
    lim = {0: (ny, nz), 1: (nx, nz), 2: (nx, ny)}[patch.axis]
    if patch.a_min < 0 or patch.b_min < 0 or patch.a_max >= lim[0] or patch.b_max >= lim[1]:
        raise ValueError(f"outflow patch out of range: {patch}")
    room.outflows.append(patch)
    ct = room.cell_type.reshape(nx, ny, nz)
    a = slice(patch.a_min, patch.a_max + 1)
    b = slice(patch.b_min, patch.b_max + 1)
    if patch.axis == 0:
        ct[0 if patch.side == 0 else nx - 1, a, b] = OUTFLOW
    elif patch.axis == 1:
        ct[a, 0 if patch.side == 0 else ny - 1, b] = OUTFLOW
    else:
        ct[a, b, 0 if patch.side == 0 else nz - 1] = OUTFLOW


def _to_cell(x: float, L: float, N: int) -> int:
    return int(x / L * N)


def obstacle_box(cfg: SceneConfig, obs: ObstacleConfig):
    """Scene._add_obstacle (scene.py:135-145)."""
    r = cfg.room
    return (_to_cell(obs.bbox_min[0], r.size[0], r.grid[0]),
            _to_cell(obs.bbox_max[0], r.size[0], r.grid[0]) - 1,
            _to_cell(obs.bbox_min[1], r.size[1], r.grid[1]),
            _to_cell(obs.bbox_max[1], r.size[1], r.grid[1]) - 1,
            _to_cell(obs.bbox_min[2], r.size[2], r.grid[2]),
            _to_cell(obs.bbox_max[2], r.size[2], r.grid[2]) - 1)


def fan_patch(cfg: SceneConfig, fan: FanConfig) -> Fan:
    """Scene._add_fan (scene.py:147-192)."""
    r = cfg.room
    ax = fan.snapped_axis()
    vx, vy, vz = fan.direction_vector()

    def span(c, rad, L, N):
        return max(0, int((c - rad) / L * N)), min(N - 1, int((c + rad) / L * N))

    def plane(c, L, N):
        return max(0, min(N - 1, _to_cell(c, L, N)))

    cx, cy, cz = fan.position
    rad = fan.radius
    vel = (vx * fan.velocity, vy * fan.velocity, vz * fan.velocity)
    if ax == 0:
        ix = plane(cx, r.size[0], r.grid[0])
        jlo, jhi = span(cy, rad, r.size[1], r.grid[1])
        klo, khi = span(cz, rad, r.size[2], r.grid[2])
        box = (ix, ix, jlo, jhi, klo, khi)
    elif ax == 1:
        ilo, ihi = span(cx, rad, r.size[0], r.grid[0])
        jy = plane(cy, r.size[1], r.grid[1])
        klo, khi = span(cz, rad, r.size[2], r.grid[2])
        box = (ilo, ihi, jy, jy, klo, khi)
    else:
        ilo, ihi = span(cx, rad, r.size[0], r.grid[0])
        jlo, jhi = span(cy, rad, r.size[1], r.grid[1])
        kz = plane(cz, r.size[2], r.grid[2])
        box = (ilo, ihi, jlo, jhi, kz, kz)
    return Fan(box, vel)


_WALLS = {"west": (0, 0), "east": (0, 1), "south": (1, 0), "north": (1, 1),
          "floor": (2, 0), "ceiling": (2, 1)}


def opening_patch(cfg: SceneConfig, op: OpeningConfig) -> Patch:
    """Scene._add_opening (scene.py:194-231)."""
    r = cfg.room
    ax, sd = _WALLS[op.wall.lower()]
    trans = {0: (1, 2), 1: (0, 2), 2: (0, 1)}[ax]
    (La, Na), (Lb, Nb) = [(r.size[t], r.grid[t]) for t in trans]

    def rng(c, w, L, N):
        return max(0, int((c - w / 2) / L * N)), min(N - 1, int((c + w / 2) / L * N))

    a0, a1 = rng(op.center[0], op.size[0], La, Na)
    b0, b1 = rng(op.center[1], op.size[1], Lb, Nb)
    T_out = op.T_outside if op.T_outside is not None else cfg.solver.T_outside
    return Patch(ax, sd, a0, a1, b0, b1, float(T_out))


def auto_outflow_patch(cfg: SceneConfig, fan: FanConfig) -> Patch:
    """Scene._add_auto_outflow (scene.py:108-133): the whole wall the first
    fan blows toward."""
    g = cfg.room.grid
    ax = fan.snapped_axis()
    side = 1 if fan.snapped_sign() > 0 else 0
    trans = {0: (1, 2), 1: (0, 2), 2: (0, 1)}[ax]
    return Patch(ax, side, 0, g[trans[0]] - 1, 0, g[trans[1]] - 1)


def heat_patch_box(cfg: SceneConfig, hp: HeatPatchConfig):
    r = cfg.room
    i0 = max(0, _to_cell(hp.x_range[0], r.size[0], r.grid[0]))
    i1 = min(r.grid[0] - 1, _to_cell(hp.x_range[1], r.size[0], r.grid[0]) - 1)
    j0 = max(0, _to_cell(hp.y_range[0], r.size[1], r.grid[1]))
    j1 = min(r.grid[1] - 1, _to_cell(hp.y_range[1], r.size[1], r.grid[1]) - 1)
    k = 0 if hp.wall.lower() == "floor" else r.grid[2] - 1
    return (i0, i1, j0, j1, k, k)


def build_room(cfg: SceneConfig) -> RoomSpec:
    """Scene._build (scene.py:72-106) in numpy."""
    r = cfg.room
    stretch = getattr(r, "stretch", 1.0) or 1.0
    room = empty_room(r.grid[0], r.grid[1], r.grid[2], r.size[0], r.size[1], r.size[2], stretch)
    for obs in cfg.obstacles:
        add_solid_box(room, obstacle_box(cfg, obs))
    for fan in cfg.fans:
        add_fan(room, fan_patch(cfg, fan))
    for op in cfg.openings:
        add_outflow(room, opening_patch(cfg, op))
    if cfg.fans and not cfg.openings:
        add_outflow(room, auto_outflow_patch(cfg, cfg.fans[0]))
    for hp in cfg.heat_patches:
        room.heats.append(HeatPatch(heat_patch_box(cfg, hp), float(hp.T)))
    return room


def build_on_core(core, room: RoomSpec):
    """Replays a RoomSpec through a ``_ffroom_core``-like module (Grid,
    BoundaryManager, FanBC, OutflowBC, OpeningBC) in Scene order and returns
    (grid, bm)."""
    g = core.Grid(room.nx, room.ny, room.nz, room.lx, room.ly, room.lz)
    if room.stretched:
        g.set_face_coords(list(room.xs), list(room.ys), list(room.zs))
    bm = core.BoundaryManager()
    for box in room.solids:
        bm.add_solid_box(g, *box)
    for fan in room.fans:
        bc = core.FanBC()
        bc.i_min, bc.i_max, bc.j_min, bc.j_max, bc.k_min, bc.k_max = fan.box
        bc.vel = list(fan.vel)
        bm.add_fan(g, bc)
    for p in room.outflows:
        ob = core.OpeningBC() if p.is_opening else core.OutflowBC()
        ob.axis, ob.side = p.axis, p.side
        ob.a_min, ob.a_max, ob.b_min, ob.b_max = p.a_min, p.a_max, p.b_min, p.b_max
        if p.is_opening:
            ob.T_outside = p.T_outside
            bm.add_opening(g, ob)
        else:
            bm.add_outflow(g, ob)
    if room.heats and hasattr(bm, "add_heat_patch"):
        for hp in room.heats:
            bm.add_heat_patch(g, *hp.box, hp.T)
    return g, bm


def solver_params(core, cfg: SceneConfig):
    """SolverBridge.run's mapping SolverConfig → FluidSolverParams
    (solver_bridge.py:108-127, 74-83)."""
    sc = cfg.solver
    p = core.FluidSolverParams()
    p.rho, p.nu, p.dt = sc.rho, sc.nu, sc.dt
    p.max_steps, p.convergence_tol = sc.max_steps, sc.convergence_tol
    p.poisson.max_iter, p.poisson.tol = sc.poisson_max_iter, sc.poisson_tol
    p.thermal = bool(cfg.openings) or sc.buoyancy or (sc.T_target is not None)
    p.T_initial = sc.T_initial
    p.T_target = sc.T_target if sc.T_target is not None else 1e30
    p.buoyancy = sc.buoyancy
    p.k_thermal, p.cp = sc.k_thermal, sc.cp
    p.beta = 1.0 / (sc.T_initial + 273.15)
    adv = (sc.advection or "upwind").lower()
    p.advection = {"quick": core.AdvectionScheme.QUICK,
                   "lax_wendroff": core.AdvectionScheme.LAX_WENDROFF}.get(adv, core.AdvectionScheme.UPWIND1)
    p.use_openmp = bool(sc.parallel)
    p.use_multigrid = (getattr(sc, "poisson_method", "cg") == "multigrid")
    return p


ADVECTION = {"upwind": 0, "quick": 1, "lax_wendroff": 2}
