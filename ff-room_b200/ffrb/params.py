"""Solver parameters shared by the C ABI, the oracle wrappers and the tests.

``FluidParams`` carries the fields of the reference ``FluidSolverParams``
(cpp/src/core/FluidSolver.hpp:11-38, including ``PoissonSolverParams``,
PoissonSolver.hpp:14-18) plus the B200 options ``precision`` ("fp64" = the
reference method in FP64, "mixed" = FP32 fields with an FP64 outer Krylov
solve) and ``poisson`` ("cg" = the reference's unpreconditioned CG,
"mgpcg" = multigrid-preconditioned CG).
"""
from __future__ import annotations

from dataclasses import dataclass, replace

from .scene import ADVECTION, SceneConfig


@dataclass
class FluidParams:
    rho: float = 1.2
    nu: float = 1.5e-5
    dt: float = 0.01
    max_steps: int = 500
    convergence_tol: float = 1.0
    poisson_max_iter: int = 1000
    poisson_tol: float = 1e-6
    advection: int = 0
    use_openmp: bool = False
    use_multigrid: bool = False
    thermal: bool = False
    T_initial: float = 20.0
    T_target: float = 1e30
    buoyancy: bool = False
    g_accel: float = 9.81
    beta: float = 1.0 / 293.0
    k_thermal: float = 0.026
    cp: float = 1005.0
    precision: str = "fp64"
    poisson: str = "cg"

    def with_(self, **kw) -> "FluidParams":
        return replace(self, **kw)


def params_from_scene(cfg: SceneConfig) -> FluidParams:
    """SolverBridge's SolverConfig → FluidSolverParams mapping
    (python/ff_room/solver_bridge.py:108-127)."""
    sc = cfg.solver
    return FluidParams(
        rho=sc.rho, nu=sc.nu, dt=sc.dt, max_steps=sc.max_steps,
        convergence_tol=sc.convergence_tol, poisson_max_iter=sc.poisson_max_iter,
        poisson_tol=sc.poisson_tol,
        advection=ADVECTION.get((sc.advection or "upwind").lower(), 0),
        use_openmp=bool(sc.parallel),
        use_multigrid=(sc.poisson_method == "multigrid"),
        thermal=bool(cfg.openings) or sc.buoyancy or (sc.T_target is not None),
        T_initial=sc.T_initial,
        T_target=sc.T_target if sc.T_target is not None else 1e30,
        buoyancy=sc.buoyancy, k_thermal=sc.k_thermal, cp=sc.cp,
        beta=1.0 / (sc.T_initial + 273.15),
        precision=getattr(sc, "precision", "fp64"),
        poisson="mgpcg" if sc.poisson_method == "multigrid" else "cg",
    )
