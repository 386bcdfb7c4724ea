"""The drop-in boundary without a GPU: library exports, module surface,
argument validation."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_available

HEADER = os.path.join(ROOT, "include", "ffroom.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ffr_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from ffrb import capi
    lib = capi.lib()
    names = declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert lib.ffr_version().decode().endswith("sm_100a")
    assert lib.ffr_status_string(1).decode() == "invalid argument"


def test_invalid_room_is_rejected_without_gpu():
    from ffrb import capi
    from ffrb.params import FluidParams
    from ffrb.scene import empty_room
    room = empty_room(4, 4, 4, 1.0, 1.0, 1.0)
    room.cell_type[0] = 9            # not a cell type
    with pytest.raises(capi.FfrError) as e:
        capi.FluidHandle(room, FluidParams())
    assert e.value.status == capi.FFR_EINVAL


def test_unsupported_options_are_reported():
    from ffrb import capi
    from ffrb.params import FluidParams
    from ffrb.scene import empty_room
    room = empty_room(4, 4, 4, 1.0, 1.0, 1.0)
    with pytest.raises(capi.FfrError) as e:
        capi.FluidHandle(room, FluidParams(dt=-1.0))
    assert e.value.status == capi.FFR_EINVAL


REF_SURFACE = {
    # cpp/src/bindings/module.cpp:19-209
    "AdvectionScheme": ["UPWIND1", "QUICK", "LAX_WENDROFF"],
    "CellType": ["FLUID", "SOLID", "INFLOW", "OUTFLOW"],
    "Grid": ["Nx", "Ny", "Nz", "dx", "dy", "dz", "u", "v", "w", "p", "u_shaped", "v_shaped", "w_shaped",
             "p_shaped", "T_shaped", "cell_type_shaped", "xs", "ys", "zs", "set_face_coords",
             "zero_velocity", "zero_pressure"],
    "FanBC": ["i_min", "i_max", "j_min", "j_max", "k_min", "k_max", "vel"],
    "OutflowBC": ["axis", "side", "a_min", "a_max", "b_min", "b_max"],
    "OpeningBC": ["axis", "side", "a_min", "a_max", "b_min", "b_max", "T_outside"],
    "BoundaryManager": ["add_solid_box", "add_fan", "add_outflow", "add_opening", "apply_noslip",
                        "apply_inflow", "apply_outflow", "apply_opening_temperature"],
    "PoissonSolverParams": ["max_iter", "tol"],
    "FluidSolverParams": ["rho", "nu", "dt", "max_steps", "convergence_tol", "poisson", "advection",
                          "use_openmp", "use_multigrid", "thermal", "T_initial", "T_target", "buoyancy",
                          "g_accel", "beta", "k_thermal", "cp"],
    "StepResult": ["step", "velocity_change", "pressure_residual", "divergence_max", "converged", "T_mean"],
    "FluidSolver": ["step", "run", "compute_divergence_max", "current_step"],
    "LBMSolver": ["step", "run", "compute_divergence_max"],
}


def test_module_has_reference_surface():
    import _ffroom_core as c
    for cls, attrs in REF_SURFACE.items():
        obj = getattr(c, cls)
        for a in attrs:
            assert hasattr(obj, a), f"{cls}.{a}"
    p = c.FluidSolverParams()
    assert (p.rho, p.nu, p.dt, p.max_steps, p.convergence_tol) == (1.2, 1.5e-5, 0.01, 500, 1.0)
    assert (p.poisson.max_iter, p.poisson.tol) == (1000, 1e-6)
    assert p.advection == c.AdvectionScheme.UPWIND1 and p.T_target == 1e30 and p.beta == 1.0 / 293.0
    p.poisson.tol = 1e-9
    assert p.poisson.tol == 1e-9           # nested struct is writable in place
    doc = c.FluidSolver.__init__.__doc__
    assert "grid" in doc and "bm" in doc and "params" in doc
    doc = c.LBMSolver.__init__.__doc__
    for a in ("tau", "max_steps", "convergence_tol", "dt"):
        assert a in doc


def test_grid_views_alias_host_memory():
    import _ffroom_core as c
    g = c.Grid(4, 5, 6, 4.0, 5.0, 6.0)
    assert g.u.shape == (150,) and g.u_shaped().shape == (5, 5, 6)
    u = g.u_shaped()
    u[1, 2, 3] = 7.0
    assert g.u[(1 * 5 + 2) * 6 + 3] == 7.0
    g.zero_velocity()
    assert not np.any(g.u)
    ct = g.cell_type_shaped()
    ct[0, 0, 0] = 3                       # a copy, as in the reference
    assert g.cell_type_shaped()[0, 0, 0] == 0
    with pytest.raises(ValueError):
        c.Grid(0, 1, 1, 1.0, 1.0, 1.0)


def test_host_boundary_appliers_match_oracle(oracle):
    """BoundaryManager.apply_* on the host copy against the oracle's restatement."""
    import _ffroom_core as c
    from ffrb import workloads
    from ffrb.scene import build_room, build_on_core
    room = build_room(workloads.basic_room())
    g, bm = build_on_core(c, room)
    rng = np.random.default_rng(0)
    u0, v0, w0 = (rng.standard_normal(g.u.size), rng.standard_normal(g.v.size), rng.standard_normal(g.w.size))
    for name in ("noslip", "inflow", "outflow"):
        g.u[:] = u0; g.v[:] = v0; g.w[:] = w0
        getattr(bm, "apply_" + name)(g)
        uo, vo, wo = u0.copy(), v0.copy(), w0.copy()
        oracle.apply_bc(name, room, uo, vo, wo)
        assert np.array_equal(np.array(g.u), uo) and np.array_equal(np.array(g.v), vo)
        assert np.array_equal(np.array(g.w), wo), name


@pytest.mark.skipif(gpu_available(), reason="checks the no-GPU error path")
def test_solver_without_gpu_fails_loudly():
    import _ffroom_core as c
    g = c.Grid(4, 4, 4, 1.0, 1.0, 1.0)
    bm = c.BoundaryManager()
    with pytest.raises(RuntimeError):
        c.FluidSolver(g, bm)
