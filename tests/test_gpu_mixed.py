"""Mixed precision (FP32 increments on FP64 state, FP32 multigrid
preconditioner, FP64 outer CG) against the FP64 reference method.

Tolerance (the stated bound for mixed precision): every field within 1e-4
max-norm relative error of the FP64 result after the same number of steps,
with the pressure solved to the same relative residual.  The MG-PCG solve
itself must reach the residual the plain CG reaches.
"""
import numpy as np
import pytest

from conftest import Golden, rel_err

pytestmark = pytest.mark.gpu

CASES = ["c1_upwind_10", "c1_quick_10", "two_fans_10", "summer_cooling_10", "edge_odd_quick_10",
         "oblique_stretch_10", "updraft_laxw_10", "vent_quick_10", "thermal_small_10"]


@pytest.mark.parametrize("poisson,precision", [("mgpcg", "fp64"), ("mgpcg", "mixed"), ("cg", "mixed")])
@pytest.mark.parametrize("name", CASES)
def test_mixed_tracks_reference(name, poisson, precision):
    from ffrb import capi
    g = Golden(name)
    p = g.params.with_(poisson=poisson, precision=precision)
    h = capi.FluidHandle(g.room, p)
    recs = h.advance(g.nsteps)
    assert len(recs) == g.nsteps
    for k in "uvwpT":
        err = rel_err(h.get(k), g.fields[k])
        assert err <= 1e-4, (k, err)
    assert all(r["pressure_residual"] < g.params.poisson_tol for r in recs if r["cg_iterations"] > 0)
    if poisson == "mgpcg":
        # far fewer iterations than the unpreconditioned CG
        assert np.mean([r["cg_iterations"] for r in recs]) < 0.35 * np.mean(g.hist["cg_iterations"])
    h.close()


def test_mgpcg_long_run_tracks_reference():
    """500 steps of the benchmark room: mixed MG-PCG stays within 1e-4."""
    from ffrb import capi
    g = Golden("c1_upwind_500")
    h = capi.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed"))
    recs = h.advance(g.nsteps)
    for k in "uvwp":
        assert rel_err(h.get(k), g.fields[k]) <= 1e-4, k
    assert rel_err([recs[-1]["velocity_change"]], [g.hist["velocity_change"][-1]]) <= 1e-3


def test_projected_divergence_is_small():
    """The projected field (before the BC re-application that the reference
    performs after the correction) is divergence-free to the solver
    tolerance: measured on FLUID cells away from BC-overwritten faces."""
    from ffrb import capi
    from ffrb.scene import build_room
    from ffrb import workloads
    cfg, prm = workloads.large_thermal(grid=(80, 64, 24))
    room = build_room(cfg)
    h = capi.FluidHandle(room, prm.with_(poisson_tol=1e-10))
    h.advance(3)
    u, v, w = h.get("u"), h.get("v"), h.get("w")
    nx, ny, nz = room.nx, room.ny, room.nz
    U = u.reshape(nx + 1, ny, nz); V = v.reshape(nx, ny + 1, nz); W = w.reshape(nx, ny, nz + 1)
    div = ((U[1:] - U[:-1]) / room.dxv[:, None, None] + (V[:, 1:] - V[:, :-1]) / room.dyv[None, :, None]
           + (W[:, :, 1:] - W[:, :, :-1]) / room.dzv[None, None, :])
    ct = room.cell_type.reshape(nx, ny, nz)
    # FLUID cells whose 6 neighbours are FLUID (no BC-overwritten face)
    inner = np.zeros_like(ct, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    for ax in range(3):
        for sh in (-1, 1):
            inner &= np.roll(ct, sh, axis=ax) == 0
    inner &= ct == 0
    assert np.abs(div[inner]).max() <= 1e-6


@pytest.mark.parametrize("name", ["c1_upwind_10", "summer_cooling_10", "oblique_stretch_10", "vent_quick_10",
                                  "thermal_small_10", "edge_odd_quick_10"])
def test_split_graph_solve_tracks_reference(name):
    """The multigrid solve recorded as one kernel per pass inside a CUDA
    graph with a device-controlled WHILE loop: same bound as above, and the
    same iteration counts as the persistent kernel (±1)."""
    from ffrb import capi
    g = Golden(name)
    p = g.params.with_(poisson="mgpcg", precision="mixed")
    a = capi.FluidHandle(g.room, p)
    ra = a.advance(g.nsteps)
    b = capi.FluidHandle(g.room, p)
    b.use_graph(True)
    rb = b.advance(g.nsteps)
    assert len(rb) == g.nsteps
    for k in "uvwpT":
        assert rel_err(b.get(k), g.fields[k]) <= 1e-4, (k, rel_err(b.get(k), g.fields[k]))
    ia = np.array([r["cg_iterations"] for r in ra])
    ib = np.array([r["cg_iterations"] for r in rb])
    assert np.abs(ia - ib).max() <= 1, (ia, ib)
    assert all(r["pressure_residual"] < p.poisson_tol for r in rb if r["cg_iterations"] > 0)
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["c1_upwind_10", "oblique_stretch_10", "thermal_small_10"])
def test_split_eager_matches_split_graph(name):
    """The split solve paced by the host (no graph) runs the same kernels on
    the same grids as the graph's WHILE loop, so fields and histories are
    bit-identical; kernels queued past convergence change nothing."""
    from ffrb import capi
    g = Golden(name)
    p = g.params.with_(poisson="mgpcg", precision="mixed")
    a = capi.FluidHandle(g.room, p)
    a.use_graph(True)
    ra = a.advance(g.nsteps)
    b = capi.FluidHandle(g.room, p)
    b.set_split(1)
    rb = b.advance(g.nsteps)
    assert [r["cg_iterations"] for r in ra] == [r["cg_iterations"] for r in rb]
    for k in "uvwpT":
        assert np.array_equal(a.get(k), b.get(k)), k
    # the pressure re-solve used for timing leaves the step state unchanged
    ms, it = b.time_pressure(2)
    assert ms > 0 and it == rb[-1]["cg_iterations"]
    assert np.array_equal(a.get("p"), b.get("p"))
    a.close()
    b.close()


@pytest.mark.parametrize("name", ["c1_upwind_10", "summer_cooling_10", "oblique_stretch_10", "thermal_small_10",
                                  "vent_quick_10"])
def test_warm_start_tracks_reference(name):
    """The multigrid solve started from the previous step's pressure (the
    default) and from zero (the reference's start) both stay within the
    mixed bound of the FP64 fixtures; the first step (zero pressure before
    it) is bit-identical, and the warm start takes no more iterations."""
    from ffrb import capi
    g = Golden(name)
    p = g.params.with_(poisson="mgpcg", precision="mixed")
    warm = capi.FluidHandle(g.room, p)
    cold = capi.FluidHandle(g.room, p)
    cold.set_warm_start(False)
    for h in (warm, cold):
        h.set_split(1)
    rw, rc = warm.advance(1), cold.advance(1)
    assert rw[0]["cg_iterations"] == rc[0]["cg_iterations"]
    for k in "uvwpT":
        assert np.array_equal(warm.get(k), cold.get(k)), k
    rw += warm.advance(g.nsteps - 1)
    rc += cold.advance(g.nsteps - 1)
    for h in (warm, cold):
        for k in "uvwpT":
            err = rel_err(h.get(k), g.fields[k])
            assert err <= 1e-4, (k, err)
    assert all(r["pressure_residual"] < g.params.poisson_tol for r in rw if r["cg_iterations"] > 0)
    assert sum(r["cg_iterations"] for r in rw) <= sum(r["cg_iterations"] for r in rc)
    warm.close()
    cold.close()


def test_time_pressure_after_batched_step_is_refused():
    """A warm-started re-solve needs the starting pressure of the last step,
    which batched steps do not keep."""
    from ffrb import capi
    g = Golden("c1_upwind_10")
    h = capi.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed"))
    h.set_split(1)
    h.advance(2)
    ms, it = h.time_pressure(2)
    assert ms > 0 and it > 0
    b = capi.BatchHandle([h])
    b.advance(1)
    with pytest.raises(capi.FfrError):
        h.time_pressure(2)
    b.close()
    h.advance(1)
    assert h.time_pressure(1)[1] > 0
    h.close()
