"""GPU projection and LBM solvers against the reference (golden fixtures).

Every call goes through the C ABI of libffroom_cuda.so (ffrb.capi) or the
drop-in pybind11 module.  FP64 tolerances (max-norm relative error of each
field): 1e-8 after 10 steps, 1e-6 after 500 steps; the CG iteration count of
every step must equal the reference's (the 500-step run may differ by one
iteration on a few steps, from reduction order).  Masks are bit-exact.
"""
import numpy as np
import pytest

from conftest import Golden, golden_names, rel_err

pytestmark = pytest.mark.gpu

FLUID = [n for n in golden_names() if not n.startswith("lbm")]
LBM = [n for n in golden_names() if n.startswith("lbm")]


@pytest.mark.parametrize("name", FLUID)
def test_fluid_fp64_matches_reference(name):
    from ffrb import capi
    g = Golden(name)
    h = capi.FluidHandle(g.room, g.params)
    recs = h.advance(g.nsteps)
    assert len(recs) == g.nsteps
    long_run = g.nsteps > 100
    tol = 1e-6 if long_run else 1e-8
    for k in "uvwpT":
        err = rel_err(h.get(k), g.fields[k])
        assert err <= tol, (k, err)
    its = np.array([r["cg_iterations"] for r in recs])
    diff = np.abs(its - g.hist["cg_iterations"])
    if long_run:
        assert diff.max() <= 1 and (diff > 0).mean() < 0.05
    else:
        assert diff.max() == 0, (its, g.hist["cg_iterations"])
    for key in ("velocity_change", "divergence_max", "T_mean"):
        got = np.array([r[key] for r in recs])
        assert rel_err(got, g.hist[key]) <= max(tol, 1e-9), key
    assert [bool(r["converged"]) for r in recs] == list(g.hist["converged"].astype(bool))
    assert h.current_step() == g.nsteps
    assert rel_err([h.divergence_max()], [g.hist["divergence_max"][-1]]) <= 1e-9
    h.close()


@pytest.mark.parametrize("name", LBM)
def test_lbm_fp64_matches_reference(name):
    from ffrb import capi
    g = Golden(name)
    L = g.lbm
    h = capi.LbmHandle(g.room, L["tau"], g.nsteps, L["tol"], L["dt"], "fp64")
    recs = h.advance(g.nsteps)
    assert len(recs) == g.nsteps
    for k in "uvwp":
        err = rel_err(h.get(k), g.fields[k])
        assert err <= 1e-10, (k, err)
    got = np.array([r["velocity_change"] for r in recs])
    assert rel_err(got, g.hist["velocity_change"]) <= 1e-9
    got = np.array([r["divergence_max"] for r in recs])
    assert rel_err(got, g.hist["divergence_max"]) <= 1e-9
    h.close()


def test_basic_room_converges_at_published_step():
    """basic_room.yaml (tol 1.0) converges at step 529 with the projection
    method (docs/developer_guide.md:426, reproduced by the reference)."""
    import os
    from conftest import ROOT
    from ffrb import capi, workloads
    from ffrb.params import params_from_scene
    from ffrb.scene import build_room
    cfg = workloads.basic_room(steps=1000, tol=1.0)
    h = capi.FluidHandle(build_room(cfg), params_from_scene(cfg))
    recs = h.advance(1000, stop_on_converge=True)
    assert len(recs) == 529 and recs[-1]["converged"] and not recs[-2]["converged"]
    assert h.current_step() == 529


def test_basic_room_lbm_converges_at_published_step():
    """basic_room.yaml with the LBM (tau 0.8) converges at step 119
    (docs/developer_guide.md:426)."""
    from ffrb import capi, workloads
    from ffrb.scene import build_room
    cfg = workloads.basic_room(steps=1000, tol=1.0)
    h = capi.LbmHandle(build_room(cfg), 0.8, 1000, 1.0, 0.01, "fp64")
    recs = h.advance(1000, stop_on_converge=True)
    assert len(recs) == 119 and recs[-1]["converged"]


@pytest.mark.parametrize("storage,tol", [("fp32", 2e-6), ("fp16", 2e-3)])
@pytest.mark.parametrize("name", ["lbm_basic_10", "lbm_small_20", "lbm_openings_10"])
def test_lbm_narrow_storage_tracks_reference(name, storage, tol):
    """FP32 / FP16 population storage (shifted populations, FP32 collision)
    against the reference's FP64 LBM fixtures.  Bound per storage: an FP32
    population carries a relative rounding of 6e-8 and an FP16 one 4.9e-4
    of the shifted value; over 10-20 steps the fields stay within about 5e-7
    (FP32) and 5e-4 (FP16) of the reference, and the bound is four times
    that."""
    from ffrb import capi
    g = Golden(name)
    L = g.lbm
    h = capi.LbmHandle(g.room, L["tau"], g.nsteps, L["tol"], L["dt"], storage)
    h.advance(g.nsteps)
    for k in "uvwp":
        err = rel_err(h.get(k), g.fields[k])
        assert err <= tol, (storage, k, err)
    h.close()


@pytest.mark.parametrize("storage,tol", [("fp32", 2e-3), ("fp16", 5e-2)])
def test_lbm_narrow_storage_tracks_fp64(storage, tol):
    """FP32 / FP16 populations (shifted, FP32 collision) against the FP64
    run on the same room; the error bound is stated per field."""
    from ffrb import capi
    g = Golden("lbm_basic_10")
    L = g.lbm
    ref = capi.LbmHandle(g.room, L["tau"], 50, L["tol"], L["dt"], "fp64")
    ref.advance(50)
    h = capi.LbmHandle(g.room, L["tau"], 50, L["tol"], L["dt"], storage)
    h.advance(50)
    for k in "uvw":
        assert rel_err(h.get(k), ref.get(k)) <= tol, (storage, k, rel_err(h.get(k), ref.get(k)))
    assert rel_err(h.get("p"), ref.get("p")) <= tol / 10


def test_dropin_module_matches_reference():
    """The reference-shaped API (_ffroom_core) with a per-step callback, a
    held numpy view and run(): same answer as the reference."""
    import _ffroom_core as c
    from ffrb.scene import build_on_core, solver_params
    g = Golden("c1_quick_10")
    grid, bm = build_on_core(c, g.room)
    params = solver_params(c, g.cfg)
    params.max_steps = g.nsteps
    params.convergence_tol = 0.0
    solver = c.FluidSolver(grid, bm, params)
    held = grid.u_shaped()            # a live view, as the reference allows
    seen = []

    def cb(res):
        seen.append((res.step, float(held[5, 10, 6])))

    final = solver.run(cb)
    assert final.step == g.nsteps and len(seen) == g.nsteps
    assert seen[-1][1] == grid.u_shaped()[5, 10, 6]
    assert rel_err(np.array(grid.u_shaped()).reshape(-1), g.fields["u"]) <= 1e-8
    assert rel_err(np.array(grid.p_shaped()).reshape(-1), g.fields["p"]) <= 1e-8
    assert rel_err(np.array(grid.T_shaped()).reshape(-1), g.fields["T"]) <= 1e-12
    assert solver.current_step == g.nsteps
    assert repr(final).startswith("StepResult(step=10, vel_change=")
    assert final.cg_iterations == int(g.hist["cg_iterations"][-1])


def test_dropin_lbm_module():
    import _ffroom_core as c
    from ffrb.scene import build_on_core
    g = Golden("lbm_openings_10")
    grid, bm = build_on_core(c, g.room)
    L = g.lbm
    s = c.LBMSolver(grid, bm, L["tau"], g.nsteps, L["tol"], L["dt"])
    for _ in range(g.nsteps):
        r = s.step()
    assert r.step == g.nsteps
    for k in "uvwp":
        assert rel_err(np.array(getattr(grid, k + "_shaped")()).reshape(-1), g.fields[k]) <= 1e-10


def test_host_write_through_view_reaches_device():
    """Writing T through Grid.T_shaped() between steps (the way a callback
    imposes a heated patch on the reference) changes the next step."""
    import _ffroom_core as c
    from ffrb.scene import build_on_core, solver_params
    g = Golden("thermal_small_10")
    grid, bm = build_on_core(c, g.room)     # heat patches registered on the bm
    p = c.FluidSolverParams()
    P = g.params
    for k in ("rho", "nu", "dt", "max_steps", "convergence_tol", "thermal", "T_initial", "T_target",
              "buoyancy", "g_accel", "beta", "k_thermal", "cp"):
        setattr(p, k, getattr(P, k))
    p.poisson.max_iter, p.poisson.tol = P.poisson_max_iter, P.poisson_tol
    s = c.FluidSolver(grid, bm, p)
    for _ in range(g.nsteps):
        s.step()
    for k in "uvwpT":
        assert rel_err(np.array(getattr(grid, k + "_shaped")()).reshape(-1), g.fields[k]) <= 1e-8, k


def test_snapshot_matches_fields():
    """The device snapshot (run_animated's cell-centred velocity and speed)
    equals the same averages taken on the host from the face fields."""
    from ffrb import capi
    g = Golden("summer_cooling_10")
    h = capi.FluidHandle(g.room, g.params)
    h.advance(3)
    snap = h.snapshot()
    nx, ny, nz = g.room.nx, g.room.ny, g.room.nz
    u = h.get("u").reshape(nx + 1, ny, nz)
    v = h.get("v").reshape(nx, ny + 1, nz)
    w = h.get("w").reshape(nx, ny, nz + 1)
    uc, vc, wc = 0.5 * (u[:-1] + u[1:]), 0.5 * (v[:, :-1] + v[:, 1:]), 0.5 * (w[:, :, :-1] + w[:, :, 1:])
    assert np.array_equal(snap["vel"], np.stack([uc, vc, wc], axis=-1))
    assert rel_err(snap["speed"], np.sqrt(uc ** 2 + vc ** 2 + wc ** 2)) <= 1e-14
    # the solve continues unchanged after a snapshot (its buffers are scratch)
    a = h.advance(2)
    b = capi.FluidHandle(g.room, g.params)
    bb = b.advance(5)
    assert [r["cg_iterations"] for r in bb[3:]] == [r["cg_iterations"] for r in a]
    for k in "uvwp":
        assert np.array_equal(h.get(k), b.get(k)), k


def test_large_field_transfers_round_trip():
    """Fields of tens of MB cross PCIe through page-locked bounce buffers in
    chunks (uploads at creation and set_field, downloads in get): every
    byte arrives, including a ragged last chunk."""
    from ffrb import capi, workloads
    from ffrb.scene import build_room
    cfg, prm = workloads.large_thermal(grid=(203, 160, 96))     # ~25 MB per cell field
    room = build_room(cfg)
    rng = np.random.default_rng(5)
    shapes = room.shapes()
    init = {k: rng.standard_normal(int(np.prod(shapes[k]))) for k in ("u", "v", "w", "p")}
    h = capi.FluidHandle(room, prm, init)
    for k in ("u", "v", "w", "p"):
        assert np.array_equal(h.get(k), init[k]), k
    t = rng.standard_normal(room.n_cells)
    h.set("T", t)
    assert np.array_equal(h.get("T"), t)
    h.close()


def test_result_files_from_a_device_room(tmp_path):
    """ResultStore-layout archive and velocity CSV written from a handle."""
    from ffrb import capi
    from ffrb.results import save_npz, save_velocity_csv
    g = Golden("summer_cooling_10")
    h = capi.FluidHandle(g.room, g.params)
    recs = h.advance(2)
    save_npz(h, g.cfg, str(tmp_path / "r.npz"), last=recs[-1], steps=len(recs))
    z = np.load(tmp_path / "r.npz", allow_pickle=True)
    assert np.array_equal(z["p_field"].ravel(), h.get("p"))
    assert np.array_equal(z["u_field"].ravel(), h.get("u"))
    assert int(z["_steps"]) == 2 and float(z["_velocity_change"]) == recs[-1]["velocity_change"]
    save_velocity_csv(h, str(tmp_path / "v.csv"))
    rows = np.loadtxt(tmp_path / "v.csv", delimiter=",", skiprows=1)
    assert np.array_equal(rows[:, 6], h.snapshot(with_velocity=False)["speed"].ravel())
    h.close()


def test_dropin_snapshot_matches_run_animated_arithmetic():
    """FluidSolver.snapshot() (device-side) gives run_animated's cell-centred
    velocity and speed (solver_bridge.py:222-238) from the same fields."""
    import _ffroom_core as c
    from ffrb.scene import build_on_core, solver_params
    g = Golden("summer_cooling_10")
    grid, bm = build_on_core(c, g.room)
    params = solver_params(c, g.cfg)
    s = c.FluidSolver(grid, bm, params)
    for _ in range(5):
        s.step()
    snap = s.snapshot()
    u, v, w = np.array(grid.u_shaped()), np.array(grid.v_shaped()), np.array(grid.w_shaped())
    uc = 0.5 * (u[:-1, :, :] + u[1:, :, :])
    vc = 0.5 * (v[:, :-1, :] + v[:, 1:, :])
    wc = 0.5 * (w[:, :, :-1] + w[:, :, 1:])
    assert np.allclose(snap["vel"], np.stack([uc, vc, wc], axis=-1), rtol=0, atol=1e-14)
    assert np.allclose(snap["speed"], np.sqrt(uc ** 2 + vc ** 2 + wc ** 2), rtol=1e-14, atol=1e-14)
    # the snapshot leaves the run unchanged
    r = s.step()
    assert r.step == 6
