"""Failure handling and checkpointing, tested without faulting the GPU.

* A bounded device wait that runs out: the self-test kernel's blocks wait at
  the library's own grid reduction for a block that never arrives; with the
  wait limit shortened to 50 ms every wait gives up, the call returns
  FFR_ETIMEDOUT, and the same process then solves a room correctly.
* A NaN seeded into one room of a batch (through the public set-field call)
  is flagged in that room only; the other rooms of the batch end exactly as
  they do alone.
* An LBM room saved (populations, step counter, fields) and loaded into a
  new handle continues as the original does: bit-identically with FP64
  populations, within 1e-6 with FP32/FP16 storage.
"""
import numpy as np
import pytest

from conftest import Golden, rel_err

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_the_context_survives():
    from ffrb import capi
    capi.set_device_wait_limit(0.05)
    try:
        status, ms = capi.selftest_device_wait(8)
    finally:
        capi.set_device_wait_limit(0.0)
    assert status == capi.FFR_ETIMEDOUT
    assert 40.0 <= ms <= 3000.0, ms
    # the context is intact: a room solves exactly as the reference did
    g = Golden("c1_upwind_10")
    h = capi.FluidHandle(g.room, g.params)
    recs = h.advance(g.nsteps)
    assert [r["cg_iterations"] for r in recs] == list(g.hist["cg_iterations"])
    for k in "uvwp":
        assert rel_err(h.get(k), g.fields[k]) <= 1e-8, k
    h.close()


def test_wait_limit_rejects_bad_values():
    from ffrb import capi
    with pytest.raises(capi.FfrError):
        capi.set_device_wait_limit(-1.0)
    with pytest.raises(capi.FfrError):
        capi.set_device_wait_limit(1e6)


def _split_handle(g, max_iter=200):
    from ffrb import capi
    h = capi.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed", poisson_max_iter=max_iter))
    h.set_split(1)
    return h


def test_nan_in_one_batched_room_stays_in_that_room():
    from ffrb import capi
    names = ["c1_upwind_10", "summer_cooling_10", "two_fans_10"]
    gs = [Golden(n) for n in names]
    steps = 3
    alone = {}
    for i in (0, 2):
        h = _split_handle(gs[i])
        alone[i] = (h.advance(steps), {k: h.get(k) for k in "uvwpT"})
        h.close()
    hs = [_split_handle(g) for g in gs]
    u = hs[1].get("u")
    u[len(u) // 2] = np.nan
    hs[1].set("u", u)
    b = capi.BatchHandle(hs)
    out = b.advance(steps)
    b.close()
    assert any(r["flags"] & capi.FFR_FLAG_NAN for r in out[1])
    for i in (0, 2):
        recs_a, fa = alone[i]
        assert len(out[i]) == steps
        for ra, rb in zip(recs_a, out[i]):
            assert not (rb["flags"] & capi.FFR_FLAG_NAN)
            for k in ("velocity_change", "pressure_residual", "cg_iterations", "T_mean"):
                assert ra[k] == rb[k], (names[i], k)
        for k in "uvwpT":
            assert np.array_equal(hs[i].get(k), fa[k]), (names[i], k)
    for h in hs:
        h.close()


@pytest.mark.parametrize("storage", ["fp64", "fp32", "fp16"])
def test_lbm_checkpoint_resume(storage):
    from ffrb import capi
    g = Golden("lbm_small_20")
    tau, dt, tol = g.lbm["tau"], g.lbm["dt"], g.lbm["tol"]
    a = capi.LbmHandle(g.room, tau, 20, tol, dt, storage)
    ra = a.advance(12)
    b = capi.LbmHandle(g.room, tau, 20, tol, dt, storage)
    b.advance(7)
    f, step = b.get_populations()
    fields = {k: b.get(k) for k in "uvwp"}
    assert step == 7 and f.shape == (19 * g.room.n_cells,) and np.isfinite(f).all()
    b.close()
    c = capi.LbmHandle(g.room, tau, 20, tol, dt, storage, init=fields)
    c.set_populations(f, step)
    f2, step2 = c.get_populations()
    assert step2 == 7 and np.array_equal(f2, f)
    rc = c.advance(5)
    assert [r["step"] for r in rc] == [r["step"] for r in ra[7:]]
    for k in "uvwp":
        if storage == "fp64":
            assert np.array_equal(c.get(k), a.get(k)), k
        else:
            assert rel_err(c.get(k), a.get(k)) <= 1e-6, k
    for x, y in zip(rc, ra[7:]):
        if storage == "fp64":
            assert x["velocity_change"] == y["velocity_change"]
    a.close()
    c.close()
