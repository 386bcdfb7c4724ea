"""Parity on the configurations the benchmark measures, not only on small rooms.

* The large thermal room itself (320x256x96, 7.86 M cells, two fans,
  buoyancy, heat patches, pressure to 1e-8): its first three steps from rest
  against the reference's own solver compiled from its sources (the
  checker library oracle/_ref, run on the host cores).  The plain FP64
  path must track it within 1e-7 max-norm relative on every field with the
  same CG iteration count on every step; the benchmark's exact path (mixed
  precision, multigrid-preconditioned CG, warm start, each step replayed
  from a CUDA graph) within the mixed bound 1e-4.
* The same room scaled down to 80x64x24 over its full 2000 steps, against a
  fixture written by the reference (tests/golden/thermal_80x64x24_2000.npz):
  the benchmark path within 1e-4 on every field after 2000 steps and the
  projected divergence of the benchmark path below 1e-6 at the benchmark's
  tolerance 1e-8 (the plain FP64 path is held to 1e-6 on this fixture by
  the golden tests of test_gpu_parity.py).
* Rooms of the serving stream and of the batch of uneven rooms, run through
  the continuous-batching server (one stream per room, and batched), against
  the FP64 oracle on the same steps: within 1e-4.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, Golden, rel_err

pytestmark = pytest.mark.gpu

MIXED_TOL = 1e-4


def bench_path(h):
    """The benchmark's default configuration of a handle: each step replayed
    from a CUDA graph (multigrid solve one kernel per pass in a WHILE node),
    warm start on (the default)."""
    h.use_graph(True)
    return h


@pytest.fixture(scope="module")
def large_thermal_reference():
    import oracle as orc
    from ffrb import workloads
    from ffrb.scene import build_room
    if not orc.ref_available():
        pytest.fail("oracle/_ref (the reference compiled from its sources) is missing")
    cfg, prm = workloads.large_thermal()
    room = build_room(cfg)
    ref = prm.with_(precision="fp64", poisson="cg")
    os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
    fields, ct, recs = orc.RefDriver().fluid_run(room, ref, 3, use_openmp=True)
    assert np.array_equal(ct, room.cell_type)
    return room, prm, fields, recs


def test_large_thermal_fp64_matches_reference_first_steps(large_thermal_reference):
    from ffrb import capi
    room, prm, fields, recs = large_thermal_reference
    h = capi.FluidHandle(room, prm.with_(precision="fp64", poisson="cg"))
    got = h.advance(3)
    assert [r["cg_iterations"] for r in got] == [r.cg_iterations for r in recs]
    for k in "uvwpT":
        err = rel_err(h.get(k), fields[k])
        assert err <= 1e-7, (k, err)
    for a, b in zip(got, recs):
        assert abs(a["velocity_change"] - b.velocity_change) <= 1e-7 * abs(b.velocity_change)
    h.close()


def test_large_thermal_bench_path_matches_reference_first_steps(large_thermal_reference):
    from ffrb import capi
    room, prm, fields, recs = large_thermal_reference
    h = bench_path(capi.FluidHandle(room, prm))
    got = h.advance(3)
    assert len(got) == 3
    for k in "uvwpT":
        err = rel_err(h.get(k), fields[k])
        assert err <= MIXED_TOL, (k, err)
    assert all(r["pressure_residual"] < prm.poisson_tol for r in got)
    h.close()


def _projected_divergence(room, u, v, w):
    nx, ny, nz = room.nx, room.ny, room.nz
    U = u.reshape(nx + 1, ny, nz)
    V = v.reshape(nx, ny + 1, nz)
    W = w.reshape(nx, ny, nz + 1)
    div = ((U[1:] - U[:-1]) / room.dxv[:, None, None] + (V[:, 1:] - V[:, :-1]) / room.dyv[None, :, None]
           + (W[:, :, 1:] - W[:, :, :-1]) / room.dzv[None, None, :])
    ct = room.cell_type.reshape(nx, ny, nz)
    # FLUID cells whose six neighbours are FLUID: no face of theirs is
    # overwritten by the boundary appliers after the correction
    inner = np.zeros_like(ct, dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    for ax in range(3):
        for sh in (-1, 1):
            inner &= np.roll(ct, sh, axis=ax) == 0
    inner &= ct == 0
    return float(np.abs(div[inner]).max())


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "thermal_80x64x24_2000.npz")),
                    reason="fixture not generated")
def test_scaled_thermal_room_2000_steps_bench_path():
    from ffrb import capi
    g = Golden("thermal_80x64x24_2000")
    prm = g.params.with_(precision="mixed", poisson="mgpcg", use_openmp=False)
    h = bench_path(capi.FluidHandle(g.room, prm))
    recs = h.advance(g.nsteps)
    assert len(recs) == g.nsteps
    for k in "uvwpT":
        err = rel_err(h.get(k), g.fields[k])
        assert err <= MIXED_TOL, (k, err)
    assert all(r["pressure_residual"] < prm.poisson_tol for r in recs)
    assert _projected_divergence(g.room, h.get("u"), h.get("v"), h.get("w")) <= 1e-6
    # the per-step histories follow the reference's to the same bound
    vc = np.array([r["velocity_change"] for r in recs])
    assert rel_err(vc[-100:], g.hist["velocity_change"][-100:]) <= 1e-3
    tm = np.array([r["T_mean"] for r in recs])
    assert rel_err(tm, g.hist["T_mean"]) <= 1e-6
    h.close()


def _served_sample():
    """Three rooms of the serving stream (one heated) and two of the batch
    of uneven rooms, the smallest of each, 12 steps each."""
    from ffrb import workloads
    from ffrb.params import params_from_scene
    from ffrb.serve import requests_from_configs
    stream = [rq for rq in workloads.serving_stream()[:64] if np.prod(rq.cfg.room.grid) <= 120_000]
    heated = [rq for rq in stream if rq.cfg.heat_patches][:1]
    plain = [rq for rq in stream if not rq.cfg.heat_patches][:2]
    batch = sorted(workloads.batch_rooms(), key=lambda c: np.prod(c.room.grid))[:2]
    cfgs = [rq.cfg for rq in plain + heated] + batch
    params = [rq.params for rq in plain + heated] + [params_from_scene(c) for c in batch]
    return requests_from_configs(cfgs, params, [0.0] * len(cfgs), 12)


@pytest.mark.parametrize("batched", [False, True])
def test_served_rooms_match_the_oracle(oracle, batched):
    import torch
    from ffrb.serve import Server
    from oracle import new_fields
    reqs = _served_sample()
    free, _ = torch.cuda.mem_get_info()
    srv = Server(mem_budget=int(free * 0.5), max_active=8, keep_fields=True, batched=batched, chunk=5)
    out = {o.rid: o for o in srv.run(reqs, realtime=False)}
    for rq in reqs:
        o = out[rq.rid]
        assert o.steps == rq.max_steps
        fl = new_fields(rq.room)
        ref = rq.params.with_(precision="fp64", poisson="cg")
        oracle.fluid_init(rq.room, ref, fl)
        oracle.fluid_run(rq.room, ref, fl, rq.max_steps)
        for k in "uvwpT":
            err = rel_err(o.fields[k], fl[k])
            assert err <= MIXED_TOL, (rq.rid, k, err)
