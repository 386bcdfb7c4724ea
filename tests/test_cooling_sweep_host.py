"""Time-to-cool sweeps on the CPU: the oracle against the reference's
recorded sweep, and the sweep's scene variants and ordering.

tests/golden/cooling_sweep.json holds, per fan placement of
summer_cooling.yaml, the step on which the reference's SolverBridge.run
stopped on its T_target test (FluidSolver.cpp:538-547) and the T_mean of
every step until then.  The target sits at least ``margin`` (> 1e-4 K)
away from every step's T_mean, so a solver within the mixed-precision bound
must stop on the same step."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

FIX = os.path.join(GOLDEN, "cooling_sweep.json")


def _fixture():
    with open(FIX) as fh:
        return json.load(fh)


def _placements(fx):
    from ffrb.sweep import Placement
    return [Placement(p["label"], p["fan"], tuple(p["position"]), tuple(p["direction"]), p["velocity"])
            for p in fx["placements"]]


def test_fixture_shape():
    fx = _fixture()
    reached = [p["reached"] for p in fx["placements"]]
    assert sum(reached) >= 3 and not all(reached)
    assert fx["margin"] > 1e-4
    for p in fx["placements"]:
        assert len(p["T_mean"]) == p["steps"] <= fx["cap"]
        tm = np.array(p["T_mean"])
        if p["reached"]:
            assert tm[-1] <= fx["T_target"] and np.all(tm[:-1] > fx["T_target"])
        else:
            assert p["steps"] == fx["cap"] and np.all(tm > fx["T_target"])


def test_oracle_reproduces_time_to_cool(oracle):
    from ffrb.params import params_from_scene
    from ffrb.scene import SceneConfig, build_room
    from ffrb.sweep import variant
    from oracle import new_fields
    fx = _fixture()
    base = SceneConfig.from_dict(fx["base"])
    for pl, want in zip(_placements(fx), fx["placements"]):
        cfg = variant(base, pl, fx["T_target"], fx["cap"])
        room, prm = build_room(cfg), params_from_scene(cfg)
        fl = new_fields(room)
        oracle.fluid_init(room, prm, fl)
        recs = oracle.fluid_run(room, prm, fl, fx["cap"], stop_on_converge=True)
        assert len(recs) == want["steps"], pl.label
        assert bool(recs[-1].converged) == want["reached"], pl.label
        got = np.array([r.T_mean for r in recs])
        assert np.max(np.abs(got - np.array(want["T_mean"]))) <= 1e-9, pl.label


def test_variants_and_requests():
    from ffrb.scene import SceneConfig
    from ffrb.sweep import Placement, placement_grid, requests, variant
    fx = _fixture()
    base = SceneConfig.from_dict(fx["base"])
    pls = placement_grid([(1.0, 2.0, 0.5), (2.0, 2.0, 0.5)], [(0.0, 0.0), (90.0, 0.0), (180.0, 0.0)])
    assert [p.label for p in pls] == ["p0_d0", "p0_d1", "p0_d2", "p1_d0", "p1_d1", "p1_d2"]
    v = variant(base, pls[4], 31.0, 50)
    assert v.fans[0].position == (2.0, 2.0, 0.5) and v.fans[0].direction == (90.0, 0.0)
    assert base.fans[0].position != v.fans[0].position          # the base is untouched
    assert v.solver.T_target == 31.0 and v.solver.max_steps == 50 and v.metadata["placement"] == "p1_d1"
    reqs = requests(base, pls[:2], 31.0, 50)
    assert [r.max_steps for r in reqs] == [50, 50]
    assert reqs[0].params.precision == "mixed" and reqs[0].params.poisson == "mgpcg"
    assert reqs[0].params.T_target == 31.0 and reqs[0].params.thermal
    nobase = SceneConfig.from_dict(fx["base"])
    nobase.solver.T_target = None
    with pytest.raises(ValueError):
        requests(nobase, [Placement("x")])
    assert requests(nobase, [Placement("x")], T_target=30.0)[0].params.T_target == 30.0


def test_sweep_orders_by_time_to_cool(monkeypatch):
    """Results come back fastest first, then the placements that never
    reached the target; times are steps × dt."""
    from ffrb import sweep
    from ffrb.scene import SceneConfig
    from ffrb.serve import Outcome
    fx = _fixture()
    base = SceneConfig.from_dict(fx["base"])
    steps = {0: (40, True), 1: (80, False), 2: (12, True), 3: (25, True)}

    class FakeServer:
        def run(self, reqs, realtime=True):
            assert not realtime
            return [Outcome(r.rid, r.room.n_cells, 0.0, 0.0, 1.0, steps[r.rid][0], steps[r.rid][1], 0.0, None, 31.0)
                    for r in reversed(reqs)]

    pls = [sweep.Placement(f"v{i}", 0, (1.0 + i, 3.8, 0.9)) for i in range(4)]
    res = sweep.cooling_sweep(base, pls, T_target=31.0, max_steps=80, server=FakeServer())
    assert [r.label for r in res] == ["v2", "v3", "v0", "v1"]
    dt = base.solver.dt
    assert [r.time_to_target_s for r in res] == [12 * dt, 25 * dt, 40 * dt, None]
