"""Continuous-batching server: results alone vs in the mix, admission by
memory footprint, asynchronous chunks and CUDA-graph replay.

A room's arithmetic depends only on its own inputs and its pressure-solve
grid size, so its fields must be bit-identical whether it ran alone or
side by side with other rooms (max |difference| == 0)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_requests(n=5, steps=12):
    from ffrb import workloads
    from ffrb.params import params_from_scene
    from ffrb.serve import requests_from_configs
    cfgs = workloads.batch_rooms(n_rooms=n, seed=3, dims=(12, 28), steps=steps)
    params = [params_from_scene(c) for c in cfgs]
    return requests_from_configs(cfgs, params, [0.0] * n, steps)


def _tuner():
    from ffrb.serve import Schedule, Tuner
    return Tuner({c: Schedule(0, 5, c % 2 == 1, 8 if c % 3 == 0 else 0) for c in range(0, 40)})


_TUNER = None


def test_results_identical_alone_and_in_mix():
    global _TUNER
    _TUNER = _tuner()
    from ffrb import capi
    from ffrb.serve import Server, Tuner, Schedule
    reqs = _small_requests()
    from ffrb.serve import apply_schedule
    alone = {}
    for rq in reqs:
        h = capi.FluidHandle(rq.room, rq.params)
        apply_schedule(h, _TUNER.schedule(rq.room), rq.room, rq.params)
        h.advance(rq.max_steps, stop_on_converge=True)
        alone[rq.rid] = {k: h.get(k) for k in "uvwpT"}
        h.close()
    srv = Server(mem_budget=8 << 30, max_active=8, tuner=_TUNER, keep_fields=True)
    out = srv.run(reqs, realtime=False)
    assert len(out) == len(reqs)
    for o in out:
        for k in "uvwpT":
            assert np.max(np.abs(o.fields[k] - alone[o.rid][k])) == 0.0, (o.rid, k)


def test_admission_by_memory_footprint():
    from ffrb.serve import Server, estimate_bytes
    reqs = _small_requests(6, steps=6)
    budget = int(2.5 * max(estimate_bytes(r.room, r.params) for r in reqs))
    srv = Server(mem_budget=budget, max_active=64)
    out = srv.run(reqs, realtime=False)
    assert len(out) == len(reqs)
    # with room for about two rooms, admissions must wait for completions
    admits = sorted(o.t_admit for o in out)
    dones = sorted(o.t_done for o in out)
    assert admits[-1] >= dones[0]


def test_graph_replay_matches_direct_launches():
    from ffrb import capi
    from conftest import Golden
    g = Golden("c1_quick_10")
    a = capi.FluidHandle(g.room, g.params)
    ra = a.advance(g.nsteps)
    b = capi.FluidHandle(g.room, g.params)
    b.use_graph(True)
    rb = b.advance(g.nsteps)
    assert [r["cg_iterations"] for r in ra] == [r["cg_iterations"] for r in rb]
    for k in "uvwpT":
        assert np.array_equal(a.get(k), b.get(k))


def test_enqueue_poll_stops_on_convergence():
    from ffrb import capi, workloads
    from ffrb.params import params_from_scene
    from ffrb.scene import build_room
    cfg = workloads.basic_room(steps=1000, tol=1.0)
    h = capi.FluidHandle(build_room(cfg), params_from_scene(cfg))
    total = 0
    while True:
        h.enqueue(100, True)
        res = None
        while res is None:
            res = h.poll()
        total += len(res)
        if len(res) < 100:
            break
    assert total == 529


@pytest.mark.parametrize("ctas", [4, 16])
def test_cluster_schedule_tracks_reference(ctas):
    """The multigrid solve inside one thread-block cluster gives the same
    answer as the reference within the mixed-precision bound (1e-4)."""
    from ffrb import capi
    from conftest import Golden, rel_err
    for name in ("c1_quick_10", "vent_quick_10", "oblique_stretch_10"):
        g = Golden(name)
        h = capi.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed"))
        h.set_cluster(ctas)
        h.use_graph(True)
        recs = h.advance(g.nsteps)
        assert len(recs) == g.nsteps
        for k in "uvwpT":
            assert rel_err(h.get(k), g.fields[k]) <= 1e-4, (name, k)
        h.close()


@pytest.mark.parametrize("cluster", [0, 16])
def test_batched_server_results_identical_alone_and_in_mix(cluster):
    """The batched engine: rooms arriving at different times join and leave
    the batch between chunks; each room's fields equal those of the room
    solved alone with the same pressure schedule (the split multigrid form,
    or one 16-block cluster per room) bit for bit."""
    from ffrb import capi
    from ffrb.serve import Server
    reqs = _small_requests(6, steps=9)
    for i, rq in enumerate(reqs):
        rq.t_arrival = 0.0 if i < 3 else 1e-3 * i    # later arrivals join running batches
        rq.max_steps = 4 + i                         # different caps: rooms leave at different chunks
    alone = {}
    for rq in reqs:
        h = capi.FluidHandle(rq.room, rq.params)
        if cluster:
            h.set_cluster(cluster)
        else:
            h.set_split(1)
        h.advance(rq.max_steps, stop_on_converge=True)
        alone[rq.rid] = {k: h.get(k) for k in "uvwpT"}
        h.close()
    srv = Server(mem_budget=8 << 30, max_active=4, keep_fields=True, batched=True, chunk=3, batch_cluster=cluster)
    out = srv.run(reqs, realtime=True)
    assert len(out) == len(reqs)
    for o in out:
        assert o.steps == reqs[o.rid].max_steps
        for k in "uvwpT":
            assert np.array_equal(o.fields[k], alone[o.rid][k]), (o.rid, k)


@pytest.mark.parametrize("precision,poisson", [("mixed", "mgpcg"), ("fp64", "cg")])
def test_cooling_sweep_stops_on_the_reference_steps(precision, poisson):
    """summer_cooling.yaml per fan placement, run to T_target on the server
    (batched for MG-PCG, one stream per room for plain CG): every placement
    stops on the reference's step, or runs to the cap where the reference
    did not reach the target, with T_mean within the mixed bound."""
    import json
    import os
    from conftest import GOLDEN
    from ffrb.scene import SceneConfig
    from ffrb.sweep import Placement, cooling_sweep
    with open(os.path.join(GOLDEN, "cooling_sweep.json")) as fh:
        fx = json.load(fh)
    base = SceneConfig.from_dict(fx["base"])
    pls = [Placement(p["label"], p["fan"], tuple(p["position"]), tuple(p["direction"]), p["velocity"])
           for p in fx["placements"]]
    res = {r.label: r for r in cooling_sweep(base, pls, fx["T_target"], fx["cap"], precision=precision,
                                             poisson=poisson)}
    tol = 1e-4 if precision == "mixed" else 1e-9
    for want in fx["placements"]:
        r = res[want["label"]]
        assert (r.steps, r.reached) == (want["steps"], want["reached"]), (want["label"], r)
        assert abs(r.T_mean - want["T_mean"][-1]) <= tol * abs(want["T_mean"][-1]), (want["label"], r.T_mean)
        if r.reached:
            assert r.time_to_target_s == pytest.approx(want["steps"] * base.solver.dt)


def test_native_server_matches_rooms_alone():
    """The C-ABI server (ffr_server_*): every room ends on exactly the step
    results of the same room run alone with the server's schedule (one
    16-block cluster, CUDA-graph steps), whatever else ran beside it and
    however its steps were chunked; a tight budget admits fewer rooms at a
    time and changes nothing."""
    from ffrb import capi
    reqs = _small_requests(n=6, steps=12)
    reqs = [type(r)(r.rid, r.t_arrival, r.room, r.params.with_(poisson="mgpcg", precision="mixed"), r.max_steps)
            for r in reqs]
    alone = {}
    for rq in reqs:
        h = capi.FluidHandle(rq.room, rq.params)
        h.set_cluster(16)
        h.use_graph(True)
        alone[rq.rid] = h.advance(rq.max_steps, stop_on_converge=True)
        h.close()
    need = max(capi.estimate_bytes(rq.room, rq.params) for rq in reqs)
    for budget, active in ((64 * need, 8), (2 * need, 8)):
        srv = capi.NativeServer(budget, active, 5)
        for rq in reqs:
            srv.submit(rq.rid, rq.room, rq.params, rq.max_steps)
        out = {o["id"]: o for o in srv.drain()}
        srv.close()
        assert sorted(out) == sorted(alone)
        for rid, recs in alone.items():
            o = out[rid]
            assert o["status"] == 0 and o["steps"] == len(recs), (rid, o)
            assert o["velocity_change"] == recs[-1]["velocity_change"] and o["T_mean"] == recs[-1]["T_mean"]
            assert bool(o["converged"]) == bool(recs[-1]["converged"])
