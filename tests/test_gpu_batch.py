"""Batched rooms (ffr_batch): one launch per stage for every room of a batch.

Each room's blocks do exactly what that room's own launches do with the
one-kernel-per-pass multigrid schedule (same block counts, same order of
every partial sum), so a room's fields and step histories must be
bit-identical whether it ran alone or in a batch, and within the mixed-
precision bound (1e-4 max-norm relative) of the FP64 oracle fixtures."""
import numpy as np
import pytest

from conftest import Golden, rel_err

pytestmark = pytest.mark.gpu

# uniform and stretched grids, openings with thermal transport, heated
# patches, QUICK / upwind / Lax-Wendroff, odd dimensions
NAMES = ["c1_upwind_10", "summer_cooling_10", "oblique_stretch_10", "thermal_small_10", "edge_odd_quick_10",
         "vent_quick_10", "updraft_laxw_10", "two_fans_10"]
HIST = ("step", "velocity_change", "pressure_residual", "divergence_max", "converged", "T_mean", "cg_iterations",
        "flags")


def _handle(g):
    from ffrb import capi
    h = capi.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed"))
    h.set_split(1)
    return h


def test_batch_matches_rooms_alone():
    from ffrb import capi
    gs = [Golden(n) for n in NAMES]
    steps = min(g.nsteps for g in gs)
    alone = []
    for g in gs:
        h = _handle(g)
        recs = h.advance(steps)
        alone.append((recs, {k: h.get(k) for k in "uvwpT"}))
        h.close()
    hs = [_handle(g) for g in gs]
    b = capi.BatchHandle(hs)
    out = b.advance(steps)
    for g, h, recs, (recs_a, fa) in zip(gs, hs, out, alone):
        assert len(recs) == steps
        for ra, rb in zip(recs_a, recs):
            for k in HIST:
                assert ra[k] == rb[k], (g.name, k, ra[k], rb[k])
        for k in "uvwpT":
            assert np.array_equal(h.get(k), fa[k]), (g.name, k)
    b.close()
    for h in hs:
        h.close()


def test_batch_tracks_oracle_across_membership_changes():
    """Chunks on one batch object whose members change between chunks (a
    subset in reverse order, then all again): every room still ends on its
    own 10-step result, within the mixed bound of the FP64 fixtures."""
    from ffrb import capi
    gs = [Golden(n) for n in NAMES]
    hs = [_handle(g) for g in gs]
    b = capi.BatchHandle(hs)
    first = b.advance(4)
    half = hs[::-2]
    b.set_rooms(half)
    mid = dict(zip([id(h) for h in half], b.advance(3)))
    b.set_rooms(hs)
    # the rooms left out of the middle chunk catch up alone
    for h in hs:
        if id(h) not in mid:
            mid[id(h)] = h.advance(3)
    last = b.advance(3)
    for g, h, r1, r3 in zip(gs, hs, first, last):
        assert [r["step"] for r in r1 + mid[id(h)] + r3] == list(range(1, 11))
        if g.nsteps != 10:
            continue
        for k in "uvwpT":
            assert rel_err(h.get(k), g.fields[k]) <= 1e-4, (g.name, k)
    b.close()


def test_batch_room_halts_on_convergence_alone():
    """A room that converges stops (stop_on_converge) while the others run on."""
    from ffrb import capi
    g1, g2 = Golden("c1_upwind_10"), Golden("thermal_small_10")
    h1 = capi.FluidHandle(g1.room, g1.params.with_(poisson="mgpcg", precision="mixed", convergence_tol=1e30))
    h2 = _handle(g2)
    h1.set_split(1)
    b = capi.BatchHandle([h1, h2])
    r1, r2 = b.advance(5, stop_on_converge=True)
    assert len(r1) == 1 and r1[0]["converged"]
    assert len(r2) == 5
    b.close()


def test_batch_rejects_rooms_it_cannot_take():
    from ffrb import capi
    g = Golden("c1_upwind_10")
    h = capi.FluidHandle(g.room, g.params)          # plain CG
    with pytest.raises(capi.FfrError):
        capi.BatchHandle([h])
    h2 = _handle(g)
    with pytest.raises(capi.FfrError):
        capi.BatchHandle([h2, h2])


def test_destroyed_member_leaves_the_batch():
    """Destroying a member removes it from its batch: the batch queues
    nothing (FfrError, before any launch) until its members are set again,
    and then runs on with the others.  A batch that kept the destroyed
    room's pointers would launch on freed memory."""
    from ffrb import capi
    g = Golden("c1_upwind_10")
    for graph in (False, True):
        h1, h2 = _handle(g), _handle(g)
        b = capi.BatchHandle([h1, h2])
        if graph:
            b.use_graph(True)
        first = b.advance(1)[1][0]["step"]
        h1.close()
        with pytest.raises(capi.FfrError):
            b.enqueue(1)
        b.set_rooms([h2])
        (recs,) = b.advance(2)
        assert [r["step"] for r in recs] == [first + 1, first + 2]
        b.close()
        h2.close()


def test_batch_graph_matches_host_paced_batch():
    """The batched step captured as one CUDA graph (the solve a WHILE node
    over the count of rooms still iterating) gives exactly the host-paced
    batch's results, across a membership change (which recaptures it)."""
    from ffrb import capi
    gs = [Golden(n) for n in NAMES]
    steps = min(g.nsteps for g in gs)
    out = {}
    for graph in (False, True):
        hs = [_handle(g) for g in gs]
        b = capi.BatchHandle(hs)
        if graph:
            b.use_graph(True)
        first = b.advance(steps // 2)
        b.set_rooms(hs[::-1])
        second = b.advance(steps - steps // 2)[::-1]
        out[graph] = ([f + s for f, s in zip(first, second)], [{k: h.get(k) for k in "uvwpT"} for h in hs])
        b.close()
        for h in hs:
            h.close()
    for g, ra, rb, fa, fb in zip(gs, out[False][0], out[True][0], out[False][1], out[True][1]):
        assert len(ra) == len(rb) == steps
        for x, y in zip(ra, rb):
            for k in HIST:
                assert x[k] == y[k], (g.name, k, x[k], y[k])
        for k in "uvwpT":
            assert np.array_equal(fa[k], fb[k]), (g.name, k)


def test_batch_of_cluster_rooms_matches_rooms_alone():
    """Rooms on the one-cluster schedule (ffr_fluid_set_cluster(16)) batched:
    every room's whole solve runs on its own cluster, all rooms in one
    launch, and each room ends exactly as when solved alone on that
    schedule, with the step graph and without it."""
    from ffrb import capi
    gs = [Golden(n) for n in NAMES]
    steps = min(g.nsteps for g in gs)

    def cl(g):
        from ffrb import capi as c
        h = c.FluidHandle(g.room, g.params.with_(poisson="mgpcg", precision="mixed"))
        h.set_cluster(16)
        return h

    alone = []
    for g in gs:
        h = cl(g)
        recs = h.advance(steps)
        alone.append((recs, {k: h.get(k) for k in "uvwpT"}))
        h.close()
    for graph in (False, True):
        hs = [cl(g) for g in gs]
        b = capi.BatchHandle(hs)
        if graph:
            b.use_graph(True)
        out = b.advance(steps)
        for g, h, recs, (recs_a, fa) in zip(gs, hs, out, alone):
            assert len(recs) == steps
            for ra, rb in zip(recs_a, recs):
                for k in HIST:
                    assert ra[k] == rb[k], (g.name, graph, k, ra[k], rb[k])
            for k in "uvwpT":
                assert np.array_equal(h.get(k), fa[k]), (g.name, graph, k)
        b.close()
        for h in hs:
            h.close()
