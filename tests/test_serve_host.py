"""Host-side parts of the server (no GPU): percentiles, sizing, tuner table."""
from ffrb.serve import Outcome, Schedule, Tuner, estimate_bytes, report, size_class
from ffrb.params import FluidParams
from ffrb.scene import empty_room


def test_report_percentiles_and_rates():
    outs = [Outcome(i, 1000, 0.0, 0.0, float(i + 1), 10, i % 2 == 0, 0.1) for i in range(100)]
    r = report(outs)
    assert r["requests"] == 100 and abs(r["p50_s"] - 50.5) < 1e-9 and abs(r["p99_s"] - 99.01) < 1e-6
    assert abs(r["room_solves_per_s"] - 1.0) < 1e-12 and r["converged_fraction"] == 0.5


def test_estimate_grows_with_cells_and_multigrid():
    small, big = empty_room(8, 8, 8, 1, 1, 1), empty_room(32, 32, 32, 1, 1, 1)
    p = FluidParams()
    assert estimate_bytes(big, p) > estimate_bytes(small, p)
    assert estimate_bytes(big, p.with_(poisson="mgpcg")) > estimate_bytes(big, p)
    assert size_class(1 << 20) == 20


def test_tuner_table_roundtrip():
    t = Tuner({14: Schedule(-4, 20, True), 20: Schedule(0, 10, False)})
    t2 = Tuner.from_json(t.to_json())
    assert t2.table == t.table
    assert t2.schedule(empty_room(16, 32, 32, 1, 1, 1)).blocks == -4


def test_default_schedule_by_room_size():
    small, big = empty_room(64, 64, 64, 1, 1, 1), empty_room(128, 128, 96, 1, 1, 1)
    t = Tuner()
    assert t.schedule(small).cluster == 16 and t.schedule(small).graph
    assert t.schedule(big).cluster == 0 and t.schedule(big).blocks == 0 and t.schedule(big).graph


class _FakeRoom:
    """Stands in for capi.FluidHandle: a chunk of n steps completes at once."""

    def __init__(self, room, params):
        self.steps = 0
        self.pending = 0
        self.split = None
        self.closed = False

    def set_split(self, mode):
        self.split = mode

    def set_cluster(self, ctas):
        self.cluster = ctas

    def set_blocks(self, blocks):
        self.blocks = blocks

    def use_graph(self, enable=True):
        self.graph = enable

    def enqueue(self, n, stop=True):
        self.pending = n

    def poll(self):
        n, self.pending = self.pending, 0
        out = [{"step": self.steps + i + 1, "converged": False, "velocity_change": 1.0, "T_mean": 20.0,
                "divergence_max": 0.0} for i in range(n)]
        self.steps += n
        return out

    def get(self, k):
        return None

    def device_bytes(self):
        return 1

    def close(self):
        self.closed = True


class _FakeBatch:
    log = []

    def __init__(self, rooms):
        self.rooms = list(rooms)
        _FakeBatch.log.append(("create", len(self.rooms)))

    def use_graph(self, enable=True):
        _FakeBatch.log.append(("graph", bool(enable)))

    def set_rooms(self, rooms):
        assert all(not r.closed for r in rooms)
        self.rooms = list(rooms)
        _FakeBatch.log.append(("set", len(self.rooms)))

    def enqueue(self, n, stop):
        assert all(not r.closed for r in self.rooms)
        for r in self.rooms:
            r.pending = n
        _FakeBatch.log.append(("enqueue", n))

    def close(self):
        pass


def test_batched_server_chunks_membership_and_admission(monkeypatch):
    """The batched server's host logic: rooms join between chunks, a chunk
    never runs a room past its cap, finished rooms leave before the next
    chunk, and admission respects the memory budget."""
    import types
    from ffrb import serve
    from ffrb.serve import Request, Server
    fake = types.SimpleNamespace(FluidHandle=_FakeRoom, BatchHandle=_FakeBatch)
    monkeypatch.setattr(serve, "capi", fake)
    _FakeBatch.log = []
    p = FluidParams(poisson="mgpcg")
    rooms = [empty_room(16, 16, 8 + i, 1, 1, 1) for i in range(6)]
    caps = [5, 12, 7, 20, 3, 9]
    reqs = [Request(i, 0.0, rooms[i], p, caps[i]) for i in range(6)]
    need = max(estimate_bytes(r, p) for r in rooms)
    for cluster in (0, 16):
        _FakeBatch.log = []
        srv = Server(mem_budget=3 * need, max_active=8, batched=True, chunk=4, batch_cluster=cluster)
        out = srv.run(reqs, realtime=False)
        assert sorted(o.rid for o in out) == list(range(6))
        for o in out:
            assert o.steps == caps[o.rid]
        sizes = [n for kind, n in _FakeBatch.log if kind in ("create", "set")]
        assert max(sizes) <= 3                       # memory admission: three rooms at a time
        assert all(n <= 4 for kind, n in _FakeBatch.log if kind == "enqueue")


def test_native_server_host_paths():
    """The C-ABI server without a GPU: footprint estimates, the budget
    check at submit, argument errors, and every request coming back as an
    outcome (on a box without a GPU, with the handle's CUDA error as its
    status) instead of a hang."""
    import pytest
    from ffrb import capi
    small, big = empty_room(8, 8, 8, 1, 1, 1), empty_room(32, 32, 32, 1, 1, 1)
    p = FluidParams(poisson="mgpcg", precision="mixed")
    assert capi.estimate_bytes(big, p) > capi.estimate_bytes(small, p)
    assert capi.estimate_bytes(big, p) > capi.estimate_bytes(big, p.with_(poisson="cg"))
    with pytest.raises(capi.FfrError) as e:
        capi.NativeServer(0, 4, 5)
    assert e.value.status == capi.FFR_EINVAL
    tiny = capi.NativeServer(capi.estimate_bytes(small, p), 4, 5)
    with pytest.raises(capi.FfrError) as e:
        tiny.submit(1, big, p, 3)
    assert e.value.status == 6                      # FFR_ERANGE: alone over the budget
    tiny.close()
    srv = capi.NativeServer(1 << 30, 2, 5)
    for i in range(3):
        srv.submit(10 + i, small, p, 4)
    out = srv.drain()
    assert sorted(o["id"] for o in out) == [10, 11, 12]
    for o in out:
        assert o["cells"] == 512 and 0 <= o["steps"] <= 4 and o["t_done"] >= o["t_admit"] >= o["t_submit"]
        assert o["status"] == 0 or o["steps"] == 0
    srv.close()


def test_admission_lets_small_rooms_pass_a_waiting_large_one_boundedly():
    """A request that does not fit lets later ones that fit pass it, at most
    MAX_PASSED of them; then admission stops until memory frees up."""
    from ffrb.serve import MAX_PASSED, Request, _Admission
    p = FluidParams()
    small, big = empty_room(8, 8, 8, 1, 1, 1), empty_room(64, 64, 64, 1, 1, 1)
    reqs = [Request(0, 0.0, small, p, 1), Request(1, 0.1, big, p, 1)]
    reqs += [Request(2 + i, 0.2 + 0.01 * i, small, p, 1) for i in range(MAX_PASSED + 4)]
    adm = _Admission(reqs)
    nb, ns = estimate_bytes(big, p), estimate_bytes(small, p)
    budget = nb + ns - 1          # the big room cannot run beside anything
    used = 0
    got = []
    while True:
        pick = adm.next_fit(1e9, True, used, budget, any_active=True)
        if pick is None:
            break
        got.append(pick[0].rid)
        used = ns                 # one small room in flight at a time
    assert got[0] == 0 and 1 not in got
    assert len(got) == 1 + MAX_PASSED
    # with nothing in flight the waiting big room is next
    pick = adm.next_fit(1e9, True, 0, budget, any_active=False)
    assert pick[0].rid == 1
    # realtime: requests that have not arrived are not admitted
    adm2 = _Admission(reqs)
    assert adm2.next_fit(0.05, True, 0, budget, any_active=False)[0].rid == 0
    assert adm2.next_fit(0.05, True, 0, budget, any_active=False) is None
