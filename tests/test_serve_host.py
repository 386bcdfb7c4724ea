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
