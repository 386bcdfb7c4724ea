"""The benchmark's reference arm on the host (no GPU needed).

`bench.py --impl reference` times the reference's own CPU solver (the
compiled reference in oracle/_ref) and prints one JSON line with the same
metric, unit and workload keys as the GPU arm.  Here it runs on a small
grid of the default workload: the line must carry the contract's keys,
describe the reference's own method, report no host/device copies, and
name the host threads the reference's OpenMP loops really ran on.  Under
torchrun only rank 0 prints.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DRIVER = os.path.join(ROOT, "oracle", "_ref", "libffr_refdriver.so")

needs_ref = pytest.mark.skipif(not os.path.exists(REF_DRIVER),
                               reason="oracle/_ref not built (reference sources absent at build time)")


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--grid", "40,32,12",
           "--steps", "2", "--warmup", "1", "--ref-budget", "5"]
    return subprocess.run(cmd, cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


@needs_ref
def test_reference_arm_line_keeps_the_contract():
    p = _run({"OMP_NUM_THREADS": "2", "RANK": "0", "WORLD_SIZE": "1"})
    assert p.returncode == 0, p.stderr[-2000:]
    line = json.loads(p.stdout.strip().splitlines()[-1])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in line, k
    assert line["impl"] == "reference"
    assert line["unit"] == "cell-steps/s" and line["value"] > 0 and line["higher_is_better"] is True
    # the steps it reports are the steps it timed (at most warm-up + steps)
    assert 1 <= line["steps"] <= 3 and line["steps"] == line["cpu_baseline"]["steps_timed"]
    assert line["ms_per_step"] == pytest.approx(40 * 32 * 12 / line["value"] * 1e3)
    cfg = line["config"]
    assert cfg["workload"] == "large_thermal" and cfg["grid"] == [40, 32, 12]
    assert (cfg["precision"], cfg["poisson"], cfg["pressure_start"]) == ("fp64", "cg", "zero")
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] == 2 and cb["value"] == line["value"]
    assert "2 threads" in cb["sample"]
    assert all(n > 0 for n in cb["cg_iterations"])
    assert line["e2e"] == {"value": line["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


@needs_ref
def test_reference_arm_other_ranks_print_nothing():
    p = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert p.returncode == 0, p.stderr[-2000:]
    assert p.stdout.strip() == ""


def test_host_threads_follow_the_openmp_setting(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("OMP_NUM_THREADS", "3")
    assert bench.host_threads() == 3
    monkeypatch.setenv("OMP_NUM_THREADS", "5,2")      # nested form: the outer level counts
    assert bench.host_threads() == 5
    monkeypatch.delenv("OMP_NUM_THREADS")
    assert bench.host_threads() == len(os.sched_getaffinity(0))


def test_clock_summary_names_the_throttle_reasons():
    """The clocks block of the line: median SM clock under load, the
    maximum, and every throttle reason seen active (nvidia-smi columns in
    the order ClockSampler.Q asks for them)."""
    sys.path.insert(0, ROOT)
    import bench
    c = bench.ClockSampler(0)
    na = "Not Active"
    c.rows = [["0", "1965", "1965", "700.1", "0x0", na, na, na, na],
              ["0", "1800", "1965", "990.0", "0x4", na, na, na, "Active"],
              ["0", "1410", "1965", "990.0", "0x8", na, na, "Active", "Active"]]
    c.stamps = [1.0, 2.0, 3.0]
    c.t_enter, c.t_exit = 1.5, 3.5
    s = c.summary()
    assert s["sm_mhz"] == 1800.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap", "sw_thermal_slowdown"]
    assert s["samples"] == 3 and s["samples_inside_region"] == 2
    assert bench.ClockSampler(0).summary()["reasons"] == ["unsampled"]


def test_solve_traffic_scales_the_measured_figures():
    sys.path.insert(0, ROOT)
    import bench
    it = bench.load_traffic("pcg_split_bytes_per_cell_iter")
    once = bench.load_traffic("pcg_split_bytes_per_cell_once")
    assert it > 0 and once > 0
    assert bench.solve_traffic(True, 1000, 7.0) == pytest.approx(1000 * (once + 7.0 * it))
    assert bench.solve_traffic(False, 1000, 10.0) == pytest.approx(1000 * 10.0 * bench.load_traffic("cg_bytes_per_cell_iter"))
