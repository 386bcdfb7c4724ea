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
