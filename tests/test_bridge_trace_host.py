"""The SolverBridge call traces (tests/golden/bridge_*.json) against the
module they were recorded on.

Replaying a trace on the reference's own compiled `_ffroom_core` (the
checker build in oracle/_ref) must reproduce every recorded value exactly:
this pins the recorder and the replayer before the GPU test uses them on
this repository's drop-in module.  Runs in a child process so that the
reference module and the drop-in module (same name) never share one."""
import glob
import json
import os
import subprocess
import sys

import pytest

from conftest import GOLDEN, ROOT

TRACES = sorted(os.path.basename(p)[:-5] for p in glob.glob(os.path.join(GOLDEN, "bridge_*.json")))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")

CHILD = r"""
import importlib.util, json, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from bridge_trace import replay
spec = importlib.util.spec_from_file_location("_ffroom_core", sys.argv[2])
mod = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mod)
ops = json.load(open(sys.argv[3] + ".json"))
arrays = np.load(sys.argv[3] + ".npz")
print(json.dumps(replay(mod, ops, arrays, rtol=0.0)))
"""


def _ref_module():
    hits = glob.glob(os.path.join(REF_DIR, "_ffroom_core*.so"))
    return hits[0] if hits else None


def test_traces_are_present():
    assert {"bridge_basic_room_run", "bridge_basic_room_animated", "bridge_summer_cooling_run",
            "bridge_basic_room_lbm_run"} <= set(TRACES)
    ops = json.load(open(os.path.join(GOLDEN, "bridge_basic_room_run.json")))
    calls = [op for op in ops if op[0] == "call" and op[5]]
    assert len(calls) == 1 and len(calls[0][5]) == 529   # run(): one callback per step


@pytest.mark.skipif(_ref_module() is None, reason="oracle/_ref not built (reference sources absent)")
@pytest.mark.parametrize("name", TRACES)
def test_trace_replays_exactly_on_the_reference_module(name):
    out = subprocess.run([sys.executable, "-c", CHILD, os.path.join(ROOT, "tests"), _ref_module(),
                          os.path.join(GOLDEN, name)], capture_output=True, text=True, timeout=600,
                         env=dict(os.environ, OMP_NUM_THREADS="1"))
    assert out.returncode == 0, out.stderr[-2000:]
    stats = json.loads(out.stdout.strip().splitlines()[-1])
    assert stats["checks"] > 0 and stats["callbacks"] > 0
