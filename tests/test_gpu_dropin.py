"""ff-room's own SolverBridge on this repository's drop-in `_ffroom_core`.

The traces in tests/golden/bridge_*.json hold every call the reference's
unmodified SolverBridge.run / run_animated (python/ff_room/solver_bridge.py:
86-281, with scene.py's Scene building the masks) made into `_ffroom_core`,
with every value the reference returned: the Grid and BoundaryManager
construction, FanBC/OutflowBC/OpeningBC set-up, FluidSolverParams with its
nested poisson parameters and the advection enum, the solver, run() with its
per-step callback (step, velocity change, divergence, T_mean read from each
StepResult), the snapshots run_animated takes inside the callback, and the
fields copied out at the end.  Replaying them on the drop-in module makes the
same calls in the same order; every value must match the reference's within
the FP64 bounds of the other parity tests: 1e-6 max-norm relative for the
projection runs (529 and 120 steps) and 1e-9 for the LBM run; integers,
flags and masks exactly.
"""
import glob
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

pytestmark = pytest.mark.gpu

TRACES = sorted(os.path.basename(p)[:-5] for p in glob.glob(os.path.join(GOLDEN, "bridge_*.json")))


@pytest.mark.parametrize("name", TRACES)
def test_solver_bridge_trace_on_the_dropin_module(name):
    import _ffroom_core as core
    from bridge_trace import replay
    assert getattr(core, "__backend__", "").startswith("b200"), "picked up a module other than the drop-in one"
    ops = json.load(open(os.path.join(GOLDEN, name + ".json")))
    arrays = np.load(os.path.join(GOLDEN, name + ".npz"))
    rtol = 1e-9 if "lbm" in name else 1e-6
    stats = replay(core, ops, arrays, rtol=rtol)
    assert stats["callbacks"] > 0 and stats["arrays"] >= 6
