"""Shared test setup: import paths, the `gpu` marker and golden-case loading."""
from __future__ import annotations

import glob
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "ff-room_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _reference_checkout() -> str:
    """The reference checkout the checker was built from: $FFR_REFERENCE, or
    the path oracle/Makefile recorded in oracle/_ref/reference_path.  Empty
    when neither is known; tests that read the reference's own Python
    sources skip then (and wherever the recorded path does not exist)."""
    env = os.environ.get("FFR_REFERENCE")
    if env:
        return env
    try:
        with open(os.path.join(ROOT, "oracle", "_ref", "reference_path")) as fh:
            return fh.read().strip()
    except OSError:
        return ""


REFERENCE = _reference_checkout()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def golden_names():
    """The solver fixtures (the bridge_* call traces are a different kind)."""
    return sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(GOLDEN, "*.npz"))
                  if not os.path.basename(p).startswith("bridge_"))


class Golden:
    """One fixture written by tests/golden/make_golden.py."""

    def __init__(self, name: str):
        from ffrb.params import FluidParams, params_from_scene
        from ffrb.scene import SceneConfig, build_room
        z = np.load(os.path.join(GOLDEN, name + ".npz"))
        self.name = name
        self.meta = json.loads(bytes(z["meta"]).decode())
        self.cfg = SceneConfig.from_dict(self.meta["config"])
        self.room = build_room(self.cfg)
        self.nsteps = int(self.meta["nsteps"])
        self.lbm = self.meta.get("lbm")
        if "params" in self.meta:
            self.params = FluidParams(**self.meta["params"])
        else:
            self.params = params_from_scene(self.cfg)
        self.cell_type = z["cell_type"]
        self.fields = {k[2:]: z[k] for k in z.files if k.startswith("f_")}
        self.hist = {k[2:]: z[k] for k in z.files if k.startswith("h_")}


@pytest.fixture(scope="session")
def oracle():
    from oracle import Oracle
    return Oracle()


def rel_err(a, b) -> float:
    """max-norm relative error |a - b|_inf / max(|b|_inf, tiny)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)) if b.size else 0.0


def gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
