"""Scene building (config -> masks, fans, outflows) and indexing contracts.

The restated scene builder (ffrb.scene) must give the reference Scene's
masks bit for bit (scene.py:72-231, BoundaryManager.cpp:6-44); the synthetic
workloads are pinned through sha256 hashes of the reference's masks.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, REFERENCE
from ffrb import workloads
from ffrb.scene import SceneConfig, build_room, empty_room, FanConfig

HASHES = json.load(open(os.path.join(GOLDEN, "mask_hashes.json")))


def _workload_cfgs():
    out = {}
    cfg, _ = workloads.large_thermal()
    out["large_thermal"] = cfg
    lcfg, _, _ = workloads.lbm_room()
    out["lbm_room"] = lcfg
    for i, c in enumerate(workloads.batch_rooms()[:16]):
        out[f"batch{i}"] = c
    for i, rq in enumerate(workloads.serving_stream()[:16]):
        out[f"serve{i}"] = rq.cfg
    return out


def test_workload_masks_match_reference_hashes():
    cfgs = _workload_cfgs()
    assert set(cfgs) == set(HASHES)
    for name, cfg in cfgs.items():
        ct = build_room(cfg).cell_type
        assert list(cfg.room.grid) == HASHES[name]["grid"]
        assert np.bincount(ct, minlength=4).tolist() == HASHES[name]["counts"], name
        assert hashlib.sha256(ct.tobytes()).hexdigest() == HASHES[name]["sha256"], name


def test_grid_sizes_and_index_uniqueness():
    # restates cpp/tests/test_grid.cpp:8-36
    r = empty_room(4, 5, 6, 4.0, 5.0, 6.0)
    sh = r.shapes()
    assert np.prod(sh["u"]) == 5 * 5 * 6 and np.prod(sh["v"]) == 4 * 6 * 6
    assert np.prod(sh["w"]) == 4 * 5 * 7 and np.prod(sh["p"]) == 4 * 5 * 6
    assert abs(r.dx - 1.0) < 1e-12
    r = empty_room(3, 4, 5, 1.0, 1.0, 1.0)
    idx = {(i * 4 + j) * 5 + k for i in range(3) for j in range(4) for k in range(5)}
    assert len(idx) == 60 and min(idx) == 0 and max(idx) == 59
    with pytest.raises(ValueError):
        empty_room(0, 1, 1, 1.0, 1.0, 1.0)


def test_fan_direction_snapping():
    # restates python/tests/test_config.py TestFanConfig
    f = FanConfig(direction=(90.0, 0.0))
    assert f.snapped_axis() == 1 and f.snapped_sign() == 1.0
    f = FanConfig(direction=(180.0, 0.0))
    assert f.snapped_axis() == 0 and f.snapped_sign() == -1.0
    f = FanConfig(direction=(0.0, 90.0))
    assert f.snapped_axis() == 2
    vx, vy, vz = FanConfig(direction=(90.0, 0.0)).direction_vector()
    assert vx != 0.0 and abs(vx) < 1e-15   # cos(90 deg) is not exactly 0 in floating point


def test_outflow_patch_out_of_range_is_rejected():
    from ffrb.scene import Patch, add_outflow
    r = empty_room(4, 4, 4, 1.0, 1.0, 1.0)
    with pytest.raises(ValueError):
        add_outflow(r, Patch(0, 1, 0, 4, 0, 3))


def test_yaml_examples_roundtrip(tmp_path):
    cfg = workloads.basic_room()
    d = cfg.to_dict()
    again = SceneConfig.from_dict(d)
    assert np.array_equal(build_room(again).cell_type, build_room(cfg).cell_type)


@pytest.mark.skipif(not os.path.isdir(os.path.join(REFERENCE, "python", "ff_room")),
                    reason="reference Python sources not present")
def test_reference_scene_on_this_module():
    """The reference's own Scene builds its masks through this package's
    _ffroom_core (the drop-in), identically to the reference build."""
    import importlib
    import sys
    sys.path.insert(0, os.path.join(REFERENCE, "python"))
    try:
        import _ffroom_core as core
        assert hasattr(core, "__backend__")
        scene_mod = importlib.import_module("ff_room.scene")
        cfg_mod = importlib.import_module("ff_room.config")
        for yml in ("basic_room.yaml", "two_fans.yaml", "summer_cooling.yaml"):
            rc = cfg_mod.SceneConfig.load_yaml(os.path.join(REFERENCE, "examples", yml))
            s = scene_mod.Scene(rc)
            mine = SceneConfig.load_yaml(os.path.join(REFERENCE, "examples", yml))
            assert np.array_equal(s.grid.cell_type_shaped().reshape(-1), build_room(mine).cell_type)
    finally:
        sys.path.remove(os.path.join(REFERENCE, "python"))
