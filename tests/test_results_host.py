"""Result files in ff-room's ResultStore layout (no GPU: a stand-in handle)."""
import json

import numpy as np

from ffrb import workloads
from ffrb.results import save_npz, save_velocity_csv
from ffrb.scene import SceneConfig, build_room


class _Handle:
    def __init__(self, room, rng):
        self.room = room
        sh = room.shapes()
        self.f = {k: rng.standard_normal(int(np.prod(sh[k]))) for k in "uvwpT"}

    def get(self, k):
        return self.f[k]

    def snapshot(self, with_velocity=True):
        nx, ny, nz = self.room.nx, self.room.ny, self.room.nz
        u = self.f["u"].reshape(nx + 1, ny, nz)
        v = self.f["v"].reshape(nx, ny + 1, nz)
        w = self.f["w"].reshape(nx, ny, nz + 1)
        vel = np.stack([0.5 * (u[:-1] + u[1:]), 0.5 * (v[:, :-1] + v[:, 1:]), 0.5 * (w[:, :, :-1] + w[:, :, 1:])],
                       axis=-1)
        return {"vel": vel, "speed": np.sqrt((vel ** 2).sum(-1))}


def test_npz_layout_matches_resultstore(tmp_path):
    cfg = workloads.basic_room()
    room = build_room(cfg)
    h = _Handle(room, np.random.default_rng(1))
    path = tmp_path / "r.npz"
    save_npz(h, cfg, str(path), last={"converged": True, "velocity_change": 0.5, "divergence_max": 0.1,
                                      "T_mean": 20.0}, steps=7, wall_time_s=1.5)
    z = np.load(path, allow_pickle=True)
    nx, ny, nz = room.nx, room.ny, room.nz
    assert z["u_field"].shape == (nx + 1, ny, nz) and z["w_field"].shape == (nx, ny, nz + 1)
    assert z["cell_type"].dtype == np.uint8 and z["cell_type"].shape == (nx, ny, nz)
    assert np.array_equal(z["v_field"].ravel(), h.f["v"])
    assert int(z["_steps"]) == 7 and bool(z["_converged"]) and float(z["_wall_time_s"]) == 1.5
    back = SceneConfig.from_dict(json.loads(str(z["_config_json"])))
    assert back.room.grid == cfg.room.grid


def test_velocity_csv_columns(tmp_path):
    cfg = workloads.basic_room()
    room = build_room(cfg)
    h = _Handle(room, np.random.default_rng(2))
    path = tmp_path / "v.csv"
    save_velocity_csv(h, str(path))
    with open(path) as fh:
        assert fh.readline().strip() == "x_m,y_m,z_m,u_ms,v_ms,w_ms,speed_ms"
    rows = np.loadtxt(path, delimiter=",", skiprows=1)
    assert rows.shape == (room.n_cells, 7)
    snap = h.snapshot()
    assert np.allclose(rows[:, 6], snap["speed"].ravel(), rtol=1e-15, atol=1e-15)
    assert abs(rows[0, 0] - room.lx / (2 * room.nx)) < 1e-15


def test_config_json_is_the_reference_dict():
    """The archive's configuration drops this build's keys when they hold
    their defaults and keeps non-default ones where the reference's
    from_dict skips them; ours reads both forms back."""
    cfg = workloads.basic_room()
    d = cfg.to_reference_dict()
    assert "precision" not in d["solver"] and "heat_patches" not in d and "precision" not in d
    assert SceneConfig.from_dict(d) == cfg
    hot, _ = workloads.large_thermal(grid=(40, 32, 12))
    hot.solver.precision = "mixed"
    d = hot.to_reference_dict()
    assert d["precision"] == "mixed" and d["heat_patches"] and "precision" not in d["solver"]
    assert SceneConfig.from_dict(d) == hot


def test_experiment_log_lines(tmp_path):
    from ffrb.results import config_hash, log_outcome
    from ffrb.serve import Outcome
    path = str(tmp_path / "log.jsonl")
    cfg = workloads.basic_room()
    o1 = Outcome(0, 6000, 0.0, 0.5, 2.5, 100, True, 0.2, None, 20.0, 0.01)
    o2 = Outcome(1, 6000, 0.0, 1.0, 1.0, 3, False, 5.0, None, 20.0, 0.02)
    h = log_outcome(path, cfg, o1, notes="a")
    assert h == config_hash(cfg) and len(h) == 8
    log_outcome(path, cfg, o2)
    with open(path) as fh:
        rows = [json.loads(x) for x in fh if x.strip()]
    assert [r["steps"] for r in rows] == [100, 3] and rows[0]["notes"] == "a"
    assert rows[0]["wall_time_s"] == 2.0 and rows[0]["cell_steps_per_s"] == 6000 * 100 / 2.0
    assert np.isnan(rows[1]["cell_steps_per_s"])
    assert rows[0]["divergence_max"] == 0.01 and rows[0]["T_mean"] == 20.0
    assert SceneConfig.from_dict(rows[0]["config"]) == cfg


def test_reference_resultstore_reads_the_archive(tmp_path):
    """With the reference sources at hand, its own ResultStore.load_npz
    reads the archive and its own hash agrees with ours."""
    import hashlib
    import os
    import sys
    import pytest
    from conftest import REFERENCE
    src = os.path.join(REFERENCE, "python")
    if not os.path.isdir(os.path.join(src, "ff_room")):
        pytest.skip("reference sources not present")
    sys.path.insert(0, src)
    try:
        from ff_room.config import SceneConfig as RefSceneConfig
        from ff_room.io import ResultStore
    finally:
        sys.path.remove(src)
    from ffrb.results import config_hash
    cfg = workloads.basic_room()
    room = build_room(cfg)
    h = _Handle(room, np.random.default_rng(3))
    path = str(tmp_path / "r.npz")
    save_npz(h, cfg, path, last={"converged": False, "velocity_change": 1.5, "divergence_max": 0.3,
                                 "T_mean": 0.0}, steps=4, wall_time_s=0.25)
    res = ResultStore.load_npz(path)
    assert res.steps == 4 and res.velocity_change == 1.5 and res.config.room.grid == tuple(cfg.room.grid)
    assert np.array_equal(res.p_field.ravel(), h.f["p"])
    ref = RefSceneConfig.from_dict(cfg.to_reference_dict())
    want = hashlib.sha256(json.dumps(ref.to_dict(), sort_keys=True).encode()).hexdigest()[:8]
    assert config_hash(cfg) == want
