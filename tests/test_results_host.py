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
