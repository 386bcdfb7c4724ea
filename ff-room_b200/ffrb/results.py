"""Result files written from a device-resident room.

The layouts are those of ff-room's ResultStore (python/ff_room/io.py:23-104),
so its own ``ResultStore.load_npz`` reads these archives back into a
SimResult and the CSV has the same columns:

* ``save_npz`` — the five fields in their shaped layouts (u (nx+1, ny, nz),
  v (nx, ny+1, nz), w (nx, ny, nz+1), p and T (nx, ny, nz)), the cell
  types, the run diagnostics and the scene configuration as JSON
  (io.py:23-42);
* ``save_velocity_csv`` — one row per cell: cell-centre coordinates,
  cell-centred velocity and speed (io.py:80-104), the velocity and speed
  formed on the device (``FluidHandle.snapshot``), so only those arrays
  cross PCIe;
* ``log_outcome`` — one JSON line per finished room in ExperimentLog's
  format (io.py:107-140: timestamp, 8-hex config hash, run diagnostics,
  notes, configuration), plus the room's cell count and throughput in
  cell-steps per second of its own residence on the server, so
  ``ExperimentLog.load_all`` reads a serving run's log.

A serving or batched run has no SolverBridge and no Grid on the host;
these writers take the room's handle directly.
"""
from __future__ import annotations

import hashlib
import json
import time
from typing import Optional

import numpy as np

from .scene import SceneConfig


def _diagnostics(last: Optional[dict], steps: int, wall_time_s: float) -> dict:
    last = last or {}
    return {
        "_steps": int(steps),
        "_converged": bool(last.get("converged", False)),
        "_velocity_change": float(last.get("velocity_change", 0.0)),
        "_divergence_max": float(last.get("divergence_max", 0.0)),
        "_T_mean": float(last.get("T_mean", 0.0)),
        "_wall_time_s": float(wall_time_s),
    }


def save_npz(handle, cfg: SceneConfig, path: str, last: Optional[dict] = None, steps: int = 0,
             wall_time_s: float = 0.0) -> None:
    """The room's fields, cell types, diagnostics (``last`` = the final step
    result) and configuration as a compressed archive in ResultStore's
    layout."""
    room = handle.room
    nx, ny, nz = room.nx, room.ny, room.nz
    np.savez_compressed(
        path,
        u_field=handle.get("u").reshape(nx + 1, ny, nz),
        v_field=handle.get("v").reshape(nx, ny + 1, nz),
        w_field=handle.get("w").reshape(nx, ny, nz + 1),
        p_field=handle.get("p").reshape(nx, ny, nz),
        T_field=handle.get("T").reshape(nx, ny, nz),
        cell_type=np.asarray(room.cell_type, dtype=np.uint8).reshape(nx, ny, nz),
        _config_json=np.array(json.dumps(cfg.to_reference_dict())),
        **_diagnostics(last, steps, wall_time_s),
    )


def save_velocity_csv(handle, path: str) -> None:
    """Cell-centred velocity and speed as CSV rows
    ``x_m,y_m,z_m,u_ms,v_ms,w_ms,speed_ms`` (cell centres of a uniform
    grid over the room, as ResultStore writes them)."""
    room = handle.room
    nx, ny, nz = room.nx, room.ny, room.nz
    snap = handle.snapshot(with_velocity=True)
    xs = np.linspace(room.lx / (2 * nx), room.lx * (1 - 1 / (2 * nx)), nx)
    ys = np.linspace(room.ly / (2 * ny), room.ly * (1 - 1 / (2 * ny)), ny)
    zs = np.linspace(room.lz / (2 * nz), room.lz * (1 - 1 / (2 * nz)), nz)
    X, Y, Z = np.meshgrid(xs, ys, zs, indexing="ij")
    vel = snap["vel"]
    rows = np.column_stack([X.ravel(), Y.ravel(), Z.ravel(), vel[..., 0].ravel(), vel[..., 1].ravel(),
                            vel[..., 2].ravel(), snap["speed"].ravel()])
    np.savetxt(path, rows, delimiter=",", header="x_m,y_m,z_m,u_ms,v_ms,w_ms,speed_ms", comments="")


def config_hash(cfg: SceneConfig) -> str:
    """First 8 hex digits of sha256 over the sorted-key JSON of the
    configuration (io.py:118-119); equal to the reference's hash for any
    scene the reference can express."""
    return hashlib.sha256(json.dumps(cfg.to_reference_dict(), sort_keys=True).encode()).hexdigest()[:8]


def log_outcome(path: str, cfg: SceneConfig, outcome, notes: str = "") -> str:
    """Appends one finished server request (``serve.Outcome``) to a JSON
    Lines experiment log and returns its config hash.  wall_time_s is the
    room's time from admission to completion."""
    wall = float(outcome.t_done - outcome.t_admit)
    entry = {
        "timestamp": time.strftime("%Y-%m-%dT%H:%M:%S"),
        "config_hash": config_hash(cfg),
        "steps": int(outcome.steps),
        "converged": bool(outcome.converged),
        "velocity_change": float(outcome.velocity_change),
        "divergence_max": float(outcome.divergence_max),
        "T_mean": float(outcome.T_mean),
        "wall_time_s": wall,
        "notes": notes,
        "config": cfg.to_reference_dict(),
        "cells": int(outcome.cells),
        "cell_steps_per_s": outcome.cells * outcome.steps / wall if wall > 0 else float("nan"),
    }
    with open(path, "a") as fh:
        fh.write(json.dumps(entry) + "\n")
    return entry["config_hash"]
