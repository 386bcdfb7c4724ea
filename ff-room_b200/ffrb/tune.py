"""Autotuning of the per-room schedules on the GPU at hand.

The streams engine of the server runs every room with a Schedule chosen by
its size class (log2 of the cell count).  The candidates
(``Tuner.CANDIDATES``) are the pressure solve one kernel per pass on the
whole GPU, or on one thread-block cluster of 4, 8 or 16 blocks per room,
each step replayed from a CUDA graph (the persistent cooperative solve is
left out: beside other rooms' kernels its grid is not co-resident).
``Tuner.tune`` times the candidates on rooms of each class running side by
side and keeps the fastest by aggregate cell-steps/s.  This module runs it on samples of the
serving stream and of the batch of uneven rooms and stores the table, so
that servers (and the benchmark) start from a tuned table instead of the
built-in defaults:

    python -m ffrb.tune --out ff-room_b200/ffrb/tuned_b200.json

``load_tuned()`` returns a Tuner with the stored table (classes it does not
cover fall back to the default schedule), or the default Tuner when no
table has been stored.
"""
from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from .serve import Tuner, size_class

TUNED_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")


def load_tuned(path: str = TUNED_TABLE) -> Tuner:
    if not os.path.exists(path):
        return Tuner()
    with open(path) as fh:
        d = json.load(fh)
    return Tuner.from_json(d.get("table", d))


def sample_rooms(n_stream: int = 400, n_batch: int = 128, per_class: int = 12):
    """Rooms of the serving stream (seed 11) and of the 256-room batch
    (seed 7): up to per_class of each size class."""
    from . import workloads
    from .params import params_from_scene
    from .scene import build_room
    picked = {}
    for rq in workloads.serving_stream()[:n_stream]:
        picked.setdefault(size_class(int(np.prod(rq.cfg.room.grid))), []).append((rq.cfg, rq.params))
    for c in workloads.batch_rooms()[:n_batch]:
        picked.setdefault(size_class(int(np.prod(c.room.grid))), []).append((c, params_from_scene(c)))
    rooms, params = [], []
    for cls in sorted(picked):
        for cfg, p in picked[cls][:per_class]:
            rooms.append(build_room(cfg))
            params.append(p)
    return rooms, params


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TUNED_TABLE)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--concurrent", type=int, default=12,
                    help="rooms of a class timed side by side (a served GPU holds many)")
    args = ap.parse_args()
    rooms, params = sample_rooms()
    t = Tuner()
    t0 = time.perf_counter()
    t.tune(rooms, params, steps=args.steps, concurrent=args.concurrent)
    took = time.perf_counter() - t0
    out = {"table": t.to_json(), "tuned_seconds": round(took, 1),
           "classes": sorted(int(k) for k in t.to_json()),
           "how": (f"Tuner.tune over {len(rooms)} rooms (serving stream seed 11, batch seed 7), up to "
                   f"{args.concurrent} rooms of a size class side by side, {args.steps} steps per candidate, "
                   f"fastest aggregate cell-steps/s")}
    with open(args.out, "w") as fh:
        json.dump(out, fh, indent=1)
    print(json.dumps(out))


if __name__ == "__main__":
    main()
