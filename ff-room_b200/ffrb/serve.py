"""Continuous-batching room server.

Room solves arrive over time; each admitted room gets its own device-resident
solver (an ``ffr_fluid`` handle on its own CUDA stream) and advances in
chunks of steps queued with ``ffr_fluid_enqueue``.  Between chunks the host
loop only polls (``ffr_fluid_poll``), so every active room's kernels are in
flight together and their work overlaps on the GPU.  A room leaves at the
chunk boundary where it converged (max|du|/dt < tol) or reached its step
cap; a waiting room is admitted as soon as a slot and enough device memory
are free (admission by footprint: each room is charged the library's
figure for its device bytes against the budget until it leaves).  Per request the server records arrival,
admission and completion times; the report gives p50/p99 time-to-converged,
room-solves/s and cell-steps/s.

Every room's arithmetic depends only on its own inputs and on the pressure-
solve grid size, which the tuner fixes per size class, so a room gives the
same result alone and in any mix.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np

from . import capi
from .params import FluidParams
from .scene import RoomSpec, SceneConfig, build_room

_library_estimate = capi.estimate_bytes


def estimate_bytes(room: RoomSpec, params: FluidParams) -> int:
    """Device bytes a handle of this room takes: the library's own figure
    (ffr_fluid_estimate_bytes: the handle's allocation plus the transient
    scratch of its multigrid set-up; host arithmetic only, no GPU needed),
    the same figure the native server charges.  Admission charges it
    against the budget while the room is in flight."""
    return _library_estimate(room, params)


def size_class(cells: int) -> int:
    return int(math.log2(max(1, cells)))


@dataclass
class Schedule:
    """How one room runs: the pressure-solve grid (0 = the whole GPU, -k = a
    k-th of its co-resident blocks), or one thread-block cluster of
    `cluster` blocks (1..16, then `blocks` is unused); steps per queued
    chunk; whether each step replays a captured CUDA graph."""
    blocks: int = 0
    chunk: int = 20
    graph: bool = False
    cluster: int = 0


class Tuner:
    """Picks a Schedule per size class (log2 of the cell count).

    ``tune`` times a few candidate schedules on rooms of the class running
    side by side and keeps the fastest by aggregate cell-steps/s; untuned
    classes get the default schedule (default_schedule).  The table can be
    saved and loaded.
    """

    # Candidates for a server, where a room shares the GPU with others: the
    # split solve on the whole GPU, or one thread-block cluster of 4-16
    # blocks per room, each step a graph replay.  The persistent grid-wide
    # solve is left out: a cooperative grid beside other rooms' kernels is
    # only co-resident once they leave room for it, and its grid barriers
    # then wait (up to the device wait limit) on blocks that are not running.
    CANDIDATES = [Schedule(0, 20, True), Schedule(0, 20, True, 16), Schedule(0, 20, True, 8),
                  Schedule(0, 20, True, 4)]

    def __init__(self, table: Optional[Dict[int, Schedule]] = None):
        self.table: Dict[int, Schedule] = dict(table or {})

    # rooms up to this size default to one 16-block cluster per room (many
    # such rooms run side by side); larger ones to the split solve on the
    # whole GPU; both replay each step from a CUDA graph
    CLUSTER_MAX_CELLS = 1 << 20

    @classmethod
    def default_schedule(cls, room: RoomSpec) -> Schedule:
        if room.n_cells <= cls.CLUSTER_MAX_CELLS:
            return Schedule(0, 20, True, 16)
        return Schedule(0, 20, True, 0)

    def schedule(self, room: RoomSpec) -> Schedule:
        return self.table.get(size_class(room.n_cells), self.default_schedule(room))

    @staticmethod
    def _blocks(sched: Schedule, cap: int) -> int:
        return sched.blocks if sched.blocks >= 0 else max(1, cap // (-sched.blocks))

    def tune(self, rooms: List[RoomSpec], params: List[FluidParams], steps: int = 6, concurrent: int = 4) -> None:
        by_class: Dict[int, List[int]] = {}
        for i, r in enumerate(rooms):
            by_class.setdefault(size_class(r.n_cells), []).append(i)
        for cls, idx in by_class.items():
            if cls in self.table:
                continue
            pick = idx[:concurrent]
            best, best_rate = Schedule(), -1.0
            for cand in self.CANDIDATES:
                hs = [capi.FluidHandle(rooms[i], params[i]) for i in pick]
                try:
                    for h, i in zip(hs, pick):
                        apply_schedule(h, cand, rooms[i], params[i])
                        h.advance(1)
                    t0 = time.perf_counter()
                    for h in hs:
                        h.enqueue(steps, False)
                    pend = list(hs)
                    while pend:
                        pend = [h for h in pend if h.poll() is None]
                    dt = time.perf_counter() - t0
                    rate = sum(rooms[i].n_cells for i in pick) * steps / dt
                finally:
                    for h in hs:
                        h.close()
                if rate > best_rate:
                    best, best_rate = cand, rate
            self.table[cls] = best

    def to_json(self) -> dict:
        return {str(k): [v.blocks, v.chunk, v.graph, v.cluster] for k, v in self.table.items()}

    @classmethod
    def from_json(cls, d: dict) -> "Tuner":
        return cls({int(k): Schedule(int(v[0]), int(v[1]), bool(v[2]), int(v[3]) if len(v) > 3 else 0)
                    for k, v in d.items()})


def apply_schedule(h, sched: Schedule, room: RoomSpec, params: FluidParams) -> None:
    """Configures a fresh handle for `sched` (cluster schedules need the
    multigrid solve; other rooms keep the grid schedule)."""
    cap = max(1, (room.n_cells + 255) // 256)
    if sched.cluster and params.poisson == "mgpcg":
        h.set_cluster(sched.cluster)
    elif sched.blocks:
        h.set_blocks(Tuner._blocks(sched, min(cap, 1184)))
    if sched.graph:
        h.use_graph(True)


@dataclass
class Request:
    rid: int
    t_arrival: float            # seconds after the start of the run
    room: RoomSpec
    params: FluidParams
    max_steps: int


@dataclass
class Outcome:
    rid: int
    cells: int
    t_arrival: float
    t_admit: float
    t_done: float
    steps: int
    converged: bool
    velocity_change: float
    fields: Optional[dict] = None
    T_mean: float = float("nan")
    divergence_max: float = float("nan")

    @property
    def latency(self) -> float:
        return self.t_done - self.t_arrival


class _Active:
    def __init__(self, req: Request, sched: Schedule, t_admit: float, keep_fields: bool, split: int = -1,
                 warm_start: bool = True):
        self.req = req
        self.sched = sched
        self.t_admit = t_admit
        self.keep_fields = keep_fields
        self.h = capi.FluidHandle(req.room, req.params)
        if not warm_start and req.params.poisson == "mgpcg":
            self.h.set_warm_start(False)
        if split != -1:
            self.h.set_split(split)
        else:
            apply_schedule(self.h, sched, req.room, req.params)
        self.bytes = self.h.device_bytes()
        self.charge = self.bytes
        self.steps = 0
        self.last = None
        self.queued = 0

    def launch(self) -> None:
        self.queued = min(self.sched.chunk, self.req.max_steps - self.steps)
        self.h.enqueue(self.queued, True)

    def poll(self) -> Optional[bool]:
        """None while running; True when the room is finished."""
        res = self.h.poll()
        if res is None:
            return None
        self.steps += len(res)
        if res:
            self.last = res[-1]
        halted = len(res) < self.queued
        done = halted or self.steps >= self.req.max_steps or (self.last is not None and self.last["converged"])
        return done


class _Group:
    """One batch of the batched engine: its members, its BatchHandle (own
    stream) and whether a chunk of it is in flight."""

    def __init__(self):
        self.members: List["_Active"] = []
        self.batch = None
        self.launched: List["_Active"] = []   # the members of the last chunk (held, so never confused with new ones)
        self.in_flight = False

    def cells(self) -> int:
        return sum(a.req.room.n_cells for a in self.members)

    def launch(self, chunk: int, graph: bool) -> None:
        same = len(self.members) == len(self.launched) and all(a is b for a, b in zip(self.members, self.launched))
        if self.batch is None:
            self.batch = capi.BatchHandle([a.h for a in self.members])
            if graph:
                self.batch.use_graph(True)
        elif not same:
            self.batch.set_rooms([a.h for a in self.members])
        self.launched = list(self.members)
        nsteps = min([chunk] + [a.req.max_steps - a.steps for a in self.members])
        self.batch.enqueue(nsteps, True)
        for a in self.members:
            a.queued = nsteps
            a.result = None
        self.in_flight = True

    def poll(self):
        """None while the chunk runs; else the members that finished (they
        leave the group)."""
        waiting = False
        for a in self.members:
            if a.result is None:
                a.result = a.poll()
                waiting |= a.result is None
        if waiting:
            return None
        self.in_flight = False
        done = [a for a in self.members if a.result]
        self.members = [a for a in self.members if not a.result]
        return done

    def close(self) -> None:
        if self.batch is not None:
            self.batch.close()
            self.batch = None


MAX_PASSED = 16       # admissions past one waiting request before it blocks the queue
SCAN_DEPTH = 256      # queued requests looked at per admission round


class _Admission:
    """Arrival-order admission in which a request that does not fit the
    memory budget lets later requests that fit pass it, at most MAX_PASSED
    of them; after that it blocks the queue until the rooms in flight
    drain enough for it (the same rule as the native server, server.cu)."""

    def __init__(self, requests: List["Request"]):
        self.queue = sorted(requests, key=lambda r: r.t_arrival)
        self.passed = [0] * len(self.queue)
        self.need = [estimate_bytes(r.room, r.params) for r in self.queue]
        self.order = list(range(len(self.queue)))

    def __bool__(self) -> bool:
        return bool(self.order)

    def next_fit(self, now: float, realtime: bool, used: int, budget: int, any_active: bool):
        """The request to admit now, or None (removed from the queue)."""
        for pos, qi in enumerate(self.order[:SCAN_DEPTH]):
            req = self.queue[qi]
            if realtime and req.t_arrival > now:
                return None
            need = self.need[qi]
            if any_active and used + need > budget:
                if self.passed[qi] >= MAX_PASSED:
                    return None
                continue
            for earlier in self.order[:pos]:
                self.passed[earlier] += 1
            del self.order[pos]
            return req, need
        return None


class Server:
    """Continuous-batching server over one GPU.

    batched=False: every room runs on its own stream with its own launches
    (the tuner's schedule per size class); batched=True: all active rooms
    advance together, one launch per stage for the whole set (ffr_batch),
    in chunks of `chunk` steps; rooms join and leave between chunks.  With
    batch_graph (default) each batched step replays one captured CUDA graph
    (recaptured when the membership changes).  batch_cluster (default 16):
    each batched room's whole pressure solve runs on its own thread-block
    cluster of that size, every room's in one launch, and rooms the tuner
    would not solve on a cluster (or above Tuner.CLUSTER_MAX_CELLS) run
    beside the batch on their own streams with the tuner's schedule;
    batch_cluster=0: every room joins the batch with the one-kernel-per-pass
    solve.  batch_groups (default 1): the batched rooms may be spread over
    that many batches, each with its own stream and chunks."""

    def __init__(self, mem_budget: int, max_active: int = 64, tuner: Optional[Tuner] = None,
                 keep_fields: bool = False, batched: bool = False, chunk: int = 10, warm_start: bool = True,
                 batch_graph: bool = True, batch_cluster: int = 16, batch_groups: int = 1):
        self.batch_graph = batch_graph
        self.batch_cluster = batch_cluster
        self.batch_groups = batch_groups
        self.mem_budget = mem_budget
        self.max_active = max_active
        self.tuner = tuner or Tuner()
        self.keep_fields = keep_fields
        self.batched = batched
        self.chunk = chunk
        self.warm_start = warm_start

    def run(self, requests: List[Request], realtime: bool = True) -> List[Outcome]:
        if self.batched:
            return self._run_batched(requests, realtime)
        return self._run_streams(requests, realtime)

    def _finish(self, a: "_Active", t0: float) -> Outcome:
        fields = {k: a.h.get(k) for k in "uvwpT"} if self.keep_fields else None
        t = time.perf_counter() - t0
        o = Outcome(a.req.rid, a.req.room.n_cells, a.req.t_arrival, a.t_admit, t, a.steps,
                    bool(a.last and a.last["converged"]),
                    float(a.last["velocity_change"]) if a.last else float("nan"), fields,
                    float(a.last["T_mean"]) if a.last else float("nan"),
                    float(a.last["divergence_max"]) if a.last else float("nan"))
        a.h.close()
        return o

    def _run_batched(self, requests: List[Request], realtime: bool) -> List[Outcome]:
        """Batch members advance together in chunks (one launch per stage);
        with batch_cluster, rooms above the one-cluster size run beside the
        batch on their own streams with the tuner's schedule.  Members are
        spread over `batch_groups` batches (each on its own stream, so one
        group's predictor and correction overlap another's solve); a member
        joins or leaves its group only between that group's chunks."""
        adm = _Admission(requests)
        groups = [_Group() for _ in range(max(1, self.batch_groups))]
        solo: List[_Active] = []
        used = 0
        out: List[Outcome] = []
        t0 = time.perf_counter()

        def n_active():
            return len(solo) + sum(len(g.members) for g in groups)

        while adm or solo or any(g.members for g in groups):
            now = time.perf_counter() - t0
            idle = [g for g in groups if not g.in_flight]
            while adm and idle and n_active() < self.max_active:
                pick = adm.next_fit(now, realtime, used, self.mem_budget, n_active() > 0)
                if pick is None:
                    break
                req, need = pick
                # the batch takes the rooms the tuner would solve on one
                # cluster; the others run beside it with their own schedule
                sched = self.tuner.schedule(req.room)
                small = (req.room.n_cells <= Tuner.CLUSTER_MAX_CELLS and req.params.poisson == "mgpcg"
                         and sched.cluster > 0)
                if self.batch_cluster and not small:
                    a = _Active(req, sched, now, self.keep_fields, warm_start=self.warm_start)
                    a.launch()
                    solo.append(a)
                else:
                    if self.batch_cluster:
                        a = _Active(req, Schedule(0, self.chunk, False, self.batch_cluster), now, self.keep_fields,
                                    warm_start=self.warm_start)
                    else:
                        a = _Active(req, Schedule(0, self.chunk, False, 0), now, self.keep_fields, split=1,
                                    warm_start=self.warm_start)
                    min(idle, key=lambda g: g.cells()).members.append(a)
                a.charge = need
                used += need
            for g in idle:
                if g.members:
                    g.launch(self.chunk, self.batch_graph)
            progressed = False
            for g in groups:
                if not g.in_flight:
                    continue
                done = g.poll()
                if done is None:
                    continue
                progressed = True
                for a in done:
                    out.append(self._finish(a, t0))
                    used -= a.charge
            still = []
            for a in solo:
                st = a.poll()
                if st is None:
                    still.append(a)
                    continue
                progressed = True
                if st:
                    out.append(self._finish(a, t0))
                    used -= a.charge
                else:
                    a.launch()
                    still.append(a)
            solo = still
            if not progressed:
                time.sleep(0.0002)
        for g in groups:
            g.close()
        return out

    def _run_streams(self, requests: List[Request], realtime: bool = True) -> List[Outcome]:
        adm = _Admission(requests)
        active: List[_Active] = []
        used = 0
        out: List[Outcome] = []
        t0 = time.perf_counter()
        while adm or active:
            now = time.perf_counter() - t0
            # admission: arrived, a free slot, and room in the memory budget
            # (smaller requests may pass a waiting large one, boundedly)
            while adm and len(active) < self.max_active:
                pick = adm.next_fit(now, realtime, used, self.mem_budget, bool(active))
                if pick is None:
                    break
                req, need = pick
                a = _Active(req, self.tuner.schedule(req.room), now, self.keep_fields, warm_start=self.warm_start)
                a.charge = need
                used += need
                a.launch()
                active.append(a)
            progressed = False
            still = []
            for a in active:
                st = a.poll()
                if st is None:
                    still.append(a)
                    continue
                progressed = True
                if st:
                    out.append(self._finish(a, t0))
                    used -= a.charge
                else:
                    a.launch()
                    still.append(a)
            active = still
            if not progressed:
                time.sleep(0.0002)
        return out


def report(outcomes: List[Outcome], makespan: Optional[float] = None) -> dict:
    if not outcomes:
        return {}
    lat = np.array([o.latency for o in outcomes])
    span = makespan if makespan is not None else max(o.t_done for o in outcomes) - min(o.t_arrival for o in outcomes)
    cs = sum(o.cells * o.steps for o in outcomes)
    return {"requests": len(outcomes), "room_solves_per_s": len(outcomes) / span,
            "cell_steps_per_s": cs / span, "p50_s": float(np.percentile(lat, 50)),
            "p99_s": float(np.percentile(lat, 99)), "converged_fraction": float(np.mean([o.converged for o in outcomes])),
            "makespan_s": span, "mean_steps": float(np.mean([o.steps for o in outcomes]))}


def serial_solve(requests: List[Request], params_override: Optional[dict] = None) -> List[Outcome]:
    """The same rooms solved one after another, each to convergence or its
    cap (the serial baseline; with params_override precision="fp64",
    poisson="cg", use_multigrid=False it is the plain FP64 GPU solver, the
    reference's method)."""
    out = []
    t0 = time.perf_counter()
    for req in sorted(requests, key=lambda r: r.t_arrival):
        p = req.params.with_(**(params_override or {}))
        ta = time.perf_counter() - t0
        h = capi.FluidHandle(req.room, p)
        res = h.advance(req.max_steps, stop_on_converge=True)
        h.close()
        out.append(Outcome(req.rid, req.room.n_cells, ta, ta, time.perf_counter() - t0, len(res),
                           bool(res and res[-1]["converged"]), float(res[-1]["velocity_change"]) if res else float("nan"),
                           None, float(res[-1]["T_mean"]) if res else float("nan"),
                           float(res[-1]["divergence_max"]) if res else float("nan")))
    return out


def requests_from_configs(cfgs: List[SceneConfig], params: List[FluidParams], arrivals: List[float],
                          max_steps: int) -> List[Request]:
    return [Request(i, t, build_room(c), p.with_(max_steps=max_steps), max_steps)
            for i, (c, p, t) in enumerate(zip(cfgs, params, arrivals))]
