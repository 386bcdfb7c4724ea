"""ctypes front-end of the checkers (TEST INFRASTRUCTURE ONLY).

* ``Oracle`` loads ``oracle/libffr_oracle.so``, the plain-C restatement of
  the reference solver (ffr_oracle.c), which needs nothing but gcc.
* ``RefDriver`` loads ``oracle/_ref/libffr_refdriver.so``, the reference's
  own C++ sources compiled by oracle/Makefile, when that build exists.

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
legs may use this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_u8p = C.POINTER(C.c_uint8)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t) if a is not None else None


class _Fan(C.Structure):
    _fields_ = [("i_min", C.c_int), ("i_max", C.c_int), ("j_min", C.c_int), ("j_max", C.c_int),
                ("k_min", C.c_int), ("k_max", C.c_int), ("vel", C.c_double * 3)]


class _Patch(C.Structure):
    _fields_ = [("axis", C.c_int), ("side", C.c_int), ("a_min", C.c_int), ("a_max", C.c_int),
                ("b_min", C.c_int), ("b_max", C.c_int)]


class _Opening(C.Structure):
    _fields_ = [("patch", _Patch), ("T_outside", C.c_double)]


class _Heat(C.Structure):
    _fields_ = [("i_min", C.c_int), ("i_max", C.c_int), ("j_min", C.c_int), ("j_max", C.c_int),
                ("k_min", C.c_int), ("k_max", C.c_int), ("T", C.c_double)]


class _Room(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int), ("dx", C.c_double),
                ("dxv", _dp), ("dyv", _dp), ("dzv", _dp), ("cell_type", _u8p),
                ("nfans", C.c_int), ("fans", C.POINTER(_Fan)),
                ("nout", C.c_int), ("outflows", C.POINTER(_Patch)),
                ("nopen", C.c_int), ("openings", C.POINTER(_Opening)),
                ("nheat", C.c_int), ("heats", C.POINTER(_Heat))]


class _Params(C.Structure):
    _fields_ = [("rho", C.c_double), ("nu", C.c_double), ("dt", C.c_double),
                ("convergence_tol", C.c_double), ("poisson_max_iter", C.c_int),
                ("poisson_tol", C.c_double), ("advection", C.c_int), ("thermal", C.c_int),
                ("T_initial", C.c_double), ("T_target", C.c_double), ("buoyancy", C.c_int),
                ("g_accel", C.c_double), ("beta", C.c_double), ("k_thermal", C.c_double),
                ("cp", C.c_double)]


class _Result(C.Structure):
    _fields_ = [("step", C.c_int), ("velocity_change", C.c_double),
                ("pressure_residual", C.c_double), ("divergence_max", C.c_double),
                ("converged", C.c_int), ("T_mean", C.c_double), ("cg_iterations", C.c_int)]


class _Fields(C.Structure):
    _fields_ = [("u", _dp), ("v", _dp), ("w", _dp), ("p", _dp), ("T", _dp)]


@dataclass
class StepRecord:
    step: int
    velocity_change: float
    pressure_residual: float
    divergence_max: float
    converged: bool
    T_mean: float
    cg_iterations: int
    seconds: float = 0.0


def _records(arr, n) -> List[StepRecord]:
    return [StepRecord(r.step, r.velocity_change, r.pressure_residual, r.divergence_max,
                       bool(r.converged), r.T_mean, r.cg_iterations, getattr(r, "seconds", 0.0))
            for r in arr[:n]]


def new_fields(room) -> dict:
    return {k: np.zeros(int(np.prod(s)), dtype=np.float64) for k, s in room.shapes().items()}


def ensure_built() -> None:
    """Builds libffr_oracle.so with gcc when it is missing (it is plain C)."""
    so = os.path.join(HERE, "libffr_oracle.so")
    src = os.path.join(HERE, "ffr_oracle.c")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        subprocess.check_call(["gcc", "-O2", "-std=c11", "-fPIC", "-shared", "-ffp-contract=off",
                               "-o", so, src, "-lm"])


class Oracle:
    """The plain-C restatement."""

    def __init__(self):
        ensure_built()
        self.lib = C.CDLL(os.path.join(HERE, "libffr_oracle.so"))
        L = self.lib
        L.ffro_fluid_init.argtypes = [C.POINTER(_Room), C.POINTER(_Params), C.POINTER(_Fields)]
        L.ffro_fluid_run.argtypes = [C.POINTER(_Room), C.POINTER(_Params), C.POINTER(_Fields),
                                     C.c_int, C.c_int, C.c_int, C.POINTER(_Result)]
        L.ffro_fluid_run.restype = C.c_int
        L.ffro_laplacian.argtypes = [C.POINTER(_Room), _dp, _dp]
        L.ffro_cg_solve.argtypes = [C.POINTER(_Room), _dp, _dp, C.c_int, C.c_double, _ip]
        L.ffro_cg_solve.restype = C.c_double
        L.ffro_divergence_max.argtypes = [C.POINTER(_Room), _dp, _dp, _dp]
        L.ffro_divergence_max.restype = C.c_double
        L.ffro_lbm_init.argtypes = [C.POINTER(_Room), C.c_double, C.c_double, _dp]
        L.ffro_lbm_run.argtypes = [C.POINTER(_Room), C.c_double, C.c_double, C.c_double, _dp, _dp,
                                   C.POINTER(_Fields), C.c_int, C.c_int, C.c_int, C.POINTER(_Result)]
        L.ffro_lbm_run.restype = C.c_int
        for name in ("ffro_apply_noslip", "ffro_apply_inflow", "ffro_apply_outflow"):
            getattr(L, name).argtypes = [C.POINTER(_Room), _dp, _dp, _dp]

    # -- marshalling
    @staticmethod
    def room(room) -> tuple:
        keep = {}
        keep["dxv"] = np.ascontiguousarray(room.dxv, dtype=np.float64)
        keep["dyv"] = np.ascontiguousarray(room.dyv, dtype=np.float64)
        keep["dzv"] = np.ascontiguousarray(room.dzv, dtype=np.float64)
        keep["ct"] = np.ascontiguousarray(room.cell_type, dtype=np.uint8)
        fans = (_Fan * max(1, len(room.fans)))()
        for i, f in enumerate(room.fans):
            fans[i] = _Fan(*f.box, (C.c_double * 3)(*f.vel))
        outs = (_Patch * max(1, len(room.outflows)))()
        for i, p in enumerate(room.outflows):
            outs[i] = _Patch(p.axis, p.side, p.a_min, p.a_max, p.b_min, p.b_max)
        ops = room.openings
        opens = (_Opening * max(1, len(ops)))()
        for i, p in enumerate(ops):
            opens[i] = _Opening(_Patch(p.axis, p.side, p.a_min, p.a_max, p.b_min, p.b_max), p.T_outside)
        heats = (_Heat * max(1, len(room.heats)))()
        for i, h in enumerate(room.heats):
            heats[i] = _Heat(*h.box, h.T)
        keep.update(fans=fans, outs=outs, opens=opens, heats=heats)
        r = _Room(room.nx, room.ny, room.nz, room.lx / room.nx,
                  _ptr(keep["dxv"]), _ptr(keep["dyv"]), _ptr(keep["dzv"]), _ptr(keep["ct"], _u8p),
                  len(room.fans), fans, len(room.outflows), outs, len(ops), opens,
                  len(room.heats), heats)
        return r, keep

    @staticmethod
    def params(p) -> _Params:
        return _Params(p.rho, p.nu, p.dt, p.convergence_tol, p.poisson_max_iter, p.poisson_tol,
                       p.advection, int(p.thermal), p.T_initial, p.T_target, int(p.buoyancy),
                       p.g_accel, p.beta, p.k_thermal, p.cp)

    @staticmethod
    def _fields(fl) -> _Fields:
        return _Fields(_ptr(fl["u"]), _ptr(fl["v"]), _ptr(fl["w"]), _ptr(fl["p"]), _ptr(fl["T"]))

    # -- API
    def fluid_init(self, room, params, fields) -> None:
        r, keep = self.room(room)
        pr = self.params(params)
        self.lib.ffro_fluid_init(C.byref(r), C.byref(pr), C.byref(self._fields(fields)))

    def fluid_run(self, room, params, fields, nsteps, step0=0, stop_on_converge=False):
        r, keep = self.room(room)
        pr = self.params(params)
        res = (_Result * max(1, nsteps))()
        n = self.lib.ffro_fluid_run(C.byref(r), C.byref(pr), C.byref(self._fields(fields)),
                                    step0, nsteps, int(stop_on_converge), res)
        return _records(res, n)

    def laplacian(self, room, x):
        r, keep = self.room(room)
        x = np.ascontiguousarray(x, dtype=np.float64)
        ax = np.empty_like(x)
        self.lib.ffro_laplacian(C.byref(r), _ptr(x), _ptr(ax))
        return ax

    def cg_solve(self, room, rhs, max_iter, tol):
        r, keep = self.room(room)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        x = np.zeros_like(rhs)
        it = C.c_int(0)
        res = self.lib.ffro_cg_solve(C.byref(r), _ptr(rhs), _ptr(x), max_iter, tol, C.byref(it))
        return x, res, it.value

    def divergence_max(self, room, u, v, w):
        r, keep = self.room(room)
        return self.lib.ffro_divergence_max(C.byref(r), _ptr(u), _ptr(v), _ptr(w))

    def apply_bc(self, which, room, u, v, w):
        r, keep = self.room(room)
        getattr(self.lib, "ffro_apply_" + which)(C.byref(r), _ptr(u), _ptr(v), _ptr(w))

    def lbm_init(self, room, tau, dt):
        r, keep = self.room(room)
        f = np.empty(19 * room.n_cells)
        self.lib.ffro_lbm_init(C.byref(r), tau, dt, _ptr(f))
        return f

    def lbm_run(self, room, tau, dt, tol, f, fields, nsteps, step0=0, stop_on_converge=False):
        r, keep = self.room(room)
        ftmp = np.empty_like(f)
        res = (_Result * max(1, nsteps))()
        n = self.lib.ffro_lbm_run(C.byref(r), tau, dt, tol, _ptr(f), _ptr(ftmp),
                                  C.byref(self._fields(fields)), step0, nsteps,
                                  int(stop_on_converge), res)
        return _records(res, n)


# ------------------------------------------------------------- reference

class _RefRoom(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("xs", _dp), ("ys", _dp), ("zs", _dp),
                ("nsolid", C.c_int), ("solids", _ip),
                ("nfans", C.c_int), ("fan_box", _ip), ("fan_vel", _dp),
                ("nopen", C.c_int), ("open_patch", _ip), ("open_T", _dp),
                ("nout", C.c_int), ("out_patch", _ip),
                ("nheat", C.c_int), ("heat_box", _ip), ("heat_T", _dp)]


class _RefParams(C.Structure):
    _fields_ = [("rho", C.c_double), ("nu", C.c_double), ("dt", C.c_double),
                ("max_steps", C.c_int), ("convergence_tol", C.c_double),
                ("poisson_max_iter", C.c_int), ("poisson_tol", C.c_double),
                ("advection", C.c_int), ("use_openmp", C.c_int), ("thermal", C.c_int),
                ("T_initial", C.c_double), ("T_target", C.c_double), ("buoyancy", C.c_int),
                ("g_accel", C.c_double), ("beta", C.c_double), ("k_thermal", C.c_double),
                ("cp", C.c_double), ("time_budget", C.c_double)]


class _RefResult(C.Structure):
    _fields_ = _Result._fields_ + [("seconds", C.c_double)]


def ref_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libffr_refdriver.so"))


class RefDriver:
    """The reference's own solver sources, compiled (oracle/_ref)."""

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libffr_refdriver.so")
        self.lib = C.CDLL(path)
        self.lib.ffref_fluid_run.argtypes = [C.POINTER(_RefRoom), C.POINTER(_RefParams), C.c_int,
                                             C.c_int, _dp, _dp, _dp, _u8p, _dp, _dp, _dp, _dp, _dp,
                                             C.POINTER(_RefResult)]
        self.lib.ffref_fluid_run.restype = C.c_int
        self.lib.ffref_lbm_run.argtypes = [C.POINTER(_RefRoom), C.c_double, C.c_double, C.c_double,
                                           C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.POINTER(_RefResult)]
        self.lib.ffref_lbm_run.restype = C.c_int
        if hasattr(self.lib, "ffref_poisson_solve"):     # absent from drivers built before it was added
            self.lib.ffref_poisson_solve.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                                     C.c_double, _u8p, _dp, C.c_int, C.c_double, _dp, _ip]
            self.lib.ffref_poisson_solve.restype = C.c_double

    @staticmethod
    def room(room):
        keep = {}

        def ints(rows):
            a = np.ascontiguousarray(np.array(rows, dtype=np.int32).reshape(-1)) if rows else np.zeros(6, np.int32)
            return a

        opens = [p for p in room.outflows if p.is_opening]
        outs = [p for p in room.outflows if not p.is_opening]
        keep["solids"] = ints([list(b) for b in room.solids])
        keep["fan_box"] = ints([list(f.box) for f in room.fans])
        keep["fan_vel"] = np.ascontiguousarray(np.array([f.vel for f in room.fans] or [[0, 0, 0]], dtype=np.float64).reshape(-1))
        keep["open_patch"] = ints([[p.axis, p.side, p.a_min, p.a_max, p.b_min, p.b_max] for p in opens])
        keep["open_T"] = np.array([p.T_outside for p in opens] or [0.0], dtype=np.float64)
        keep["out_patch"] = ints([[p.axis, p.side, p.a_min, p.a_max, p.b_min, p.b_max] for p in outs])
        keep["heat_box"] = ints([list(h.box) for h in room.heats])
        keep["heat_T"] = np.array([h.T for h in room.heats] or [0.0], dtype=np.float64)
        if room.stretched:
            keep["xs"], keep["ys"], keep["zs"] = (np.ascontiguousarray(room.xs), np.ascontiguousarray(room.ys),
                                                  np.ascontiguousarray(room.zs))
        # The driver adds openings before outflows (Scene order); a RoomSpec
        # whose outflows precede its openings cannot be replayed that way.
        if opens and outs and room.outflows.index(outs[0]) < room.outflows.index(opens[-1]):
            raise ValueError("reference driver replays openings before plain outflows")
        r = _RefRoom(room.nx, room.ny, room.nz, room.lx, room.ly, room.lz,
                     _ptr(keep.get("xs")), _ptr(keep.get("ys")), _ptr(keep.get("zs")),
                     len(room.solids), _ptr(keep["solids"], _ip),
                     len(room.fans), _ptr(keep["fan_box"], _ip), _ptr(keep["fan_vel"]),
                     len(opens), _ptr(keep["open_patch"], _ip), _ptr(keep["open_T"]),
                     len(outs), _ptr(keep["out_patch"], _ip),
                     len(room.heats), _ptr(keep["heat_box"], _ip), _ptr(keep["heat_T"]))
        return r, keep

    def fluid_run(self, room, params, nsteps, stop_on_converge=False, init=None, use_openmp=None,
                  time_budget=0.0):
        """Runs the reference FluidSolver; with time_budget > 0 the run stops
        before the first step that starts after that many seconds of stepping
        (each record's ``seconds`` is the wall time of its step())."""
        r, keep = self.room(room)
        omp = params.use_openmp if use_openmp is None else use_openmp
        pr = _RefParams(params.rho, params.nu, params.dt, params.max_steps, params.convergence_tol,
                        params.poisson_max_iter, params.poisson_tol, params.advection, int(omp),
                        int(params.thermal), params.T_initial, params.T_target, int(params.buoyancy),
                        params.g_accel, params.beta, params.k_thermal, params.cp, float(time_budget))
        fl = new_fields(room)
        ct = np.zeros(room.n_cells, dtype=np.uint8)
        res = (_RefResult * max(1, nsteps))()
        init = init or {}
        n = self.lib.ffref_fluid_run(C.byref(r), C.byref(pr), nsteps, int(stop_on_converge),
                                     _ptr(init.get("u")), _ptr(init.get("v")), _ptr(init.get("w")),
                                     _ptr(ct, _u8p), _ptr(fl["u"]), _ptr(fl["v"]), _ptr(fl["w"]),
                                     _ptr(fl["p"]), _ptr(fl["T"]), res)
        return fl, ct, _records(res, n)

    def poisson_solve(self, room, rhs, max_iter, tol):
        """The reference PoissonSolver on the room's cell types as given
        (no BoundaryManager replay): returns (p, residual, iterations)."""
        ct = np.ascontiguousarray(room.cell_type, dtype=np.uint8)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        p = np.zeros(room.n_cells)
        it = C.c_int(0)
        res = self.lib.ffref_poisson_solve(room.nx, room.ny, room.nz, room.lx, room.ly, room.lz, _ptr(ct, _u8p),
                                           _ptr(rhs), max_iter, tol, _ptr(p), C.byref(it))
        return p, res, it.value

    def lbm_run(self, room, tau, dt, tol, nsteps, stop_on_converge=False):
        r, keep = self.room(room)
        fl = new_fields(room)
        res = (_RefResult * max(1, nsteps))()
        n = self.lib.ffref_lbm_run(C.byref(r), tau, dt, tol, nsteps, int(stop_on_converge),
                                   _ptr(fl["u"]), _ptr(fl["v"]), _ptr(fl["w"]), _ptr(fl["p"]), res)
        return fl, _records(res, n)
