"""ctypes binding of libffroom_cuda.so (include/ffroom.h).

This is the reference-side binding a ctypes caller would add for the C ABI;
``_ffroom_core`` (the pybind11 module) is the other front-end.  The library
is loaded from this package directory and must exist: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import List, Optional

import numpy as np

from .params import FluidParams
from .scene import RoomSpec

PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG, "libffroom_cuda.so")

FFR_OK, FFR_EINVAL, FFR_ENOMEM, FFR_ECUDA, FFR_ETIMEDOUT, FFR_ENOTSUP, FFR_ERANGE = range(7)
FIELD = {"u": 0, "v": 1, "w": 2, "p": 3, "T": 4}
FFR_FLAG_NAN, FFR_FLAG_CG_MAXITER, FFR_FLAG_CG_BREAKDOWN, FFR_FLAG_TIMEOUT = 1, 2, 4, 8
PREC = {"fp64": 0, "mixed": 1}
POISSON = {"cg": 0, "mgpcg": 1}
LBM_STORAGE = {"fp64": 0, "fp32": 1, "fp16": 2}

_dp = C.POINTER(C.c_double)


class FfrError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"[{status}] {msg}")
        self.status = status


class Fan(C.Structure):
    _fields_ = [("i_min", C.c_int), ("i_max", C.c_int), ("j_min", C.c_int), ("j_max", C.c_int),
                ("k_min", C.c_int), ("k_max", C.c_int), ("vel", C.c_double * 3)]


class Patch(C.Structure):
    _fields_ = [("axis", C.c_int), ("side", C.c_int), ("a_min", C.c_int), ("a_max", C.c_int),
                ("b_min", C.c_int), ("b_max", C.c_int), ("is_opening", C.c_int),
                ("T_outside", C.c_double)]


class HeatPatch(C.Structure):
    _fields_ = [("i_min", C.c_int), ("i_max", C.c_int), ("j_min", C.c_int), ("j_max", C.c_int),
                ("k_min", C.c_int), ("k_max", C.c_int), ("T", C.c_double)]


class RoomDesc(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("lx", C.c_double), ("ly", C.c_double), ("lz", C.c_double),
                ("dxv", _dp), ("dyv", _dp), ("dzv", _dp), ("cell_type", C.POINTER(C.c_uint8)),
                ("nfans", C.c_int), ("fans", C.POINTER(Fan)),
                ("npatches", C.c_int), ("patches", C.POINTER(Patch)),
                ("nheat", C.c_int), ("heats", C.POINTER(HeatPatch))]


class FluidParamsC(C.Structure):
    _fields_ = [("rho", C.c_double), ("nu", C.c_double), ("dt", C.c_double),
                ("max_steps", C.c_int), ("convergence_tol", C.c_double),
                ("poisson_max_iter", C.c_int), ("poisson_tol", C.c_double),
                ("advection", C.c_int), ("use_multigrid", C.c_int), ("thermal", C.c_int),
                ("T_initial", C.c_double), ("T_target", C.c_double), ("buoyancy", C.c_int),
                ("g_accel", C.c_double), ("beta", C.c_double), ("k_thermal", C.c_double),
                ("cp", C.c_double), ("precision", C.c_int), ("poisson", C.c_int)]


class StepResultC(C.Structure):
    _fields_ = [("step", C.c_int), ("velocity_change", C.c_double),
                ("pressure_residual", C.c_double), ("divergence_max", C.c_double),
                ("converged", C.c_int), ("T_mean", C.c_double), ("cg_iterations", C.c_int),
                ("flags", C.c_int)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Fields(C.Structure):
    _fields_ = [("u", _dp), ("v", _dp), ("w", _dp), ("p", _dp)]


_lib = None


class OutcomeC(C.Structure):
    _fields_ = [("id", C.c_longlong), ("cells", C.c_longlong), ("status", C.c_int), ("steps", C.c_int),
                ("converged", C.c_int), ("velocity_change", C.c_double), ("divergence_max", C.c_double),
                ("T_mean", C.c_double), ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


def lib():
    """Loads the library once; raises when it is missing (no CPU fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run ff-room_b200/build.py")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        sigs = {
            "ffr_status_string": ([C.c_int], C.c_char_p),
            "ffr_last_error": ([], C.c_char_p),
            "ffr_version": ([], C.c_char_p),
            "ffr_launch_count": ([], C.c_ulonglong),
            "ffr_fluid_create": ([C.POINTER(RoomDesc), C.POINTER(FluidParamsC), C.POINTER(Fields), C.POINTER(vp)], C.c_int),
            "ffr_fluid_destroy": ([vp], C.c_int),
            "ffr_fluid_step": ([vp, C.POINTER(StepResultC)], C.c_int),
            "ffr_fluid_advance": ([vp, C.c_int, C.c_int, C.POINTER(StepResultC), C.POINTER(C.c_int)], C.c_int),
            "ffr_fluid_divergence_max": ([vp, _dp], C.c_int),
            "ffr_fluid_current_step": ([vp, C.POINTER(C.c_int)], C.c_int),
            "ffr_fluid_get_field": ([vp, C.c_int, _dp], C.c_int),
            "ffr_fluid_set_field": ([vp, C.c_int, _dp], C.c_int),
            "ffr_fluid_field_dev": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
            "ffr_fluid_synchronize": ([vp], C.c_int),
            "ffr_poisson_create": ([C.POINTER(RoomDesc), C.c_int, C.c_double, C.POINTER(vp)], C.c_int),
            "ffr_poisson_destroy": ([vp], C.c_int),
            "ffr_poisson_solve_dev": ([vp, vp, vp, vp, _dp, C.POINTER(C.c_int)], C.c_int),
            "ffr_poisson_solve": ([vp, _dp, _dp, _dp, C.POINTER(C.c_int)], C.c_int),
            "ffr_poisson_apply": ([vp, _dp, _dp], C.c_int),
            "ffr_lbm_create": ([C.POINTER(RoomDesc), C.c_double, C.c_int, C.c_double, C.c_double, C.c_int,
                                C.POINTER(Fields), C.POINTER(vp)], C.c_int),
            "ffr_lbm_destroy": ([vp], C.c_int),
            "ffr_lbm_step": ([vp, C.POINTER(StepResultC)], C.c_int),
            "ffr_lbm_advance": ([vp, C.c_int, C.c_int, C.POINTER(StepResultC), C.POINTER(C.c_int)], C.c_int),
            "ffr_lbm_divergence_max": ([vp, _dp], C.c_int),
            "ffr_lbm_current_step": ([vp, C.POINTER(C.c_int)], C.c_int),
            "ffr_lbm_get_field": ([vp, C.c_int, _dp], C.c_int),
            "ffr_lbm_set_field": ([vp, C.c_int, _dp], C.c_int),
            "ffr_lbm_synchronize": ([vp], C.c_int),
            "ffr_fluid_stream": ([vp, C.POINTER(vp)], C.c_int),
            "ffr_fluid_profile": ([vp, C.c_int], C.c_int),
            "ffr_fluid_profile_read": ([vp, _dp, C.POINTER(C.c_longlong)], C.c_int),
            "ffr_lbm_stream": ([vp, C.POINTER(vp)], C.c_int),
            "ffr_lbm_profile": ([vp, C.c_int], C.c_int),
            "ffr_lbm_profile_read": ([vp, _dp, C.POINTER(C.c_longlong)], C.c_int),
            "ffr_fluid_enqueue": ([vp, C.c_int, C.c_int], C.c_int),
            "ffr_fluid_poll": ([vp, C.POINTER(StepResultC), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)], C.c_int),
            "ffr_fluid_set_blocks": ([vp, C.c_int], C.c_int),
            "ffr_fluid_device_bytes": ([vp, C.POINTER(C.c_size_t)], C.c_int),
            "ffr_fluid_use_graph": ([vp, C.c_int], C.c_int),
            "ffr_fluid_set_cluster": ([vp, C.c_int], C.c_int),
            "ffr_fluid_time_pressure": ([vp, C.c_int, _dp, C.POINTER(C.c_int)], C.c_int),
            "ffr_fluid_set_split": ([vp, C.c_int], C.c_int),
            "ffr_fluid_set_warm_start": ([vp, C.c_int], C.c_int),
            "ffr_fluid_snapshot": ([vp, _dp, _dp, _dp, _dp], C.c_int),
            "ffr_batch_create": ([C.POINTER(vp), C.c_int, C.POINTER(vp)], C.c_int),
            "ffr_batch_destroy": ([vp], C.c_int),
            "ffr_batch_set_rooms": ([vp, C.POINTER(vp), C.c_int], C.c_int),
            "ffr_batch_size": ([vp, C.POINTER(C.c_int)], C.c_int),
            "ffr_batch_enqueue": ([vp, C.c_int, C.c_int], C.c_int),
            "ffr_batch_use_graph": ([vp, C.c_int], C.c_int),
            "ffr_fluid_estimate_bytes": ([C.POINTER(RoomDesc), C.POINTER(FluidParamsC), C.POINTER(C.c_size_t)],
                                         C.c_int),
            "ffr_server_create": ([C.c_size_t, C.c_int, C.c_int, C.POINTER(vp)], C.c_int),
            "ffr_server_destroy": ([vp], C.c_int),
            "ffr_server_submit": ([vp, C.c_longlong, C.POINTER(RoomDesc), C.POINTER(FluidParamsC), C.c_int],
                                  C.c_int),
            "ffr_server_progress": ([vp, C.POINTER(OutcomeC), C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)],
                                    C.c_int),
            "ffr_server_drain": ([vp, C.POINTER(OutcomeC), C.c_int, C.POINTER(C.c_int)], C.c_int),
            "ffr_set_device_wait_limit": ([C.c_double], C.c_int),
            "ffr_selftest_device_wait": ([C.c_int, _dp], C.c_int),
            "ffr_lbm_get_populations": ([vp, _dp, C.POINTER(C.c_int)], C.c_int),
            "ffr_lbm_field_dev": ([vp, C.c_int, C.POINTER(vp)], C.c_int),
            "ffr_lbm_set_populations": ([vp, _dp, C.c_int], C.c_int),
            "ffr_poisson_solve_noalloc": ([C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, vp, vp, vp, C.c_int,
                                           C.c_double, vp, _dp, C.POINTER(C.c_int)], C.c_int),
        }
        for name, (args, res) in sigs.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != FFR_OK:
        L = lib()
        raise FfrError(status, f"{L.ffr_status_string(status).decode()}: {L.ffr_last_error().decode()}")


class DeviceArray:
    """A device buffer of this library seen through __cuda_array_interface__
    (torch.as_tensor(DeviceArray(ptr, n), device="cuda") wraps it without a
    copy); the owning handle must outlive the view."""

    def __init__(self, ptr: int, n: int, typestr: str = "<f8"):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 3}


def launch_count() -> int:
    return int(lib().ffr_launch_count())


def set_device_wait_limit(seconds: float) -> None:
    """Bound of the device-side waits on the current device (0: 4 s)."""
    check(lib().ffr_set_device_wait_limit(float(seconds)))


def selftest_device_wait(blocks: int = 8):
    """(status, elapsed_ms) of the bounded-wait self-test kernel."""
    ms = C.c_double(0.0)
    st = lib().ffr_selftest_device_wait(int(blocks), C.byref(ms))
    return st, ms.value


class _RoomMarshal:
    """Keeps the numpy/ctypes buffers of a RoomDesc alive."""

    def __init__(self, room: RoomSpec):
        self.dxv = np.ascontiguousarray(room.dxv, dtype=np.float64)
        self.dyv = np.ascontiguousarray(room.dyv, dtype=np.float64)
        self.dzv = np.ascontiguousarray(room.dzv, dtype=np.float64)
        self.ct = np.ascontiguousarray(room.cell_type, dtype=np.uint8)
        self.fans = (Fan * max(1, len(room.fans)))()
        for i, f in enumerate(room.fans):
            self.fans[i] = Fan(*f.box, (C.c_double * 3)(*f.vel))
        self.patches = (Patch * max(1, len(room.outflows)))()
        for i, p in enumerate(room.outflows):
            self.patches[i] = Patch(p.axis, p.side, p.a_min, p.a_max, p.b_min, p.b_max,
                                    int(p.is_opening), p.T_outside if p.is_opening else 0.0)
        self.heats = (HeatPatch * max(1, len(room.heats)))()
        for i, h in enumerate(room.heats):
            self.heats[i] = HeatPatch(*h.box, h.T)
        self.desc = RoomDesc(room.nx, room.ny, room.nz, room.lx, room.ly, room.lz,
                             self.dxv.ctypes.data_as(_dp), self.dyv.ctypes.data_as(_dp),
                             self.dzv.ctypes.data_as(_dp),
                             self.ct.ctypes.data_as(C.POINTER(C.c_uint8)),
                             len(room.fans), self.fans, len(room.outflows), self.patches,
                             len(room.heats), self.heats)


def _params(p: FluidParams) -> FluidParamsC:
    return FluidParamsC(p.rho, p.nu, p.dt, p.max_steps, p.convergence_tol, p.poisson_max_iter,
                        p.poisson_tol, p.advection, int(p.use_multigrid), int(p.thermal), p.T_initial,
                        p.T_target, int(p.buoyancy), p.g_accel, p.beta, p.k_thermal, p.cp,
                        PREC[p.precision], POISSON[p.poisson])


def _fields(init: Optional[dict]):
    keep = {}
    if not init:
        return None, keep
    for k in ("u", "v", "w", "p"):
        if init.get(k) is not None:
            keep[k] = np.ascontiguousarray(init[k], dtype=np.float64).reshape(-1)
    f = Fields(*[keep[k].ctypes.data_as(_dp) if k in keep else None for k in ("u", "v", "w", "p")])
    return f, keep


class FluidHandle:
    """One projection solver (ffr_fluid)."""
    _pfx = "ffr_fluid"
    _groups = ("predict", "pressure", "correct", "thermal")
    _ngroups = 4

    def stream(self) -> int:
        p = C.c_void_p()
        check(getattr(lib(), self._pfx + "_stream")(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        check(getattr(lib(), self._pfx + "_profile")(self.h, int(enable)))

    def profile_read(self):
        n = self._ngroups
        ms = (C.c_double * n)()
        la = (C.c_longlong * n)()
        check(getattr(lib(), self._pfx + "_profile_read")(self.h, ms, la))
        return {g: (ms[i], la[i]) for i, g in enumerate(self._groups)}

    def __init__(self, room: RoomSpec, params: FluidParams, init: Optional[dict] = None):
        self.room = room
        self.params = params
        self._m = _RoomMarshal(room)
        pc = _params(params)
        f, keep = _fields(init)
        h = C.c_void_p()
        check(lib().ffr_fluid_create(C.byref(self._m.desc), C.byref(pc), C.byref(f) if f else None,
                                     C.byref(h)))
        self.h = h

    def close(self) -> None:
        if self.h:
            lib().ffr_fluid_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> dict:
        r = StepResultC()
        check(lib().ffr_fluid_step(self.h, C.byref(r)))
        return r.as_dict()

    def advance(self, nsteps: int, stop_on_converge: bool = False, want_results: bool = True) -> List[dict]:
        res = (StepResultC * max(1, nsteps))() if want_results else None
        done = C.c_int(0)
        check(lib().ffr_fluid_advance(self.h, nsteps, int(stop_on_converge), res, C.byref(done)))
        return [res[i].as_dict() for i in range(done.value)] if want_results else [None] * done.value

    def enqueue(self, nsteps: int, stop_on_converge: bool = True) -> None:
        check(lib().ffr_fluid_enqueue(self.h, nsteps, int(stop_on_converge)))
        self._pending = nsteps

    def poll(self):
        """None while the queued chunk runs, else the list of step results."""
        n = max(1, getattr(self, "_pending", 0))
        res = (StepResultC * n)()
        got, ready = C.c_int(0), C.c_int(0)
        check(lib().ffr_fluid_poll(self.h, res, n, C.byref(got), C.byref(ready)))
        if not ready.value:
            return None
        self._pending = 0
        return [res[i].as_dict() for i in range(got.value)]

    def set_blocks(self, blocks: int) -> None:
        check(lib().ffr_fluid_set_blocks(self.h, int(blocks)))

    def snapshot(self, with_velocity: bool = True) -> dict:
        """run_animated's snapshot from the device: {"speed": (nx, ny, nz),
        "vel": (nx, ny, nz, 3)} (vel only with with_velocity)."""
        shape = (self.room.nx, self.room.ny, self.room.nz)
        n = int(np.prod(shape))
        speed = np.empty(n)
        comps = [np.empty(n) for _ in range(3)] if with_velocity else [None, None, None]
        ptr = lambda a: a.ctypes.data_as(_dp) if a is not None else None
        check(lib().ffr_fluid_snapshot(self.h, ptr(comps[0]), ptr(comps[1]), ptr(comps[2]), ptr(speed)))
        out = {"speed": speed.reshape(shape)}
        if with_velocity:
            out["vel"] = np.stack([c.reshape(shape) for c in comps], axis=-1)
        return out

    def set_split(self, mode: int) -> None:
        """Multigrid schedule: 1 kernel per pass, 0 persistent, -1 split in graphs."""
        check(lib().ffr_fluid_set_split(self.h, mode))

    def set_warm_start(self, enable: bool) -> None:
        """Multigrid-PCG start: extrapolated from the last two pressures (default) or zero."""
        check(lib().ffr_fluid_set_warm_start(self.h, int(enable)))

    def time_pressure(self, nrep: int = 3):
        """(mean ms per pressure solve, iterations) re-solving the last step."""
        ms, it = C.c_double(), C.c_int()
        check(lib().ffr_fluid_time_pressure(self.h, nrep, C.byref(ms), C.byref(it)))
        return ms.value, it.value

    def set_cluster(self, ctas: int) -> None:
        check(lib().ffr_fluid_set_cluster(self.h, int(ctas)))

    def use_graph(self, enable: bool = True) -> None:
        check(lib().ffr_fluid_use_graph(self.h, int(enable)))

    def device_bytes(self) -> int:
        b = C.c_size_t(0)
        check(lib().ffr_fluid_device_bytes(self.h, C.byref(b)))
        return b.value

    def get(self, field: str) -> np.ndarray:
        shape = self.room.shapes()[field]
        out = np.empty(int(np.prod(shape)), dtype=np.float64)
        check(lib().ffr_fluid_get_field(self.h, FIELD[field], out.ctypes.data_as(_dp)))
        return out

    def set(self, field: str, arr) -> None:
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(-1)
        check(lib().ffr_fluid_set_field(self.h, FIELD[field], a.ctypes.data_as(_dp)))

    def field_dev(self, field: str) -> int:
        p = C.c_void_p()
        check(lib().ffr_fluid_field_dev(self.h, FIELD[field], C.byref(p)))
        return p.value

    def divergence_max(self) -> float:
        d = C.c_double()
        check(lib().ffr_fluid_divergence_max(self.h, C.byref(d)))
        return d.value

    def current_step(self) -> int:
        s = C.c_int()
        check(lib().ffr_fluid_current_step(self.h, C.byref(s)))
        return s.value

    def synchronize(self) -> None:
        check(lib().ffr_fluid_synchronize(self.h))


class BatchHandle:
    """Several rooms advanced together (ffr_batch): one launch per stage for
    all of them.  Each room's results are polled on its own FluidHandle."""

    def __init__(self, rooms: List["FluidHandle"]):
        self.rooms = list(rooms)
        arr = (C.c_void_p * len(self.rooms))(*[r.h for r in self.rooms])
        h = C.c_void_p()
        check(lib().ffr_batch_create(arr, len(self.rooms), C.byref(h)))
        self.h = h

    def set_rooms(self, rooms: List["FluidHandle"]) -> None:
        arr = (C.c_void_p * len(rooms))(*[r.h for r in rooms])
        check(lib().ffr_batch_set_rooms(self.h, arr, len(rooms)))
        self.rooms = list(rooms)

    def use_graph(self, enable: bool = True) -> None:
        check(lib().ffr_batch_use_graph(self.h, int(enable)))

    def enqueue(self, nsteps: int, stop_on_converge: bool = True) -> None:
        check(lib().ffr_batch_enqueue(self.h, nsteps, int(stop_on_converge)))
        for r in self.rooms:
            r._pending = nsteps

    def advance(self, nsteps: int, stop_on_converge: bool = False) -> List[List[dict]]:
        """Runs nsteps on every room; the step results of each room."""
        self.enqueue(nsteps, stop_on_converge)
        out = []
        for r in self.rooms:
            res = None
            while res is None:
                res = r.poll()
            out.append(res)
        return out

    def close(self) -> None:
        if self.h:
            lib().ffr_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PoissonHandle:
    """ffr_poisson: the pressure solve bound to one room."""

    def __init__(self, room: RoomSpec, max_iter: int, tol: float):
        self.room = room
        self._m = _RoomMarshal(room)
        h = C.c_void_p()
        check(lib().ffr_poisson_create(C.byref(self._m.desc), max_iter, tol, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().ffr_poisson_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def solve(self, rhs):
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        p = np.empty_like(rhs)
        res, it = C.c_double(), C.c_int()
        check(lib().ffr_poisson_solve(self.h, rhs.ctypes.data_as(_dp), p.ctypes.data_as(_dp),
                                      C.byref(res), C.byref(it)))
        return p, res.value, it.value

    def solve_dev(self, rhs_ptr: int, p_ptr: int, stream: int = 0):
        res, it = C.c_double(), C.c_int()
        check(lib().ffr_poisson_solve_dev(self.h, C.c_void_p(rhs_ptr), C.c_void_p(p_ptr),
                                          C.c_void_p(stream) if stream else None, C.byref(res),
                                          C.byref(it)))
        return res.value, it.value

    def apply(self, x):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.empty_like(x)
        check(lib().ffr_poisson_apply(self.h, x.ctypes.data_as(_dp), y.ctypes.data_as(_dp)))
        return y


class LbmHandle:
    """ffr_lbm: the D3Q19 solver."""
    _pfx = "ffr_lbm"
    _groups = ("stream_collide", "faces")
    _ngroups = 2

    def stream(self) -> int:
        p = C.c_void_p()
        check(getattr(lib(), self._pfx + "_stream")(self.h, C.byref(p)))
        return p.value or 0

    def profile(self, enable: bool = True) -> None:
        check(getattr(lib(), self._pfx + "_profile")(self.h, int(enable)))

    def profile_read(self):
        n = self._ngroups
        ms = (C.c_double * n)()
        la = (C.c_longlong * n)()
        check(getattr(lib(), self._pfx + "_profile_read")(self.h, ms, la))
        return {g: (ms[i], la[i]) for i, g in enumerate(self._groups)}

    def __init__(self, room: RoomSpec, tau: float, max_steps: int, tol: float, dt: float,
                 storage: str = "fp64", init: Optional[dict] = None):
        self.room = room
        self._m = _RoomMarshal(room)
        f, keep = _fields(init)
        h = C.c_void_p()
        check(lib().ffr_lbm_create(C.byref(self._m.desc), tau, max_steps, tol, dt, LBM_STORAGE[storage],
                                   C.byref(f) if f else None, C.byref(h)))
        self.h = h

    def close(self):
        if self.h:
            lib().ffr_lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self) -> dict:
        r = StepResultC()
        check(lib().ffr_lbm_step(self.h, C.byref(r)))
        return r.as_dict()

    def advance(self, nsteps: int, stop_on_converge: bool = False) -> List[dict]:
        res = (StepResultC * max(1, nsteps))()
        done = C.c_int(0)
        check(lib().ffr_lbm_advance(self.h, nsteps, int(stop_on_converge), res, C.byref(done)))
        return [res[i].as_dict() for i in range(done.value)]

    def get(self, field: str) -> np.ndarray:
        shape = self.room.shapes()[field]
        out = np.empty(int(np.prod(shape)), dtype=np.float64)
        check(lib().ffr_lbm_get_field(self.h, FIELD[field], out.ctypes.data_as(_dp)))
        return out

    def field_dev(self, field: str) -> int:
        p = C.c_void_p()
        check(lib().ffr_lbm_field_dev(self.h, FIELD[field], C.byref(p)))
        return p.value

    def get_populations(self):
        """(f, step): the kept populations as FP64 f[q*N + c] and the step counter."""
        f = np.empty(19 * self.room.n_cells, dtype=np.float64)
        step = C.c_int(0)
        check(lib().ffr_lbm_get_populations(self.h, f.ctypes.data_as(_dp), C.byref(step)))
        return f, step.value

    def set_populations(self, f, step: int) -> None:
        f = np.ascontiguousarray(f, dtype=np.float64)
        assert f.size == 19 * self.room.n_cells
        check(lib().ffr_lbm_set_populations(self.h, f.ctypes.data_as(_dp), int(step)))

    def divergence_max(self) -> float:
        d = C.c_double()
        check(lib().ffr_lbm_divergence_max(self.h, C.byref(d)))
        return d.value

    def synchronize(self) -> None:
        check(lib().ffr_lbm_synchronize(self.h))


def poisson_solve_noalloc(room: RoomSpec, cell_type_ptr: int, rhs_ptr: int, p_ptr: int, max_iter: int,
                          tol: float, stream: int = 0):
    """ffr_poisson_solve_noalloc on device buffers (cell types, rhs, p)."""
    dxv = np.ascontiguousarray(room.dxv, dtype=np.float64)
    dyv = np.ascontiguousarray(room.dyv, dtype=np.float64)
    dzv = np.ascontiguousarray(room.dzv, dtype=np.float64)
    res, it = C.c_double(), C.c_int()
    check(lib().ffr_poisson_solve_noalloc(room.nx, room.ny, room.nz, dxv.ctypes.data_as(_dp),
                                          dyv.ctypes.data_as(_dp), dzv.ctypes.data_as(_dp),
                                          C.c_void_p(cell_type_ptr), C.c_void_p(rhs_ptr), C.c_void_p(p_ptr),
                                          max_iter, tol, C.c_void_p(stream) if stream else None,
                                          C.byref(res), C.byref(it)))
    return res.value, it.value


def estimate_bytes(room: RoomSpec, params: FluidParams) -> int:
    """Device bytes a FluidHandle of this room would take (ffr_fluid_estimate_bytes)."""
    m = _RoomMarshal(room)
    pc = _params(params)
    b = C.c_size_t()
    check(lib().ffr_fluid_estimate_bytes(C.byref(m.desc), C.byref(pc), C.byref(b)))
    return int(b.value)


class NativeServer:
    """The continuous-batching server of the C ABI (ffr_server_*): rooms are
    submitted, admitted by device memory, advanced in chunks on their own
    streams and returned as outcome dicts by progress() / drain()."""

    def __init__(self, mem_budget: int, max_active: int = 64, chunk: int = 20):
        h = C.c_void_p()
        check(lib().ffr_server_create(int(mem_budget), int(max_active), int(chunk), C.byref(h)))
        self.h = h
        self._buf = (OutcomeC * 256)()

    def submit(self, rid: int, room: RoomSpec, params: FluidParams, max_steps: int) -> None:
        m = _RoomMarshal(room)          # the server copies the arrays
        pc = _params(params)
        check(lib().ffr_server_submit(self.h, int(rid), C.byref(m.desc), C.byref(pc), int(max_steps)))

    def progress(self):
        """One non-blocking round: (finished outcomes, requests still pending)."""
        n, pend = C.c_int(), C.c_int()
        check(lib().ffr_server_progress(self.h, self._buf, len(self._buf), C.byref(n), C.byref(pend)))
        return [self._buf[i].as_dict() for i in range(n.value)], pend.value

    def drain(self):
        """Runs every submitted request to the end; all their outcomes."""
        out = []
        while True:
            n = C.c_int()
            check(lib().ffr_server_drain(self.h, self._buf, len(self._buf), C.byref(n)))
            out += [self._buf[i].as_dict() for i in range(n.value)]
            if n.value < len(self._buf):
                break
        rest, pend = self.progress()
        return out + rest

    def close(self) -> None:
        if self.h:
            lib().ffr_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
