"""Call traces of ff-room's SolverBridge against a `_ffroom_core` module.

The reference's Python front end (python/ff_room/solver_bridge.py:86-281,
scene.py:62-235) cannot run where the reference sources are absent, but
every call it makes into `_ffroom_core` can be recorded where they are
present and replayed anywhere.  ``Recorder`` stands in for the module while
the unmodified ``SolverBridge.run`` / ``run_animated`` execute on the
reference's own compiled module: it forwards every call and records the
sequence -- constructors, attribute reads and writes, method calls, the
per-step callbacks of ``run`` with what the callback read from each
StepResult and which views it took -- with every value the reference
returned.  ``replay`` performs the same sequence on another module (this
repository's drop-in `_ffroom_core`) and compares each returned value with
the recorded one: integers, booleans and strings exactly, floats and arrays
within a relative max-norm tolerance.

Trace format: a JSON list of operations; arrays live in a companion .npz.
  ["attr",  dst, src, name]            dst = src.name       (src -1: the module)
  ["set",   obj, name, value]          obj.name = value
  ["call",  dst, fn, args, kwargs, invocations]
                                       dst = fn(*args, **kwargs); invocations
                                       holds, per callback call made during it,
                                       [arg_id, [ops...]]
  ["check", obj, value]                the value obj stood for when recorded
Values: ["v", x] plain, ["arr", key] array, ["obj", id] an object,
["list", [...]], ["cb", k] a Python callable passed in.
"""
from __future__ import annotations

import json
from typing import Any, Dict, List

import numpy as np

PLAIN = (type(None), bool, int, float, str)


class _Proxy:
    __slots__ = ("_rec", "_id", "_obj")

    def __init__(self, rec, oid, obj):
        object.__setattr__(self, "_rec", rec)
        object.__setattr__(self, "_id", oid)
        object.__setattr__(self, "_obj", obj)

    def __getattr__(self, name):
        return self._rec._attr(self, name)

    def __setattr__(self, name, value):
        self._rec._set(self, name, value)

    def __call__(self, *args, **kwargs):
        return self._rec._call(self, args, kwargs)

    def __repr__(self):
        return self._rec._call(self._rec._attr(self, "__repr__"), (), {})

    def __array__(self, dtype=None, copy=None):
        a = np.asarray(self._obj)
        return a.astype(dtype) if dtype is not None else a


class Recorder:
    """Stands in for the `_ffroom_core` module (install it in sys.modules)."""

    def __init__(self, real_module):
        self._real = real_module
        self.ops: List[list] = []
        self.arrays: Dict[str, np.ndarray] = {}
        self._stack = [self.ops]
        self._n = 0
        self._cbs = 0

    # the module's attributes
    def __getattr__(self, name):
        if name.startswith("__"):
            raise AttributeError(name)
        return self._attr(None, name)

    def _new(self, obj) -> Any:
        """The value a caller sees for a result: plain values as they are
        (recorded), arrays as copies (recorded), everything else a proxy."""
        if isinstance(obj, PLAIN):
            return obj
        if isinstance(obj, np.ndarray):
            return obj
        self._n += 1
        return _Proxy(self, self._n, obj)

    def _enc(self, v):
        if isinstance(v, _Proxy):
            return ["obj", v._id]
        if isinstance(v, bool) or v is None or isinstance(v, (int, str)):
            return ["v", v]
        if isinstance(v, (float, np.floating)):
            return ["v", float(v)]
        if isinstance(v, np.integer):
            return ["v", int(v)]
        if isinstance(v, np.ndarray):
            key = f"a{len(self.arrays)}"
            self.arrays[key] = np.array(v)
            return ["arr", key]
        if isinstance(v, (list, tuple)):
            return ["list", [self._enc(x) for x in v]]
        raise TypeError(f"cannot record a value of type {type(v)}")

    @staticmethod
    def _raw(v):
        if isinstance(v, _Proxy):
            return v._obj
        if isinstance(v, (list, tuple)):
            return type(v)(Recorder._raw(x) for x in v)
        return v

    def _result(self, dst_op: list, raw):
        out = self._new(raw)
        if isinstance(out, _Proxy):
            dst_op[1] = out._id
        else:
            dst_op[1] = 0
            self._stack[-1].append(["check", 0, self._enc(out)])
        return out

    def _attr(self, obj, name):
        src = -1 if obj is None else obj._id
        raw = getattr(self._real if obj is None else obj._obj, name)
        op = ["attr", None, src, name]
        self._stack[-1].append(op)
        return self._result(op, raw)

    def _set(self, obj, name, value):
        self._stack[-1].append(["set", obj._id, name, self._enc(value)])
        setattr(obj._obj, name, self._raw(value))

    def _call(self, fn, args, kwargs):
        invocations: List[list] = []
        enc_args, raw_args = [], []
        for a in args:
            if callable(a) and not isinstance(a, _Proxy):
                k = self._cbs
                self._cbs += 1
                enc_args.append(["cb", k])
                raw_args.append(self._wrap_cb(a, invocations))
            else:
                enc_args.append(self._enc(a))
                raw_args.append(self._raw(a))
        enc_kw = {k: self._enc(v) for k, v in kwargs.items()}
        op = ["call", None, fn._id, enc_args, enc_kw, invocations]
        self._stack[-1].append(op)
        raw = fn._obj(*raw_args, **{k: self._raw(v) for k, v in kwargs.items()})
        return self._result(op, raw)

    def _wrap_cb(self, f, invocations):
        def cb(res):
            p = self._new(res)
            ops: List[list] = []
            invocations.append([p._id if isinstance(p, _Proxy) else 0, ops])
            self._stack.append(ops)
            try:
                return f(p)
            finally:
                self._stack.pop()
        return cb

    def save(self, path_json: str, path_npz: str) -> None:
        with open(path_json, "w") as fh:
            json.dump(self.ops, fh)
        np.savez_compressed(path_npz, **self.arrays)


class Mismatch(AssertionError):
    pass


def replay(module, ops: List[list], arrays, rtol: float = 1e-6, on_value=None) -> Dict[str, int]:
    """Performs the recorded operations on `module`; raises Mismatch at the
    first returned value that differs from the recorded one.  Returns counts
    of the operations and checks performed."""
    objs: Dict[int, Any] = {}
    stats = {"ops": 0, "checks": 0, "callbacks": 0, "arrays": 0}
    last = [None]

    def dec(v, cbs=None):
        kind, x = v
        if kind == "v":
            return x
        if kind == "arr":
            return np.array(arrays[x])
        if kind == "obj":
            return objs[x]
        if kind == "list":
            return [dec(y, cbs) for y in x]
        if kind == "cb":
            return cbs[x]
        raise ValueError(kind)

    def check(got, want_enc):
        stats["checks"] += 1
        kind, x = want_enc
        if kind == "arr":
            stats["arrays"] += 1
            want = np.asarray(arrays[x])
            g = np.asarray(got)
            if g.shape != want.shape:
                raise Mismatch(f"array shape {g.shape} != {want.shape}")
            if want.dtype.kind in "fc":
                scale = max(float(np.max(np.abs(want))) if want.size else 0.0, 1e-300)
                err = float(np.max(np.abs(g - want))) / scale if want.size else 0.0
                if err > rtol:
                    raise Mismatch(f"array differs: max-norm relative {err:.3e} > {rtol:g}")
            elif not np.array_equal(g, want):
                raise Mismatch("integer array differs")
            if on_value is not None:
                on_value(g, want)
            return
        want = dec(want_enc)
        if isinstance(want, float) and not isinstance(got, bool):
            got = float(got)
            if np.isnan(want) and np.isnan(got):
                return
            if abs(got - want) > rtol * max(abs(want), 1e-300) and not (want == 0.0 and abs(got) < 1e-300):
                raise Mismatch(f"value {got!r} != {want!r}")
        elif isinstance(want, str):
            if str(got) != want:
                raise Mismatch(f"text {got!r} != {want!r}")
        elif got != want:
            raise Mismatch(f"value {got!r} != {want!r}")

    def run(op_list):
        for op in op_list:
            stats["ops"] += 1
            kind = op[0]
            if kind == "attr":
                _, dst, src, name = op
                base = module if src == -1 else objs[src]
                val = getattr(base, name)
                last[0] = val
                if dst:
                    objs[dst] = val
            elif kind == "set":
                _, oid, name, v = op
                setattr(objs[oid], name, dec(v))
            elif kind == "call":
                _, dst, fn, args, kwargs, invocations = op
                queue = list(invocations)
                cbs = {}

                def make_cb():
                    def cb(res):
                        if not queue:
                            raise Mismatch("more callbacks than recorded")
                        arg_id, ops_in = queue.pop(0)
                        stats["callbacks"] += 1
                        if arg_id:
                            objs[arg_id] = res
                        run(ops_in)
                    return cb
                for a in args:
                    if a[0] == "cb":
                        cbs[a[1]] = make_cb()
                val = objs[fn](*[dec(a, cbs) for a in args], **{k: dec(v, cbs) for k, v in kwargs.items()})
                if queue:
                    raise Mismatch(f"{len(queue)} recorded callbacks did not happen")
                last[0] = val
                if dst:
                    objs[dst] = val
            elif kind == "check":
                check(last[0], op[2])
            else:
                raise ValueError(kind)

    run(ops)
    return stats
