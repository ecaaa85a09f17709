"""Serving form: continuously batched viscous solves (pt_server_* in the C ABI).

A ``Server`` takes requests -- A11 u = f on a one-rank box with its own
coordinates, Gauss-point viscosity and Dirichlet mask -- as they arrive,
admits them against a device-memory budget, and advances every admitted
request together with one batched flexible-CG iteration (FP64 residuals,
Chebyshev-Jacobi preconditioner in FP32 or FP64).  There is no counterpart in
the reference, which runs one solve per process; the per-request solve is the
reference's viscous-block configuration (src/ptatin_driver_linear_ts.c).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi


def default_opts(**kw):
    o = _capi.ServerOpts()
    _capi.load().pt_server_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Server:
    """Request loop on the current CUDA device."""

    def __init__(self, **opts):
        self.opts = default_opts(**opts)
        h = ctypes.c_void_p()
        _capi.call("pt_server_create", ctypes.byref(self.opts), ctypes.byref(h))
        self._h = h
        self._held = {}   # id -> arrays that must outlive the request

    def time(self) -> float:
        """Seconds on the server clock."""
        return _capi.load().pt_server_time(self._h)

    def submit(self, rid: int, dims, coords, eta, mask, f) -> np.ndarray:
        """Queue a request; returns the array that receives its solution."""
        mx, my, mz = (int(v) for v in dims)
        coords = np.ascontiguousarray(coords, dtype=np.float64)
        eta = np.ascontiguousarray(eta, dtype=np.float64)
        f = np.ascontiguousarray(f, dtype=np.float64)
        mask = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
        n = 3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1)
        if coords.size != n or f.size != n or eta.size != 27 * mx * my * mz or (mask is not None and mask.size != n):
            raise ValueError("array sizes do not match the box")
        x = np.zeros(n)
        d = _capi.MeshDesc(mx, my, mz, 0, 0, 0, 0, 0, 0)
        _capi.call("pt_server_submit", self._h, int(rid), ctypes.byref(d), coords.ctypes.data, eta.ctypes.data,
                   None if mask is None else mask.ctypes.data, f.ctypes.data, x.ctypes.data)
        self._held[int(rid)] = (coords, eta, mask, f, x)
        return x

    def step(self, iterations: int = 1):
        """Run `iterations` batched iterations; returns (active, queued)."""
        a, q = ctypes.c_int32(), ctypes.c_int32()
        _capi.call("pt_server_step", self._h, int(iterations), ctypes.byref(a), ctypes.byref(q))
        return a.value, q.value

    def done(self):
        """Finished requests since the last call: list of dicts with 'x'."""
        out = []
        while True:
            r = _capi.ServerResult()
            _capi.call("pt_server_next_done", self._h, ctypes.byref(r))
            if r.id < 0:
                return out
            d = {k: getattr(r, k) for k, _ in _capi.ServerResult._fields_}
            d["x"] = self._held.pop(int(r.id))[4]
            out.append(d)

    def stats(self):
        it, la, by = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _capi.call("pt_server_stats", self._h, ctypes.byref(it), ctypes.byref(la), ctypes.byref(by))
        t = [ctypes.c_double() for _ in range(4)]
        _capi.call("pt_server_timers", self._h, *[ctypes.byref(v) for v in t])
        return {"iterations": it.value, "launches": la.value, "bytes_in_use": by.value,
                "host_s": {k: v.value for k, v in zip(("enqueue", "admit", "wait", "retire"), t)}}

    def destroy(self):
        if getattr(self, "_h", None):
            _capi.call("pt_server_destroy", self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.destroy()

    def __del__(self):  # pragma: no cover
        try:
            self.destroy()
        except Exception:
            pass
