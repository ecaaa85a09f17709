"""Krylov solve of A11 u = f on the device (pt_solver_* in the C ABI).

``KSPSolveA11`` mirrors how the reference drives the A11 shell inside its
viscous-block solve (FGMRES outer, Chebyshev-Jacobi smoothing with the
eigenvalue window 0.2..1.1 of the estimated lambda_max; see
src/ptatin_driver_linear_ts.c:559-883), with the smoother optionally in FP32.
``pc="cheby_jacobi"`` smooths the fine level only; ``pc="mg"`` is the
reference's geometric V-cycle over re-discretised Q2 levels (coordinates
injected, Gauss-point viscosity projected, the same kernels on each level).
"""
from __future__ import annotations

import ctypes

from . import _capi
from .operator import _dptr

KSP = {"fgmres": 0, "fcg": 1}
PC = {"none": 0, "jacobi": 1, "cheby_jacobi": 2, "mg": 3}


def default_opts(**kw):
    o = _capi.SolveOpts()
    _capi.load().pt_solve_opts_default(ctypes.byref(o))
    for k, v in kw.items():
        if k == "ksp":
            v = KSP[v] if isinstance(v, str) else v
        if k == "pc":
            v = PC[v] if isinstance(v, str) else v
        setattr(o, k, v)
    return o


class KSPSolveA11:
    """A solver bound to one MatStokesMF (its stream, mask and viscosity)."""

    def __init__(self, op, **opts):
        self.op = op
        self.opts = default_opts(**opts)
        h = ctypes.c_void_p()
        _capi.call("pt_solver_create", op.handle, ctypes.byref(self.opts), ctypes.byref(h))
        self._h = h

    def solve(self, b, x):
        """b, x: contiguous float64 CUDA tensors; x is the initial guess and
        receives the solution.  Returns a dict of statistics."""
        import torch
        st = _capi.SolveStats()
        _capi.call("pt_solver_solve_d", self._h, _dptr(b, torch.float64), _dptr(x, torch.float64), ctypes.byref(st))
        return {f: getattr(st, f) for f, _ in _capi.SolveStats._fields_}

    def apply_pc(self, r, z):
        """z = P r (PCApply) with the configured preconditioner; float64 CUDA
        tensors on the op's device."""
        import torch
        _capi.call("pt_solver_apply_pc_d", self._h, _dptr(r, torch.float64), _dptr(z, torch.float64))

    def destroy(self):
        if getattr(self, "_h", None):
            _capi.call("pt_solver_destroy", self._h)
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
