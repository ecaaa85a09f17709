"""Host-side mirror of pTatin3D's matrix-free Stokes operator interface.

``MatStokesMF`` plays the role of the reference's ``MatA11MF`` / ``MatStokesMF``
contexts (include/stokes_operators.h:34-64) for one rank: it is created with
an ``a11_op`` name (the ``-a11_op`` switch of src/stokes_operators.c:123-154),
set up with the mesh data, and exposes

* the SpMVOp-level element loops under the reference's names
  (``MFStokesWrapper_A11``, ``MFStokesWrapper_diagA11``, ``MFStokesWrapper_A12``,
  ``MFStokesWrapper_A21``): caller-zeroed Dirichlet input, unassembled output;
* the MatShell-level operators (``MatMult_MFStokes_A11``,
  ``MatGetDiagonal_MFStokes_A11``, ``MatMult_MFStokes_A12``,
  ``MatMult_MFStokes_A21``) with the reference's BC semantics.

Vectors may be numpy arrays (host path: the library copies in and out) or
CUDA ``torch`` tensors (device path, asynchronous on the op's stream unless
``sync=True``).  Every call goes through libpt_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi

try:  # torch is plumbing only (device memory, streams); optional on CPU hosts
    import torch
except Exception:  # pragma: no cover
    torch = None

A11_OPS = ("b200", "b200_stream", "b200_ebe", "b200_colour")


def _is_dev(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _hptr(a: np.ndarray, dtype):
    if not isinstance(a, np.ndarray) or a.dtype != dtype or not a.flags["C_CONTIGUOUS"]:
        raise TypeError(f"expected a C-contiguous numpy {np.dtype(dtype).name} array")
    return ctypes.c_void_p(a.ctypes.data)


def _dptr(t, dtype):
    if t.dtype != dtype or not t.is_contiguous():
        raise TypeError(f"expected a contiguous CUDA tensor of {dtype}")
    return ctypes.c_void_p(t.data_ptr())


class MatStokesMF:
    """One rank's Q2-P1disc Stokes operator on a structured box of mx*my*mz elements."""

    def __init__(self, mx: int, my: int, mz: int, a11_op: str = "b200", stream=None, node_box=None):
        """node_box = (nx, ny, nz, ox, oy, oz): the rank's ghosted local node box
        and the offset of its first element's first node in it (the
        DMDAGetGhostCorners / DMDAGetCornersElementQ2 layout of a multi-rank
        run); None = a one-rank box."""
        self._lib = _capi.load()
        self.dims = (int(mx), int(my), int(mz))
        h = ctypes.c_void_p()
        nb = tuple(int(v) for v in node_box) if node_box is not None else (0, 0, 0, 0, 0, 0)
        _capi.call("pt_op_create", ctypes.byref(_capi.MeshDesc(*self.dims, *nb)), ctypes.byref(h))
        self._h = h
        nv, npr, nel = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _capi.call("pt_op_get_sizes", h, ctypes.byref(nv), ctypes.byref(npr), ctypes.byref(nel))
        self.nvel, self.npres, self.nel = nv.value, npr.value, nel.value
        self.set_a11_op(a11_op)
        if stream is None and torch is not None and torch.cuda.is_available():
            # order device-pointer calls with torch's work on the current stream
            stream = torch.cuda.current_stream()
        if stream is not None:
            self.set_stream(stream)

    # -- lifecycle ---------------------------------------------------------
    def Destroy(self):
        if getattr(self, "_h", None):
            _capi.call("pt_op_destroy", self._h)
            self._h = None

    def __del__(self):  # pragma: no cover
        try:
            self.Destroy()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Destroy()

    @property
    def handle(self):
        return self._h

    def set_stream(self, stream):
        """Use a torch.cuda.Stream (or a raw cudaStream_t int) for all work."""
        raw = stream.cuda_stream if hasattr(stream, "cuda_stream") else int(stream)
        self.stream = stream
        _capi.call("pt_op_set_stream", self._h, ctypes.c_void_p(raw))

    def set_a11_op(self, name: str):
        _capi.call("pt_op_set_a11_kernel", self._h, name.encode())

    @property
    def a11_op(self) -> str:
        return self._lib.pt_op_get_a11_kernel(self._h).decode()

    def set_tiling(self, lz: int):
        """Element layers per z-chunk of the streaming kernel's tiles (0 = default)."""
        _capi.call("pt_op_set_tiling", self._h, int(lz))

    @property
    def tiling(self) -> int:
        return int(self._lib.pt_op_get_tiling(self._h))

    def autotune_tiling(self, X, candidates=(0, 2, 3, 4, 5, 6, 7, 8, 10, 12, 16), reps=5):
        """Pick the z-chunk depth that makes MatMult_MFStokes_A11 fastest on the
        device vector X (CUDA events); leaves it set.  Returns (lz, {lz: ms})."""
        import torch
        Y = torch.empty_like(X)
        st = getattr(self, "stream", None)
        st = st if hasattr(st, "record_event") else torch.cuda.current_stream()
        times = {}
        for lz in candidates:
            self.set_tiling(lz)
            if lz == 0:
                lz = self.tiling
            if lz in times:
                continue
            self.MatMult_MFStokes_A11(X, Y)
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            for _ in range(reps):
                self.MatMult_MFStokes_A11(X, Y)
            b.record(st)
            b.synchronize()
            times[lz] = a.elapsed_time(b) / reps
        best = min(times, key=times.get)
        self.set_tiling(best)
        return best, times

    def launch_count(self) -> int:
        return int(self._lib.pt_op_launch_count(self._h))

    def reset_launch_count(self):
        self._lib.pt_op_reset_launch_count(self._h)

    # -- setup (MatA11MFSetup / SpMVOp_SetUp) -----------------------------
    def SetUp(self, coords, eta=None, mask=None):
        self.set_coords(coords)
        if eta is not None:
            self.set_eta(eta)
        self.set_bc_mask(mask)
        return self

    def set_coords(self, coords):
        if _is_dev(coords):
            _capi.call("pt_op_set_coords_d", self._h, _dptr(coords, torch.float64))
        else:
            c = np.ascontiguousarray(coords, dtype=np.float64)
            if c.size != self.nvel:
                raise ValueError(f"coords has {c.size} entries, expected {self.nvel}")
            _capi.call("pt_op_set_coords_h", self._h, _hptr(c, np.float64))

    def set_eta(self, eta):
        if _is_dev(eta):
            _capi.call("pt_op_set_eta_d", self._h, _dptr(eta, torch.float64))
        else:
            e = np.ascontiguousarray(eta, dtype=np.float64)
            if e.size != 27 * self.nel:
                raise ValueError(f"eta has {e.size} entries, expected {27 * self.nel}")
            _capi.call("pt_op_set_eta_h", self._h, _hptr(e, np.float64))

    def set_bc_mask(self, mask):
        if mask is None:
            _capi.call("pt_op_set_bc_mask_h", self._h, ctypes.c_void_p(None))
            return
        m = np.ascontiguousarray(mask, dtype=np.uint8)
        if m.size != self.nvel:
            raise ValueError(f"mask has {m.size} entries, expected {self.nvel}")
        _capi.call("pt_op_set_bc_mask_h", self._h, _hptr(m, np.uint8))

    # -- generic dispatch ----------------------------------------------------
    def _apply(self, base: str, x, nout: int, out=None, dtype=np.float64):
        if _is_dev(x):
            tdt = torch.float64 if dtype == np.float64 else torch.float32
            if out is None:
                out = torch.empty(nout, dtype=tdt, device=x.device)
            _capi.call(base + "_d", self._h, _dptr(x, tdt), _dptr(out, tdt))
            return out
        x = np.ascontiguousarray(x, dtype=np.float64)
        if out is None:
            out = np.empty(nout, dtype=np.float64)
        _capi.call(base + "_h", self._h, _hptr(x, np.float64), _hptr(out, np.float64))
        return out

    def _check_len(self, x, n, what):
        if (x.numel() if _is_dev(x) else np.size(x)) != n:
            raise ValueError(f"{what} has the wrong length (expected {n})")

    # -- SpMVOp level --------------------------------------------------------
    def MFStokesWrapper_A11(self, ufield, Yu=None):
        self._check_len(ufield, self.nvel, "ufield")
        if _is_dev(ufield) and ufield.dtype == torch.float32:
            if Yu is None:
                Yu = torch.empty_like(ufield)
            _capi.call("pt_a11_apply_f32_d", self._h, _dptr(ufield, torch.float32), _dptr(Yu, torch.float32))
            return Yu
        return self._apply("pt_a11_apply", ufield, self.nvel, Yu)

    def MFStokesWrapper_diagA11(self, Yu=None):
        if Yu is not None and _is_dev(Yu):
            _capi.call("pt_a11_diag_d", self._h, _dptr(Yu, torch.float64))
            return Yu
        out = np.empty(self.nvel) if Yu is None else Yu
        _capi.call("pt_a11_diag_h", self._h, _hptr(out, np.float64))
        return out

    def MFStokesWrapper_A12(self, Xp, Yu=None):
        self._check_len(Xp, self.npres, "Xp")
        return self._apply("pt_a12_apply", Xp, self.nvel, Yu)

    def MFStokesWrapper_A21(self, Xu, Yp=None):
        self._check_len(Xu, self.nvel, "Xu")
        return self._apply("pt_a21_apply", Xu, self.npres, Yp)

    # -- MatShell level ------------------------------------------------------
    def _apply2(self, base: str, u, p, Yu=None, Yp=None):
        self._check_len(u, self.nvel, "u")
        self._check_len(p, self.npres, "p")
        if _is_dev(u):
            Yu = torch.empty_like(u) if Yu is None else Yu
            Yp = torch.empty(self.npres, dtype=torch.float64, device=u.device) if Yp is None else Yp
            _capi.call(base + "_d", self._h, _dptr(u, torch.float64), _dptr(p, torch.float64),
                       _dptr(Yu, torch.float64), _dptr(Yp, torch.float64))
            return Yu, Yp
        u = np.ascontiguousarray(u, dtype=np.float64)
        p = np.ascontiguousarray(p, dtype=np.float64)
        Yu = np.empty(self.nvel) if Yu is None else Yu
        Yp = np.empty(self.npres) if Yp is None else Yp
        _capi.call(base + "_h", self._h, _hptr(u, np.float64), _hptr(p, np.float64), _hptr(Yu, np.float64),
                   _hptr(Yp, np.float64))
        return Yu, Yp

    def ProjectMarkers(self, wil, xi, eta, rho, install=True):
        """Gauss-point (eta, rho) from material points by the reference's Q1
        projection (SwarmUpdateGaussPropertiesLocalL2Projection_Q1_MPntPStokes
        on one rank); install=True also makes eta the op's viscosity.  Device
        tensors in, device tensors out; numpy in, numpy out."""
        n = len(wil)
        if _is_dev(xi):
            eq = torch.empty(27 * self.nel, dtype=torch.float64, device=xi.device)
            rq = torch.empty_like(eq)
            w = wil.to(torch.int32).contiguous()
            _capi.call("pt_project_markers_d", self._h, n, ctypes.c_void_p(w.data_ptr()),
                       _dptr(xi.reshape(-1), torch.float64), _dptr(eta, torch.float64), _dptr(rho, torch.float64),
                       _dptr(eq, torch.float64), _dptr(rq, torch.float64), int(install))
            return eq, rq
        w = np.ascontiguousarray(wil, dtype=np.int32)
        x = np.ascontiguousarray(xi, dtype=np.float64).reshape(-1)
        e = np.ascontiguousarray(eta, dtype=np.float64)
        r = np.ascontiguousarray(rho, dtype=np.float64)
        eq = np.empty(27 * self.nel)
        rq = np.empty(27 * self.nel)
        _capi.call("pt_project_markers_h", self._h, n, w.ctypes.data, x.ctypes.data, e.ctypes.data, r.ctypes.data,
                   eq.ctypes.data, rq.ctypes.data, int(install))
        return eq, rq

    def set_body_force(self, fu):
        """Gauss-point body force QPntVolCoefStokes.Fu, [27 nel][3] (numpy or
        a CUDA float64 tensor)."""
        self._check_len(fu, 3 * 27 * self.nel, "fu")
        if _is_dev(fu):
            _capi.call("pt_op_set_body_force_d", self._h, _dptr(fu, torch.float64))
        else:
            f = np.ascontiguousarray(fu, dtype=np.float64)
            _capi.call("pt_op_set_body_force_h", self._h, _hptr(f, np.float64))

    def FormFunctionLocal_U(self, ufield, pfield, Ru=None):
        """The unassembled local momentum residual A11 u + A12 p - body force
        (FormFunctionLocal_U, src/stokes_form_function.c:99-243); u as given,
        with the Dirichlet values inserted by the caller."""
        self._check_len(ufield, self.nvel, "u")
        self._check_len(pfield, self.npres, "p")
        if _is_dev(ufield):
            Ru = torch.empty_like(ufield) if Ru is None else Ru
            _capi.call("pt_residual_u_d", self._h, _dptr(ufield, torch.float64), _dptr(pfield, torch.float64),
                       _dptr(Ru, torch.float64))
            return Ru
        u = np.ascontiguousarray(ufield, dtype=np.float64)
        p = np.ascontiguousarray(pfield, dtype=np.float64)
        Ru = np.empty(self.nvel) if Ru is None else Ru
        _capi.call("pt_residual_u_h", self._h, _hptr(u, np.float64), _hptr(p, np.float64), _hptr(Ru, np.float64))
        return Ru

    def MFStokesWrapper_A(self, ufield, pfield, Yu=None, Yp=None):
        """The whole Stokes operator, unassembled and without BCs:
        (A11 u + A12 p, A21 u) (MFStokesWrapper_A_AVX)."""
        return self._apply2("pt_stokes_a_apply", ufield, pfield, Yu, Yp)

    def MatMult_MFStokes_A(self, Xu, Xp, Yu=None, Yp=None):
        """MatMult_MFStokes_A on one rank (Dirichlet columns zeroed, rows
        copied); returns (Yu, Yp)."""
        return self._apply2("pt_matmult_a", Xu, Xp, Yu, Yp)

    def MatMult_MFStokes_A11(self, X, Y=None):
        self._check_len(X, self.nvel, "X")
        if _is_dev(X) and X.dtype == torch.float32:
            if Y is None:
                Y = torch.empty_like(X)
            _capi.call("pt_matmult_a11_f32_d", self._h, _dptr(X, torch.float32), _dptr(Y, torch.float32))
            return Y
        return self._apply("pt_matmult_a11", X, self.nvel, Y)

    def MatGetDiagonal_MFStokes_A11(self, X=None):
        if X is not None and _is_dev(X):
            _capi.call("pt_getdiag_a11_d", self._h, _dptr(X, torch.float64))
            return X
        out = np.empty(self.nvel) if X is None else X
        _capi.call("pt_getdiag_a11_h", self._h, _hptr(out, np.float64))
        return out

    def MatMult_MFStokes_A12(self, X, Y=None):
        self._check_len(X, self.npres, "X")
        return self._apply("pt_matmult_a12", X, self.nvel, Y)

    def MatMult_MFStokes_A21(self, X, Y=None):
        self._check_len(X, self.nvel, "X")
        return self._apply("pt_matmult_a21", X, self.npres, Y)
