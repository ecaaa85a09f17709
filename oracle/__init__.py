"""CPU oracle for the Q2-P1disc matrix-free Stokes operator.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import this package, and only as the
checker (or the timed CPU reference arm), never as the thing measured or
shipped.  The product path (``ptatin-gene_b200``) never imports it.

Two checkers live here:

* ``Oracle``   -- ``liboracle.so``, a plain-C restatement of the reference's
  CPU arithmetic (``pt_oracle.c``; each routine cites the reference file:line
  it restates).
* ``RefCPU``   -- ``_ref/libptref.so``, the reference's own
  ``stokes_operators_{tensor,avx,mf}.c`` and ``element_utils_q{1,2}.c``
  compiled unmodified against the PETSc stand-in headers in ``ref_stub/``
  (``ref_glue.c`` only marshals arrays).  Present where the reference tree was
  available at build time.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ORA_SO = os.path.join(_HERE, "liboracle.so")
_REF_SO = os.path.join(_HERE, "_ref", "libptref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_u8p = ctypes.POINTER(ctypes.c_uint8)
_i32p = ctypes.POINTER(ctypes.c_int32)


def reference_tree():
    """The reference source tree to compile Route A from: $PTATIN_REF_DIR, else
    a ``reference`` directory beside this repository; None when neither has
    the reference's ``src/``."""
    cands = [os.environ.get("PTATIN_REF_DIR", ""),
             os.path.join(os.path.dirname(os.path.dirname(_HERE)), "reference")]
    for c in cands:
        if c and os.path.isdir(os.path.join(c, "src")):
            return c
    return None


def build(quiet: bool = True) -> None:
    """Compile liboracle.so (and _ref/libptref.so where the reference exists)."""
    cmd = ["make", "-C", _HERE, "all"]
    ref = reference_tree()
    if ref:
        cmd.append(f"REF={ref}")
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _mask(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


class Oracle:
    """ctypes front-end of liboracle.so (Route B restatement)."""

    def __init__(self, path: str = _ORA_SO):
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        i = ctypes.c_int
        for name in ("ora_a11_tensor", "ora_a11_ref"):
            getattr(L, name).argtypes = [i, i, i, _dp, _dp, _dp, _dp]
        L.ora_a11_diag.argtypes = [i, i, i, _dp, _dp, _dp]
        for name in ("ora_a21_ref", "ora_a12_ref", "ora_a12_tensor"):
            getattr(L, name).argtypes = [i, i, i, _dp, _dp, _dp]
        L.ora_elements_q2.argtypes = [i, i, i, _i32p]
        L.ora_gauss3.argtypes = [_dp, _dp]
        L.ora_matmult_a11.argtypes = [i, i, i, _dp, _dp, _u8p, _dp, _dp, i]
        L.ora_getdiag_a11.argtypes = [i, i, i, _dp, _dp, _u8p, _dp]
        L.ora_matmult_a12.argtypes = [i, i, i, _dp, _u8p, _dp, _dp, i]
        L.ora_matmult_a21.argtypes = [i, i, i, _dp, _u8p, _dp, _dp]
        L.ora_a11_flops.argtypes = [ctypes.c_int64]
        L.ora_residual_u.argtypes = [i, i, i, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ora_marker_project.argtypes = [i, i, i, ctypes.c_int64, _i32p, _dp, _dp, _dp, _dp, _dp]
        L.ora_a11_flops.restype = ctypes.c_double
        L.ora_num_threads.restype = ctypes.c_int

    # element-loop kernels (y = 0 + contributions, unassembled semantics)
    def a11(self, dims, coords, eta, u, variant="tensor"):
        mx, my, mz = dims
        y = np.zeros_like(_f64(u))
        fn = self.lib.ora_a11_tensor if variant == "tensor" else self.lib.ora_a11_ref
        fn(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)), _ptr(_f64(u)), _ptr(y))
        return y

    def diag(self, dims, coords, eta):
        mx, my, mz = dims
        y = np.zeros(3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
        self.lib.ora_a11_diag(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)), _ptr(y))
        return y

    def a21(self, dims, coords, u):
        mx, my, mz = dims
        y = np.zeros(4 * mx * my * mz)
        self.lib.ora_a21_ref(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(u)), _ptr(y))
        return y

    def a12(self, dims, coords, p, variant="tensor"):
        mx, my, mz = dims
        y = np.zeros(3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
        fn = self.lib.ora_a12_tensor if variant == "tensor" else self.lib.ora_a12_ref
        fn(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(p)), _ptr(y))
        return y

    # MatShell-level operators (BC semantics of stokes_operators.c)
    def matmult_a11(self, dims, coords, eta, mask, x, variant="tensor"):
        mx, my, mz = dims
        y = np.zeros_like(_f64(x))
        self.lib.ora_matmult_a11(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)),
                                 _ptr(_mask(mask), _u8p), _ptr(_f64(x)), _ptr(y),
                                 0 if variant == "tensor" else 1)
        return y

    def getdiag_a11(self, dims, coords, eta, mask):
        mx, my, mz = dims
        y = np.zeros(len(mask))
        self.lib.ora_getdiag_a11(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)),
                                 _ptr(_mask(mask), _u8p), _ptr(y))
        return y

    def matmult_a12(self, dims, coords, mask, p, variant="tensor"):
        mx, my, mz = dims
        y = np.zeros(len(mask))
        self.lib.ora_matmult_a12(mx, my, mz, _ptr(_f64(coords)), _ptr(_mask(mask), _u8p),
                                 _ptr(_f64(p)), _ptr(y), 0 if variant == "tensor" else 1)
        return y

    def matmult_a21(self, dims, coords, mask, u):
        mx, my, mz = dims
        y = np.zeros(4 * mx * my * mz)
        self.lib.ora_matmult_a21(mx, my, mz, _ptr(_f64(coords)), _ptr(_mask(mask), _u8p),
                                 _ptr(_f64(u)), _ptr(y))
        return y

    # The whole Stokes operator (restated as the sum of its blocks, which is
    # what MFStokesWrapper_A computes in one element loop:
    # src/stokes_operators_mf.c:711-790, src/stokes_operators_avx.c:439-636)
    def stokes_a(self, dims, coords, eta, u, p):
        """Unassembled local Yu = A11 u + A12 p, Yp = A21 u (SpMVOp level)."""
        yu = self.a11(dims, coords, eta, u) + self.a12(dims, coords, p)
        return yu, self.a21(dims, coords, u)

    def matmult_a(self, dims, coords, eta, mask, u, p):
        """MatMult_MFStokes_A (src/stokes_operators.c:893-979): Dirichlet
        columns of u zeroed, Yu = A11 u + A12 p, Yp = A21 u, then Yu_k = u_k on
        Dirichlet dofs (no pressure BCs)."""
        m = _mask(mask).astype(bool)
        uz = _f64(u).copy()
        uz[m] = 0.0
        yu, yp = self.stokes_a(dims, coords, eta, uz, p)
        yu[m] = _f64(u)[m]
        return yu, yp

    def residual_u(self, dims, coords, eta, fu, u, p):
        """FormFunctionLocal_U (src/stokes_form_function.c:99-243): unassembled
        local Ru = A11 u + A12 p - body force; fu is [27 nel][3]."""
        mx, my, mz = dims
        ru = np.zeros_like(_f64(u))
        self.lib.ora_residual_u(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)), _ptr(_f64(fu)), _ptr(_f64(u)),
                                _ptr(_f64(p)), _ptr(ru))
        return ru

    def marker_project(self, dims, wil, xi, eta, rho):
        """Gauss-point (eta, rho) from markers (restatement of the reference's
        Q1 projection, src/material_point_utils.c:957-1190)."""
        mx, my, mz = dims
        w = np.ascontiguousarray(wil, dtype=np.int32)
        eq = np.zeros(27 * mx * my * mz)
        rq = np.zeros(27 * mx * my * mz)
        self.lib.ora_marker_project(mx, my, mz, len(w), _ptr(w, _i32p), _ptr(_f64(xi)), _ptr(_f64(eta)),
                                    _ptr(_f64(rho)), _ptr(eq), _ptr(rq))
        return eq, rq

    def elements(self, dims):
        mx, my, mz = dims
        e = np.zeros(27 * mx * my * mz, dtype=np.int32)
        self.lib.ora_elements_q2(mx, my, mz, _ptr(e, _i32p))
        return e.reshape(-1, 27)

    def gauss3(self):
        x = np.zeros(3)
        w = np.zeros(3)
        self.lib.ora_gauss3(_ptr(x), _ptr(w))
        return x, w

    def a11_flops(self, nel):
        return self.lib.ora_a11_flops(nel)

    def num_threads(self):
        return self.lib.ora_num_threads()


class RefCPU:
    """ctypes front-end of _ref/libptref.so (the reference's own sources)."""

    KINDS = {"tensor": 0, "avx": 1, "ref": 2}

    def __init__(self, path: str = _REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        i = ctypes.c_int
        L.ref_a11.argtypes = [i, i, i, i, _dp, _dp, _dp, _dp]
        L.ref_diag.argtypes = [i, i, i, _dp, _dp, _dp]
        L.ref_a21.argtypes = [i, i, i, _dp, _dp, _dp]
        L.ref_a12.argtypes = [i, i, i, i, _dp, _dp, _dp]
        L.ref_stokes_a.argtypes = [i, i, i, i, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_marker_project.argtypes = [i, i, i, i, ctypes.POINTER(ctypes.c_int), _dp, _dp, _dp, _dp, _dp]
        L.ref_residual_u.argtypes = [i, i, i, _dp, _dp, _dp, _dp, _dp, _dp]
        L.ref_has_avx.restype = i
        L.ref_set_threads.argtypes = [i]
        L.ref_set_threads.restype = i

    @staticmethod
    def available() -> bool:
        return os.path.exists(_REF_SO)

    def set_threads(self, n: int) -> int:
        """OpenMP threads of the reference's operators; returns the count in effect."""
        return int(self.lib.ref_set_threads(int(n)))

    def _check(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"reference {what} returned PetscErrorCode {rc}")

    def a11(self, dims, coords, eta, u, kind="tensor"):
        mx, my, mz = dims
        u = _f64(u).copy()
        y = np.zeros_like(u)
        self._check(self.lib.ref_a11(self.KINDS[kind], mx, my, mz, _ptr(_f64(coords)),
                                     _ptr(_f64(eta)), _ptr(u), _ptr(y)), "A11")
        return y

    def diag(self, dims, coords, eta):
        mx, my, mz = dims
        y = np.zeros(3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
        self._check(self.lib.ref_diag(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)), _ptr(y)), "diag")
        return y

    def stokes_a(self, dims, coords, eta, u, p, kind="avx"):
        """Yu = A11 u + A12 p, Yp = A21 u (MFStokesWrapper_A[_AVX])."""
        mx, my, mz = dims
        u = _f64(u).copy()
        p = _f64(p).copy()
        yu = np.zeros_like(u)
        yp = np.zeros_like(p)
        self._check(self.lib.ref_stokes_a(self.KINDS[kind], mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)),
                                          _ptr(u), _ptr(p), _ptr(yu), _ptr(yp)), "Stokes A")
        return yu, yp

    def marker_project(self, dims, wil, xi, eta, rho):
        """Gauss-point (eta, rho) from markers by the reference's Q1 projection
        (material_point_utils.c: _SwarmUpdateGaussPropertiesLocalL2ProjectionQ1_*)."""
        mx, my, mz = dims
        w = np.ascontiguousarray(wil, dtype=np.int32)
        eq = np.zeros(27 * mx * my * mz)
        rq = np.zeros(27 * mx * my * mz)
        self._check(self.lib.ref_marker_project(mx, my, mz, len(w), w.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                                _ptr(_f64(xi)), _ptr(_f64(eta)), _ptr(_f64(rho)), _ptr(eq),
                                                _ptr(rq)), "marker projection")
        return eq, rq

    def residual_u(self, dims, coords, eta, fu, u, p):
        """The reference's own FormFunctionLocal_U (src/stokes_form_function.c:
        99-243) compiled unmodified: unassembled local Ru = A11 u + A12 p -
        body force, with fu the Gauss-point QPntVolCoefStokes.Fu ([27 nel][3])."""
        mx, my, mz = dims
        u = _f64(u).copy()
        p = _f64(p).copy()
        ru = np.zeros_like(u)
        self._check(self.lib.ref_residual_u(mx, my, mz, _ptr(_f64(coords)), _ptr(_f64(eta)), _ptr(_f64(fu)),
                                            _ptr(u), _ptr(p), _ptr(ru)), "FormFunctionLocal_U")
        return ru

    def a21(self, dims, coords, u):
        mx, my, mz = dims
        u = _f64(u).copy()
        y = np.zeros(4 * mx * my * mz)
        self._check(self.lib.ref_a21(mx, my, mz, _ptr(_f64(coords)), _ptr(u), _ptr(y)), "A21")
        return y

    def a12(self, dims, coords, p, kind="avx"):
        mx, my, mz = dims
        p = _f64(p).copy()
        y = np.zeros(3 * (2 * mx + 1) * (2 * my + 1) * (2 * mz + 1))
        self._check(self.lib.ref_a12(self.KINDS[kind], mx, my, mz, _ptr(_f64(coords)),
                                     _ptr(p), _ptr(y)), "A12")
        return y

    # ---- MatShell level: the reference's element loops with the BC rules of
    # src/stokes_operators.c (one rank, so local = global) -------------------
    def matmult_a11(self, dims, coords, eta, mask, x, kind="avx"):
        """MatMult_MFStokes_A11 (stokes_operators.c:1156-1222): Dirichlet entries
        of the local input zeroed (BCListInsertLocalZero), the back-end's
        element loop, then y_k = x_k on Dirichlet dofs
        (BCListInsertDirichlet_MatMult, scale 1)."""
        m = _mask(mask).astype(bool)
        xz = _f64(x).copy()
        xz[m] = 0.0
        y = self.a11(dims, coords, eta, xz, kind)
        y[m] = _f64(x)[m]
        return y

    def getdiag_a11(self, dims, coords, eta, mask):
        """MatGetDiagonal_MFStokes_A11 (stokes_operators.c:1072-1113): the
        element diagonal, 1.0 in Dirichlet slots
        (BCListInsertValueIntoDirichletSlot)."""
        d = self.diag(dims, coords, eta)
        d[_mask(mask).astype(bool)] = 1.0
        return d

    def matmult_a12(self, dims, coords, mask, p, kind="avx"):
        """MatMult_MFStokes_A12 (stokes_operators.c:1301-1370): B^T p with the
        velocity Dirichlet rows zeroed (BCListInsertZero)."""
        y = self.a12(dims, coords, p, kind)
        y[_mask(mask).astype(bool)] = 0.0
        return y

    def matmult_a21(self, dims, coords, mask, u):
        """MatMult_MFStokes_A21 (stokes_operators.c:1444-1509): B u with the
        Dirichlet entries of u zeroed; no pressure BC."""
        uz = _f64(u).copy()
        uz[_mask(mask).astype(bool)] = 0.0
        return self.a21(dims, coords, uz)

    def matmult_a(self, dims, coords, eta, mask, u, p, kind="avx"):
        """MatMult_MFStokes_A (stokes_operators.c:893-979): Dirichlet columns of
        u zeroed, Yu = A11 u + A12 p and Yp = A21 u in one element loop
        (MFStokesWrapper_A[_AVX]), then Yu_k = u_k on Dirichlet dofs."""
        m = _mask(mask).astype(bool)
        uz = _f64(u).copy()
        uz[m] = 0.0
        yu, yp = self.stokes_a(dims, coords, eta, uz, p, kind)
        yu[m] = _f64(u)[m]
        return yu, yp
