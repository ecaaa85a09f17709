"""The PETSc plug-in (ptatin-gene_b200/shim/stokes_operators_b200.c) executed on
the GPU: compiled unmodified against the reference's headers with
oracle/shim_host.c standing in for PETSc (test library oracle/_ref/
libshimtest.so), its entry points are called the way pTatin3D calls them and
checked against the reference's own outputs (golden fixtures), and its
upload rules are checked through the op's launch counter:

* the A11 shell and the diag / B / B^T / whole-operator calls share one op;
* after the first calls, further MatMults with unchanged coordinates and
  viscosity launch only the operator kernels (no geometry, element-matrix or
  divergence-block set-up);
* moving the mesh (new coordinate Vec state) or new viscosity with a new Mat
  state re-uploads, and the results follow the new data;
* the viscosity is read from the 48-byte QPntVolCoefStokes records (strided
  upload), bitwise the same as a contiguous upload.
"""
import ctypes
import os

import numpy as np
import pytest

from conftest import REPO, golden_names, load_golden, relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
LIB = os.path.join(REPO, "oracle", "_ref", "libshimtest.so")
vp = ctypes.c_void_p


@pytest.fixture(scope="module")
def shim():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    if not os.path.exists(LIB):
        import oracle
        oracle.build()
    from pt_b200 import _capi
    _capi.load()
    L = ctypes.CDLL(LIB)
    L.shimtest_create.restype = vp
    L.shimtest_create.argtypes = [ctypes.c_int] * 9 + [vp, vp]
    for name, n in (("shimtest_a11", 3), ("shimtest_diag", 2), ("shimtest_a12", 3), ("shimtest_a21", 3),
                    ("shimtest_stokes_a", 5)):
        getattr(L, name).argtypes = [vp] * n
    L.shimtest_move.argtypes = [vp, vp]
    L.shimtest_set_eta.argtypes = [vp, vp, ctypes.c_int]
    L.shimtest_op.restype = vp
    L.shimtest_op.argtypes = [vp]
    L.shimtest_destroy.argtypes = [vp]
    return L


def _p(a):
    return vp(a.ctypes.data)


class Plugin:
    """One DM + quadrature + A11 shell driven through the plug-in."""

    def __init__(self, L, m, eta):
        self.L, self.m = L, m
        self.coords = np.ascontiguousarray(m.coords, dtype=np.float64)
        self.h = L.shimtest_create(*m.dims, 0, 0, 0, 0, 0, 0, _p(self.coords), _p(np.ascontiguousarray(eta)))
        assert self.h, "shimtest_create failed"
        from pt_b200 import _capi
        self.capi = _capi.load()

    def launches(self):
        return int(self.capi.pt_op_launch_count(vp(self.L.shimtest_op(self.h))))

    def a11(self, u):
        y = np.zeros(self.m.nvel)
        assert self.L.shimtest_a11(self.h, _p(u), _p(y)) == 0
        return y

    def diag(self):
        y = np.zeros(self.m.nvel)
        assert self.L.shimtest_diag(self.h, _p(y)) == 0
        return y

    def a12(self, p):
        y = np.zeros(self.m.nvel)
        assert self.L.shimtest_a12(self.h, _p(p), _p(y)) == 0
        return y

    def a21(self, u):
        y = np.zeros(self.m.npres)
        assert self.L.shimtest_a21(self.h, _p(u), _p(y)) == 0
        return y

    def stokes(self, u, p):
        yu, yp = np.zeros(self.m.nvel), np.zeros(self.m.npres)
        assert self.L.shimtest_stokes_a(self.h, _p(u), _p(p), _p(yu), _p(yp)) == 0
        return yu, yp

    def close(self):
        assert self.L.shimtest_destroy(self.h) == 0


@pytest.mark.parametrize("name", golden_names())
def test_plugin_matches_reference(shim, name):
    g = load_golden(name)
    m = M.BoxMesh(*(int(v) for v in g["dims"]), g["coords"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    p = np.ascontiguousarray(g["p"])
    pl = Plugin(shim, m, g["eta"])
    try:
        assert relerr(pl.a11(uz), g["a11_avx"]) < TOL64
        assert relerr(pl.diag(), g["diag"]) < TOL64
        assert relerr(pl.a21(uz), g["a21"]) < TOL64
        assert relerr(pl.a12(p), g["a12_avx"]) < TOL64
        yu, yp = pl.stokes(uz, p)
        assert relerr(yu, g["a_u_avx"]) < TOL64
        assert relerr(yp, g["a_p_avx"]) < TOL64
    finally:
        pl.close()


@pytest.mark.parametrize("workload", ["box:6,5,4", "box:40,9,7"])
def test_plugin_uploads_only_on_change(shim, ora, workload):
    m, eta, mask = M.problem(workload, seed=13)
    u = M.uniform_vec(m.nvel, 1)
    u[mask.astype(bool)] = 0.0
    p = M.uniform_vec(m.npres, 2)
    pl = Plugin(shim, m, eta)
    try:
        # first round: uploads and set-up
        pl.a11(u), pl.diag(), pl.a12(p), pl.a21(u), pl.stokes(u, p)
        # steady state: the same launches call after call, no set-up kernels
        counts = []
        for _ in range(3):
            c0 = pl.launches()
            yu, yp = pl.stokes(u, p)
            counts.append(pl.launches() - c0)
        assert counts[0] == counts[1] == counts[2]
        c0 = pl.launches()
        y = pl.a11(u)
        n_a11 = pl.launches() - c0
        c0 = pl.launches()
        pl.a11(u)
        assert pl.launches() - c0 == n_a11
        assert relerr(y, ora.a11(m.dims, m.coords, eta, u)) < TOL64
        ru = ora.a11(m.dims, m.coords, eta, u) + ora.a12(m.dims, m.coords, p)
        assert relerr(yu, ru) < TOL64
        assert relerr(yp, ora.a21(m.dims, m.coords, u)) < TOL64

        # new viscosity without a Mat state change: not uploaded (the
        # reference CUDA back-end's rule); with one: uploaded, results follow
        eta2 = eta * np.exp(np.sin(np.arange(eta.size)))
        shim.shimtest_set_eta(pl.h, _p(eta2), 0)
        c0 = pl.launches()
        assert np.array_equal(pl.a11(u), y)
        assert pl.launches() - c0 == n_a11
        shim.shimtest_set_eta(pl.h, _p(eta2), 1)
        c0 = pl.launches()
        y2 = pl.a11(u)
        assert pl.launches() - c0 > n_a11  # geometry rebuilt once
        assert relerr(y2, ora.a11(m.dims, m.coords, eta2, u)) < TOL64
        yu2, _ = pl.stokes(u, p)
        assert relerr(yu2, ora.a11(m.dims, m.coords, eta2, u) + ora.a12(m.dims, m.coords, p)) < TOL64

        # the mesh moves: new coordinate Vec state
        c2 = M.make_mesh(*m.dims, perturb=0.1, seed=99).coords
        pl.coords2 = np.ascontiguousarray(c2)
        shim.shimtest_move(pl.h, _p(pl.coords2))
        assert relerr(pl.a21(u), ora.a21(m.dims, c2, u)) < TOL64
        assert relerr(pl.a11(u), ora.a11(m.dims, c2, eta2, u)) < TOL64
        assert relerr(pl.diag(), ora.diag(m.dims, c2, eta2)) < TOL64
    finally:
        pl.close()


def test_strided_viscosity_upload_is_bitwise_the_contiguous_one():
    """pt_op_set_eta_strided_h over 48-byte records (eta at offset 0, rho, Fu,
    Fp around it) gives bitwise the apply of pt_op_set_eta_h; the box is large
    enough for several pinned staging chunks (27 * nel > 2^19)."""
    from pt_b200 import MatStokesMF, _capi
    lib = _capi.load()
    m, eta, mask = M.problem("box:40,30,20", seed=5)
    rec = np.full((eta.size, 6), -7.0)
    rec[:, 0] = eta
    x = M.uniform_vec(m.nvel, 3)
    with MatStokesMF(*m.dims) as a, MatStokesMF(*m.dims) as b:
        a.SetUp(m.coords, eta, mask)
        b.set_coords(m.coords)
        b.set_bc_mask(mask)
        assert lib.pt_op_set_eta_strided_h(b.handle, vp(rec.ctypes.data), ctypes.c_int64(6)) == 0, \
            lib.pt_last_error()
        assert np.array_equal(a.MatMult_MFStokes_A11(x), b.MatMult_MFStokes_A11(x))
        assert np.array_equal(a.MatGetDiagonal_MFStokes_A11(), b.MatGetDiagonal_MFStokes_A11())
