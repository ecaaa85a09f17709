"""The momentum residual on the GPU (pt_residual_u_[dh], Python
MatStokesMF.FormFunctionLocal_U) against the reference's own
FormFunctionLocal_U (src/stokes_form_function.c:99-243, compiled unmodified
into oracle/_ref): golden fixtures, a 64^3 box checked against the reference
directly, the body force read from the 48-byte QPntVolCoefStokes records, and
the load vector following coordinate changes.

Tolerance: 1e-12 relative in the max norm (FP64).
"""
import numpy as np
import pytest

from conftest import load_golden, relerr, residual_golden_names
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


@pytest.fixture(scope="module")
def ref():
    import os

    import oracle
    if not oracle.RefCPU.available():
        oracle.build()
    r = oracle.RefCPU()
    r.set_threads(os.cpu_count())
    return r


@pytest.mark.parametrize("a11_op", ["b200", "b200_stream", "b200_colour"])
@pytest.mark.parametrize("name", residual_golden_names())
def test_residual_matches_reference(name, a11_op):
    import torch

    from pt_b200 import MatStokesMF
    g = load_golden(name)
    m = M.BoxMesh(*(int(v) for v in g["dims"]), g["coords"])
    with MatStokesMF(*m.dims, a11_op=a11_op) as op:
        op.SetUp(m.coords, g["eta"], M.bc_mask_freeslip(*m.dims))  # the residual applies no BC rule
        op.set_body_force(g["fu"])
        assert relerr(op.FormFunctionLocal_U(g["u"], g["p"]), g["ru"]) < TOL64
        ud, pd = torch.from_numpy(g["u"]).cuda(), torch.from_numpy(g["p"]).cuda()
        rd = op.FormFunctionLocal_U(ud, pd)
        torch.cuda.synchronize()
        assert relerr(rd.cpu().numpy(), g["ru"]) < TOL64


def test_residual_at_64cubed(ref):
    """64^3 sinker box (streaming A11, stored divergence blocks, colour-ordered
    body-force load) against the reference's FormFunctionLocal_U."""
    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem("c1", seed=0)
    u = M.uniform_vec(m.nvel, 5)
    p = M.uniform_vec(m.npres, 6)
    rho = 1.0 + 0.5 * M.uniform_vec(27 * m.nel, 7)
    fu = np.zeros((27 * m.nel, 3))
    fu[:, 2] = -9.81 * rho          # gravity body force rho g
    fu = fu.reshape(-1)
    with MatStokesMF(*m.dims) as op:
        op.SetUp(m.coords, eta, mask)
        op.set_body_force(fu)
        ru = op.FormFunctionLocal_U(u, p)
    assert relerr(ru, ref.residual_u(m.dims, m.coords, eta, fu, u, p)) < TOL64


def test_body_force_from_records_and_moving_mesh(ora):
    """Fu read in place from 48-byte QPntVolCoefStokes records (eta, rho,
    Fu[3], Fp) equals the contiguous upload bitwise; after the coordinates
    change, the load vector follows them."""
    import ctypes

    from pt_b200 import MatStokesMF, _capi
    lib = _capi.load()
    m, eta, mask = M.problem("box:9,7,5", seed=9)
    u = M.uniform_vec(m.nvel, 1)
    p = M.uniform_vec(m.npres, 2)
    fu = M.uniform_vec(3 * 27 * m.nel, 3)
    rec = np.full((27 * m.nel, 6), 5.0)
    rec[:, 0] = eta
    rec[:, 2:5] = fu.reshape(-1, 3)
    with MatStokesMF(*m.dims) as a, MatStokesMF(*m.dims) as b:
        a.SetUp(m.coords, eta, mask)
        a.set_body_force(fu)
        b.SetUp(m.coords, eta, mask)
        assert lib.pt_op_set_body_force_strided_h(b.handle, ctypes.c_void_p(rec[:, 2:].ctypes.data),
                                                  ctypes.c_int64(6)) == 0, lib.pt_last_error()
        ra = a.FormFunctionLocal_U(u, p)
        assert np.array_equal(ra, b.FormFunctionLocal_U(u, p))
        assert relerr(ra, ora.residual_u(m.dims, m.coords, eta, fu, u, p)) < TOL64
        c2 = M.make_mesh(*m.dims, perturb=0.1, seed=77).coords
        a.set_coords(c2)
        assert relerr(a.FormFunctionLocal_U(u, p), ora.residual_u(m.dims, c2, eta, fu, u, p)) < TOL64


def test_residual_needs_a_body_force():
    from pt_b200 import MatStokesMF, PtError
    m, eta, mask = M.problem("box:2,2,2", seed=1)
    with MatStokesMF(*m.dims) as op:
        op.SetUp(m.coords, eta, mask)
        with pytest.raises(PtError, match="body force"):
            op.FormFunctionLocal_U(np.zeros(op.nvel), np.zeros(op.npres))
