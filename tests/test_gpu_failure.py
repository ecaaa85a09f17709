"""Failure paths injected on the host (no GPU fault): viscosity that is
negative or NaN at a Gauss point, and inverted elements.

The streaming and stored-matrix kernels need c = w*eta/detJ > 0 at every Gauss
point (they store sqrt(c)); when the set-up kernel counts a point that is not,
the op falls back to the 8-colour kernel, which evaluates the reference's
arithmetic for any sign.  These tests check that the fallback is taken (launch
counts: 8 colour launches plus the Dirichlet-row copy per MatMult instead of
the streaming kernel's 4 colour passes), that its results still match the
oracle at 1e-12, and that the no-allocation entry point, which has no fallback,
refuses such input with PT_ERR_BAD_ARG.
"""
import ctypes

import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12


def _problem(kind):
    m, eta, mask = M.problem("box:5,4,3", seed=11)
    coords = m.coords.copy()
    eta = eta.copy()
    if kind == "negative_eta":
        eta[27 * 7 + 13] = -0.5
    elif kind == "nan_eta":
        eta[27 * 9 + 4] = np.nan
    elif kind == "mirrored":
        # x -> 1 - x: every element inverted (detJ < 0 at every Gauss point)
        c = coords.reshape(-1, 3)
        c[:, 0] = 1.0 - c[:, 0]
    elif kind == "one_inverted":
        # the interior node of element (1, 1, 1) pushed through the element's
        # +x face: detJ < 0 at some of its Gauss points
        X, Y = 2 * m.mx + 1, 2 * m.my + 1
        n = 3 + 3 * X + 3 * X * Y
        coords[3 * n] += 3.0 / m.mx
    return M.BoxMesh(*m.dims, coords), eta, mask


def _launches_per_matmult(op, x):
    op.MatMult_MFStokes_A11(x)
    op.reset_launch_count()
    op.MatMult_MFStokes_A11(x)
    return op.launch_count()


@pytest.mark.parametrize("a11_op", ["b200", "b200_stream"])
@pytest.mark.parametrize("kind", ["negative_eta", "mirrored", "one_inverted"])
def test_fallback_matches_oracle(ora, kind, a11_op):
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = _problem(kind)
    x = M.uniform_vec(m.nvel, 3)
    with MatStokesMF(*m.dims, a11_op=a11_op) as op:
        op.SetUp(m.coords, eta, mask)
        xd = torch.from_numpy(x).cuda()
        assert _launches_per_matmult(op, xd) == 9  # 8 colours + Dirichlet rows
        y = op.MatMult_MFStokes_A11(x)
        d = op.MatGetDiagonal_MFStokes_A11()
    assert relerr(y, ora.matmult_a11(m.dims, m.coords, eta, mask, x)) < TOL64
    assert relerr(d, ora.getdiag_a11(m.dims, m.coords, eta, mask)) < TOL64


def test_valid_input_keeps_the_fast_path():
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = _problem("none")
    with MatStokesMF(*m.dims, a11_op="b200_stream") as op:
        op.SetUp(m.coords, eta, mask)
        # 4 colour passes + the Dirichlet rows
        assert _launches_per_matmult(op, torch.from_numpy(M.uniform_vec(m.nvel, 3)).cuda()) == 5


def test_nan_viscosity_stays_local(ora):
    """NaN at one Gauss point of element 9: the op falls back, NaN shows up in
    y, only on dofs of that element's 27 nodes, and every other dof matches
    the oracle.  (Which of the element's dofs turn NaN differs between
    algorithms: the sum-factorised kernels skip the basis weights that are
    exactly zero at the middle Gauss point, the reference multiplies by them.)"""
    from pt_b200 import MatStokesMF
    m, eta, mask = _problem("nan_eta")
    x = M.uniform_vec(m.nvel, 5)
    with MatStokesMF(*m.dims) as op:
        op.SetUp(m.coords, eta, mask)
        y = op.MatMult_MFStokes_A11(x)
    ref = ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    elem = np.zeros(m.nvel, dtype=bool)
    for n in ora.elements(m.dims)[9]:
        elem[3 * n:3 * n + 3] = True
    assert np.isnan(y).any() and not np.isnan(y[~elem]).any()
    assert not np.isnan(ref[~elem]).any()
    assert relerr(y[~elem], ref[~elem]) < TOL64


@pytest.mark.parametrize("kind", ["negative_eta", "nan_eta", "mirrored"])
def test_noalloc_refuses_invalid_geometry(kind):
    import torch

    from pt_b200 import _capi
    lib = _capi.load()
    m, eta, _ = _problem(kind)
    c = torch.from_numpy(m.coords).cuda()
    e = torch.from_numpy(eta).cuda()
    u = torch.from_numpy(M.uniform_vec(m.nvel, 2)).cuda()
    y = torch.empty_like(u)
    desc = _capi.MeshDesc(*m.dims, 0, 0, 0, 0, 0, 0)
    st = lib.pt_a11_apply_noalloc_d(ctypes.byref(desc), ctypes.c_void_p(c.data_ptr()), ctypes.c_void_p(e.data_ptr()),
                                    ctypes.c_void_p(u.data_ptr()), ctypes.c_void_p(y.data_ptr()),
                                    ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert st == 1
    assert b"w*eta/detJ" in lib.pt_last_error()
