"""GPU parity at the benchmarked size of the plain FP64 drop-in: the 64^3 sinker
box (6.44M velocity dofs, 1.05M pressure dofs, free-slip box BCs), every
MatShell-level operator through the C ABI against the reference's own CPU
code (oracle/_ref: MFStokesWrapper_A11_AVX, MFStokesWrapper_diagA11,
MFStokesWrapper_A21, MFStokesWrapper_A12_AVX, MFStokesWrapper_A_AVX compiled
from the reference sources) with the BC rules of src/stokes_operators.c.

At this size B u and B^T p run from the stored divergence blocks and A11 from
the streaming kernel, so these tests pin the kernels the bench times.

Tolerances (relative, ||y - y_ref||_inf / ||y_ref||_inf):
  FP64 operators  1e-12
  FP32 A11        5e-5 on a 1e6-contrast field (layered viscosity 1e3 / 1 /
                  1e-1 plus inclusions 1e-3..1e3): FP32 arithmetic and
                  accumulation; the measured error sits near 1e-6.
"""
import os

import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 5e-5


@pytest.fixture(scope="module")
def ref():
    import oracle
    if not oracle.RefCPU.available():
        oracle.build()
    r = oracle.RefCPU()
    r.set_threads(os.cpu_count())
    return r


@pytest.fixture(scope="module")
def c1(ref):
    import torch

    from pt_b200 import MatStokesMF
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    m, eta, mask = M.problem("c1", seed=0)
    x = M.uniform_vec(m.nvel, 7)
    p = M.uniform_vec(m.npres, 8)
    op = MatStokesMF(*m.dims)
    op.SetUp(m.coords, eta, mask)
    yield m, eta, mask, x, p, op
    op.Destroy()


def test_c1_a11_matmult(c1, ref):
    m, eta, mask, x, p, op = c1
    assert op.a11_op == "b200_stream"
    y = op.MatMult_MFStokes_A11(x)
    assert relerr(y, ref.matmult_a11(m.dims, m.coords, eta, mask, x)) < TOL64
    bc = mask.astype(bool)
    assert np.array_equal(y[bc], x[bc])


def test_c1_diagonal(c1, ref):
    m, eta, mask, x, p, op = c1
    assert relerr(op.MatGetDiagonal_MFStokes_A11(), ref.getdiag_a11(m.dims, m.coords, eta, mask)) < TOL64


def test_c1_divergence_and_gradient(c1, ref):
    """B u and B^T p from the stored 4x81 divergence blocks (5.4 GB at 128^3,
    0.68 GB here) against the reference's element loops."""
    m, eta, mask, x, p, op = c1
    assert relerr(op.MatMult_MFStokes_A21(x), ref.matmult_a21(m.dims, m.coords, mask, x)) < TOL64
    assert relerr(op.MatMult_MFStokes_A12(p), ref.matmult_a12(m.dims, m.coords, mask, p)) < TOL64


def test_c1_whole_stokes_operator(c1, ref):
    m, eta, mask, x, p, op = c1
    yu, yp = op.MatMult_MFStokes_A(x, p)
    ru, rp = ref.matmult_a(m.dims, m.coords, eta, mask, x, p)
    assert relerr(yu, ru) < TOL64
    assert relerr(yp, rp) < TOL64


@pytest.mark.parametrize("workload", ["layered:24,24,24", "layered:40,33,17"])
def test_fp32_apply_on_1e6_contrast(ref, workload):
    """The FP32 A11 (FP32 factors, arithmetic and accumulation) on the
    precision workload's viscosity structure, against the reference's FP64
    apply: within 5e-5 of ||y||_inf (measured about 1e-6)."""
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem(workload, seed=3)
    assert eta.max() / eta.min() > 1e5
    x = M.uniform_vec(m.nvel, 4)
    y_ref = ref.matmult_a11(m.dims, m.coords, eta, mask, x)
    for a11_op in ("b200", "b200_stream"):
        with MatStokesMF(*m.dims, a11_op=a11_op) as op:
            op.SetUp(m.coords, eta, mask)
            y32 = op.MatMult_MFStokes_A11(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
        assert relerr(y32, y_ref) < TOL32, a11_op
