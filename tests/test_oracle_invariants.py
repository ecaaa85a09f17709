"""Invariants of the operator, checked on the oracle (CPU): the properties
the reference's operator tests rely on (MF == assembled, symmetric A11,
A12 == A21^T, diag == assembled diagonal)."""
import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M


def assembled(ora, m, eta, fn):
    n = m.nvel
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = fn(e)
    return A


@pytest.mark.parametrize("dims", [(1, 1, 1), (2, 1, 1)])
def test_a11_symmetric_and_diag_matches(ora, dims):
    m = M.make_mesh(*dims, perturb=0.1, seed=3)
    eta = M.eta_loguniform_qp(m, seed=4)
    A = assembled(ora, m, eta, lambda e: ora.a11(m.dims, m.coords, eta, e))
    assert np.abs(A - A.T).max() / np.abs(A).max() < 1e-13
    assert relerr(ora.diag(m.dims, m.coords, eta), np.diag(A)) < 1e-13
    # positive semi-definite
    assert np.linalg.eigvalsh(0.5 * (A + A.T)).min() > -1e-10 * np.abs(A).max()


def test_rigid_body_modes_in_kernel(ora):
    """sym(grad u) = 0 for translations and rotations, which the isoparametric
    Q2 space represents exactly, so A11 u = 0."""
    m = M.make_mesh(3, 2, 2, perturb=0.1, seed=5)
    eta = M.eta_loguniform_qp(m, seed=6)
    x = m.coords.reshape(-1, 3)
    scale = np.abs(ora.a11(m.dims, m.coords, eta, M.uniform_vec(m.nvel, 1))).max()
    for omega in ([1.0, 0, 0], [0, 1.0, 0], [0, 0, 1.0]):
        u = np.cross(np.array(omega)[None, :], x).reshape(-1)
        assert np.abs(ora.a11(m.dims, m.coords, eta, u)).max() < 1e-12 * scale
    for t in range(3):
        u = np.zeros((x.shape[0], 3))
        u[:, t] = 1.0
        assert np.abs(ora.a11(m.dims, m.coords, eta, u.reshape(-1))).max() < 1e-12 * scale


def test_a12_is_a21_transpose(ora):
    m = M.make_mesh(3, 2, 2, perturb=0.1, seed=7)
    u = M.uniform_vec(m.nvel, 8)
    p = M.uniform_vec(m.npres, 9)
    lhs = p @ ora.a21(m.dims, m.coords, u)
    rhs = ora.a12(m.dims, m.coords, p) @ u
    assert abs(lhs - rhs) < 1e-13 * (abs(lhs) + abs(rhs))


def test_matshell_bc_semantics(ora):
    m, eta, mask = M.problem("box:3,2,2")
    x = M.uniform_vec(m.nvel, 10)
    bc = mask.astype(bool)
    y = ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    assert np.array_equal(y[bc], x[bc])                       # rows: y_k = x_k
    xz = x.copy()
    xz[bc] = 0.0
    assert relerr(y[~bc], ora.a11(m.dims, m.coords, eta, xz)[~bc]) < 1e-15  # columns zeroed
    d = ora.getdiag_a11(m.dims, m.coords, eta, mask)
    assert np.all(d[bc] == 1.0)
    yu = ora.matmult_a12(m.dims, m.coords, mask, M.uniform_vec(m.npres, 11))
    assert np.all(yu[bc] == 0.0)
