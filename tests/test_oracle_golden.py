"""The oracle (plain-C restatement) against golden vectors made by the
reference's own operator sources (tests/golden/make_golden.py)."""
import numpy as np
import pytest

from conftest import golden_names, load_golden, relerr, residual_golden_names

# Bar for two FP64 implementations of the same operator with different
# evaluation orders (the reference's own back-ends agree to ~1e-15).
TOL = 1e-13


@pytest.mark.parametrize("name", golden_names())
def test_oracle_matches_reference_goldens(ora, name):
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    assert relerr(ora.a11(dims, g["coords"], g["eta"], uz, "tensor"), g["a11_tensor"]) < TOL
    assert relerr(ora.a11(dims, g["coords"], g["eta"], uz, "ref"), g["a11_ref"]) < TOL
    assert relerr(ora.diag(dims, g["coords"], g["eta"]), g["diag"]) < TOL
    assert relerr(ora.a21(dims, g["coords"], uz), g["a21"]) < TOL
    assert relerr(ora.a12(dims, g["coords"], g["p"], "tensor"), g["a12_avx"]) < TOL
    assert relerr(ora.a12(dims, g["coords"], g["p"], "ref"), g["a12_ref"]) < TOL


@pytest.mark.parametrize("name", golden_names())
def test_reference_backends_agree(name):
    """The cross-back-end invariant of the reference's operator tests:
    tensor, avx and ref A11 (and avx/ref A12) agree to ~1e-13."""
    g = load_golden(name)
    assert relerr(g["a11_avx"], g["a11_tensor"]) < TOL
    assert relerr(g["a11_ref"], g["a11_tensor"]) < TOL
    assert relerr(g["a12_ref"], g["a12_avx"]) < TOL


def test_goldens_reproduce_from_reference_build():
    """Where the reference build (oracle/_ref) exists, the fixtures are what it
    computes now."""
    import oracle
    if not oracle.RefCPU.available():
        pytest.skip("oracle/_ref not built")
    r = oracle.RefCPU()
    g = load_golden("box_3x2x4")
    dims = tuple(int(v) for v in g["dims"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    assert relerr(r.a11(dims, g["coords"], g["eta"], uz, "tensor"), g["a11_tensor"]) < 1e-15
    assert relerr(r.diag(dims, g["coords"], g["eta"]), g["diag"]) < 1e-15


def test_gauss_rule(ora):
    x, w = ora.gauss3()
    assert np.allclose(x, [-np.sqrt(0.6), 0, np.sqrt(0.6)], rtol=0, atol=1e-16)
    assert np.allclose(w, [5 / 9, 8 / 9, 5 / 9], rtol=0, atol=1e-16)


def test_element_table_matches_reference_layout(ora):
    from pt_b200 import mesh as M
    for dims in [(1, 1, 1), (3, 2, 4), (5, 1, 2)]:
        assert np.array_equal(ora.elements(dims), M.element_table(*dims))


@pytest.mark.parametrize("name", golden_names())
def test_oracle_stokes_operator_matches_reference(ora, name):
    """The whole Stokes operator (Yu = A11 u + A12 p, Yp = A21 u) of the
    restatement against the reference's own MFStokesWrapper_A_AVX / _A."""
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    yu, yp = ora.stokes_a(dims, g["coords"], g["eta"], uz, g["p"])
    for kind in ("avx", "ref"):
        assert relerr(yu, g["a_u_" + kind]) < 1e-13
        assert relerr(yp, g["a_p_" + kind]) < 1e-13


@pytest.mark.parametrize("name", __import__("conftest").marker_golden_names())
def test_oracle_marker_projection_matches_reference(ora, name):
    """Marker -> Gauss-point (eta, rho) of the restatement against the
    reference's own Q1 projection (src/material_point_utils.c, Route A)."""
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    eq, rq = ora.marker_project(dims, g["wil"], g["xi"], g["eta"], g["rho"])
    assert relerr(eq, g["eta_qp"]) < 1e-13
    assert relerr(rq, g["rho_qp"]) < 1e-13
    # values stay inside each element's node-value range (the clamp)
    assert np.all(eq >= g["eta"].min() * (1 - 1e-12)) and np.all(eq <= g["eta"].max() * (1 + 1e-12))


@pytest.mark.parametrize("name", residual_golden_names())
def test_oracle_residual_matches_reference(ora, name):
    """The restated momentum residual against the reference's own
    FormFunctionLocal_U (src/stokes_form_function.c:99-243), and the residual
    as the sum of its parts: A11 u + A12 p minus the body-force load."""
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    ru = ora.residual_u(dims, g["coords"], g["eta"], g["fu"], g["u"], g["p"])
    assert relerr(ru, g["ru"]) < TOL
    zero = ora.residual_u(dims, g["coords"], g["eta"], np.zeros_like(g["fu"]), g["u"], g["p"])
    parts = ora.a11(dims, g["coords"], g["eta"], g["u"], "ref") + ora.a12(dims, g["coords"], g["p"], "ref")
    assert relerr(zero, parts) < TOL
