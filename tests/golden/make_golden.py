"""Generates the golden fixtures in this directory from the reference's own code.

The outputs come from oracle/_ref/libptref.so, i.e. the reference's
src/stokes_operators_{tensor,avx,mf}.c and src/element_utils_q{1,2}.c compiled
unmodified (oracle/Makefile, Route A).  Inputs are seeded synthetic box meshes
(ptatin-gene_b200/pt_b200/mesh.py).  Re-run after changing either:

    python tests/golden/make_golden.py          (markers and residual fixtures; operator fixtures if absent)
    python tests/golden/make_golden.py --all    (all fixtures)

Each fixture stores the inputs and the reference outputs of
  A11 via "tensor", "avx" and "ref" (MFStokesWrapper_A11_*),
  diag(A11) (MFStokesWrapper_diagA11),
  A21 = B u (MFStokesWrapper_A21),
  A12 = B^T p via "avx" and "ref" (MFStokesWrapper_A12_AVX / MFStokesWrapper_A12),
  the whole Stokes operator (Yu = A11 u + A12 p, Yp = A21 u) via "avx" and "ref"
  (MFStokesWrapper_A_AVX / MFStokesWrapper_A),
all as unassembled local sums on one rank (local == global numbering).

The residual fixtures (residual_*) store the inputs and output of the
reference's momentum residual FormFunctionLocal_U
(src/stokes_form_function.c:99-243): u with arbitrary values on Dirichlet dofs
(the caller inserts boundary values, it does not zero them), p, the
Gauss-point body force fu ([27 nel][3], QPntVolCoefStokes.Fu) and
ru = A11 u + A12 p - body force, unassembled.
The reference's OpenMP scatter ("omp critical") sums in thread order, so a
re-run reproduces the A11 outputs only to ~1e-16 relative.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, REPO)
sys.path.insert(0, os.path.join(REPO, "ptatin-gene_b200"))

import oracle  # noqa: E402
from pt_b200 import mesh as M  # noqa: E402

CASES = {
    # name: (workload, u seed, p seed, use the reference's X+Y+Z+c+3 vector)
    "c0_8x8x8": ("c0", 11, 12, False),
    "box_3x2x4": ("box:3,2,4", 21, 22, False),
    "box_1x1x3": ("box:1,1,3", 31, 32, False),
    "box_5x1x2_refvec": ("box:5,1,2", 41, 42, True),
}


RESIDUAL_CASES = {
    # name: (workload, u seed, p seed, body-force seed)
    "residual_c0_8x8x8": ("c0", 61, 62, 63),
    "residual_box_3x2x4": ("box:3,2,4", 71, 72, 73),
    "residual_box_1x1x3": ("box:1,1,3", 81, 82, 83),
}


MARKER_CASES = {
    # name: (workload, markers per element, seed)
    "markers_c0_8x8x8": ("c0", 6, 51),
    "markers_box_3x2x4": ("box:3,2,4", 11, 52),
}


def make_markers(name, workload, per_element, seed):
    """Gauss-point (eta, rho) from seeded markers by the reference's Q1
    projection (src/material_point_utils.c:957-1190)."""
    m, _, _ = M.problem(workload)
    wil, xi, x, eta, rho = M.markers(m, per_element, seed=seed)
    eq, rq = oracle.RefCPU().marker_project(m.dims, wil, xi, eta, rho)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array(m.dims, dtype=np.int32), wil=wil, xi=xi,
                        eta=eta, rho=rho, eta_qp=eq, rho_qp=rq)


def make_residual(name, workload, useed, pseed, fseed):
    """FormFunctionLocal_U of the reference (src/stokes_form_function.c:99-243)."""
    m, eta, _ = M.problem(workload)
    u = M.uniform_vec(m.nvel, useed)
    p = M.uniform_vec(m.npres, pseed)
    fu = M.uniform_vec(3 * 27 * m.nel, fseed)
    ru = oracle.RefCPU().residual_u(m.dims, m.coords, eta, fu, u, p)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), dims=np.array(m.dims, dtype=np.int32), coords=m.coords,
                        eta=eta, fu=fu, u=u, p=p, ru=ru)


def make(name, workload, useed, pseed, refvec):
    m, eta, mask = M.problem(workload)
    u = M.reference_test_vector(m) if refvec else M.uniform_vec(m.nvel, useed)
    p = M.uniform_vec(m.npres, pseed)
    uz = u.copy()
    uz[mask.astype(bool)] = 0.0
    r = oracle.RefCPU()
    out = dict(
        dims=np.array(m.dims, dtype=np.int32), coords=m.coords, eta=eta, mask=mask, u=u, p=p,
        a11_tensor=r.a11(m.dims, m.coords, eta, uz, "tensor"),
        a11_avx=r.a11(m.dims, m.coords, eta, uz, "avx"),
        a11_ref=r.a11(m.dims, m.coords, eta, uz, "ref"),
        diag=r.diag(m.dims, m.coords, eta),
        a21=r.a21(m.dims, m.coords, uz),
        a12_avx=r.a12(m.dims, m.coords, p, "avx"),
        a12_ref=r.a12(m.dims, m.coords, p, "ref"),
    )
    out["a_u_avx"], out["a_p_avx"] = r.stokes_a(m.dims, m.coords, eta, uz, p, "avx")
    out["a_u_ref"], out["a_p_ref"] = r.stokes_a(m.dims, m.coords, eta, uz, p, "ref")
    np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


if __name__ == "__main__":
    if not oracle.RefCPU.available():
        oracle.build()
    for name, args in CASES.items():
        if not os.path.exists(os.path.join(HERE, name + ".npz")) or "--all" in sys.argv:
            make(name, *args)
            print("wrote", name)
    for name, args in MARKER_CASES.items():
        make_markers(name, *args)
        print("wrote", name)
    for name, args in RESIDUAL_CASES.items():
        make_residual(name, *args)
        print("wrote", name)
