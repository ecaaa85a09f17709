"""The kernels' per-element arithmetic (csrc/q2_core.cuh) compiled for the host
with g++ and checked against the oracle -- the GPU kernels' algorithm is
validated here without a GPU."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from conftest import PKG_ROOT, REPO, relerr
from pt_b200 import mesh as M


@pytest.fixture(scope="module")
def core(tmp_path_factory):
    out = tmp_path_factory.mktemp("core") / "libcore.so"
    src = os.path.join(REPO, "tests", "core_host_check.cpp")
    subprocess.run(["g++", "-O2", "-fPIC", "-shared", "-I", os.path.join(PKG_ROOT, "csrc"), src, "-o", str(out)],
                   check=True)
    lib = ctypes.CDLL(str(out))
    dp = ctypes.POINTER(ctypes.c_double)
    for f in ("core_a11_f64", "core_a11_f32", "core_a11_plane_f64", "core_a11_plane_f32"):
        getattr(lib, f).argtypes = [ctypes.c_int] * 3 + [dp] * 4
    return lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


@pytest.mark.parametrize("workload", ["c0", "box:1,1,1", "box:3,2,4", "box:5,1,2"])
def test_core_a11_matches_oracle(core, ora, workload):
    m, eta, _ = M.problem(workload)
    u = M.uniform_vec(m.nvel, 3)
    ref = ora.a11(m.dims, m.coords, eta, u)
    y = np.zeros(m.nvel)
    core.core_a11_f64(*m.dims, _p(m.coords), _p(eta), _p(u), _p(y))
    assert relerr(y, ref) < 1e-13
    y32 = np.zeros(m.nvel)
    core.core_a11_f32(*m.dims, _p(m.coords), _p(eta), _p(u), _p(y32))
    assert relerr(y32, ref) < 5e-5


@pytest.mark.parametrize("workload", ["c0", "box:1,1,1", "box:3,2,4"])
def test_stream_kernel_algorithm_matches_oracle(core, ora, workload):
    """Per-plane algorithm of the streaming kernel with the precomputed
    geometry factor K (csrc/q2_plane.cuh)."""
    m, eta, _ = M.problem(workload)
    u = M.uniform_vec(m.nvel, 4)
    ref = ora.a11(m.dims, m.coords, eta, u)
    y = np.zeros(m.nvel)
    assert core.core_a11_plane_f64(*m.dims, _p(m.coords), _p(eta), _p(u), _p(y)) == 0
    assert relerr(y, ref) < 1e-13
    y32 = np.zeros(m.nvel)
    assert core.core_a11_plane_f32(*m.dims, _p(m.coords), _p(eta), _p(u), _p(y32)) == 0
    assert relerr(y32, ref) < 5e-5


def test_stream_geometry_flags_nonpositive_viscosity(core):
    m, eta, _ = M.problem("box:2,2,2")
    eta = eta.copy()
    eta[5] = -1.0
    y = np.zeros(m.nvel)
    u = M.uniform_vec(m.nvel, 4)
    assert core.core_a11_plane_f64(*m.dims, _p(m.coords), _p(eta), _p(u), _p(y)) == 1


@pytest.mark.parametrize("workload", ["c0", "box:1,1,1", "box:3,2,4"])
def test_stream_diag_algorithm_matches_oracle(core, ora, workload):
    """Sum-factorised diagonal from the Gauss-point factor K (the streaming
    diag kernel's per-plane arithmetic, q2::diag_form_plane)."""
    m, eta, _ = M.problem(workload)
    ref = ora.diag(m.dims, m.coords, eta)
    d = np.zeros(m.nvel)
    core.core_diag_plane_f64.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_double)] * 3
    assert core.core_diag_plane_f64(*m.dims, _p(m.coords), _p(eta), _p(d)) == 0
    assert relerr(d, ref) < 1e-13
