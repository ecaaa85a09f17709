"""pt_a11_apply_noalloc_d: the A11 apply for callers that cannot allocate
device memory when they need it (a process that gave the GPU to its own
fixed-size pool, or runs under an exhausted memory cap, or must not stall on
the allocator).  It keeps its geometry scratch in a fixed device array, so it
is checked here against the op-based entry point that allocates (pt_a11_apply_d)
and against the oracle's A11 (the reference's tensor-path arithmetic) on two
calls in a row -- the scratch keeps the previous call's contents, which must
not leak into the next result.  This file is collected last on purpose."""
import ctypes

import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M

TOL64 = 1e-12


def _desc(dims):
    from pt_b200 import _capi
    return _capi.MeshDesc(*dims, 0, 0, 0, 0, 0, 0)


@pytest.mark.gpu
def test_noalloc_apply_matches_op_apply_twice(ora):
    import torch

    from pt_b200 import MatStokesMF, _capi
    assert torch.cuda.is_available()
    lib = _capi.load()
    stream = torch.cuda.current_stream()
    # two different meshes and inputs in a row through the same scratch
    for workload, seed in (("box:16,16,16", 3), ("box:9,5,7", 4)):
        m, eta, _ = M.problem(workload, seed=seed)
        uh = M.uniform_vec(m.nvel, seed + 10)
        u = torch.from_numpy(uh).cuda()
        c = torch.from_numpy(m.coords).cuda()
        e = torch.from_numpy(eta).cuda()
        y = torch.full((m.nvel,), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.pt_a11_apply_noalloc_d(ctypes.byref(_desc(m.dims)), ctypes.c_void_p(c.data_ptr()),
                                        ctypes.c_void_p(e.data_ptr()), ctypes.c_void_p(u.data_ptr()),
                                        ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert st == 0, lib.pt_last_error()
        with MatStokesMF(*m.dims) as op:
            op.SetUp(m.coords, eta, None)
            ref = op.MFStokesWrapper_A11(u)
        torch.cuda.synchronize()
        assert relerr(y.cpu().numpy(), ref.cpu().numpy()) < TOL64
        assert relerr(y.cpu().numpy(), ora.a11(m.dims, m.coords, eta, uh)) < TOL64


def test_noalloc_rejects_meshes_beyond_its_scratch():
    """Size check happens before any CUDA call."""
    from pt_b200 import _capi
    lib = _capi.load()
    st = lib.pt_a11_apply_noalloc_d(ctypes.byref(_desc((40, 40, 40))), ctypes.c_void_p(8), ctypes.c_void_p(8),
                                    ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert st == 1
    assert b"geometry scratch" in lib.pt_last_error()
