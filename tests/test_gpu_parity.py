"""GPU parity: libpt_b200.so (through its C ABI) against the reference's own
outputs (golden fixtures) and the oracle.

Tolerances (relative, ||y - y_ref||_inf / ||y_ref||_inf):
  FP64 operators  1e-12   (the project's parity bar)
  FP32 A11        5e-5    (FP32 arithmetic and accumulation, eta contrast <= 1e4)
"""
import numpy as np
import pytest

from conftest import golden_names, load_golden, relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 5e-5


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA device required for -m gpu tests")
    return torch


def make_op(m, eta=None, mask=None, a11_op="b200"):
    from pt_b200 import MatStokesMF
    op = MatStokesMF(*m.dims, a11_op=a11_op)
    op.SetUp(m.coords, eta, mask)
    return op


@pytest.mark.parametrize("a11_op", ["b200_stream", "b200_ebe", "b200_colour"])
@pytest.mark.parametrize("name", golden_names())
def test_spmvop_level_matches_reference(torch_cuda, name, a11_op):
    g = load_golden(name)
    m = M.BoxMesh(*(int(v) for v in g["dims"]), g["coords"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    with make_op(m, g["eta"], None, a11_op) as op:
        assert relerr(op.MFStokesWrapper_A11(uz), g["a11_tensor"]) < TOL64
        assert relerr(op.MFStokesWrapper_A11(uz), g["a11_avx"]) < TOL64
        assert relerr(op.MFStokesWrapper_diagA11(), g["diag"]) < TOL64
        assert relerr(op.MFStokesWrapper_A21(uz), g["a21"]) < TOL64
        assert relerr(op.MFStokesWrapper_A12(g["p"]), g["a12_avx"]) < TOL64


# shapes exercising the streaming kernel's tiling: partial warps, 1-3 x-tiles
# (x-colouring), single rows, many z-chunks (z-colouring)
@pytest.mark.parametrize("workload", ["c0", "box:3,2,4", "box:1,1,1", "box:1,2,3", "box:7,5,3", "box:33,2,2",
                                      "box:2,40,1", "box:64,3,1", "box:130,2,3", "box:257,1,2", "box:3,2,40",
                                      "box:65,9,7", "box:128,3,5", "box:100,4,11"])
@pytest.mark.parametrize("a11_op", ["b200", "b200_stream"])
def test_matshell_level_matches_oracle(torch_cuda, ora, workload, a11_op):
    m, eta, mask = M.problem(workload, seed=5)
    x = M.uniform_vec(m.nvel, 6)
    p = M.uniform_vec(m.npres, 7)
    with make_op(m, eta, mask, a11_op) as op:
        assert relerr(op.MatMult_MFStokes_A11(x), ora.matmult_a11(m.dims, m.coords, eta, mask, x)) < TOL64
        assert relerr(op.MatGetDiagonal_MFStokes_A11(), ora.getdiag_a11(m.dims, m.coords, eta, mask)) < TOL64
        assert relerr(op.MatMult_MFStokes_A12(p), ora.matmult_a12(m.dims, m.coords, mask, p)) < TOL64
        assert relerr(op.MatMult_MFStokes_A21(x), ora.matmult_a21(m.dims, m.coords, mask, x)) < TOL64
        # Dirichlet rows are exact copies (BCListInsertDirichlet_MatMult, scale 1)
        y = op.MatMult_MFStokes_A11(x)
        bc = mask.astype(bool)
        assert np.array_equal(y[bc], x[bc])


def test_device_and_host_paths_agree_bitwise(torch_cuda):
    torch = torch_cuda
    m, eta, mask = M.problem("box:9,6,5", seed=2)
    x = M.uniform_vec(m.nvel, 3)
    with make_op(m, eta, mask) as op:
        yh = op.MatMult_MFStokes_A11(x)
        xd = torch.from_numpy(x).cuda()
        yd = op.MatMult_MFStokes_A11(xd)
        torch.cuda.synchronize()
        assert np.array_equal(yh, yd.cpu().numpy())


def test_apply_is_deterministic(torch_cuda):
    """No atomics: repeated applies are bitwise identical."""
    torch = torch_cuda
    m, eta, mask = M.problem("box:17,9,6", seed=4)
    with make_op(m, eta, mask) as op:
        xd = torch.from_numpy(M.uniform_vec(m.nvel, 5)).cuda()
        y1 = op.MatMult_MFStokes_A11(xd).clone()
        y2 = op.MatMult_MFStokes_A11(xd).clone()
        torch.cuda.synchronize()
        assert torch.equal(y1, y2)


def test_stream_diag_runs_on_the_streaming_tiles(torch_cuda, ora):
    """diag(A11) of a streaming op is the sum-factorised kernel on the
    streaming tiles: one launch per colour class of tiles (4 for a box one
    tile wide), not the 8-colour element kernel; bitwise repeatable, and
    equal to the oracle and to the 8-colour kernel to FP64 rounding."""
    torch = torch_cuda
    m, eta, _ = M.problem("box:17,9,6", seed=6)
    with make_op(m, eta, None, "b200_stream") as a, make_op(m, eta, None, "b200_colour") as b:
        d1 = a.MFStokesWrapper_diagA11(torch.empty(m.nvel, dtype=torch.float64, device="cuda")).clone()
        a.reset_launch_count()
        d2 = a.MFStokesWrapper_diagA11(torch.empty(m.nvel, dtype=torch.float64, device="cuda"))
        torch.cuda.synchronize()
        assert a.launch_count() == 4
        assert torch.equal(d1, d2)
        dc = b.MFStokesWrapper_diagA11(torch.empty(m.nvel, dtype=torch.float64, device="cuda"))
        torch.cuda.synchronize()
        d = d2.cpu().numpy()
        assert relerr(d, ora.diag(m.dims, m.coords, eta)) < TOL64
        assert relerr(d, dc.cpu().numpy()) < 1e-14


@pytest.mark.parametrize("other", ["b200_colour", "b200_ebe"])
@pytest.mark.parametrize("workload", ["box:40,7,5", "box:150,3,9", "box:128,4,6"])
def test_kernels_agree(torch_cuda, workload, other):
    """The streaming kernel, the stored element matrices and the 8-colour
    kernel agree to FP64 rounding."""
    torch = torch_cuda
    m, eta, mask = M.problem(workload, seed=8)
    xd = torch.from_numpy(M.uniform_vec(m.nvel, 9)).cuda()
    with make_op(m, eta, mask, "b200_stream") as a, make_op(m, eta, mask, other) as b:
        ya = a.MatMult_MFStokes_A11(xd).cpu().numpy()
        yb = b.MatMult_MFStokes_A11(xd).cpu().numpy()
        assert relerr(ya, yb) < 1e-14


@pytest.mark.parametrize("workload", ["c0", "box:7,5,3"])
def test_fp32_apply(torch_cuda, ora, workload):
    torch = torch_cuda
    m, eta, mask = M.problem(workload, seed=1)
    x = M.uniform_vec(m.nvel, 2)
    ref = ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    with make_op(m, eta, mask) as op:
        y32 = op.MatMult_MFStokes_A11(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
        assert relerr(y32, ref) < TOL32


def test_unknown_a11_op_rejected(torch_cuda):
    from pt_b200 import MatStokesMF, PtError
    with pytest.raises(PtError, match="No -a11_op"):
        MatStokesMF(2, 2, 2, a11_op="avx")


def test_apply_before_setup_is_an_error(torch_cuda):
    from pt_b200 import MatStokesMF, PtError
    with MatStokesMF(2, 2, 2) as op:
        with pytest.raises(PtError, match="PT_ERR_STATE"):
            op.MFStokesWrapper_A11(np.zeros(op.nvel))


def test_large_mesh_properties(torch_cuda, ora):
    """At 64^3 (6.4M velocity dofs, sinker viscosity): direct oracle
    comparison plus the size-independent invariants: symmetry of A11,
    linearity, rigid-body null space, A12 = A21^T."""
    torch = torch_cuda
    m, eta, mask = M.problem("c1", seed=0)
    u = M.uniform_vec(m.nvel, 1)
    v = M.uniform_vec(m.nvel, 2)
    p = M.uniform_vec(m.npres, 3)
    with make_op(m, eta, None) as op:
        ud, vd = torch.from_numpy(u).cuda(), torch.from_numpy(v).cuda()
        Au = op.MFStokesWrapper_A11(ud)
        Av = op.MFStokesWrapper_A11(vd)
        # symmetry: v.(A u) == u.(A v)
        a, b = float(torch.dot(vd, Au)), float(torch.dot(ud, Av))
        assert abs(a - b) <= 1e-12 * (abs(a) + abs(b))
        # linearity
        Aw = op.MFStokesWrapper_A11(2.0 * ud - 3.0 * vd)
        assert relerr(Aw.cpu().numpy(), (2.0 * Au - 3.0 * Av).cpu().numpy()) < 1e-12
        # rigid rotation about z is in the kernel
        x = m.coords.reshape(-1, 3)
        rot = np.cross(np.array([0.0, 0.0, 1.0])[None, :], x).reshape(-1)
        Ar = op.MFStokesWrapper_A11(torch.from_numpy(rot).cuda())
        assert float(Ar.abs().max()) < 1e-12 * float(Au.abs().max())
        # adjointness of B and B^T
        Bu = op.MFStokesWrapper_A21(ud)
        Btp = op.MFStokesWrapper_A12(torch.from_numpy(p).cuda())
        lhs = float(torch.dot(torch.from_numpy(p).cuda(), Bu))
        rhs = float(torch.dot(Btp, ud))
        assert abs(lhs - rhs) <= 1e-12 * (abs(lhs) + abs(rhs))
        # direct comparison with the oracle at this size
        assert relerr(Au.cpu().numpy(), ora.a11(m.dims, m.coords, eta, u)) < TOL64


def test_tiling_schedules_agree_with_the_oracle(ora):
    """Every z-chunk depth gives the oracle's result to 1e-12 (schedules only
    reorder the node sums), and set_tiling(0) restores the default."""
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem("box:40,9,13", seed=21)
    x = M.uniform_vec(m.nvel, 22)
    ref = ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    with MatStokesMF(*m.dims, a11_op="b200_stream") as op:
        op.SetUp(m.coords, eta, mask)
        default = op.tiling
        xd = torch.from_numpy(x).cuda()
        for lz in (1, 2, 3, 5, 13, 40):
            op.set_tiling(lz)
            assert op.tiling == min(lz, m.mz)
            y = op.MatMult_MFStokes_A11(xd).cpu().numpy()
            assert relerr(y, ref) < 1e-12, lz
        op.set_tiling(0)
        assert op.tiling == default
        best, table = op.autotune_tiling(xd, candidates=(0, 2, 4))
        assert op.tiling == best and best in table


@pytest.mark.parametrize("lz", [0, 3])
def test_pipelined_host_apply_is_bitwise_the_device_apply(lz):
    """With pinned host arrays the host-pointer applies overlap their copies
    with the compute group by group; the result is bitwise the device apply's
    (MatShell and SpMVOp level), and pageable arrays give the same."""
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem("box:24,10,30", seed=23)
    x = M.uniform_vec(m.nvel, 24)
    with MatStokesMF(*m.dims, a11_op="b200_stream") as op:
        op.SetUp(m.coords, eta, mask)
        op.set_tiling(lz)
        xd = torch.from_numpy(x).cuda()
        y_dev = op.MatMult_MFStokes_A11(xd).cpu().numpy()
        a_dev = op.MFStokesWrapper_A11(xd).cpu().numpy()
        xp = torch.from_numpy(x).pin_memory()
        yp = torch.empty(m.nvel, dtype=torch.float64).pin_memory()
        op.MatMult_MFStokes_A11(xp.numpy(), yp.numpy())
        assert np.array_equal(yp.numpy(), y_dev)
        op.MFStokesWrapper_A11(xp.numpy(), yp.numpy())
        assert np.array_equal(yp.numpy(), a_dev)
        assert np.array_equal(op.MatMult_MFStokes_A11(x.copy()), y_dev)


@pytest.mark.parametrize("a11_op", ["b200_stream", "b200_ebe", "b200_colour"])
@pytest.mark.parametrize("name", golden_names())
def test_stokes_operator_matches_reference(torch_cuda, name, a11_op):
    """The whole Stokes operator (Yu = A11 u + A12 p, Yp = A21 u) against the
    reference's own MFStokesWrapper_A_AVX and MFStokesWrapper_A."""
    g = load_golden(name)
    m = M.BoxMesh(*(int(v) for v in g["dims"]), g["coords"])
    uz = g["u"].copy()
    uz[g["mask"].astype(bool)] = 0.0
    with make_op(m, g["eta"], None, a11_op) as op:
        yu, yp = op.MFStokesWrapper_A(uz, g["p"])
        for kind in ("avx", "ref"):
            assert relerr(yu, g["a_u_" + kind]) < TOL64
            assert relerr(yp, g["a_p_" + kind]) < TOL64


@pytest.mark.parametrize("workload", ["c0", "box:3,2,4", "box:7,5,3", "box:65,9,7", "box:40,20,9", "box:130,3,4"])
@pytest.mark.parametrize("a11_op", ["b200", "b200_stream"])
def test_matmult_stokes_a_matches_oracle(torch_cuda, ora, workload, a11_op):
    """MatMult_MFStokes_A on one rank (device and host paths) against the
    oracle's restatement of its BC semantics, with the default op (stored
    element matrices on these small boxes) and with the streaming kernel."""
    torch = torch_cuda
    m, eta, mask = M.problem(workload, seed=31)
    u = M.uniform_vec(m.nvel, 32)
    p = M.uniform_vec(m.npres, 33)
    ru, rp = ora.matmult_a(m.dims, m.coords, eta, mask, u, p)
    with make_op(m, eta, mask, a11_op) as op:
        yu, yp = op.MatMult_MFStokes_A(u, p)
        assert relerr(yu, ru) < TOL64 and relerr(yp, rp) < TOL64
        du, dp = op.MatMult_MFStokes_A(torch.from_numpy(u).cuda(), torch.from_numpy(p).cuda())
        assert np.array_equal(du.cpu().numpy(), yu) and np.array_equal(dp.cpu().numpy(), yp)
        bc = mask.astype(bool)
        assert np.array_equal(yu[bc], u[bc])


@pytest.mark.parametrize("a11_op", ["b200", "b200_colour"])
@pytest.mark.parametrize("part", [((1, 2), (0, 3), (2, 4)), ((0, 5), (1, 4), (0, 2)), ((2, 3), (0, 1), (1, 3))])
def test_ghosted_rank_box_matches_oracle(torch_cuda, ora, part, a11_op):
    """One rank of a multi-rank run: the op owns an element sub-box inside a
    ghosted local node box (stencil width 2, clipped at the global boundary).
    The SpMVOp-level applies read and write the ghosted local arrays and give
    the owned elements' unassembled contributions, as the oracle on the
    sub-box embedded in the ghosted box."""
    from pt_b200 import MatStokesMF
    torch = torch_cuda
    m, eta, mask = M.problem("box:5,4,4", seed=41)
    G = [2 * d + 1 for d in m.dims]                      # global nodes per axis
    (ex0, ex1), (ey0, ey1), (ez0, ez1) = part            # owned elements [e0, e1)
    lo = [max(0, 2 * e0 - 2) for e0 in (ex0, ey0, ez0)]  # ghosted node box
    hi = [min(g, 2 * e1 + 1 + 2) for e1, g in zip((ex1, ey1, ez1), G)]
    nb = [h - l for h, l in zip(hi, lo)]
    off = [2 * e0 - l for e0, l in zip((ex0, ey0, ez0), lo)]
    sub = (ex1 - ex0, ey1 - ey0, ez1 - ez0)
    c = m.coords.reshape(G[2], G[1], G[0], 3)
    cg = np.ascontiguousarray(c[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]].reshape(-1))
    e = eta.reshape(m.mz, m.my, m.mx, 27)[ez0:ez1, ey0:ey1, ex0:ex1].reshape(-1).copy()
    u = M.uniform_vec(3 * nb[0] * nb[1] * nb[2], 42)
    p = M.uniform_vec(4 * sub[0] * sub[1] * sub[2], 43)
    # oracle: the sub-box on its own node block, embedded at the offset
    ug = u.reshape(nb[2], nb[1], nb[0], 3)
    sl = tuple(slice(o, o + 2 * n + 1) for o, n in zip(off[::-1], sub[::-1]))
    cs = np.ascontiguousarray(cg.reshape(nb[2], nb[1], nb[0], 3)[sl].reshape(-1))
    us = np.ascontiguousarray(ug[sl].reshape(-1))
    ref_a11 = np.zeros_like(ug)
    ref_a11[sl] = ora.a11(sub, cs, e, us).reshape(ref_a11[sl].shape)
    ref_a12 = np.zeros_like(ug)
    ref_a12[sl] = ora.a12(sub, cs, p).reshape(ref_a12[sl].shape)
    with MatStokesMF(*sub, a11_op=a11_op, node_box=(*nb, *off)) as op:
        op.set_coords(cg)
        op.set_eta(e)
        y = op.MFStokesWrapper_A11(torch.from_numpy(u).cuda()).cpu().numpy()
        assert relerr(y, ref_a11.reshape(-1)) < TOL64
        assert relerr(op.MFStokesWrapper_A21(u), ora.a21(sub, cs, us)) < TOL64
        assert relerr(op.MFStokesWrapper_A12(p), ref_a12.reshape(-1)) < TOL64
        d = op.MFStokesWrapper_diagA11()
        dref = np.zeros_like(ug)
        dref[sl] = ora.diag(sub, cs, e).reshape(dref[sl].shape)
        assert relerr(d, dref.reshape(-1)) < TOL64


@pytest.mark.parametrize("name", __import__("conftest").marker_golden_names())
def test_marker_projection_matches_reference(torch_cuda, name):
    """Gauss-point (eta, rho) from markers against the reference's own Q1
    projection (src/material_point_utils.c); installing the result makes the
    op's A11 equal to the oracle's with that viscosity."""
    torch = torch_cuda
    from pt_b200 import MatStokesMF
    g = load_golden(name)
    dims = tuple(int(v) for v in g["dims"])
    m, _, mask = M.problem("c0" if dims == (8, 8, 8) else "box:%d,%d,%d" % dims)
    with MatStokesMF(*dims) as op:
        op.set_coords(m.coords)
        eq, rq = op.ProjectMarkers(g["wil"], g["xi"], g["eta"], g["rho"])
        assert relerr(eq, g["eta_qp"]) < TOL64 and relerr(rq, g["rho_qp"]) < TOL64
        # device path, markers in another order: the same values
        perm = np.random.default_rng(3).permutation(len(g["wil"]))
        t = lambda a: torch.from_numpy(np.ascontiguousarray(a[perm])).cuda()
        deq, drq = op.ProjectMarkers(t(g["wil"]), t(g["xi"]), t(g["eta"]), t(g["rho"]))
        assert relerr(deq.cpu().numpy(), g["eta_qp"]) < TOL64
        x = M.uniform_vec(m.nvel, 9)
        y = op.MFStokesWrapper_A11(x)
    from oracle import Oracle
    assert relerr(y, Oracle().a11(dims, m.coords, deq.cpu().numpy(), x)) < TOL64


def test_marker_projection_rejects_markers_outside_the_box(torch_cuda):
    from pt_b200 import MatStokesMF, PtError
    m, eta, mask = M.problem("box:3,2,2")
    wil, xi, x, e, r = M.markers(m, 4, seed=5)
    wil[7] = 12  # element count is 12
    with MatStokesMF(*m.dims) as op:
        op.set_coords(m.coords)
        with pytest.raises(PtError, match="1 markers have an element index outside"):
            op.ProjectMarkers(wil, xi, e, r, install=False)
        wil[3] = -1
        wil[11] = 1 << 30
        with pytest.raises(PtError, match="3 markers have an element index outside"):
            op.ProjectMarkers(wil, xi, e, r, install=False)


def test_divergence_blocks_follow_coordinate_updates(torch_cuda, ora):
    """B u and B^T p use element blocks stored from the coordinates: after new
    coordinates they are rebuilt (a viscosity update keeps them), so both
    applies still match the oracle on the new mesh."""
    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem("box:6,5,4", seed=8)
    m2 = M.make_mesh(*m.dims, perturb=0.1, seed=99)
    x = M.uniform_vec(m.nvel, 3)
    p = M.uniform_vec(m.npres, 4)
    with MatStokesMF(*m.dims) as op:
        op.SetUp(m.coords, eta, mask)
        assert relerr(op.MFStokesWrapper_A21(x), ora.a21(m.dims, m.coords, x)) < TOL64
        op.set_eta(eta[::-1].copy())
        assert relerr(op.MFStokesWrapper_A12(p), ora.a12(m.dims, m.coords, p)) < TOL64
        op.set_coords(m2.coords)
        assert relerr(op.MFStokesWrapper_A21(x), ora.a21(m.dims, m2.coords, x)) < TOL64
        assert relerr(op.MFStokesWrapper_A12(p), ora.a12(m.dims, m2.coords, p)) < TOL64
        assert relerr(op.MatMult_MFStokes_A12(p), ora.matmult_a12(m.dims, m2.coords, mask, p)) < TOL64
