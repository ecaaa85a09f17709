"""Device Krylov solves of A11 u = f (FP64 outer, FP64 or FP32 Chebyshev-Jacobi
inner), checked with the oracle's operator: the true FP64 residual, a dense
direct solve on a tiny mesh, agreement of the FP32-smoothed and FP64 solves,
and bitwise repeatability."""
import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu


def setup(workload, seed=0):
    import torch

    from pt_b200 import MatStokesMF
    m, eta, mask = M.problem(workload, seed=seed)
    f = M.uniform_vec(m.nvel, seed + 100)
    f[mask.astype(bool)] = 0.0
    op = MatStokesMF(*m.dims)
    op.SetUp(m.coords, eta, mask)
    return m, eta, mask, f, op, torch.from_numpy(f).cuda()


def true_relres(ora, m, eta, mask, f, x):
    r = f - ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    return np.linalg.norm(r) / np.linalg.norm(f)


@pytest.mark.parametrize("ksp", ["fgmres", "fcg"])
@pytest.mark.parametrize("fp32", [0, 1])
def test_solve_reaches_rtol(ora, ksp, fp32):
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:10,8,6", seed=3)
    x = torch.zeros_like(fd)
    with op, KSPSolveA11(op, ksp=ksp, cheby_fp32=fp32, rtol=1e-8, max_it=3000) as ksp_:
        st = ksp_.solve(fd, x)
        assert st["converged"] == 1, st
        assert st["rnorm"] <= 1e-8 * st["rnorm0"] * (1 + 1e-6)
        assert true_relres(ora, m, eta, mask, f, x.cpu().numpy()) < 2e-8
        if fp32:
            assert st["a11_f32"] > 0
        else:
            assert st["a11_f32"] == 0


def test_solve_matches_dense_direct_solve(ora):
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:2,2,2", seed=4)
    n = m.nvel
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = ora.matmult_a11(m.dims, m.coords, eta, mask, e)
    xref = np.linalg.solve(A, f)
    x = torch.zeros_like(fd)
    with op, KSPSolveA11(op, rtol=1e-12, max_it=2000) as ksp_:
        st = ksp_.solve(fd, x)
    assert st["converged"] == 1
    assert relerr(x.cpu().numpy(), xref) < 1e-9


def test_fp32_smoothed_matches_fp64_solution():
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("c0", seed=5)
    with op:
        x64 = torch.zeros_like(fd)
        x32 = torch.zeros_like(fd)
        with KSPSolveA11(op, cheby_fp32=0) as k64:
            s64 = k64.solve(fd, x64)
        with KSPSolveA11(op, cheby_fp32=1) as k32:
            s32 = k32.solve(fd, x32)
        assert s64["converged"] and s32["converged"]
        # both meet rtol 1e-8 on the FP64 residual; the solutions agree to the
        # conditioning of A11 times that
        assert relerr(x32.cpu().numpy(), x64.cpu().numpy()) < 1e-5


def test_solve_is_bitwise_repeatable():
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:7,6,5", seed=6)
    with op, KSPSolveA11(op) as k:
        x1 = torch.zeros_like(fd)
        x2 = torch.zeros_like(fd)
        s1 = k.solve(fd, x1)
        s2 = k.solve(fd, x2)
        torch.cuda.synchronize()
        assert s1["its"] == s2["its"]
        assert torch.equal(x1, x2)


@pytest.mark.parametrize("ksp", ["fgmres", "fcg"])
@pytest.mark.parametrize("fp32", [0, 1])
def test_mg_solve_reaches_rtol(ora, ksp, fp32):
    """Geometric V-cycle (re-discretised Q2 levels 16 -> 8 -> 4 -> 2) as the
    preconditioner: converges to rtol 1e-8 on the true FP64 residual."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:16,16,16", seed=7)
    x = torch.zeros_like(fd)
    with op, KSPSolveA11(op, ksp=ksp, pc="mg", cheby_fp32=fp32, rtol=1e-8, max_it=500) as k:
        st = k.solve(fd, x)
        assert st["converged"] == 1, st
        assert st["mg_levels"] == 4
        assert st["a11_coarse"] > 0
        assert true_relres(ora, m, eta, mask, f, x.cpu().numpy()) < 2e-8
        assert (st["a11_f32"] > 0) == bool(fp32)


def test_mg_needs_far_fewer_iterations_than_single_level():
    """A correct coarse-grid correction (prolongation, restriction, coarse
    operators) cuts the outer iteration count several-fold against the
    single-level Chebyshev-Jacobi preconditioner of the same degree."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:16,16,16", seed=8)
    with op:
        x1 = torch.zeros_like(fd)
        x2 = torch.zeros_like(fd)
        with KSPSolveA11(op, pc="cheby_jacobi", max_it=5000) as k:
            s1 = k.solve(fd, x1)
        with KSPSolveA11(op, pc="mg", max_it=5000) as k:
            s2 = k.solve(fd, x2)
        assert s1["converged"] and s2["converged"], (s1, s2)
        assert s2["its"] * 4 <= s1["its"], (s1["its"], s2["its"])
        assert relerr(x2.cpu().numpy(), x1.cpu().numpy()) < 1e-5


def test_mg_is_bitwise_repeatable_and_handles_odd_meshes(ora):
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:12,9,8", seed=9)   # 9 is odd: one level
    with op, KSPSolveA11(op, pc="mg", ksp="fcg", max_it=3000) as k:
        x1 = torch.zeros_like(fd)
        x2 = torch.zeros_like(fd)
        s1 = k.solve(fd, x1)
        s2 = k.solve(fd, x2)
        torch.cuda.synchronize()
        assert s1["converged"] and s1["mg_levels"] == 1
        assert s1["its"] == s2["its"] and torch.equal(x1, x2)
        assert true_relres(ora, m, eta, mask, f, x1.cpu().numpy()) < 2e-8


def test_mg_vcycle_is_symmetric_and_graph_replay_is_bitwise():
    """With FP64 smoothing the V-cycle is a symmetric operator (restriction is
    the transpose of prolongation, pre- and post-smoother are the same
    polynomial), and the captured-graph replay gives bitwise the eager result."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("layered:16,16,8", seed=10)
    free = torch.from_numpy((mask == 0).astype(np.float64)).cuda()
    g = torch.Generator(device="cpu").manual_seed(3)
    r1 = (torch.rand(m.nvel, generator=g, dtype=torch.float64) - 0.5).cuda() * free
    r2 = (torch.rand(m.nvel, generator=g, dtype=torch.float64) - 0.5).cuda() * free
    with op:
        z = {}
        for graph in (0, 1):
            with KSPSolveA11(op, pc="mg", cheby_fp32=0, pc_graph=graph) as k:
                z1 = torch.empty_like(r1)
                z2 = torch.empty_like(r2)
                k.apply_pc(r1, z1)
                k.apply_pc(r2, z2)
                k.apply_pc(r1, z1)   # second replay of the same input
                torch.cuda.synchronize()
                z[graph] = (z1, z2)
        assert torch.equal(z[0][0], z[1][0]) and torch.equal(z[0][1], z[1][1])
        a = torch.dot(z[1][0], r2).item()
        b = torch.dot(r1, z[1][1]).item()
        assert abs(a - b) <= 1e-10 * max(abs(a), abs(b)), (a, b)
        assert torch.dot(z[1][0], r1).item() > 0.0


def test_pc_setup_follows_viscosity_changes(ora):
    """A solver set up for one viscosity re-does its set-up (diagonal,
    eigenvalue estimates, level hierarchy) after the op's viscosity changes,
    and then gives bitwise the result of a fresh solver."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("layered:8,8,8", seed=11)
    eta2 = eta * np.exp(np.sin(np.arange(eta.size) * 0.37))
    with op:
        with KSPSolveA11(op, pc="mg") as k:
            x = torch.zeros_like(fd)
            k.solve(fd, x)
            op.set_eta(eta2)
            x1 = torch.zeros_like(fd)
            s1 = k.solve(fd, x1)
        with KSPSolveA11(op, pc="mg") as k2:
            x2 = torch.zeros_like(fd)
            s2 = k2.solve(fd, x2)
        torch.cuda.synchronize()
        assert s1["converged"] and s1["its"] == s2["its"] and torch.equal(x1, x2)
        assert true_relres(ora, m, eta2, mask, f, x1.cpu().numpy()) < 2e-8


def test_mg_assembled_levels_match_matrix_free_levels():
    """Element-matrix levels apply the same operator as the matrix-free
    kernels: with FP64 smoothing the V-cycles agree to rounding."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("layered:8,8,8", seed=12)
    with op:
        z = {}
        for asm in (0, 1):
            with KSPSolveA11(op, pc="mg", cheby_fp32=0, mg_levels=2, mg_assembled=asm) as k:
                out = torch.empty_like(fd)
                k.apply_pc(fd, out)
                torch.cuda.synchronize()
                z[asm] = out.cpu().numpy()
        assert relerr(z[1], z[0]) < 1e-11


def test_mg_galerkin_levels_equal_rediscretised_levels_where_exact():
    """On an undeformed box with constant viscosity the Q2 spaces are nested
    and both quadratures are exact, so P^T A P equals the re-discretised
    coarse operator (Dirichlet dofs included: a coarse free dof interpolates
    to zero on a fine Dirichlet face).  The Galerkin levels (first one from
    the fine level's quadrature, the next from stored matrices, the 2^3
    coarsest by its dense inverse) then give the re-discretised V-cycle to
    rounding."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200.solver import KSPSolveA11
    m = M.make_mesh(8, 8, 8, perturb=0.0)
    eta = np.full(27 * m.nel, 3.7)
    mask = M.bc_mask_freeslip(*m.dims)
    r = M.uniform_vec(m.nvel, 21)
    r[mask.astype(bool)] = 0.0
    rd = torch.from_numpy(r).cuda()
    with MatStokesMF(*m.dims) as op:
        op.SetUp(m.coords, eta, mask)
        z = {}
        for asm in (1, 2):
            with KSPSolveA11(op, pc="mg", cheby_fp32=0, mg_levels=3, mg_assembled=asm) as k:
                out = torch.empty_like(rd)
                k.apply_pc(rd, out)
                torch.cuda.synchronize()
                z[asm] = out.cpu().numpy()
    assert relerr(z[2], z[1]) < 1e-10


@pytest.mark.parametrize("fp32", [0, 1])
def test_mg_galerkin_solve_converges_and_agrees(ora, fp32):
    """Galerkin coarse levels on a high-contrast perturbed box: the solve
    reaches rtol on the true residual, in no more iterations than the
    re-discretised hierarchy, and both solutions agree."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("layered:16,16,16", seed=5)
    xs, its = {}, {}
    with op:
        for asm in (1, 2):
            x = torch.zeros_like(fd)
            with KSPSolveA11(op, pc="mg", ksp="fcg", cheby_fp32=fp32, mg_assembled=asm, rtol=1e-9,
                             max_it=4000) as k:
                st = k.solve(fd, x)
            assert st["converged"] == 1, st
            xs[asm], its[asm] = x.cpu().numpy(), st["its"]
    assert its[2] <= its[1], its
    assert true_relres(ora, m, eta, mask, f, xs[2]) < 2e-9
    assert relerr(xs[2], xs[1]) < 1e-6


def test_mg_dense_coarsest_level_is_an_exact_solve(ora):
    """One level of 2^3 elements (375 dofs) is solved by its dense inverse:
    the preconditioned iteration converges at once to the direct solution."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:2,2,2", seed=13)
    n = m.nvel
    A = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        A[:, j] = ora.matmult_a11(m.dims, m.coords, eta, mask, e)
    xref = np.linalg.solve(A, f)
    with op, KSPSolveA11(op, pc="mg", ksp="fcg", mg_levels=1, cheby_fp32=0, rtol=1e-10) as k:
        x = torch.zeros_like(fd)
        st = k.solve(fd, x)
    assert st["converged"] and st["its"] <= 2, st
    assert relerr(x.cpu().numpy(), xref) < 1e-10


def test_mg_fp16_coarse_matrices_keep_convergence(ora):
    """FP32 smoothing with the Galerkin levels' element matrices in FP16
    (scaled per element, mg_coarse_half=1, the default) against FP32 copies
    (mg_coarse_half=0) on a 1e6-contrast layered box: both reach rtol on the
    true residual of the reference's own A11, in about the same number of
    iterations, and the solutions agree."""
    import torch

    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("layered:16,16,16", seed=5)
    xs, its = {}, {}
    with op:
        for half in (0, 1):
            x = torch.zeros_like(fd)
            with KSPSolveA11(op, pc="mg", ksp="fcg", cheby_fp32=1, mg_coarse_half=half, rtol=1e-9,
                             max_it=4000) as k:
                st = k.solve(fd, x)
            assert st["converged"] == 1, (half, st)
            xs[half], its[half] = x.cpu().numpy(), st["its"]
    assert its[1] <= 1.1 * its[0] + 2, its
    assert true_relres(ora, m, eta, mask, f, xs[1]) < 2e-9
    assert relerr(xs[1], xs[0]) < 1e-6


def test_mg_coarse_half_option_is_checked():
    from pt_b200 import PtError
    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f, op, fd = setup("box:8,8,8", seed=2)
    with op:
        with pytest.raises(PtError, match="mg_coarse_half"):
            KSPSolveA11(op, pc="mg", mg_coarse_half=2)
