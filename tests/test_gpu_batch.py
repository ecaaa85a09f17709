"""Batched A11 over independent boxes: with each op's own tiling a problem's
result is bitwise the result of its own apply (FP64 and FP32, SpMVOp and
MatShell level), for a mix of tile widths (rows of <=32, <=64 and >64
elements); other z-chunk depths change only the summation order on chunk
boundary planes (agreement to rounding)."""
import pytest

from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu

SHAPES = [(8, 8, 8), (12, 16, 8), (32, 24, 16), (40, 5, 7), (70, 3, 4), (17, 9, 33)]


@pytest.fixture(scope="module")
def problems():
    import torch

    from pt_b200 import MatStokesMF
    ops, us = [], []
    for i, (mx, my, mz) in enumerate(SHAPES):
        m = M.make_mesh(mx, my, mz, perturb=0.05, seed=i)
        eta = M.eta_per_element(m, contrast=10.0 ** (2 + 2 * (i % 3)), seed=i)
        op = MatStokesMF(mx, my, mz, a11_op="b200_stream")
        op.SetUp(m.coords, eta, M.bc_mask_freeslip(mx, my, mz))
        ops.append(op)
        us.append(torch.from_numpy(M.uniform_vec(m.nvel, 50 + i)).cuda())
    yield ops, us
    for op in ops:
        op.Destroy()


@pytest.mark.parametrize("lz", [None, 1, 3])
@pytest.mark.parametrize("masked", [True, False])
@pytest.mark.parametrize("fp32", [False, True])
def test_batched_equals_individual(problems, lz, masked, fp32):
    import torch

    from pt_b200.batch import BatchA11
    ops, us = problems
    if fp32:
        us = [u.float() for u in us]
    ys = [torch.full_like(u, float("nan")) for u in us]
    with BatchA11(ops, lz=lz) as b:
        b.apply(us, ys, masked=masked)
        torch.cuda.synchronize()
        assert b.launches_per_apply >= 1
    for op, u, y in zip(ops, us, ys):
        ref = op.MatMult_MFStokes_A11(u) if masked else op.MFStokesWrapper_A11(u)
        torch.cuda.synchronize()
        if lz is None:
            assert torch.equal(y, ref)
        else:
            tol = 1e-5 if fp32 else 1e-14
            assert float((y - ref).abs().max()) <= tol * float(ref.abs().max())


def test_batched_matches_oracle(problems, ora):
    """The batched work-list against the oracle directly (MatShell level, FP64),
    not only against each box's own apply."""
    import torch

    from conftest import relerr
    from pt_b200.batch import BatchA11
    ops, us = problems
    ys = [torch.full_like(u, float("nan")) for u in us]
    with BatchA11(ops) as b:
        b.apply(us, ys, masked=True)
        torch.cuda.synchronize()
    for i, ((mx, my, mz), u, y) in enumerate(zip(SHAPES, us, ys)):
        m = M.make_mesh(mx, my, mz, perturb=0.05, seed=i)
        eta = M.eta_per_element(m, contrast=10.0 ** (2 + 2 * (i % 3)), seed=i)
        ref = ora.matmult_a11(m.dims, m.coords, eta, M.bc_mask_freeslip(mx, my, mz), u.cpu().numpy())
        assert relerr(y.cpu().numpy(), ref) < 1e-12, (mx, my, mz)


@pytest.mark.parametrize("fp32", [False, True])
def test_masked_batch_mixes_boxes_with_and_without_a_mask(fp32):
    """A MatShell-level (masked) batched apply over boxes of which some carry
    no Dirichlet mask: those get the plain apply, the others the column and
    row rules, each bitwise its own op's MatMult (the served form submits
    requests with or without a mask into one masked batch)."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200.batch import BatchA11
    ops, us = [], []
    try:
        for i, (mx, my, mz) in enumerate([(8, 8, 8), (12, 6, 9), (20, 4, 5)]):
            m = M.make_mesh(mx, my, mz, perturb=0.05, seed=40 + i)
            eta = M.eta_per_element(m, contrast=1e4, seed=40 + i)
            op = MatStokesMF(mx, my, mz, a11_op="b200_stream")
            op.SetUp(m.coords, eta, M.bc_mask_freeslip(mx, my, mz) if i != 1 else None)
            ops.append(op)
            u = torch.from_numpy(M.uniform_vec(m.nvel, 60 + i)).cuda()
            us.append(u.float() if fp32 else u)
        ys = [torch.full_like(u, float("nan")) for u in us]
        with BatchA11(ops) as b:
            b.apply(us, ys, masked=True)
            torch.cuda.synchronize()
        for op, u, y in zip(ops, us, ys):
            ref = op.MatMult_MFStokes_A11(u)
            torch.cuda.synchronize()
            assert torch.equal(y, ref)
    finally:
        for op in ops:
            op.Destroy()
