"""Serving form: continuously batched viscous solves.  Each request reaches
rtol on the true FP64 residual (oracle operator), its result is bitwise the
same alone and in a mix that changes while it runs, and admission respects
the memory budget."""
import numpy as np
import pytest

from conftest import relerr
from pt_b200 import mesh as M

pytestmark = pytest.mark.gpu


def request(kind_dims, seed):
    m, eta, mask = M.problem(kind_dims, seed=seed)
    f = M.uniform_vec(m.nvel, seed + 1000)
    f[mask.astype(bool)] = 0.0
    return m, eta, mask, f


def true_relres(ora, m, eta, mask, f, x):
    r = f - ora.matmult_a11(m.dims, m.coords, eta, mask, x)
    return np.linalg.norm(r) / np.linalg.norm(f)


def run(server, reqs, joins, iters=4, limit=200000):
    """reqs: {id: (m, eta, mask, f)}; joins: {step index: [ids]} submitted then."""
    out, k = {}, 0
    pending = dict(joins)
    while True:
        for rid in pending.pop(k, []):
            m, eta, mask, f = reqs[rid]
            server.submit(rid, m.dims, m.coords, eta, mask, f)
        act, queued = server.step(iters)
        for d in server.done():
            out[d["id"]] = d
        k += 1
        if not pending and act == 0 and queued == 0:
            return out
        assert k < limit


@pytest.mark.parametrize("fp32", [1, 0])
def test_served_requests_reach_rtol(ora, fp32):
    from pt_b200.serve import Server
    reqs = {0: request("box:6,5,4", 1), 1: request("layered:8,8,8", 2), 2: request("box:3,7,5", 3)}
    with Server(cheby_fp32=fp32, rtol=1e-8, max_it=5000) as s:
        out = run(s, reqs, {0: [0, 1], 2: [2]})
    assert sorted(out) == [0, 1, 2]
    for rid, d in out.items():
        m, eta, mask, f = reqs[rid]
        assert d["converged"] == 1, d
        assert d["rnorm"] <= 1e-8 * d["rnorm0"] * (1 + 1e-9)
        assert true_relres(ora, m, eta, mask, f, d["x"]) < 1e-7
        assert d["t_submit"] <= d["t_admit"] <= d["t_done"]


def test_result_is_bitwise_the_same_alone_and_in_the_mix():
    from pt_b200.serve import Server
    reqs = {0: request("layered:8,8,6", 4), 1: request("box:6,6,6", 5), 2: request("box:9,4,5", 6),
            3: request("layered:12,8,8", 7), 4: request("box:4,4,4", 8)}
    with Server(rtol=1e-8, max_it=5000) as s:
        alone = run(s, {0: reqs[0]}, {0: [0]})[0]
    # request 0 runs while others join at different iterations and leave
    with Server(rtol=1e-8, max_it=5000) as s:
        mixed = run(s, reqs, {0: [1, 2], 1: [0], 3: [3], 5: [4]}, iters=3)
    assert mixed[0]["its"] == alone["its"]
    assert np.array_equal(mixed[0]["x"], alone["x"])
    with Server(rtol=1e-8, max_it=5000) as s:
        solo3 = run(s, {3: reqs[3]}, {0: [3]})[3]
    assert np.array_equal(mixed[3]["x"], solo3["x"])


def test_admission_respects_memory_budget():
    """With a budget that holds one request at a time the requests are served
    one after another, and all of them finish."""
    from pt_b200.serve import Server
    reqs = {i: request("box:6,6,6", 20 + i) for i in range(3)}
    with Server(rtol=1e-8, memory_budget_bytes=6 << 20) as s:
        for rid, (m, eta, mask, f) in reqs.items():
            s.submit(rid, m.dims, m.coords, eta, mask, f)
        seen_active, out = [], {}
        while len(out) < 3:
            act, queued = s.step(4)
            seen_active.append(act)
            for d in s.done():
                out[d["id"]] = d
            assert s.stats()["bytes_in_use"] <= 6 << 20
    assert max(seen_active) == 1
    assert all(d["converged"] for d in out.values())
    # FIFO: admitted in submission order
    assert out[0]["t_admit"] <= out[1]["t_admit"] <= out[2]["t_admit"]


def test_serving_matches_single_solver(ora):
    """The served FP32-smoothed CG and the single-op device solver (same
    preconditioner) both meet rtol 1e-8; their solutions agree to it."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200.serve import Server
    from pt_b200.solver import KSPSolveA11
    m, eta, mask, f = request("layered:10,8,6", 9)
    with Server(rtol=1e-8) as s:
        d = run(s, {0: (m, eta, mask, f)}, {0: [0]})[0]
    op = MatStokesMF(*m.dims)
    op.SetUp(m.coords, eta, mask)
    with op, KSPSolveA11(op, ksp="fcg", pc="cheby_jacobi", cheby_fp32=1, rtol=1e-8) as k:
        x = torch.zeros(m.nvel, dtype=torch.float64, device="cuda")
        st = k.solve(torch.from_numpy(f).cuda(), x)
    assert st["converged"]
    assert relerr(d["x"], x.cpu().numpy()) < 1e-6


def test_request_without_a_mask_shares_the_batch():
    """A request submitted without a Dirichlet mask runs in the same masked
    batch as the others (plain apply for it, no mask read): it finishes with
    finite values, and a masked request beside it is bitwise what it is alone."""
    from pt_b200.serve import Server
    m, eta, mask, f = request("box:6,5,4", 7)
    m2, eta2, _, f2 = request("box:5,4,4", 8)
    with Server(cheby_fp32=1, rtol=1e-8, max_it=300) as s:
        alone = run(s, {0: (m, eta, mask, f)}, {0: [0]})
    with Server(cheby_fp32=1, rtol=1e-8, max_it=300) as s:
        mixed = run(s, {0: (m, eta, mask, f), 1: (m2, eta2, None, f2)}, {0: [0, 1]})
    assert sorted(mixed) == [0, 1]
    assert alone[0]["converged"] == 1
    assert np.array_equal(mixed[0]["x"], alone[0]["x"])
    assert np.isfinite(mixed[1]["x"]).all()
