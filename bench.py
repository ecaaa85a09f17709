"""Benchmark of the B200 Q2-P1disc Stokes operator (pTatin3D hot path).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload c2|c1|c0] [--no-cpu-baseline]

One step = one FP64 A11 apply (MatMult_MFStokes_A11: Dirichlet columns zeroed,
rows copied) over the whole 128^3 Q2 box of the precision workload (257^3
nodes, 50.9M velocity dofs; nodes perturbed +-0.05h; three viscosity layers
1e3/1/1e-1 plus 64 inclusions 1e-3..1e3; free-slip box BCs).  Inputs are
resident in HBM and larger than L2 (u, y 407 MB each; eta 453 MB), so no L2
flush is needed between steps.

value     = 3N / t_apply in GDoF/s, the device-timed apply (CUDA events on the
            op's stream), whole job over all ranks (replicas: each rank runs
            the same problem; the operator is single-GPU by design).
e2e       = the same metric through the public host-pointer API
            (pt_matmult_a11_h): pinned host x -> device, apply, device -> host y.
roofline  = algorithmic bytes of one apply / its device time against the
            measured HBM copy bandwidth (MEASURED_PEAKS.json).
cpu_baseline = the reference's own AVX A11 (oracle/_ref, compiled from the
            reference sources) on a 128x128x16 slab of the same workload,
            on all host cores.
--impl reference times that reference CPU path only and prints its line.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "ptatin-gene_b200"))

METRIC = "Q2 A11 GDoF/s FP64 vs FP32 @128³; batched solves/s & p99 @rtol 1e-8"

WORKLOAD_TEXT = {
    "c2": "perturbed +-0.05h, layered eta + 64 inclusions (1e6 contrast)",
    "c1": "undeformed, sinker eta (16 spheres r 0.08, 1e4)",
    "c0": "perturbed +-0.1h, log-uniform Gauss-point eta [1e-2, 1e2]",
    "box": "perturbed +-0.1h, log-uniform Gauss-point eta [1e-2, 1e2]",
    "sinker": "perturbed +-0.05h, sinker eta",
    "layered": "perturbed +-0.05h, layered eta + inclusions",
}
# DRAM bytes per element of one FP64 streaming apply (K 1.94 KB + u/y tiles),
# measured with ncu on the 96^3 box: 2 colour launches averaged 0.730 GB for
# 96^3/4 elements.
TRAFFIC_PER_ELEMENT_F64 = 4 * 0.730e9 / 96 ** 3
UNIT = "GDoF/s"


def algorithmic_bytes(m, s=8):
    """u + coords + y (3N each) + eta (27 nel), s bytes per value."""
    return (9 * m.nnodes + 27 * m.nel) * s


def load_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            # the timed region starts once samples flow
            t_end = time.time() + 3.0
            while not self.lines and time.time() < t_end:
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(x, pg, device):
    if pg is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    import torch
    if pg is not None:
        t = torch.zeros(1, device=device)
        pg.all_reduce(t)
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def reference_sample_problem(workload):
    """The CPU sample of a workload: the whole problem when it has at most
    300k elements, else a 16-layer z-slab of it (same generators)."""
    from pt_b200 import mesh as M
    m, eta, mask = M.problem(workload, seed=0) if workload != "c2" else (None, None, None)
    if m is not None and m.nel <= 300_000:
        return m, eta, mask, f"the whole {m.mx}x{m.my}x{m.mz} problem"
    if m is None or workload == "c2":
        m = M.make_mesh(128, 128, 16, perturb=0.05, seed=0)
        eta = M.eta_layered(m, seed=1)
        return m, eta, M.bc_mask_freeslip(*m.dims), "a 128x128x16 slab of the 128^3 workload"
    mx, my, mz = m.dims
    ms = M.make_mesh(mx, my, 16, perturb=0.05, seed=0)
    from pt_b200.mesh import eta_loguniform_qp
    return ms, eta_loguniform_qp(ms, seed=1), M.bc_mask_freeslip(*ms.dims), f"a {mx}x{my}x16 slab"


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def cpu_reference_sample(workload="c2", seconds=12.0, kind="avx", ops=False):
    """Time the reference's own A11 (oracle/_ref, all host cores) on the
    workload's CPU sample; with ops=True also its diag, B and B^T."""
    import oracle
    from pt_b200 import mesh as M
    if not oracle.RefCPU.available():
        oracle.build()
    r = oracle.RefCPU()
    m, eta, mask, what = reference_sample_problem(workload)
    x = M.uniform_vec(m.nvel, 7)
    x[mask.astype(bool)] = 0.0
    p = M.uniform_vec(m.npres, 8)

    def best_of(fn, budget):
        fn()  # warm-up
        times, t_end = [], time.perf_counter() + budget
        while time.perf_counter() < t_end or len(times) < 2:
            t0 = time.perf_counter()
            fn()
            times.append(time.perf_counter() - t0)
        return min(times), len(times)

    nthreads = r.set_threads(os.cpu_count())
    best, nrep = best_of(lambda: r.a11(m.dims, m.coords, eta, x, kind), seconds)
    # one thread as well: the reference's element loop scatters under `omp critical`
    r.set_threads(1)
    best1, nrep1 = best_of(lambda: r.a11(m.dims, m.coords, eta, x, kind), max(1.0, seconds / 4))
    r.set_threads(nthreads)
    out = {
        "value": m.nvel / best / 1e9,
        "unit": UNIT,
        "cores": nthreads,
        "kind": "reference",
        "sample": f"reference {kind} A11 (MFStokesWrapper_A11_AVX, OpenMP {nthreads} threads) on "
                  f"{what}, best of {nrep} applies",
        "seconds_per_apply": best,
        "one_thread": {"value": m.nvel / best1 / 1e9, "seconds_per_apply": best1, "applies": nrep1},
        "cpu_model": cpu_model(),
    }
    if ops:
        budget = max(1.0, seconds / 4)
        out["ops_seconds"] = {
            "diag": best_of(lambda: r.diag(m.dims, m.coords, eta), budget)[0],
            "a21": best_of(lambda: r.a21(m.dims, m.coords, x), budget)[0],
            "a12": best_of(lambda: r.a12(m.dims, m.coords, p, "avx"), budget)[0],
            "stokes_a": best_of(lambda: r.stokes_a(m.dims, m.coords, eta, x, p, "avx"), budget)[0],
        }
        out["ops_gdofs"] = {k: (m.nvel + (m.npres if k == "stokes_a" else 0)) / v / 1e9
                            for k, v in out["ops_seconds"].items()}
    return out


def run_reference(args):
    ws, rank, local, pg = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0, None
    if rank != 0:
        return 0
    try:
        import oracle
        if not oracle.RefCPU.available():
            oracle.build()
        oracle.RefCPU()
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build missing: {e}"}))
        return 0
    from pt_b200 import mesh as M
    r = oracle.RefCPU()
    m, eta, mask, what = reference_sample_problem(args.workload)
    x = M.uniform_vec(m.nvel, 7)
    x[mask.astype(bool)] = 0.0
    for _ in range(args.warmup):
        r.a11(m.dims, m.coords, eta, x, "avx")
    t0 = time.perf_counter()
    for _ in range(args.steps):
        r.a11(m.dims, m.coords, eta, x, "avx")
    dt = (time.perf_counter() - t0) / args.steps
    v = m.nvel / dt / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"A11 FP64 apply on {what} ({args.workload}), reference CPU (oracle/_ref, avx)",
                   "global_batch": 1, "seq_len": 0, "parallelism": "cpu-openmp"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                         "sample": f"{what}, MFStokesWrapper_A11_AVX compiled from the reference sources"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200 import mesh as M

    ws, rank, local, pg = dist_setup(args)
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)

    m, eta, mask = M.problem(args.workload, seed=0)
    stream = torch.cuda.Stream(device=dev)
    op = MatStokesMF(*m.dims, a11_op=args.a11_op, stream=stream)
    op.SetUp(m.coords, eta, mask)
    x = torch.from_numpy(M.uniform_vec(m.nvel, 7)).to(dev)
    y = torch.empty_like(x)
    x32, y32 = x.float(), torch.empty(m.nvel, dtype=torch.float32, device=dev)
    p = torch.from_numpy(M.uniform_vec(m.npres, 8)).to(dev)
    yp = torch.empty(m.npres, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    def timed(fn, k):
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(k):
                fn()
            ev1.record(stream)
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / 1e3

    # ---- tile schedule by the autotuner (untimed), then the headline --------
    tiling = {"lz": op.tiling, "autotune": None}
    if not args.no_autotune and op.a11_op in ("b200_stream", "b200_tmem"):
        best, table = op.autotune_tiling(x)
        tiling = {"lz": best, "autotune_ms": {str(k): round(v, 4) for k, v in table.items()}}
    # ---- headline: FP64 A11 (MatShell level), device resident ----------------
    for _ in range(max(args.warmup, 3)):
        op.MatMult_MFStokes_A11(x, y)
    barrier(pg, dev)
    op.reset_launch_count()
    with ClockSampler(local) as clk:
        t = timed(lambda: op.MatMult_MFStokes_A11(x, y), args.steps)
    launches = op.launch_count()
    t = max_over_ranks(t, pg, dev)
    t_apply = t / args.steps
    value = ws * m.nvel / t_apply / 1e9

    # ---- roofline of the A11 apply ---------------------------------------------
    peak, peak_kind = load_peaks()
    bytes_alg = algorithmic_bytes(m)
    achieved = bytes_alg / t_apply / 1e9

    # ---- other operators and FP32 (device resident) ------------------------------
    extra = {}
    if not args.quick:
        def rate(fn, n):
            for _ in range(2):
                fn()
            dt = timed(fn, max(2, args.steps // 2)) / max(2, args.steps // 2)
            return n / dt / 1e9, dt * 1e3
        extra["a11_fp32_gdofs"], extra["a11_fp32_ms"] = rate(lambda: op.MatMult_MFStokes_A11(x32, y32), m.nvel)
        extra["diag_gdofs"], extra["diag_ms"] = rate(lambda: op.MatGetDiagonal_MFStokes_A11(y), m.nvel)
        extra["a21_gdofs"], extra["a21_ms"] = rate(lambda: op.MatMult_MFStokes_A21(x, yp), m.nvel)
        extra["a12_gdofs"], extra["a12_ms"] = rate(lambda: op.MatMult_MFStokes_A12(p, y), m.nvel)
        # the whole Stokes operator (A11 u + A12 p, A21 u), rate over velocity + pressure dofs
        extra["stokes_a_gdofs"], extra["stokes_a_ms"] = rate(lambda: op.MatMult_MFStokes_A(x, p, y, yp),
                                                             m.nvel + m.npres)
        extra["a11_flops_per_element_ref_count"] = 17253

    # ---- e2e through the host-pointer API (pinned buffers) ----------------------------
    xh = torch.empty(m.nvel, dtype=torch.float64, pin_memory=True)
    xh.copy_(x.cpu())
    yh = torch.empty(m.nvel, dtype=torch.float64, pin_memory=True)
    xn, yn = xh.numpy(), yh.numpy()
    op.MatMult_MFStokes_A11(xn, yn)
    k_e2e = max(2, min(args.steps, 5))
    barrier(pg, dev)
    t0 = time.perf_counter()
    for _ in range(k_e2e):
        op.MatMult_MFStokes_A11(xn, yn)
    t_e2e = max_over_ranks((time.perf_counter() - t0) / k_e2e, pg, dev)
    e2e = {"value": ws * m.nvel / t_e2e / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * m.nvel,
           "d2h_bytes_per_step": 8 * m.nvel, "ms_per_step": t_e2e * 1e3,
           "path": "pt_matmult_a11_h (MatMult_MFStokes_A11 on pinned numpy arrays)"}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_reference_sample(args.workload, seconds=args.cpu_seconds, ops=not args.quick)
        except Exception as e:  # pragma: no cover
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"unavailable: {e}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": t_apply * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"A11 FP64 MatMult, {m.mx}x{m.my}x{m.mz} Q2 box ({m.nvel} velocity dofs), "
                                   f"{WORKLOAD_TEXT.get(args.workload.split(':')[0], args.workload)}, free-slip BCs",
                       "global_batch": 1, "seq_len": 0, "parallelism": f"replicas{ws}",
                       "a11_op": op.a11_op, "tiling": tiling, "l2": "inputs larger than L2 (no flush)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": TRAFFIC_PER_ELEMENT_F64 * m.nel,
                         "traffic_source": "ncu dram__bytes_read+write of the 4 colour launches of one 96^3 apply "
                                           "(profiles/a11_stream_96cubed.md), scaled by the element count",
                         "peak_kind": peak_kind, "algorithmic_bytes_per_apply": bytes_alg},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "extra": extra,
        }
        print(json.dumps(line))
    op.Destroy()
    if pg is not None:
        pg.destroy_process_group()
    return 0


def run_solve(args):
    """Precision form: A11 u = f with f uniform [-1, 1] on free dofs, FP64
    outer Krylov to rtol 1e-8, preconditioned by the geometric V-cycle with
    Chebyshev-Jacobi smoothing (or single-level Chebyshev-Jacobi, --pc) in
    FP64 vs FP32.  Prints one JSON line with both solves and the solutions'
    difference."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200 import mesh as M
    from pt_b200.solver import KSPSolveA11
    torch.cuda.set_device(0)
    m, eta, mask = M.problem(args.workload, seed=0)
    f = M.uniform_vec(m.nvel, 11)
    f[mask.astype(bool)] = 0.0
    fd = torch.from_numpy(f).cuda()
    op = MatStokesMF(*m.dims)
    op.SetUp(m.coords, eta, mask)
    # the fine level's tile schedule from the autotuner, as in the apply bench
    lz, _ = op.autotune_tiling(fd) if not args.no_autotune else (op.tiling, None)
    out = {"mode": "solve", "workload": args.workload, "nvel": m.nvel, "ksp": args.ksp, "pc": args.pc,
           "cheby_degree": args.cheby_degree, "rtol": args.rtol, "tiling_lz": lz}
    sols = {}
    for name, fp32 in (("fp64", 0), ("fp32_smoothed", 1)):
        x = torch.zeros_like(fd)
        with KSPSolveA11(op, ksp=args.ksp, pc=args.pc, cheby_degree=args.cheby_degree, cheby_fp32=fp32,
                         rtol=args.rtol, max_it=args.max_it, restart=args.restart) as k:
            first = k.solve(fd, x)   # builds levels, estimates eigenvalues, warms up
            x.zero_()
            st = k.solve(fd, x)
            st["first_solve_seconds_incl_setup"] = first["seconds"]
        sols[name] = x
        out[name] = st
    d = (sols["fp32_smoothed"] - sols["fp64"]).abs().max().item() / sols["fp64"].abs().max().item()
    out["solution_relerr_fp32_vs_fp64"] = d
    out["time_to_solution_speedup"] = out["fp64"]["seconds"] / out["fp32_smoothed"]["seconds"]
    print(json.dumps(out))
    op.Destroy()
    return 0


def batched_problems(n=256, seed=0):
    """The batched workload: n boxes with axes drawn from {8,12,16,24,32},
    per-element log-uniform eta with contrast drawn from {1e2,1e4,1e6},
    nodes perturbed +-0.05h, free-slip box BCs."""
    from pt_b200 import mesh as M
    rng = np.random.default_rng(seed)
    axes = np.array([8, 12, 16, 24, 32])
    out = []
    for i in range(n):
        mx, my, mz = (int(v) for v in rng.choice(axes, size=3))
        c = float(rng.choice([1e2, 1e4, 1e6]))
        m = M.make_mesh(mx, my, mz, perturb=0.05, seed=seed * 100003 + i)
        eta = M.eta_per_element(m, contrast=c, seed=seed * 100003 + i)
        out.append((m, eta, M.bc_mask_freeslip(mx, my, mz)))
    return out


def run_batched(args):
    """Batched form: one batched A11 apply over all problems (work-list
    launches) vs the same problems applied one after another, FP64 and FP32."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200.batch import BatchA11, autotune_lz
    torch.cuda.set_device(0)
    probs = batched_problems(args.nbatch, seed=0)
    ops, us64 = [], []
    for i, (m, eta, mask) in enumerate(probs):
        op = MatStokesMF(*m.dims)
        op.SetUp(m.coords, eta, mask)
        ops.append(op)
        us64.append(torch.from_numpy(M_uniform(m.nvel, 1000 + i)).cuda())
    ndof = sum(m.nvel for m, _, _ in probs)
    out = {"mode": "batched", "problems": len(probs), "velocity_dofs": ndof,
           "elements": int(sum(m.nel for m, _, _ in probs))}

    def timed(fn, k):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record()
        for _ in range(k):
            fn()
        ev1.record()
        ev1.synchronize()
        return ev0.elapsed_time(ev1) / k

    for prec, us in (("fp64", us64), ("fp32", [u.float() for u in us64])):
        ys = [torch.empty_like(u) for u in us]
        best, table = autotune_lz(ops, us, ys)
        with BatchA11(ops, lz=best if best else None) as b:
            t_b = timed(lambda: b.apply(us, ys, masked=True), args.steps)
            launches = b.launches_per_apply
        # sequential baselines: each box's own default apply ("b200": stored element
        # matrices up to 32^3, else streaming), and the streaming kernel the batch runs
        t_s = timed(lambda: [op.MatMult_MFStokes_A11(u, y) for op, u, y in zip(ops, us, ys)], max(2, args.steps // 4))
        for op in ops:
            op.set_a11_op("b200_stream")
        t_ss = timed(lambda: [op.MatMult_MFStokes_A11(u, y) for op, u, y in zip(ops, us, ys)], max(2, args.steps // 4))
        for op in ops:
            op.set_a11_op("b200")
        out[prec] = {"batched_ms": t_b, "sequential_ms": t_s, "batched_gdofs": ndof / t_b / 1e6,
                     "sequential_gdofs": ndof / t_s / 1e6, "speedup": t_s / t_b,
                     "sequential_stream_ms": t_ss, "speedup_vs_sequential_stream": t_ss / t_b,
                     "launches_per_apply": launches, "autotune_lz": best, "autotune_ms": table}
    print(json.dumps(out))
    for op in ops:
        op.Destroy()
    return 0


def serve_requests(n, seed=0, sizes=(8, 48)):
    """The served stream: cubic boxes m^3, m uniform over sizes; nodes
    perturbed +-0.05h; viscosity 1 with 8 seeded inclusions (radius 0.1), four
    at c^(1/2) and four at c^(-1/2), c log-uniform in [1e2, 1e6]; free-slip box
    BCs; f uniform [-1, 1] on free dofs."""
    from pt_b200 import mesh as M
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        m = int(rng.integers(sizes[0], sizes[1] + 1))
        c = 10.0 ** rng.uniform(2.0, 6.0)
        mesh = M.make_mesh(m, m, m, perturb=0.05, seed=seed * 1000003 + i)
        r = np.random.default_rng(seed * 7919 + i + 1)
        centres = r.uniform(0.0, 1.0, size=(8, 3))
        vals = [c ** 0.5] * 4 + [c ** -0.5] * 4
        eta = M.eta_spheres(mesh, centres, [0.1] * 8, vals)
        mask = M.bc_mask_freeslip(m, m, m)
        f = M_uniform(mesh.nvel, seed * 31 + i)
        f[mask.astype(bool)] = 0.0
        out.append((mesh, eta, mask, f, c))
    return out


def serve_run(reqs, arrivals, iters, **opts):
    """Serve reqs arriving at the given times (seconds on the server clock,
    relative to the first arrival).  Returns (results by id, stats)."""
    from pt_b200.serve import Server
    res, max_active, max_bytes = {}, 0, 0
    with Server(**opts) as s:
        t0 = s.time()
        nxt = 0
        while len(res) < len(reqs):
            now = s.time() - t0
            while nxt < len(reqs) and arrivals[nxt] <= now:
                m, eta, mask, f, _ = reqs[nxt]
                s.submit(nxt, m.dims, m.coords, eta, mask, f)
                nxt += 1
            act, queued = s.step(iters)
            max_active = max(max_active, act)
            max_bytes = max(max_bytes, s.stats()["bytes_in_use"])
            for d in s.done():
                d["t_done"] -= t0
                d["t_submit"] -= t0
                d["t_admit"] -= t0
                res[d["id"]] = d
            if act == 0 and queued == 0 and nxt < len(reqs):
                time.sleep(max(0.0, min(0.01, arrivals[nxt] - (s.time() - t0))))
        st = s.stats()
    st.update(max_active=max_active, max_bytes_in_use=max_bytes)
    return res, st


def run_serve(args):
    """Serving form: Poisson arrivals at ~80% of the measured capacity, solves
    of A11 u = f to rtol 1e-8 by FP32 Chebyshev(3)-Jacobi-preconditioned FP64
    CG, continuously batched; p50/p99 latency and solves/s against serial
    plain FP64 solves of the same requests."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200.solver import KSPSolveA11
    torch.cuda.set_device(0)
    t_gen = time.time()
    cal = serve_requests(args.ncal, seed=1)
    reqs = serve_requests(args.nreq, seed=0)
    t_gen = time.time() - t_gen
    # tile schedule (tile width, z-chunk depth) by the autotuner, on the
    # calibration requests' FP32 applies
    from pt_b200.batch import autotune
    ops = []
    for m, eta, mask, _, _ in cal:
        op = MatStokesMF(*m.dims)
        op.SetUp(m.coords, eta, mask)
        ops.append(op)
    us = [torch.ones(op.nvel, dtype=torch.float32, device="cuda") for op in ops]
    ys = [torch.empty_like(u) for u in us]
    (lz, tile_x), table = autotune(ops, us, ys, lz_candidates=(1, 2, 0), tile_candidates=(0, 64, 128))
    for op in ops:
        op.Destroy()
    opts = dict(rtol=args.rtol, max_it=args.max_it, cheby_fp32=1, cheby_degree=args.cheby_degree,
                memory_budget_bytes=120 << 30, max_active=256, lz=lz, tile_x=tile_x)
    # capacity: a saturated queue (everything arrives at once)
    res_cal, _ = serve_run(cal, [0.0] * len(cal), args.serve_iters, **opts)
    capacity = len(cal) / max(d["t_done"] for d in res_cal.values())
    rate = 0.8 * capacity
    rng = np.random.default_rng(12345)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(reqs)))
    arrivals -= arrivals[0]
    res, st = serve_run(reqs, arrivals, args.serve_iters, **opts)
    lat = np.array([res[i]["t_done"] - arrivals[i] for i in range(len(reqs))])
    wall = max(d["t_done"] for d in res.values())
    its = np.array([res[i]["its"] for i in range(len(reqs))])
    conv = all(res[i]["converged"] for i in range(len(reqs)))
    # true FP64 residual of a sample of served results
    relres = []
    for i in range(0, len(reqs), max(1, len(reqs) // 8)):
        m, eta, mask, f, _ = reqs[i]
        with MatStokesMF(*m.dims) as op:
            op.SetUp(m.coords, eta, mask)
            y = op.MatMult_MFStokes_A11(torch.from_numpy(res[i]["x"]).cuda()).cpu().numpy()
        relres.append(float(np.linalg.norm(f - y) / np.linalg.norm(f)))
    # serial plain FP64 solves (one request at a time, set-up included)
    serial = []
    for i in np.linspace(0, len(reqs) - 1, min(args.nserial, len(reqs))).astype(int):
        m, eta, mask, f, _ = reqs[i]
        torch.cuda.synchronize()
        t = time.time()
        with MatStokesMF(*m.dims) as op:
            op.SetUp(m.coords, eta, mask)
            fd = torch.from_numpy(f).cuda()
            x = torch.zeros_like(fd)
            with KSPSolveA11(op, ksp="fcg", pc="cheby_jacobi", cheby_fp32=0, cheby_degree=args.cheby_degree,
                             rtol=args.rtol, max_it=args.max_it) as k:
                sst = k.solve(fd, x)
            x.cpu()
        serial.append({"seconds": time.time() - t, "its": sst["its"], "converged": sst["converged"],
                       "elements": m.nel, "served_its": res[int(i)]["its"]})
    serial_rate = len(serial) / sum(d["seconds"] for d in serial)
    out = {"mode": "serve", "requests": len(reqs), "sizes": "m^3, m uniform 8..48",
           "contrast": "log-uniform [1e2, 1e6]", "rtol": args.rtol, "iterations_per_step": args.serve_iters,
           "capacity_solves_per_s": capacity, "arrival_rate_per_s": rate, "calibration_requests": len(cal),
           "solves_per_s": len(reqs) / wall, "p50_latency_s": float(np.percentile(lat, 50)),
           "p99_latency_s": float(np.percentile(lat, 99)), "mean_its": float(its.mean()),
           "max_its": int(its.max()), "all_converged": conv, "true_relres_sample_max": max(relres),
           "serial_fp64_solves_per_s": serial_rate, "serial_sample": len(serial),
           "serial_mean_its": float(np.mean([d["its"] for d in serial])),
           "serial_mean_served_its_same_requests": float(np.mean([d["served_its"] for d in serial])),
           "speedup_solves_per_s": (len(reqs) / wall) / serial_rate, "server": st,
           "autotune": {"lz": lz, "tile_x": tile_x, "ms": {f"lz{a}_tx{b}": v for (a, b), v in table.items()}},
           "host_generation_s": t_gen}
    print(json.dumps(out))
    return 0


def run_markers(args):
    """Coefficient producer: Gauss-point (eta, rho) from material points by the
    reference's Q1 projection, device-resident markers (CUDA events) and the
    host path, against the reference's own CPU projection on the same markers."""
    import torch

    from pt_b200 import MatStokesMF
    from pt_b200 import mesh as M
    torch.cuda.set_device(0)
    m, _, _ = M.problem(args.workload, seed=0)
    wil, xi, _, eta, rho = M.markers(m, args.markers_per_element, seed=3)
    n = len(wil)
    op = MatStokesMF(*m.dims)
    op.set_coords(m.coords)
    dw, dx = torch.from_numpy(wil).cuda(), torch.from_numpy(xi).cuda()
    de, dr = torch.from_numpy(eta).cuda(), torch.from_numpy(rho).cuda()
    for _ in range(max(args.warmup, 3)):
        op.ProjectMarkers(dw, dx, de, dr, install=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        op.ProjectMarkers(dw, dx, de, dr, install=False)
    torch.cuda.synchronize()
    t_dev = (time.perf_counter() - t0) / args.steps
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 4)):
        eq, rq = op.ProjectMarkers(wil, xi, eta, rho, install=False)
    t_host = (time.perf_counter() - t0) / max(1, args.steps // 4)
    out = {"mode": "markers", "workload": args.workload, "elements": m.nel, "markers": n,
           "gpu_ms": t_dev * 1e3, "gpu_markers_per_s": n / t_dev, "e2e_ms": t_host * 1e3}
    if not args.no_cpu_baseline:
        import oracle
        if not oracle.RefCPU.available():
            oracle.build()
        r = oracle.RefCPU()
        t0 = time.perf_counter()
        req, rrq = r.marker_project(m.dims, wil, xi, eta, rho)
        t_cpu = time.perf_counter() - t0
        rel = float(np.abs(eq - req).max() / np.abs(req).max())
        out.update(cpu_ms=t_cpu * 1e3, cpu_kind="reference (material_point_utils.c, one thread: its loops are serial)",
                   speedup=t_cpu / t_dev, relerr_vs_reference=rel)
    op.Destroy()
    print(json.dumps(out))
    return 0


def M_uniform(n, seed):
    return np.random.default_rng(seed).uniform(-1.0, 1.0, size=n)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c2")
    ap.add_argument("--a11-op", default="b200")
    ap.add_argument("--quick", action="store_true", help="headline A11 only")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="apply: keep the default tile schedule")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--mode", default="apply", choices=["apply", "solve", "batched", "serve", "markers"])
    ap.add_argument("--markers-per-element", type=int, default=8)
    ap.add_argument("--nreq", type=int, default=200, help="serve: requests in the measured stream")
    ap.add_argument("--ncal", type=int, default=48, help="serve: requests of the capacity calibration")
    ap.add_argument("--nserial", type=int, default=12, help="serve: requests solved one at a time")
    ap.add_argument("--serve-iters", type=int, default=8, help="serve: iterations per server step")
    ap.add_argument("--nbatch", type=int, default=256)
    ap.add_argument("--ksp", default="fgmres")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--max-it", type=int, default=20000)
    ap.add_argument("--restart", type=int, default=30)
    ap.add_argument("--pc", default="mg", choices=["mg", "cheby_jacobi", "jacobi", "none"])
    ap.add_argument("--cheby-degree", type=int, default=3)
    args = ap.parse_args()
    if args.mode == "solve":
        return run_solve(args)
    if args.mode == "batched":
        return run_batched(args)
    if args.mode == "serve":
        return run_serve(args)
    if args.mode == "markers":
        return run_markers(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
