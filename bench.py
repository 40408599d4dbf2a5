"""Benchmark of the GLU numeric phase on B200: batched FP64 sparse-LU refactorization + solve.

Workload (default): one n = 20,000 MNA pattern (netlist generator, seed 2) x 512 Monte Carlo
value sets (conductances x lognormal(0, 0.1), controlled sources x U[0.8, 1.2], seed 1234 + rank),
b_k = A_k * 1.  One step = ingest the 512 value sets, refactor all 512, solve all 512, i.e. one
replay of the CUDA graph that holds the whole batch.  The preprocessing (NICSLU MC64 + AMD) of
the pattern is the reference's, read from tests/golden/nicslu_mna20000_s2.npz; the symbolic
analysis is this package's bit-exact fast version.  Synthetic data stands in for the UFL circuit
matrices the reference quotes (not available).

Printed JSON line (rank 0): value = matrices/s over all ranks (weak scaling: every rank runs its
own 512 instances); e2e = the same through host buffers (H2D values + RHS, replay, D2H x);
plain = the same kernels one matrix per launch without a graph; roofline = the dense trailing
update kernel (FP64 DMMA) against the FP64 DGEMM peak measured in the same run; cpu_baseline =
the reference's NICSLU CPU refactorization (+ solve) on a bounded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--count C]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 sparse LU refactor/s batched vs plain at resid<=1e-12; adjoint/forward time"
PATTERN = dict(name="mna20000_s2", n=20000, seed=2)
FIXTURE = os.path.join(ROOT, "tests", "golden", "nicslu_mna20000_s2.npz")
INST_SEED = 1234
MEASURED_PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
# dram__bytes_read.sum + dram__bytes_write.sum of one trailing-update launch (group 0, 8 instances,
# K = 512) divided by its algorithmic bytes (2.162 GB / 2.207 GB), measured with ncu on that launch
DRAM_OVER_ALG = 0.980


# ---------------------------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)

    def summary(self) -> dict:
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace('.', '', 1).isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace('.', '', 1).isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": sorted(reasons),
                "samples": len(self.rows)}


def dist_setup():
    import torch
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if torch.cuda.is_available():
        torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(ws, v: float) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def shard_of(count: int, ws: int, rank: int) -> tuple:
    """Weak scaling: the job factors ONE global batch of count * ws instances; rank r takes the
    contiguous block [r * count, (r + 1) * count) of it (glu_public_b200.shard.instance_range)."""
    from glu_public_b200 import shard
    return shard.instance_range(count * ws, ws, rank)


def workload_values(count: int, rank: int, ws: int = 1):
    """The generated pattern and this rank's shard of the global batch: instance values (instance
    i drawn from its own generator seeded with (1234, i)) and right-hand sides b_k = A_k * 1.
    Uses the generator only, so it loads no native library."""
    import scipy.sparse as sp
    from glu_public_b200 import gen
    c = gen.mna_netlist(PATTERN["n"], PATTERN["seed"])
    first, cnt = shard_of(count, ws, rank)
    vals = c.instance_values_indexed(first, cnt, INST_SEED)
    rows = sp.csr_matrix((np.ones(c.nnz), (c.indices, np.arange(c.nnz))), shape=(c.n, c.nnz))
    B = np.ascontiguousarray((rows @ vals.T).T)
    return c, vals, B


def workload_config(c, count: int, ws: int) -> dict:
    """The `config` of both arms' JSON lines (identical by construction)."""
    return {"workload": f"batched_mna20000_x{count}", "pattern": PATTERN,
            "instances_per_gpu": count, "global_batch": count * ws, "nrhs": 1, "nnz_a": c.nnz,
            "instance_seeds": f"instance i of the global batch: default_rng(({INST_SEED}, i))",
            "l2": f"inputs larger than L2 ({count} value sets of {c.nnz * 8 / 1e6:.2f} MB plus "
                  f"their factors per step)"}


def build_workload(count: int, rank: int, ws: int = 1):
    """Pattern, preprocessing, fast symbolic, this rank's instance values and right-hand sides."""
    from glu_public_b200 import glu
    c, vals, B = workload_values(count, rank, ws)
    nic = glu.NicsluArrays.from_npz(FIXTURE)
    import hashlib
    h = hashlib.sha256()
    for a in (c.indptr.astype(np.int64), c.indices.astype(np.int32), c.data):
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    if str(np.load(FIXTURE)["matrix_digest"]) != h.hexdigest():
        raise RuntimeError("preprocessing fixture does not belong to the generated pattern")
    ap, ai, ax = nic.preprocess(c.indptr, c.indices, c.data)
    sym = glu.SymbolicMatrix(c.n).analyze(ai, ap)
    return c, nic, sym, vals, B


def hbm_peak_gbs() -> tuple:
    try:
        return float(json.load(open(MEASURED_PEAKS))["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs"
    except (OSError, ValueError, KeyError):
        return 6650.0, "fallback 6.65 TB/s"


def solve_roofline(st: dict, count: int, ms: float) -> dict:
    byts = count * (8.0 * st["nnz"] + 16.0 * st["n"])
    peak, src = hbm_peak_gbs()
    gbs = byts / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
            "alg_bytes": byts, "peak_source": src, "vectors": count}


def dense_update_model(ntp: int, nb: int, depth: int) -> dict:
    """Algorithmic FLOPs and bytes of the dense update products of one instance, as the library
    issues them (launch_dense_factor): per group of `depth` panels, two thin products per panel
    after the first (its column block and row block, K = the group's panels before it) and one
    trailing product with K = depth * nb.  Bytes: C read and written once, A and B read once."""
    flops = byts = 0.0
    launches, trailing = 0, []
    def gemm(m, n, k):
        nonlocal flops, byts, launches
        if m <= 0 or n <= 0 or k <= 0:
            return
        flops += 2.0 * m * n * k
        byts += 8.0 * (2 * m * n + m * k + k * n)
        launches += 1
    for k0 in range(0, ntp, depth * nb):
        dd = min(depth, (ntp - k0) // nb)
        for j in range(1, dd):
            c = k0 + j * nb
            gemm(ntp - c, nb, c - k0)
            gemm(nb, ntp - c - nb, c - k0)
        m = ntp - k0 - dd * nb
        if m > 0:
            trailing.append((m, m, dd * nb, 2.0 * m * m * dd * nb, 8.0 * (2 * m * m + 2 * m * dd * nb)))
        gemm(m, m, dd * nb)
    return {"flops": flops, "bytes": byts, "launches": launches, "trailing": trailing}


def measure_cublas_shape(torch, m: int, n: int, k: int, cnt: int) -> float:
    """cuBLAS (torch.baddbmm) FP64 throughput on C -= A B of the given batched shape, best of 5."""
    a = torch.randn(cnt, m, k, dtype=torch.float64, device="cuda")
    b = torch.randn(cnt, k, n, dtype=torch.float64, device="cuda")
    c = torch.randn(cnt, m, n, dtype=torch.float64, device="cuda")
    torch.baddbmm(c, a, b, alpha=-1.0, out=c)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.baddbmm(c, a, b, alpha=-1.0, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b, c
    torch.cuda.empty_cache()
    return 2.0 * m * n * k * cnt / (best * 1e-3) / 1e12


def measure_dgemm_peak(torch) -> float:
    """cuBLAS FP64 GEMM throughput (TFLOP/s), best of 5, as the FP64 tensor-pipe reference."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    best = 0.0
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = max(best, 2.0 * n ** 3 / (e0.elapsed_time(e1) * 1e-3) / 1e12)
    del a, b, c
    torch.cuda.empty_cache()
    return best


def cpu_baseline(c, vals, B, budget_s: float = 25.0, threads: int | None = None) -> dict:
    """The reference's NICSLU CPU refactorization + solve on a bounded sample of instances."""
    from oracle import oracle as O
    if not O.have_ref():
        return {"value": None, "unavailable": "oracle/_ref/libglu_ref.so not built"}
    threads = threads or os.cpu_count() or 1
    ref = O.RefPipeline.from_csc(c.n, c.indptr, c.indices, c.data)
    st = ref.nicslu_factorize()
    if st < 0:
        return {"value": None, "unavailable": f"NicsLU_Factorize returned {st}"}
    mt = threads > 1 and ref.nicslu_create_threads(threads) >= 0
    done, t_total, t1 = 0, 0.0, None
    worst = 0.0
    while done < vals.shape[0] and (done == 0 or t_total < budget_s):
        t0 = time.perf_counter()
        ref.nicslu_refactorize(vals[done], mt)
        x = ref.nicslu_solve(B[done])
        dt = time.perf_counter() - t0
        t_total += dt
        worst = max(worst, O.residual(c.n, c.indptr, c.indices, vals[done], x, B[done]))
        done += 1
    # one single-thread refactorization for comparison (NICSLU's MT scheduler can be slower)
    if mt:
        t0 = time.perf_counter()
        ref.nicslu_refactorize(vals[0], False)
        ref.nicslu_solve(B[0])
        t1 = time.perf_counter() - t0
    ref.close()
    return {"value": done / t_total, "unit": "matrices/s", "cores": threads if mt else 1,
            "kind": "reference",
            "sample": f"NicsLU_ReFactorize{'_MT' if mt else ''} + NicsLU_Solve on {done} of the "
                      f"instances ({t_total:.1f}s); single-thread refactor+solve "
                      f"{'%.3fs' % t1 if t1 else 'n/a'}",
            "max_residual": worst}


# ---------------------------------------------------------------------------------------------
# arms
# ---------------------------------------------------------------------------------------------

def run_reference(args, ws, rank):
    """The reference's own CPU path on the host cores: NICSLU's multithreaded refactorization +
    solve (NicsLU_ReFactorize_MT + NicsLU_Solve, src/nicslu/source/nicslu_refact_parallel.c),
    after NicsLU_Analyze + one NicsLU_Factorize of the pattern outside the timed region.  One step
    = one instance of the benchmark's batch (instances 0, 1, 2, ... of rank 0's shard, in order);
    W untimed steps, then K timed steps.  Loads only the oracle's build of the reference
    (oracle/_ref), never this package's library."""
    if rank != 0:
        return
    from oracle import oracle as O
    c, vals, B = workload_values(args.count, 0, args.gpus)
    config = workload_config(c, args.count, args.gpus)
    if not O.have_ref():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libglu_ref.so not built"}))
        return
    threads = os.cpu_count() or 1
    ref = O.RefPipeline.from_csc(c.n, c.indptr, c.indices, c.data)
    st = ref.nicslu_factorize()
    if st < 0:
        print(json.dumps({"impl": "reference", "unavailable": f"NicsLU_Factorize returned {st}"}))
        return
    mt = threads > 1 and ref.nicslu_create_threads(threads) >= 0
    xs = []

    def step(i):
        ref.nicslu_refactorize(vals[i % vals.shape[0]], mt)
        xs.append((i % vals.shape[0], ref.nicslu_solve(B[i % vals.shape[0]])))

    for i in range(args.warmup):
        step(i)
    xs.clear()
    t0 = time.perf_counter()
    for i in range(args.warmup, args.warmup + args.steps):
        step(i)
    total = time.perf_counter() - t0
    worst = max(O.residual(c.n, c.indptr, c.indices, vals[i], x, B[i]) for i, x in xs)
    ref.close()
    v = args.steps / total
    sample = (f"NicsLU_ReFactorize{'_MT' if mt else ''} + NicsLU_Solve, one instance per step "
              f"(instances {args.warmup}..{args.warmup + args.steps - 1} of the batch), "
              f"{total:.1f}s for {args.steps} steps")
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "matrices/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded MNA netlist generator; reference NICSLU preprocessing)",
            "config": config,
            "cpu_baseline": {"value": v, "unit": "matrices/s", "cores": threads if mt else 1,
                             "kind": "reference", "sample": sample, "max_residual": worst},
            "e2e": {"value": v, "unit": "matrices/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def run_ours(args, ws, rank, local):
    import torch
    from glu_public_b200 import glu
    from glu_public_b200 import build as _b  # noqa: F401  (library must already be built)

    t_setup = time.time()
    c, nic, sym, vals, B = build_workload(args.count, rank, ws)
    dev = torch.device("cuda", local)
    opts = dict(json.loads(args.options)) if args.options else {}
    if args.panel:
        opts["panel"] = args.panel
    if args.gemm is not None:
        opts["gemm_variant"] = args.gemm
    if args.depth:
        opts["update_depth"] = args.depth
    tuned = None
    if args.tune and not opts:
        from glu_public_b200 import autotune
        sample = torch.as_tensor(vals[:min(args.count, args.tune_sample)], device=dev)
        t_tune = time.time()
        opts = autotune.autotune(sym, sample, nic=nic, indptr=c.indptr, indices=c.indices,
                                 count_hint=args.count, cache=None)
        tuned = {"options": opts, "seconds": time.time() - t_tune, "sample": int(sample.shape[0])}
        del sample
    plan = glu.Plan(sym, **opts)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, nic)
    plan.set_solve_maps(nic)
    plan.set_original_csc(c.indptr, c.indices)
    st = plan.stats()
    count, n = args.count, c.n
    a_host = torch.from_numpy(vals).pin_memory()
    b_host = torch.from_numpy(B.reshape(count, 1, n)).pin_memory()
    x_host = torch.empty((count, 1, n), dtype=torch.float64).pin_memory()
    a_dev = a_host.to(dev)
    b_dev = b_host.to(dev)
    x_dev = torch.empty_like(b_dev)
    batch = glu.Batch(plan, count)

    # correctness gate on this exact workload: status flags and the residual of every instance,
    # before and after the refinement round the timed step includes
    batch.load_values(a_dev)
    batch.refactor(0.0)
    batch.solve(b_dev, out=x_dev)
    res0 = batch.residual(a_dev, b_dev, x_dev)
    res1 = batch.refine(a_dev, b_dev, x_dev, steps=args.refine, with_residual=True) \
        if args.refine else res0
    torch.cuda.synchronize()
    flags = batch.status()
    worst_unrefined = float(res0.max().item())
    worst = float(res1.max().item())
    from scipy.sparse import csc_matrix
    xs = x_dev.cpu().numpy()
    for i in sorted(set([0, count // 2, count - 1])):      # host cross-check of the device norm
        A = csc_matrix((vals[i], c.indices, c.indptr), shape=(n, n))
        r = A @ xs[i, 0] - B[i]
        an = np.abs(A).sum(axis=1).max()
        host = float(np.abs(r).max() / (an * np.abs(xs[i, 0]).max() + np.abs(B[i]).max()))
        worst = max(worst, host)

    # live roofline of the dominant kernel: per-phase device time of one refactorization
    batch.load_values(a_dev)
    phases = batch.refactor_timed(0.0)
    ntp, nb, depth = int(st["ntp"]), int(st["panel"]), int(st["update_depth"])
    upd = dense_update_model(ntp, nb, depth)
    # the trailing products of the groups (phase "update"; the thin in-group ones are "strips")
    trail_flops = sum(t[3] for t in upd["trailing"]) * count
    trail_bytes = sum(t[4] for t in upd["trailing"]) * count
    upd_ms, upd_launches = phases["update"]

    batch.capture(a_dev, b_dev, x_dev, pert=0.0, refine=args.refine)
    launches_per_step = batch.launches
    torch.cuda.synchronize()
    for _ in range(args.warmup):
        batch.replay()
    torch.cuda.synchronize()

    # ---- timed region: K graph replays (inputs 512 x 141 MB per step >> L2) ----
    with ClockSampler(local) as clk:
        barrier(ws)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s = torch.cuda.current_stream()
        e0.record(s)
        for _ in range(args.steps):
            batch.replay()
        e1.record(s)
        torch.cuda.synchronize()
        barrier(ws)
    ms = max_over_ranks(ws, e0.elapsed_time(e1)) / args.steps
    value = ws * count / (ms * 1e-3)

    # ---- end to end through host buffers ----
    for _ in range(2):
        a_dev.copy_(a_host, non_blocking=True)
        b_dev.copy_(b_host, non_blocking=True)
        batch.replay()
        x_host.copy_(x_dev, non_blocking=True)
    barrier(ws)
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        a_dev.copy_(a_host, non_blocking=True)
        b_dev.copy_(b_host, non_blocking=True)
        batch.replay()
        x_host.copy_(x_dev, non_blocking=True)
    f1.record()
    torch.cuda.synchronize()
    barrier(ws)
    e2e_ms = max_over_ranks(ws, f0.elapsed_time(f1)) / args.steps
    e2e = ws * count / (e2e_ms * 1e-3)

    # ---- adjoint vs forward solve on the factors of the whole batch ----
    # forward: X = A^-1 B (triangular solves); adjoint: lambda = A^-T G (transposed solves) plus
    # dLoss/dA = -lambda x^T on A's nonzeros (glu_grad_a), as in the autograd backward
    g_dev = torch.randn_like(b_dev)
    lam_dev = torch.empty_like(b_dev)
    for _ in range(2):
        batch.solve(b_dev, out=x_dev)
        batch.solve(g_dev, transpose=True, out=lam_dev)
        ga = batch.grad_a(lam_dev, x_dev)
    torch.cuda.synchronize()
    q0, q1, q2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    reps = 5
    q0.record()
    for _ in range(reps):
        batch.solve(b_dev, out=x_dev)
    q1.record()
    for _ in range(reps):
        batch.solve(g_dev, transpose=True, out=lam_dev)
        batch.grad_a(lam_dev, x_dev, out=ga)
    q2.record()
    torch.cuda.synchronize()
    fwd_ms = q0.elapsed_time(q1) / reps
    adj_ms = q1.elapsed_time(q2) / reps
    del ga, g_dev, lam_dev

    # ---- plain path: same kernels, one matrix per launch sequence, no graph ----
    plain_n = min(args.plain, count)
    b1 = glu.Batch(plan, 1)
    def plain_one(i):
        b1.load_values(a_dev[i:i + 1])
        b1.refactor(0.0)
        b1.solve(b_dev[i:i + 1], out=x_dev[i:i + 1])
        if args.refine:
            b1.refine(a_dev[i:i + 1], b_dev[i:i + 1], x_dev[i:i + 1], steps=args.refine)

    for i in range(2):
        plain_one(i)
    torch.cuda.synchronize()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    for i in range(plain_n):
        plain_one(i)
    p1.record()
    torch.cuda.synchronize()
    plain = plain_n / (p0.elapsed_time(p1) * 1e-3)
    # where the one-matrix time goes: ingest, refactor, solve, refinement (device time each)
    plain_parts = {
        "ingest_ms": timed(torch, lambda: b1.load_values(a_dev[:1]), 3),
        "refactor_ms": timed(torch, lambda: b1.refactor(0.0), 3),
        "solve_ms": timed(torch, lambda: b1.solve(b_dev[:1], out=x_dev[:1]), 3),
        "refine_ms": timed(torch, lambda: b1.refine(a_dev[:1], b_dev[:1], x_dev[:1],
                                                    steps=args.refine), 3) if args.refine else 0.0,
        "launches_refactor": None}
    b1.refactor(0.0)
    plain_parts["launches_refactor"] = b1.launches
    del b1

    # single-instance phase profile (the plain path's device time per phase)
    b1 = glu.Batch(plan, 1)
    b1.load_values(a_dev[:1])
    plain_phases = b1.refactor_timed(0.0)
    del b1

    peak = measure_dgemm_peak(torch)
    m0, _, k0, _, _ = upd["trailing"][0]
    cublas_shape = measure_cublas_shape(torch, m0, m0, k0, 8)
    achieved = trail_flops / (upd_ms * 1e-3) / 1e12
    gv = int(st["gemm_variant"])
    refactor_ms = sum(v[0] for v in phases.values())
    out = {
        "metric": METRIC, "value": value, "unit": "matrices/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded MNA netlist generator; reference NICSLU preprocessing)",
        "config": workload_config(c, count, ws),
        "pattern_stats": {"nnz_lu": int(st["nnz"]), "levels": int(sym.num_lev),
                          "dense_tail": int(st["nt"]), "sparse_levels": int(st["sparse_levels"]),
                          "flops_per_refactor": st["flops"],
                          "factor_mb_per_instance": st["slots"] * 8 / 1e6},
        "plain": {"value": plain, "unit": "matrices/s", "sample": plain_n,
                  "note": "same kernels, one matrix per launch sequence, no CUDA graph",
                  "parts": plain_parts},
        "batched_over_plain": value / ws / plain,
        # HBM roofline of the forward solve: every factor entry read once per vector, the vector
        # read and written (algorithmic bytes 8 nnz_LU + 16 n per vector)
        "solve_roofline": solve_roofline(st, count, fwd_ms),
        "adjoint": {"forward_solve_ms": fwd_ms, "adjoint_ms": adj_ms,
                    "adjoint_over_forward": adj_ms / fwd_ms, "instances": count, "nrhs": 1,
                    "note": "transposed solves + gradient over A's nonzeros vs the forward solve, "
                            "same factors"},
        "max_residual": worst, "max_residual_unrefined": worst_unrefined,
        "refine_steps": args.refine, "status_flags_nonzero": int((flags != 0).sum()),
        "roofline": {"bound": "tensor",
                     "kernel": ("k_gemm_sub16" if gv in (5, 6, 7, 8, 9, 10, 13) else "k_gemm_sub") +
                               f" variant {gv} (dense trailing update of a group, FP64 DMMA)",
                     "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": achieved / peak,
                     "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (MEASURED_PEAKS.json "
                                    "has no FP64 figure)",
                     "cublas_same_shape_tflops": cublas_shape,
                     "cublas_same_shape": f"torch.baddbmm, {m0} x {m0} x {k0}, 8 instances",
                     "alg_bytes_per_launch": trail_bytes / max(upd_launches, 1),
                     # DRAM bytes per launch: the ncu capture of one such launch (8 instances)
                     # measured DRAM_OVER_ALG x its algorithmic bytes; scaled by the units processed
                     "traffic": DRAM_OVER_ALG * trail_bytes / max(upd_launches, 1),
                     "traffic_unit": "bytes per launch", "launches": upd_launches,
                     "share_of_refactor": upd_ms / refactor_ms if refactor_ms else None},
        "refactor_phase_ms": {k: v[0] for k, v in phases.items()},
        "plain_phase_ms": {k: v[0] for k, v in plain_phases.items()},
        "plan": {k: st[k] for k in ("t", "ntp", "hubs", "dense_updates", "hub_updates",
                                    "pull_entries", "panel", "sparse_slots", "slots", "fronts",
                                    "lsolve_levels", "usolve_levels", "unit_levels")},
        "plan_options": opts, "autotune": tuned,
        "refactor_alg_tflops": st["flops"] * count / (refactor_ms * 1e-3) / 1e12,
        "e2e": {"value": e2e, "unit": "matrices/s",
                "h2d_bytes_per_step": int(a_host.numel() * 8 + b_host.numel() * 8),
                "d2h_bytes_per_step": int(x_host.numel() * 8)},
        "gpu_launches": int(launches_per_step * args.steps),
        "clocks": clk.summary(),
        "setup_s": time.time() - t_setup,
    }
    if rank == 0 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(c, vals[:8], B[:8], budget_s=20.0)
    if rank == 0:
        print(json.dumps(out))


# ---------------------------------------------------------------------------------------------
# further configurations (one JSON line each; the default workload is the batched one above)
# ---------------------------------------------------------------------------------------------

def load_pattern(name: str):
    """Generator + the reference's NICSLU preprocessing fixture + fast symbolic for a pattern name
    like 'mna20000_s2' or 'grid512_s1'."""
    import hashlib
    from glu_public_b200 import gen, glu
    kind, seed = name.split("_s")
    if kind.startswith("mna"):
        c = gen.mna_netlist(int(kind[3:]), int(seed))
    else:
        c = gen.power_grid(int(kind[4:]), int(seed))
    path = os.path.join(ROOT, "tests", "golden", f"nicslu_{name}.npz")
    h = hashlib.sha256()
    for a in (c.indptr.astype(np.int64), c.indices.astype(np.int32), c.data):
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    if str(np.load(path)["matrix_digest"]) != h.hexdigest():
        raise RuntimeError(f"preprocessing fixture {path} does not belong to the generated pattern")
    nic = glu.NicsluArrays.from_npz(path)
    ap, ai, _ = nic.preprocess(c.indptr, c.indices, c.data)
    t0 = time.time()
    sym = glu.SymbolicMatrix(c.n).analyze(ai, ap)
    return c, nic, sym, time.time() - t0


def make_plan(c, nic, sym, **opts):
    from glu_public_b200 import glu
    plan = glu.Plan(sym, **opts)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, nic)
    plan.set_solve_maps(nic)
    plan.set_original_csc(c.indptr, c.indices)
    return plan


def rowsum_rhs(c, vals):
    import scipy.sparse as sp
    rows = sp.csr_matrix((np.ones(c.nnz), (c.indices, np.arange(c.nnz))), shape=(c.n, c.nnz))
    return np.ascontiguousarray((rows @ vals.T).T)


def timed(torch, fn, reps):
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def base_line(args, workload, value, unit, ms, extra):
    line = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generators; reference NICSLU preprocessing)",
            "config": {"workload": workload}}
    line.update(extra)
    return line


MULTI_SPECS = [("mna2000_s3", 1024), ("mna50000_s4", 64), ("grid512_s1", 4)]


def run_multi(args, ws=1, rank=0, local=0):
    """Uneven multi-pattern batch: n=2,000 x1,024, n=50,000 x64, power-grid mesh x4, in one graph
    per rank (one branch per pattern), with per-pattern autotuned schedules.  With N ranks the
    batch is bin-packed by cost (F_alg per instance, glu_public_b200.shard.plan_shards): every
    rank factors its shards of it, and the time is the max over ranks."""
    import torch
    from glu_public_b200 import autotune, glu, shard
    dev = torch.device("cuda", local)
    loaded = {name: load_pattern(name) for name, _ in MULTI_SPECS}
    cost = {name: loaded[name][2].flops() for name, _ in MULTI_SPECS}
    mine = shard.plan_shards([(name, cnt, cost[name]) for name, cnt in MULTI_SPECS], ws)[rank]
    batches, vals, Bs, Xs, per = [], [], [], [], {}
    for sh in mine:
        k = [nm for nm, _ in MULTI_SPECS].index(sh.name)
        c, nic, sym, t_sym = loaded[sh.name]
        count = sh.count
        v = c.instance_values_indexed(sh.first, count, INST_SEED + k)
        B = rowsum_rhs(c, v).reshape(count, 1, c.n)
        vt = torch.as_tensor(v, device=dev)
        opts = {}
        if args.tune:
            sample = vt[:min(count, 16)]
            saved = dict(autotune.SPACE)
            autotune.SPACE.clear()
            autotune.SPACE.update({"gemm_variant": [12, 11, 13], "update_depth": [8, 4, 2]})
            try:
                opts = autotune.autotune(sym, sample, nic=nic, indptr=c.indptr, indices=c.indices,
                                         count_hint=count, cache=None, repeats=1)
            finally:
                autotune.SPACE.clear()
                autotune.SPACE.update(saved)
        plan = make_plan(c, nic, sym, **opts)
        b = glu.Batch(plan, count)
        Bt = torch.as_tensor(B, device=dev)
        Xt = torch.zeros_like(Bt)
        # per-pattern graph on the same batch, timed alone
        b.load_values(vt)
        b.refactor()
        b.solve(Bt, out=Xt)
        b.refine(vt, Bt, Xt, steps=1)
        b.capture(vt, Bt, Xt, refine=1)
        for _ in range(args.warmup):
            b.replay()
        ms = timed(torch, b.replay, args.steps)
        res = b.residual(vt, Bt, Xt)
        st = plan.stats()
        per[f"{sh.name}[{sh.first}:{sh.first + count}]"] = {
            "instances": count, "n": c.n, "nnz_lu": int(st["nnz"]), "dense": int(st["nt"]),
            "sparse_levels": int(st["sparse_levels"]), "options": opts, "ms_alone": ms,
            "matrices_per_s_alone": count / (ms * 1e-3), "max_residual": float(res.max().item()),
            "symbolic_s": t_sym}
        batches.append(b)
        vals.append(vt)
        Bs.append(Bt)
        Xs.append(Xt)
    group = glu.Group(batches, vals, Bs, Xs, refine=1)
    for _ in range(args.warmup):
        group.launch()
    with ClockSampler(local) as clk:
        barrier(ws)
        ms_local = timed(torch, group.launch, args.steps)
        barrier(ws)
    ms = max_over_ranks(ws, ms_local)
    worst = max(float(batches[k].residual(vals[k], Bs[k], Xs[k]).max().item())
                for k in range(len(batches)))
    worst = max_over_ranks(ws, worst)
    total = sum(cnt for _, cnt in MULTI_SPECS)
    if rank == 0:
        line = base_line(args, "multi_pattern[mna2000x1024,mna50000x64,grid512x4]",
                         total / (ms * 1e-3), "matrices/s", ms,
                         {"whole_batch_ms": ms, "patterns_rank0": per, "max_residual": worst,
                          "shards": [[(s.name, s.first, s.count) for s in p]
                                     for p in shard.plan_shards(
                                         [(nm, cnt, cost[nm]) for nm, cnt in MULTI_SPECS], ws)],
                          "gpu_launches": int(group.launches * args.steps),
                          "clocks": clk.summary()})
        line["n_gpus"] = ws
        line["scaling"] = "strong"
        print(json.dumps(line))


def run_mesh(args):
    """Plain path at scale: the two-layer power-grid mesh (n = 524,352), one factorization plus
    4 right-hand sides b_k = A r_k.  Timed with the default options (the fronts of a level
    processed together, runs of front-free levels in one cooperative launch) and, for
    comparison, with one launch chain per front and one launch per level."""
    import torch
    from glu_public_b200 import glu
    c, nic, sym, t_sym = load_pattern("grid512_s1")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(INST_SEED)
    R = rng.standard_normal((4, c.n))
    B = np.stack([c.to_scipy() @ R[k] for k in range(4)])[None]
    vt = torch.as_tensor(c.data[None, :], device=dev)
    Bt = torch.as_tensor(B, device=dev)

    def variant(**opts):
        plan = make_plan(c, nic, sym, **opts)
        b = glu.Batch(plan, 1)
        b.load_values(vt)
        b.refactor()
        X = b.solve(Bt)
        b.refine(vt, Bt, X, steps=1)
        phases = b.refactor_timed(0.0)

        def step():
            b.load_values(vt)
            b.refactor()
            b.solve(Bt, out=X)
            b.refine(vt, Bt, X, steps=1)

        for _ in range(args.warmup):
            step()
        out = {"step_ms": timed(torch, step, args.steps)}
        b.load_values(vt)
        out["refactor_ms"] = timed(torch, b.refactor, args.steps)
        out["refactor_launches"] = b.launches
        out["solve_ms_4rhs"] = timed(torch, lambda: b.solve(Bt, out=X), args.steps)
        # the same step as one CUDA graph
        b.capture(vt, Bt, X, refine=1)
        b.replay()
        out["graph_replay_ms"] = timed(torch, b.replay, args.steps)
        out["launches_per_graph"] = b.launches
        out["refactor_phase_ms"] = {k: v[0] for k, v in phases.items()}
        out["max_residual"] = float(b.residual(vt, Bt, X).max().item())
        out["max_abs_err_vs_r"] = float(np.abs(X.cpu().numpy()[0] - R).max())
        return plan, b, out

    plan, b, _ = variant()                     # warm-up pass
    st = plan.stats()
    del b, plan
    torch.cuda.empty_cache()
    _, b2, chain = variant(front_batch=0, sparse_persistent=0)
    del b2
    torch.cuda.empty_cache()
    with ClockSampler(0) as clk:
        plan, b, again = variant()
    ms = again["step_ms"]
    print(json.dumps(base_line(args, "mesh_grid2x512x512_plus_pads (n=524,352), 4 RHS",
                               1000.0 / ms, "factorizations/s", ms,
                               {"solves_per_s": 4 * 1000.0 / again["solve_ms_4rhs"],
                                "default": again,
                                "one_chain_per_front_one_launch_per_level": chain,
                                "graph_factorizations_per_s": 1000.0 / again["graph_replay_ms"],
                                "plan": {k: st[k] for k in ("nnz", "nt", "sparse_levels",
                                                            "lsolve_levels", "usolve_levels",
                                                            "flops", "fronts")},
                                "symbolic_s": t_sym, "clocks": clk.summary()})))


def run_adjoint(args):
    """Adjoint through torch.autograd at n = 100,000 with 32 right-hand sides (loss = sum w*X),
    and 256 Monte Carlo n = 20,000 instances with per-instance gradients."""
    import torch
    from glu_public_b200 import autograd
    dev = torch.device("cuda", 0)
    out = {}
    for name, count, nrhs in (("mna100000_s6", 1, 32), ("mna20000_s2", 256, 1)):
        c, nic, sym, t_sym = load_pattern(name)
        plan = make_plan(c, nic, sym)
        rng = np.random.default_rng(INST_SEED)
        vals = c.instance_values(count, seed=INST_SEED) if count > 1 else c.data[None, :]
        a = torch.tensor(vals, device=dev, requires_grad=True)
        Bt = torch.tensor(rng.standard_normal((count, nrhs, c.n)), device=dev, requires_grad=True)
        W = torch.tensor(rng.standard_normal((count, nrhs, c.n)), device=dev)
        # forward solve alone vs adjoint alone on the same factors
        from glu_public_b200 import glu
        batch = glu.Batch(plan, count)
        batch.load_values(a.detach())
        batch.refactor()
        X = batch.solve(Bt.detach())
        lam = torch.empty_like(X)
        ga = batch.grad_a(batch.solve(W, transpose=True), X)
        fwd = timed(torch, lambda: batch.solve(Bt.detach(), out=X), args.steps)

        def adj():
            batch.solve(W, transpose=True, out=lam)
            batch.grad_a(lam, X, out=ga)

        adjm = timed(torch, adj, args.steps)
        del batch, ga, lam
        torch.cuda.empty_cache()
        # the whole autograd step (refactor + solve + refine, then transposed solves + gradient)
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        torch.cuda.synchronize()
        e0.record()
        Xa = autograd.sparse_solve(a, Bt, plan)
        loss = (W * Xa).sum()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        out[name] = {"instances": count, "nrhs": nrhs, "forward_solve_ms": fwd, "adjoint_ms": adjm,
                     "adjoint_over_forward": adjm / fwd,
                     "autograd_forward_ms": e0.elapsed_time(e1),
                     "autograd_backward_ms": e1.elapsed_time(e2),
                     "grad_finite": bool(torch.isfinite(a.grad).all().item()),
                     "symbolic_s": t_sym}
        del a, Bt, W, Xa, loss
        torch.cuda.empty_cache()
    worst = max(v["adjoint_over_forward"] for v in out.values())
    print(json.dumps(base_line(args, "adjoint[mna100000 x32rhs, mna20000 x256]", worst,
                               "adjoint/forward time", out["mna100000_s6"]["adjoint_ms"],
                               {"higher_is_better": False, "cases": out})))


def run_plain4960(args):
    """Plain GLU pipeline: one n = 4,960 matrix, one factorization + solve (b = A*1).  Also
    timed: the sparse levels one launch each instead of the cooperative level launch, and the
    matrix factored with no dense trailing block at all (the reference's long tail of
    one-column levels, walked by the cooperative launch or level by level)."""
    import torch
    from glu_public_b200 import glu
    c, nic, sym, t_sym = load_pattern("mna4960_s0")
    dev = torch.device("cuda", 0)
    vt = torch.as_tensor(c.data[None, :], device=dev)
    Bt = torch.as_tensor(rowsum_rhs(c, c.data[None, :]).reshape(1, 1, c.n), device=dev)

    def variant(**opts):
        plan = make_plan(c, nic, sym, **opts)
        b = glu.Batch(plan, 1)
        X = torch.zeros_like(Bt)

        def step():
            b.load_values(vt)
            b.refactor()
            b.solve(Bt, out=X)
            b.refine(vt, Bt, X, steps=1)

        for _ in range(args.warmup):
            step()
        out = {"step_ms": timed(torch, step, args.steps)}
        b.load_values(vt)
        out["refactor_ms"] = timed(torch, b.refactor, args.steps)
        out["refactor_launches"] = b.launches
        b.capture(vt, Bt, X, refine=1)
        b.replay()
        out["graph_replay_ms"] = timed(torch, b.replay, args.steps)
        out["launches_per_graph"] = b.launches
        out["max_residual"] = float(b.residual(vt, Bt, X).max().item())
        out["sparse_levels"] = int(plan.stat("sparse_levels"))
        b.load_values(vt)
        out["refactor_phase_ms"] = {k: v[0] for k, v in b.refactor_timed(0.0).items()}
        return out

    cases = {"default": variant(),
             "levels_one_launch_each": variant(sparse_persistent=0),
             "no_dense_block_cooperative": variant(dense_threshold=2.0),
             "no_dense_block_one_launch_per_level": variant(dense_threshold=2.0,
                                                            sparse_persistent=0)}
    d = cases["default"]
    print(json.dumps(base_line(args, "plain_mna4960 (one factorization + solve)",
                               1000.0 / d["step_ms"], "factorizations/s", d["step_ms"],
                               {"graph_replay_ms": d["graph_replay_ms"],
                                "max_residual": d["max_residual"], "symbolic_s": t_sym,
                                "variants": cases})))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--count", type=int, default=512)
    ap.add_argument("--plain", type=int, default=16)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--panel", type=int, default=0, help="dense panel width (64/128); skips tuning")
    ap.add_argument("--gemm", type=int, default=None, help="DMMA tile variant 0..10; skips tuning")
    ap.add_argument("--depth", type=int, default=0,
                    help="dense panels per trailing update (1/2/4); skips tuning")
    ap.add_argument("--options", default="",
                    help="plan options as a JSON object (e.g. the autotuner's choice); skips tuning")
    ap.add_argument("--tune", type=int, default=1, help="autotune plan options (default on)")
    ap.add_argument("--tune-sample", type=int, default=128)
    ap.add_argument("--refine", type=int, default=1, help="iterative refinement rounds per step")
    ap.add_argument("--workload", default="batched",
                    choices=["batched", "multi", "mesh", "adjoint", "plain4960"])
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            import torch
            # every launch, capture, replay and event of this arm goes to one explicit stream
            stream = torch.cuda.Stream()
            with torch.cuda.stream(stream):
                if args.workload == "batched":
                    run_ours(args, ws, rank, local)
                elif args.workload == "multi":
                    run_multi(args, ws, rank, local)
                elif rank == 0:
                    {"mesh": run_mesh, "adjoint": run_adjoint,
                     "plain4960": run_plain4960}[args.workload](args)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
