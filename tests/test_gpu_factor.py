"""GPU parity of the numeric phase against the oracle (CUDA path through the C ABI).

Tolerances (from the numeric-phase contract):
  * L/U values: max-norm per column relative difference <= 1e-12 against the oracle's
    right-looking FP64 factorization on the same preprocessed values -- or, on Monte Carlo
    instances whose trailing pivots lose digits to cancellation, <= 8x the difference between
    two valid rounding orders of the oracle itself (tests.common.lu_tolerance);
  * solves: ||A x - b||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= 1e-12 on the ORIGINAL matrix.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import case, column_rel_err, have_add32, lu_tolerance

pytestmark = pytest.mark.gpu

LU_TOL = 1e-12
RES_TOL = 1e-12

CASES = ["mna:200,3", "mna:2000,5", "mna:4960,1", "grid:48,2"]


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("variant", list(range(14)))
def test_dmma_gemm_matches_torch(built_lib, cuda, variant):
    torch = _torch()
    import ctypes as C
    from glu_public_b200 import _lib
    g = torch.Generator(device="cpu").manual_seed(0)
    for (M, N, K, cnt) in [(64, 64, 64, 1), (192, 128, 64, 3), (96, 160, 32, 2), (130, 70, 48, 1),
                           (256, 320, 128, 2)]:
        lda, ldb, ldc = M + 2, K + 4, M + 6
        A = torch.randn(cnt, K, lda, generator=g, dtype=torch.float64).to(cuda)
        B = torch.randn(cnt, N, ldb, generator=g, dtype=torch.float64).to(cuda)
        Cm = torch.randn(cnt, N, ldc, generator=g, dtype=torch.float64).to(cuda)
        Am = A.transpose(1, 2)[:, :M, :]           # [cnt, M, K] column-major view
        Bm = B.transpose(1, 2)[:, :K, :]           # [cnt, K, N]
        expect = Cm.transpose(1, 2)[:, :M, :] - Am @ Bm
        st = _lib.lib().glu_debug_gemm_sub(M, N, K, A.data_ptr(), lda, B.data_ptr(), ldb,
                                           Cm.data_ptr(), ldc, cnt, K * lda, N * ldb, N * ldc,
                                           variant,
                                           C.c_void_p(torch.cuda.current_stream().cuda_stream))
        assert st == 0
        got = Cm.transpose(1, 2)[:, :M, :]
        err = (got - expect).abs().max().item()
        assert err <= 1e-12 * max(1.0, expect.abs().max().item()), (M, N, K, err)


@pytest.mark.parametrize("name", CASES + (["add32"] if have_add32() else []))
def test_lu_on_device_matches_oracle(built_lib, cuda, name):
    from glu_public_b200 import glu
    cs = case(name)
    A = cs.sym
    A.val = cs.sym_ref.val.copy()
    expect, st = O.factor(cs.sym_ref, cs.sym_ref.val)
    assert st == 0
    glu.LUonDevice(A)
    err = column_rel_err(A, A.val, expect)
    assert err <= LU_TOL, err
    # solve through the Symbolic_Matrix::solve mirror, b = A*1
    c = cs.circuit
    b = c.to_scipy() @ np.ones(c.n)
    x = A.solve(cs.nic, b)
    res = O.residual(c.n, c.indptr, c.indices, c.data, x, b)
    assert res <= RES_TOL, res
    # the GPU solve against Symbolic_Matrix::solve on the same (GPU) factors: only the
    # summation order of the triangular solves differs
    x_ref = cs.ref.solve(A.val, b)
    assert np.max(np.abs(x - x_ref)) <= 1e-6 * max(1.0, np.max(np.abs(x_ref)))


@pytest.mark.parametrize("name", ["mna:2000,5", "grid:48,2"])
def test_batched_instances_match_oracle(built_lib, cuda, name):
    torch = _torch()
    from glu_public_b200 import glu
    cs = case(name)
    c = cs.circuit
    count = 6
    vals = c.instance_values(count, seed=11)
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    batch = glu.Batch(plan, count)
    batch.load_values(torch.as_tensor(vals, device=cuda))
    batch.refactor(0.0)
    assert np.all(batch.status() == 0)
    ones = np.ones(c.n)
    B = np.stack([c.to_scipy(vals[i]) @ ones for i in range(count)])[:, None, :]
    X = batch.solve(torch.as_tensor(B, device=cuda)).cpu().numpy()
    for i in range(count):
        lu = batch.get_lu(i).cpu().numpy()
        v = cs.lu_val(vals[i])
        expect, st = O.factor(cs.sym_ref, v)
        assert column_rel_err(cs.sym, lu, expect) <= lu_tolerance(cs, v)
        res = O.residual(c.n, c.indptr, c.indices, vals[i], X[i, 0], B[i, 0])
        assert res <= RES_TOL, (i, res)


def test_native_autotuner_returns_valid_options(built_lib, cuda):
    """glu_autotune (the C-ABI autotuner) returns options from its search space, a positive
    time, leaves the plan usable, and a plan built with the options gives the oracle's factors."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:2000,5")
    c = cs.circuit
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    vals = c.instance_values(3, seed=23)
    a = torch.as_tensor(vals, device=cuda)
    opts, ms = plan.autotune(a, repeats=1)
    assert ms > 0.0
    assert opts["gemm_variant"] in (12, 11, 13, 0, 6, 5) and opts["panel"] in (64, 128)
    assert opts["update_depth"] in (8, 4, 2, 1) and opts["sparse_warps_per_col"] in (0, 1, 2, 4, 8)
    assert opts["dense_threshold"] in (0.9, 0.8, 0.95, 0.99)
    assert opts["sparse_cols_per_warp"] in (1, 2, 4) and opts["sparse_block"] in (128, 256)
    assert opts["wide_level_cols"] in (592, 148, 2368) and opts["sparse_persistent"] in (0, 2)
    assert opts["sparse_col_lanes"] in (32, 0, 16, 8)
    assert opts["level_warps_per_sm"] in (64, 0, 24, 48)
    tuned = glu.Plan(cs.sym, **opts)
    tuned.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    for p_ in (plan, tuned):
        batch = glu.Batch(p_, 3)
        batch.load_values(a)
        batch.refactor(0.0)
        for i in range(3):
            v = cs.lu_val(vals[i])
            expect, _ = O.factor(cs.sym_ref, v)
            assert column_rel_err(cs.sym, batch.get_lu(i).cpu().numpy(), expect) <= \
                lu_tolerance(cs, v)


def test_mixed_and_partial_loads_over_stale_factors(built_lib, cuda):
    """The dense block is assembled by the refactorization for instances loaded in original
    order (not cleared by the load) and cleared for instances loaded in filled-pattern order;
    partial loads of either kind over the factors of an earlier round give the oracle's factors
    for every instance."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:2000,5")
    c = cs.circuit
    plan = glu.Plan(cs.sym)
    assert plan.stat("ntp") > 0
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    count = 4
    batch = glu.Batch(plan, count)
    first = c.instance_values(count, seed=5)
    batch.load_values(torch.as_tensor(first, device=cuda))
    batch.refactor(0.0)                       # leaves factors in every dense block
    vals = c.instance_values(count, seed=6)
    lu_vals = np.stack([cs.lu_val(vals[i]) for i in range(count)])
    batch.load_values(torch.as_tensor(vals[0:2], device=cuda), first=0)
    batch.load_lu_values(torch.as_tensor(lu_vals[2:3], device=cuda), first=2)
    batch.load_values(torch.as_tensor(vals[3:4], device=cuda), first=3)
    batch.refactor(0.0)
    assert np.all(batch.status() == 0)
    for i in range(count):
        expect, _ = O.factor(cs.sym_ref, lu_vals[i])
        got = batch.get_lu(i).cpu().numpy()
        assert column_rel_err(cs.sym, got, expect) <= lu_tolerance(cs, lu_vals[i]), i
    # and the other way round: filled-pattern values first, one instance reloaded in original order
    batch.load_lu_values(torch.as_tensor(np.stack([cs.lu_val(v) for v in first]), device=cuda))
    batch.load_values(torch.as_tensor(vals[1:2], device=cuda), first=1)
    batch.refactor(0.0)
    for i in range(count):
        v = lu_vals[1] if i == 1 else cs.lu_val(first[i])
        expect, _ = O.factor(cs.sym_ref, v)
        assert column_rel_err(cs.sym, batch.get_lu(i).cpu().numpy(), expect) <= lu_tolerance(cs, v)


@pytest.mark.parametrize("name,opts", [("mna:2000,5", {}), ("grid:48,2", {}),
                                       ("grid:48,2", dict(front_min_flops=0.0)),
                                       ("grid:64,3", dict(front_min_w=4, front_min_flops=0.0))])
def test_transposed_solve_matches_oracle(built_lib, cuda, name, opts):
    """Transposed solves (the adjoint's U^T then L^T), also through supernodal fronts."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case(name)
    c = cs.circuit
    plan = glu.Plan(cs.sym, **opts)
    if opts:
        assert plan.stat("fronts") > 0
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    batch = glu.Batch(plan, 1)
    batch.load_values(torch.as_tensor(c.data[None, :], device=cuda))
    batch.refactor(0.0)
    rng = np.random.default_rng(3)
    G = rng.standard_normal((1, 3, c.n))
    lam = batch.solve(torch.as_tensor(G, device=cuda), transpose=True).cpu().numpy()
    lu = batch.get_lu(0).cpu().numpy()
    AT = c.to_scipy().T.tocsc()
    for k in range(3):
        ref = O.solve_transpose(cs.sym_ref, lu, cs.pre, G[0, k])
        assert np.max(np.abs(lam[0, k] - ref)) <= 1e-9 * max(1.0, np.max(np.abs(ref)))
        res = O.residual(c.n, AT.indptr.astype(np.int64), AT.indices, AT.data, lam[0, k], G[0, k])
        assert res <= RES_TOL


def test_perturbation_matches_oracle(built_lib, cuda):
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:2000,5")
    val = cs.sym_ref.val.copy()
    pert = O.perturbation(cs.sym_ref, val)
    # shrink a few pivots so the clamp fires, in the sparse part and in the dense block
    lp = np.asarray(cs.sym.l_col_ptr, np.int64)
    for c in [3, 700, 1900, 1990]:
        val[lp[c]] = 1e-3 * pert
    expect, _ = O.factor(cs.sym_ref, val, pert)
    plan = glu.Plan(cs.sym)
    batch = glu.Batch(plan, 1)
    batch.load_lu_values(torch.as_tensor(val[None, :], device=cuda))
    batch.refactor(-1.0)
    lu = batch.get_lu(0).cpu().numpy()
    assert column_rel_err(cs.sym, lu, expect) <= LU_TOL
    assert batch.status()[0] & 4


def test_zero_pivot_is_flagged_per_instance(built_lib, cuda):
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:200,3")
    good = cs.sym_ref.val.copy()
    bad = good.copy()
    bad[np.asarray(cs.sym.l_col_ptr, np.int64)[0]] = 0.0
    plan = glu.Plan(cs.sym)
    batch = glu.Batch(plan, 3)
    batch.load_lu_values(torch.as_tensor(np.stack([good, bad, good]), device=cuda))
    batch.refactor(0.0)
    st = batch.status()
    assert st[0] == 0 and st[2] == 0 and (st[1] & 1)


def test_nan_and_inf_pivots_are_flagged_per_instance(built_lib, cuda):
    """A NaN or infinite pivot sets GLU_INST_NAN_PIVOT (2) on its instance only, whether the pivot
    is in the sparse phase (first column) or in the dense trailing block (last column); the other
    instances of the batch are unaffected (the reference's NaN / singular checks:
    src/nicslu/source/nicslu_refact.c:151-158)."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:2000,5")
    lp = np.asarray(cs.sym.l_col_ptr, np.int64)
    good = cs.sym_ref.val.copy()
    bad = []
    for pos, v in ((lp[0], np.nan), (lp[-1], np.nan), (lp[0], np.inf), (lp[-1], -np.inf)):
        b = good.copy()
        b[pos] = v
        bad.append(b)
    plan = glu.Plan(cs.sym)
    assert plan.stat("nt") > 0                      # the last column is in the dense block
    batch = glu.Batch(plan, 6)
    batch.load_lu_values(torch.as_tensor(np.stack([good] + bad + [good]), device=cuda))
    batch.refactor(0.0)
    st = batch.status()
    assert st[0] == 0 and st[5] == 0, st
    for i in range(1, 5):
        assert st[i] & 2, (i, st)
    expect, _ = O.factor(cs.sym_ref, good)
    assert column_rel_err(cs.sym, batch.get_lu(5).cpu().numpy(), expect) <= LU_TOL


def test_device_allocation_failure_is_reported_and_recoverable(built_lib, cuda):
    """A batch larger than the device returns GLU_MEMORY_OVERFLOW (-3) with a message; the plan
    and the library stay usable."""
    torch = _torch()
    from glu_public_b200 import _lib, glu
    from tests.common import bench_case
    cs = bench_case("mna20000_s2")
    plan = glu.Plan(cs.sym)
    per = glu.Batch.slots_per_instance(plan) * 8
    total = torch.cuda.get_device_properties(0).total_memory
    count = min(65535, int(2 * total // per) + 1)          # twice the device's memory
    with pytest.raises(_lib.GluError) as ei:
        glu.Batch(plan, count)
    assert ei.value.status == -3
    c = cs.circuit
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    b = glu.Batch(plan, 1)
    b.load_values(torch.as_tensor(c.data[None, :], device=cuda))
    b.refactor(0.0)
    assert b.status()[0] == 0


def test_graph_replay_matches_direct(built_lib, cuda):
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:2000,5")
    c = cs.circuit
    count = 4
    vals = torch.as_tensor(c.instance_values(count, seed=5), device=cuda)
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    B = torch.ones((count, 1, c.n), dtype=torch.float64, device=cuda)
    X1 = torch.zeros_like(B)
    b1 = glu.Batch(plan, count)
    b1.load_values(vals)
    b1.refactor()
    b1.solve(B, out=X1)
    b2 = glu.Batch(plan, count)
    X2 = torch.zeros_like(B)
    b2.load_values(vals)
    b2.refactor()
    b2.solve(B, out=X2)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        b2.capture(vals, B, X2, stream=s)
        for _ in range(3):
            b2.replay(stream=s)
    s.synchronize()
    # atomics make the summation order of the sparse levels run-dependent: compare factors with
    # the rounding-order tolerance and the solutions through their residuals
    vh = vals.cpu().numpy()
    for i in range(count):
        tol = lu_tolerance(cs, cs.lu_val(vh[i]))
        assert column_rel_err(cs.sym, b2.get_lu(i).cpu().numpy(), b1.get_lu(i).cpu().numpy()) <= tol
        b = np.ones(c.n)
        for X in (X1, X2):
            res = O.residual(c.n, c.indptr, c.indices, vh[i], X[i, 0].cpu().numpy(), b)
            assert res <= RES_TOL


@pytest.mark.parametrize("opts", [dict(hub_min_frac=1e-9), dict(hub_min_frac=10.0),
                                  dict(panel=128), dict(gemm_variant=4, panel=128),
                                  dict(sparse_warps_per_col=1), dict(sparse_warps_per_col=8),
                                  dict(sparse_warps_per_col=2, sparse_persistent=0),
                                  dict(sparse_warps_per_col=4, sparse_cols_per_warp=2,
                                       sparse_persistent=0),
                                  dict(sparse_cols_per_warp=4, sparse_block=128,
                                       sparse_persistent=0),
                                  dict(wide_level_cols=16, narrow_col_work=8,
                                       sparse_persistent=0),
                                  dict(sparse_col_lanes=8, sparse_persistent=0),
                                  dict(sparse_col_lanes=16, sparse_cols_per_warp=2,
                                       sparse_persistent=0),
                                  dict(sparse_col_lanes=0, sparse_block=128),
                                  dict(level_warps_per_sm=0), dict(level_warps_per_sm=48),
                                  dict(level_warps_per_sm=24, sparse_block=128),
                                  dict(dense_threshold=0.8), dict(dense_threshold=0.99),
                                  dict(update_depth=1), dict(update_depth=2),
                                  dict(update_depth=8),
                                  dict(update_depth=4, panel=128, gemm_variant=9)])
def test_plan_options_match_oracle(built_lib, cuda, opts):
    """Every hub split (all / none), panel width, update grouping and kernel mode gives the
    oracle's factors."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:4960,1")
    v = cs.sym_ref.val
    expect, _ = O.factor(cs.sym_ref, v)
    plan = glu.Plan(cs.sym, **opts)
    batch = glu.Batch(plan, 2)
    batch.load_lu_values(torch.as_tensor(np.stack([v, v]), device=cuda))
    batch.refactor(0.0)
    for i in range(2):
        assert column_rel_err(cs.sym, batch.get_lu(i).cpu().numpy(), expect) <= lu_tolerance(cs, v)


def test_pull_chunks_match_oracle(built_lib, cuda):
    """Dense columns whose pulls carry far more updates than the average hand their later entries
    to extra CTAs (global atomics after the column is written) when the batch is one or a few
    matrices; the factors still match the oracle's, and at least one case has such chunks."""
    torch = _torch()
    from glu_public_b200 import glu
    chunks = 0
    for name in ("mna:4960,1", "mna:2000,5", "grid:64,3"):
        cs = case(name)
        v = cs.sym_ref.val
        expect, _ = O.factor(cs.sym_ref, v)
        plan = glu.Plan(cs.sym)
        chunks += int(plan.stat("pull_chunks"))
        batch = glu.Batch(plan, 1)
        batch.load_lu_values(torch.as_tensor(v[None, :], device=cuda))
        batch.refactor(0.0)
        assert column_rel_err(cs.sym, batch.get_lu(0).cpu().numpy(), expect) <= lu_tolerance(cs, v)
    assert chunks > 0


@pytest.mark.parametrize("transpose", [False, True])
def test_refinement_reaches_1e12_on_monte_carlo_instances(built_lib, cuda, transpose):
    """Static pivoting leaves some instances marginal (the oracle itself gives ~3e-12 on
    n = 20,000 instances); one refinement round on the original matrix brings every residual,
    computed on the device and cross-checked on the host, to <= 1e-12."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case("mna:4960,1")
    c = cs.circuit
    count = 8
    vals = c.instance_values(count, seed=21)
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    plan.set_original_csc(c.indptr, c.indices)
    batch = glu.Batch(plan, count)
    a = torch.as_tensor(vals, device=cuda)
    batch.load_values(a)
    batch.refactor(0.0)
    rng = np.random.default_rng(4)
    B = torch.as_tensor(rng.standard_normal((count, 2, c.n)), device=cuda)
    X = batch.solve(B, transpose=transpose)
    res = batch.refine(a, B, X, steps=2, transpose=transpose, with_residual=True).cpu().numpy()
    assert res.max() <= RES_TOL, res
    Xh = X.cpu().numpy()
    for i in range(count):
        A = c.to_scipy(vals[i])
        M = A.T.tocsc() if transpose else A
        for k in range(2):
            host = O.residual(c.n, M.indptr.astype(np.int64), M.indices, M.data, Xh[i, k],
                              B[i, k].cpu().numpy())
            assert host <= RES_TOL
            assert abs(host - res[i, k]) <= 0.05 * host + 1e-17


@pytest.mark.parametrize("name", ["grid:48,2", "grid:64,3"])
@pytest.mark.parametrize("opts", [dict(front_min_flops=0.0), dict(front_min_w=0),
                                  dict(front_min_w=4, front_min_flops=0.0, panel=128),
                                  dict(front_min_flops=0.0, update_depth=4),
                                  dict(front_min_flops=0.0, front_batch=0),
                                  dict(front_min_w=4, front_min_flops=0.0, front_batch=1,
                                       sparse_persistent=0),
                                  dict(front_min_flops=0.0, sparse_col_lanes=8),
                                  dict(front_min_w=0, sparse_col_lanes=0)])
def test_supernodal_fronts_match_oracle(built_lib, cuda, name, opts):
    """Mesh patterns: separator runs factored as dense fronts (forced down to small runs here;
    by default only runs whose update costs >= 1e6 flops) and, for comparison, without fronts,
    give the oracle's factors across instances of a batch."""
    torch = _torch()
    from glu_public_b200 import glu
    cs = case(name)
    c = cs.circuit
    plan = glu.Plan(cs.sym, **opts)
    if opts.get("front_min_w", 16) > 0:
        assert plan.stat("fronts") > 0
    else:
        assert plan.stat("fronts") == 0
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    plan.set_original_csc(c.indptr, c.indices)
    vals = c.instance_values(3, seed=17)
    a = torch.as_tensor(vals, device=cuda)
    batch = glu.Batch(plan, 3)
    batch.load_values(a)
    batch.refactor(0.0)
    assert np.all(batch.status() == 0)
    B = torch.as_tensor(np.stack([c.to_scipy(vals[i]) @ np.ones(c.n) for i in range(3)])[:, None, :],
                        device=cuda)
    X = batch.solve(B)
    res = batch.refine(a, B, X, steps=1, with_residual=True).cpu().numpy()
    assert res.max() <= RES_TOL
    for i in range(3):
        v = cs.lu_val(vals[i])
        expect, _ = O.factor(cs.sym_ref, v)
        assert column_rel_err(cs.sym, batch.get_lu(i).cpu().numpy(), expect) <= lu_tolerance(cs, v)
