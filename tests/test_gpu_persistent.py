"""The cooperative persistent level kernel (k_sparse_persistent) against the oracle, and its
bounded device-side waits.

Runs of consecutive sparse levels without fronts are factored by ONE cooperative launch whose
CTA groups meet at device-side barriers between levels (option sparse_persistent; 0 = one
launch per level).  Checked: the same factors as the oracle (and as per-level launches) for one
instance (one group spanning the grid), a few instances (several groups) and groups of one CTA;
the long tail of one-column levels
when the dense trailing block is switched off; graph capture of the cooperative launch; and the
failure path -- a barrier made unreachable on purpose gives up after its bound, flags every
instance GLU_INST_TIMEOUT, returns GLU_TIMEOUT, and the context stays usable.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import case, column_rel_err, lu_tolerance

pytestmark = pytest.mark.gpu


def _factor(cs, vals, cuda, **opts):
    import torch
    from glu_public_b200 import glu
    c = cs.circuit
    plan = glu.Plan(cs.sym, **opts)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    batch = glu.Batch(plan, vals.shape[0])
    batch.load_values(torch.as_tensor(vals, device=cuda))
    batch.refactor(0.0)
    return plan, batch


@pytest.mark.parametrize("name,count,opts", [
    ("mna:2000,5", 1, {}),
    ("mna:2000,5", 3, {}),
    ("mna:200,3", 200, {"dense_threshold": 2.0, "sparse_warps_per_col": 1}),  # CTA groups of one
    ("mna:4960,1", 1, {"dense_threshold": 2.0}),           # the long tail of one-column levels
    ("mna:4960,1", 2, {"dense_threshold": 2.0, "sparse_warps_per_col": 8}),
    ("grid:48,2", 2, {}),                                  # runs broken by fronts
])
def test_persistent_levels_match_oracle_and_per_level_launches(built_lib, cuda, name, count,
                                                               opts):
    cs = case(name)
    vals = cs.circuit.instance_values(count, seed=31)
    _, b_pers = _factor(cs, vals, cuda, sparse_persistent=2, **opts)
    _, b_lev = _factor(cs, vals, cuda, sparse_persistent=0, **opts)
    assert np.all(b_pers.status() == 0) and np.all(b_lev.status() == 0)
    for i in sorted({0, count // 2, count - 1}):
        v = cs.lu_val(vals[i])
        expect, st = O.factor(cs.sym_ref, v)
        tol = lu_tolerance(cs, v)
        got = b_pers.get_lu(i).cpu().numpy()
        assert column_rel_err(cs.sym, got, expect) <= tol, (i, column_rel_err(cs.sym, got, expect))
        ref = b_lev.get_lu(i).cpu().numpy()
        assert column_rel_err(cs.sym, got, ref) <= tol


def test_persistent_launch_reduces_launches(built_lib, cuda):
    cs = case("mna:4960,1")
    vals = cs.circuit.instance_values(1, seed=2)
    plan, b_pers = _factor(cs, vals, cuda, sparse_persistent=2, dense_threshold=2.0)
    n_pers = b_pers.launches
    _, b_lev = _factor(cs, vals, cuda, sparse_persistent=0, dense_threshold=2.0)
    n_lev = b_lev.launches
    assert plan.stat("sparse_levels") > 1000
    assert n_pers < 10 < n_lev, (n_pers, n_lev)


def test_persistent_launch_in_a_cuda_graph(built_lib, cuda):
    import torch
    from glu_public_b200 import glu
    cs = case("mna:4960,1")
    c = cs.circuit
    vals = torch.as_tensor(c.instance_values(2, seed=5), device=cuda)
    plan = glu.Plan(cs.sym, dense_threshold=2.0)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    batch = glu.Batch(plan, 2)
    B = torch.ones((2, 1, c.n), dtype=torch.float64, device=cuda)
    X = torch.zeros_like(B)
    batch.load_values(vals)
    batch.refactor(0.0)
    batch.solve(B, out=X)
    batch.capture(vals, B, X)
    for _ in range(2):
        batch.replay()
    torch.cuda.synchronize()
    for i in range(2):
        v = cs.lu_val(vals[i].cpu().numpy())
        expect, _ = O.factor(cs.sym_ref, v)
        assert column_rel_err(cs.sym, batch.get_lu(i).cpu().numpy(), expect) <= lu_tolerance(cs, v)


@pytest.mark.parametrize("name,count,opts", [
    ("mna:4960,1", 1, {"dense_threshold": 2.0}),                                # one group
    ("mna:200,3", 200, {"dense_threshold": 2.0, "sparse_warps_per_col": 1})])  # groups of one CTA
def test_unreachable_barrier_times_out_and_context_survives(built_lib, cuda, name, count, opts):
    import ctypes as C
    import time
    import torch
    from glu_public_b200 import _lib
    cs = case(name)
    vals = cs.circuit.instance_values(count, seed=7)
    plan, batch = _factor(cs, vals, cuda, **opts)
    _, per_level = _factor(cs, vals, cuda, sparse_persistent=0, **opts)
    assert batch.launches < per_level.launches          # the plan has cooperative level runs
    L = _lib.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    t0 = time.time()
    st = L.glu_debug_refactor_unreachable_barrier(batch.h, 5.0, stream)
    elapsed = time.time() - t0
    assert st == -101, L.glu_last_error()
    assert b"gave up" in L.glu_last_error()
    assert np.all(batch.status() & 8)                 # GLU_INST_TIMEOUT on every instance
    assert elapsed < 30.0
    # the context is still usable: a normal refactorization gives the oracle's factors
    batch.load_values(torch.as_tensor(vals, device=cuda))
    batch.refactor(0.0)
    assert np.all(batch.status() == 0)
    v = cs.lu_val(vals[0])
    expect, _ = O.factor(cs.sym_ref, v)
    assert column_rel_err(cs.sym, batch.get_lu(0).cpu().numpy(), expect) <= lu_tolerance(cs, v)
