"""Deterministic mode (glu_options.deterministic = 1): ownership instead of FP64 atomics.

Every target is written by one warp or CTA that adds its contributions in a fixed order (the
sparse levels' update pairs grouped by target column, the sparse-to-dense pull entry by entry,
row-wise forward solves), fronts and the cooperative level launch are off.  Two runs on the same
values must give the same bits -- factors, solutions, refined solutions -- and the factors must
still match the oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import bench_case, case, column_rel_err, lu_tolerance

pytestmark = pytest.mark.gpu


def _run(sym, c, nic, vals, B, cuda, **opts):
    import torch
    from glu_public_b200 import glu
    plan = glu.Plan(sym, **opts)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, nic)
    plan.set_solve_maps(nic)
    plan.set_original_csc(c.indptr, c.indices)
    batch = glu.Batch(plan, vals.shape[0])
    a = torch.as_tensor(vals, device=cuda)
    Bt = torch.as_tensor(B, device=cuda)
    batch.load_values(a)
    batch.refactor(0.0)
    X = batch.solve(Bt)
    Xr = X.clone()
    batch.refine(a, Bt, Xr, steps=1)
    lus = [batch.get_lu(i).cpu().numpy() for i in range(vals.shape[0])]
    return lus, X.cpu().numpy(), Xr.cpu().numpy(), batch.status()


@pytest.mark.parametrize("name", ["mna:2000,5", "mna:4960,1", "grid:48,2"])
def test_deterministic_mode_repeats_bits_and_matches_oracle(built_lib, cuda, name):
    cs = case(name)
    c = cs.circuit
    vals = c.instance_values(3, seed=41)
    rng = np.random.default_rng(3)
    B = np.stack([c.to_scipy(vals[i]) @ rng.standard_normal((c.n, 2)) for i in range(3)])
    B = np.ascontiguousarray(B.transpose(0, 2, 1))
    r1 = _run(cs.sym, c, cs.nic, vals, B, cuda, deterministic=1)
    r2 = _run(cs.sym, c, cs.nic, vals, B, cuda, deterministic=1)
    assert np.all(r1[3] == 0)
    for i in range(3):
        assert np.array_equal(r1[0][i], r2[0][i]), i
        v = cs.lu_val(vals[i])
        expect, _ = O.factor(cs.sym_ref, v)
        assert column_rel_err(cs.sym, r1[0][i], expect) <= lu_tolerance(cs, v)
    assert np.array_equal(r1[1], r2[1]) and np.array_equal(r1[2], r2[2])
    for i in range(3):
        for k in range(2):
            assert O.residual(c.n, c.indptr, c.indices, vals[i], r1[2][i, k], B[i, k]) <= 1e-12


def test_deterministic_mode_on_the_benchmark_pattern(built_lib, cuda):
    """n = 20,000 with the benchmark's tuned options: bit-identical over two runs."""
    cs = bench_case("mna20000_s2")
    c = cs.circuit
    vals = c.instance_values(4, seed=99)
    B = np.stack([c.to_scipy(vals[i]) @ np.ones(c.n) for i in range(4)])[:, None, :]
    opts = dict(gemm_variant=11, update_depth=8, deterministic=1)
    r1 = _run(cs.sym, c, cs.nic, vals, B, cuda, **opts)
    r2 = _run(cs.sym, c, cs.nic, vals, B, cuda, **opts)
    for i in range(4):
        assert np.array_equal(r1[0][i], r2[0][i]), i
    assert np.array_equal(r1[2], r2[2])
    for i in range(4):
        assert O.residual(c.n, c.indptr, c.indices, vals[i], r1[2][i, 0], B[i, 0]) <= 1e-12
