"""glu_residual_noalloc, the allocation-free residual check, against glu_residual.

The entry point exists for callers that may not allocate device memory between solves (a
simulator loop whose device memory belongs to its own pool, or a section where a cudaMalloc --
which can synchronize the device -- is not allowed).  Its scratch is a fixed array in the
library's static device memory.  This file is collected last on purpose: if it fails, a run that
stops at the first failure has already run every other test.  It also passes when run alone.
"""
import ctypes as C

import numpy as np
import pytest

from tests.common import case

pytestmark = pytest.mark.gpu


def test_residual_noalloc_matches_residual_on_two_calls(built_lib, cuda):
    import torch
    from glu_public_b200 import _lib, glu
    cs = case("mna:2000,5")
    c = cs.circuit
    count, nrhs = 4, 3
    vals = torch.as_tensor(c.instance_values(count, seed=8), device=cuda)
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    plan.set_original_csc(c.indptr, c.indices)
    batch = glu.Batch(plan, count)
    batch.load_values(vals)
    batch.refactor(0.0)
    rng = np.random.default_rng(12)
    B = torch.as_tensor(rng.standard_normal((count, nrhs, c.n)), device=cuda)
    X = batch.solve(B)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L = _lib.lib()
    for call in range(2):             # second call: refined X, so every norm changes
        if call == 1:
            batch.refine(vals, B, X, steps=1)
        expect = batch.residual(vals, B, X).reshape(-1)
        got = torch.full((count * nrhs,), -1.0, dtype=torch.float64, device=cuda)
        st = L.glu_residual_noalloc(batch.h, nrhs, vals.data_ptr(), B.data_ptr(), X.data_ptr(), 0,
                                    got.data_ptr(), stream)
        assert st == 0, L.glu_last_error()
        torch.cuda.synchronize()
        e, g = expect.cpu().numpy(), got.cpu().numpy()
        assert np.all(g >= 0.0)
        assert np.allclose(g, e, rtol=1e-12, atol=0.0), (call, g, e)


def test_residual_noalloc_rejects_too_many_vectors(built_lib, cuda):
    import torch
    from glu_public_b200 import _lib, glu
    cs = case("mna:200,3")
    c = cs.circuit
    plan = glu.Plan(cs.sym)
    plan.set_original_csc(c.indptr, c.indices)
    batch = glu.Batch(plan, 2)
    a = torch.zeros((2, c.nnz), dtype=torch.float64, device=cuda)
    B = torch.zeros((2, 40000, 1), dtype=torch.float64, device=cuda)   # 80,000 vectors of n=1
    st = _lib.lib().glu_residual_noalloc(batch.h, 40000, a.data_ptr(), B.data_ptr(), B.data_ptr(),
                                         0, B.data_ptr(), None)
    assert st == -102
    assert b"at most" in _lib.lib().glu_last_error()
