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

MAX_VECTORS = 65536          # GLU_NOALLOC_MAX_VECTORS in include/glu_b200.h


def _batch(cs, count, cuda, seed=8):
    import torch
    from glu_public_b200 import glu
    c = cs.circuit
    vals = torch.as_tensor(c.instance_values(count, seed=seed), device=cuda)
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    plan.set_original_csc(c.indptr, c.indices)
    batch = glu.Batch(plan, count)
    batch.load_values(vals)
    batch.refactor(0.0)
    return plan, batch, vals


def _noalloc(batch, nrhs, vals, B, X, transpose, out):
    import torch
    from glu_public_b200 import _lib
    L = _lib.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    return L.glu_residual_noalloc(batch.h, nrhs, vals.data_ptr(), B.data_ptr(), X.data_ptr(),
                                  int(transpose), out.data_ptr(), stream)


@pytest.mark.parametrize("transpose", [False, True])
def test_residual_noalloc_matches_residual_on_two_calls(built_lib, cuda, transpose):
    import torch
    from glu_public_b200 import _lib
    cs = case("mna:2000,5")
    count, nrhs = 4, 3
    plan, batch, vals = _batch(cs, count, cuda)
    rng = np.random.default_rng(12)
    B = torch.as_tensor(rng.standard_normal((count, nrhs, cs.n)), device=cuda)
    X = batch.solve(B, transpose=transpose)
    for call in range(2):             # second call: refined X, so every norm changes
        if call == 1:
            batch.refine(vals, B, X, steps=1, transpose=transpose)
        expect = batch.residual(vals, B, X, transpose=transpose).reshape(-1)
        got = torch.full((count * nrhs,), -1.0, dtype=torch.float64, device=cuda)
        st = _noalloc(batch, nrhs, vals, B, X, transpose, got)
        assert st == 0, _lib.lib().glu_last_error()
        torch.cuda.synchronize()
        e, g = expect.cpu().numpy(), got.cpu().numpy()
        assert np.all(g >= 0.0)
        assert np.allclose(g, e, rtol=1e-12, atol=0.0), (call, g, e)


def test_residual_noalloc_leaves_free_device_memory_unchanged(built_lib, cuda):
    """After the first call (which looks up the scratch address), further calls of different
    sizes leave the device's free memory exactly as it was: nothing is allocated."""
    import torch
    from glu_public_b200 import _lib
    cs = case("mna:2000,5")
    count = 4
    plan, batch, vals = _batch(cs, count, cuda, seed=9)
    rng = np.random.default_rng(3)
    Bs = [torch.as_tensor(rng.standard_normal((count, k, cs.n)), device=cuda) for k in (1, 5, 16)]
    Xs = [batch.solve(B) for B in Bs]
    outs = [torch.empty(count * B.shape[1], dtype=torch.float64, device=cuda) for B in Bs]
    assert _noalloc(batch, 1, vals, Bs[0], Xs[0], False, outs[0]) == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for rep in range(3):
        for B, X, out in zip(Bs, Xs, outs):
            st = _noalloc(batch, B.shape[1], vals, B, X, rep % 2 == 1, out)
            assert st == 0, _lib.lib().glu_last_error()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_residual_noalloc_at_and_past_its_limit(built_lib, cuda):
    """count * nrhs = GLU_NOALLOC_MAX_VECTORS runs (every vector the same, so every residual
    equals glu_residual's for that one vector); one vector more is refused."""
    import torch
    from glu_public_b200 import _lib
    cs = case("mna:200,3")
    count = 2
    plan, batch, vals = _batch(cs, count, cuda, seed=4)
    vals = vals[:1].expand(count, -1).contiguous()          # both instances the same values
    batch.load_values(vals)
    batch.refactor(0.0)
    rng = np.random.default_rng(5)
    b1 = torch.as_tensor(rng.standard_normal((1, 1, cs.n)), device=cuda)
    x1 = batch.solve(b1.expand(count, 1, cs.n).contiguous())[:1]
    expect = float(batch.residual(vals, b1.expand(count, 1, cs.n).contiguous(),
                                  x1.expand(count, 1, cs.n).contiguous()).reshape(-1)[0].item())
    nrhs = MAX_VECTORS // count
    B = b1.expand(count, nrhs, cs.n).contiguous()
    X = x1.expand(count, nrhs, cs.n).contiguous()
    out = torch.full((count * nrhs,), -1.0, dtype=torch.float64, device=cuda)
    st = _noalloc(batch, nrhs, vals, B, X, False, out)
    assert st == 0, _lib.lib().glu_last_error()
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    assert np.allclose(got, expect, rtol=1e-12, atol=0.0), (got.min(), got.max(), expect)
    del B, X, out
    torch.cuda.empty_cache()
    # one vector more: 3 instances x 21,846 right-hand sides of the same pattern = 65,538 > limit
    plan3, batch3, vals3 = _batch(cs, 3, cuda, seed=4)
    nr = MAX_VECTORS // 3 + 1
    Bz = torch.zeros((3, nr, cs.n), dtype=torch.float64, device=cuda)
    outz = torch.zeros(3 * nr, dtype=torch.float64, device=cuda)
    st = _noalloc(batch3, nr, vals3, Bz, Bz, False, outz)
    assert st == -102
    assert b"at most" in _lib.lib().glu_last_error()


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
