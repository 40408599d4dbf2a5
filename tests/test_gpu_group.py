"""Multi-pattern batch in one CUDA graph (glu_group_capture): three patterns of uneven sizes,
each branch checked against the same batch run on its own, and against the residual bound."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.common import case, column_rel_err, lu_tolerance

pytestmark = pytest.mark.gpu


def test_group_of_uneven_patterns_matches_separate_batches(built_lib, cuda):
    import torch
    from glu_public_b200 import glu
    specs = [("mna:2000,5", 16), ("grid:48,2", 3), ("mna:4960,1", 2)]
    plans, batches, vals, Bs, Xs, refs = [], [], [], [], [], []
    for k, (name, count) in enumerate(specs):
        cs = case(name)
        c = cs.circuit
        plan = glu.Plan(cs.sym)
        plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
        plan.set_solve_maps(cs.nic)
        plan.set_original_csc(c.indptr, c.indices)
        v = c.instance_values(count, seed=40 + k)
        B = np.stack([c.to_scipy(v[i]) @ np.ones(c.n) for i in range(count)])[:, None, :]
        vt = torch.as_tensor(v, device=cuda)
        Bt = torch.as_tensor(B, device=cuda)
        # the same work run on its own, for comparison
        sep = glu.Batch(plan, count)
        sep.load_values(vt)
        sep.refactor(0.0)
        Xsep = sep.solve(Bt)
        sep.refine(vt, Bt, Xsep, steps=1)
        refs.append((cs, sep, Xsep))
        plans.append(plan)
        batches.append(glu.Batch(plan, count))
        vals.append(vt)
        Bs.append(Bt)
        Xs.append(torch.zeros_like(Bt))
    group = glu.Group(batches, vals, Bs, Xs, refine=1)
    assert group.launches > 0
    for _ in range(2):
        group.launch()
    torch.cuda.synchronize()
    for k, (cs, sep, Xsep) in enumerate(refs):
        c = cs.circuit
        vh = vals[k].cpu().numpy()
        for i in range(batches[k].count):
            v = cs.lu_val(vh[i])
            tol = lu_tolerance(cs, v)
            assert column_rel_err(cs.sym, batches[k].get_lu(i).cpu().numpy(),
                                  sep.get_lu(i).cpu().numpy()) <= tol
            res = O.residual(c.n, c.indptr, c.indices, vh[i], Xs[k][i, 0].cpu().numpy(),
                             Bs[k][i, 0].cpu().numpy())
            assert res <= 1e-12, (k, i, res)
