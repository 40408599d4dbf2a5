"""Adjoint (torch.autograd.Function over the C ABI) against dense FP64 and finite differences.

Loss = sum(w * X) with X = A^-1 B for a batch of Monte Carlo instances.  Checks:
  * dLoss/dA on A's nonzeros and dLoss/dB against a dense FP64 reference gradient (numpy,
    lambda = A^-T w, dA = -lambda x^T on the pattern), n = 2,000;
  * central finite differences with step 1e-6 * |a_ij| on 200 random nonzeros;
  * the recompute-instead-of-keep path (factors not kept) gives the same gradient.
"""
import numpy as np
import pytest

from tests.common import case

pytestmark = pytest.mark.gpu


def _setup(name, count, nrhs, seed):
    import torch
    from glu_public_b200 import glu
    cs = case(name)
    c = cs.circuit
    plan = glu.Plan(cs.sym)
    plan.set_ingest_from_nicslu(c.indptr, c.indices, cs.nic)
    plan.set_solve_maps(cs.nic)
    plan.set_original_csc(c.indptr, c.indices)
    rng = np.random.default_rng(seed)
    vals = c.instance_values(count, seed=seed)
    B = rng.standard_normal((count, nrhs, c.n))
    W = rng.standard_normal((count, nrhs, c.n))
    dev = torch.device("cuda:0")
    return cs, plan, vals, B, W, dev


def _grads(plan, vals, B, W, dev, chunk=None):
    import torch
    from glu_public_b200 import autograd
    a = torch.tensor(vals, device=dev, requires_grad=True)
    b = torch.tensor(B, device=dev, requires_grad=True)
    X = autograd.sparse_solve(a, b, plan, chunk=chunk)
    loss = (torch.tensor(W, device=dev) * X).sum()
    loss.backward()
    return X.detach().cpu().numpy(), a.grad.cpu().numpy(), b.grad.cpu().numpy()


def test_adjoint_matches_dense_fp64_gradient(built_lib, cuda):
    cs, plan, vals, B, W, dev = _setup("mna:2000,5", 2, 3, 31)
    c = cs.circuit
    X, gA, gB = _grads(plan, vals, B, W, dev)
    rows = c.indices.astype(np.int64)
    cols = np.repeat(np.arange(c.n), np.diff(c.indptr))
    for i in range(2):
        A = c.to_scipy(vals[i]).toarray()
        Xd = np.linalg.solve(A, B[i].T)                 # [n, nrhs]
        lam = np.linalg.solve(A.T, W[i].T)              # [n, nrhs]
        ref_gA = -(lam[rows] * Xd[cols]).sum(axis=1)
        assert np.max(np.abs(X[i].T - Xd)) <= 1e-6 * np.max(np.abs(Xd))
        assert np.max(np.abs(gB[i].T - lam)) <= 1e-6 * np.max(np.abs(lam))
        assert np.max(np.abs(gA[i] - ref_gA)) <= 1e-6 * np.max(np.abs(ref_gA))


def test_adjoint_matches_central_finite_differences(built_lib, cuda):
    import torch
    from glu_public_b200 import glu
    cs, plan, vals, B, W, dev = _setup("mna:2000,5", 1, 2, 7)
    c = cs.circuit
    _, gA, _ = _grads(plan, vals, B, W, dev)
    batch = glu.Batch(plan, 1)
    Bt = torch.tensor(B, device=dev)
    Wt = torch.tensor(W, device=dev)

    def loss(v):
        a = torch.tensor(v[None, :], device=dev)
        batch.load_values(a)
        batch.refactor(0.0)
        x = batch.solve(Bt)
        batch.refine(a, Bt, x, steps=2)
        return float((Wt * x).sum().item())

    rng = np.random.default_rng(3)
    picks = rng.choice(c.nnz, size=200, replace=False)
    fd = np.empty(200)
    for q, e in enumerate(picks):
        h = 1e-6 * abs(vals[0, e])
        vp = vals[0].copy()
        vm = vals[0].copy()
        vp[e] += h
        vm[e] -= h
        fd[q] = (loss(vp) - loss(vm)) / (2 * h)
    an = gA[0, picks]
    scale = np.max(np.abs(an))
    err = np.abs(fd - an)
    # central differences carry O(h^2) truncation and O(eps |loss| / h) rounding error
    assert np.median(err / scale) <= 1e-6
    assert np.max(err / scale) <= 1e-3


def test_recompute_path_matches_kept_factors(built_lib, cuda):
    cs, plan, vals, B, W, dev = _setup("mna:2000,5", 4, 2, 19)
    X1, gA1, gB1 = _grads(plan, vals, B, W, dev)              # whole batch kept
    X2, gA2, gB2 = _grads(plan, vals, B, W, dev, chunk=1)     # factors recomputed per instance
    for a, b in ((X1, X2), (gA1, gA2), (gB1, gB2)):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(a))
