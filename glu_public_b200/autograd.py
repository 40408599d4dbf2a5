"""Adjoint of the sparse solve as a ``torch.autograd.Function`` over the C ABI.

Forward: X_i = A_i^-1 B_i for every instance i of a batch (ingest of the original-order values,
refactorization, solve, optional refinement).  Backward, given G_i = dLoss/dX_i:

    lambda_i = A_i^-T G_i            (transposed solves on the forward's factors: U^T, then L^T,
                                      with the row/column permutations and MC64 scalings undone)
    dLoss/dB_i = lambda_i
    dLoss/dA_i[e] = -sum_k lambda_i[k][row(e)] * X_i[k][col(e)]   for every nonzero e of A_i

(glu_solve with transpose = 1, glu_grad_a).  When the factors of the whole batch do not fit the
device memory budget, the forward keeps only its inputs and the backward refactors each chunk of
instances again before the transposed solve ("recompute instead of keep").
"""
from __future__ import annotations

from typing import Optional

import torch

from . import glu


class SparseLUSolve(torch.autograd.Function):
    """X = solve(A(values), B) for a batch of value sets of one pattern."""

    @staticmethod
    def forward(ctx, values: torch.Tensor, B: torch.Tensor, plan: glu.Plan, chunk: int,
                refine: int, pert: float):
        count = values.shape[0]
        X = torch.empty_like(B)
        keep = chunk >= count
        batch = glu.Batch(plan, min(chunk, count))
        for s in range(0, count, batch.count):
            e = min(count, s + batch.count)
            if e - s != batch.count:
                batch = glu.Batch(plan, e - s)
            v = values[s:e].contiguous()
            b = B[s:e].contiguous()
            batch.load_values(v)
            batch.refactor(pert)
            x = batch.solve(b)
            if refine:
                batch.refine(v, b, x, steps=refine)
            X[s:e] = x
        ctx.plan, ctx.chunk, ctx.refine, ctx.pert = plan, chunk, refine, pert
        ctx.batch = batch if keep else None       # factors kept only if the whole batch fits
        ctx.save_for_backward(values, B, X)
        return X

    @staticmethod
    def backward(ctx, gX: torch.Tensor):
        values, B, X = ctx.saved_tensors
        plan: glu.Plan = ctx.plan
        count = values.shape[0]
        gX = gX.contiguous()
        lam = torch.empty_like(gX)
        gA = torch.empty_like(values) if ctx.needs_input_grad[0] else None
        batch = ctx.batch
        step = batch.count if batch is not None else min(ctx.chunk, count)
        for s in range(0, count, step):
            e = min(count, s + step)
            v = values[s:e].contiguous()
            if ctx.batch is None:                  # recompute the factors of this chunk
                if batch is None or batch.count != e - s:
                    batch = glu.Batch(plan, e - s)
                batch.load_values(v)
                batch.refactor(ctx.pert)
            g = gX[s:e]
            lm = batch.solve(g, transpose=True)
            if ctx.refine:
                batch.refine(v, g, lm, steps=ctx.refine, transpose=True)
            lam[s:e] = lm
            if gA is not None:
                gA[s:e] = batch.grad_a(lm, X[s:e].contiguous())
        return gA, (lam if ctx.needs_input_grad[1] else None), None, None, None, None


def sparse_solve(values: torch.Tensor, B: torch.Tensor, plan: glu.Plan, *,
                 chunk: Optional[int] = None, refine: int = 1, pert: float = 0.0,
                 budget_bytes: Optional[int] = None) -> torch.Tensor:
    """Differentiable batched sparse solve.

    values: [count, nnz_a] original-order values (the plan needs its ingest map, solve maps and
    original pattern); B: [count, nrhs, n].  ``chunk`` instances are factored at a time; by
    default the whole batch, unless its factors would exceed ``budget_bytes`` (default: 80 % of
    the free device memory), in which case the largest chunk that fits is used and the backward
    recomputes the factors.
    """
    if not plan.grad_pattern:
        raise RuntimeError("the plan needs set_original_pattern / set_original_csc for gradients")
    count = values.shape[0]
    if chunk is None:
        per = glu.Batch.slots_per_instance(plan) * 8
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(values.device)
            budget_bytes = int(0.8 * free)
        chunk = max(1, min(count, budget_bytes // max(per, 1)))
    return SparseLUSolve.apply(values, B, plan, int(chunk), int(refine), float(pert))
