"""Autotuner for the numeric phase: picks the plan options that minimise the measured device time
of one refactorization of a batch, and caches the choice per sparsity pattern.

Knobs (``glu_options``): the density threshold of the dense trailing block, dense panel width
(64 / 128), panels per trailing update (1 / 2 / 4 / 8), DMMA GEMM tile variant (0..13), hub
threshold of the sparse-to-dense contributions, and for the sparse levels: warps per column
(1 / 2 / 4 / 8, or by level), columns per warp group (1 / 2 / 4), lanes per column (32 / 16 / 8,
or by level), the wide-level threshold in columns, the block size (128 / 256), the warps per SM
the level launches aim for, and whether runs of levels go into one cooperative launch.
The reference hard-codes its equivalents (level-width thresholds 896 / 448 / 16 and block sizes
64 / 128 / 1024, src/numeric.cu:423-545).

Search: coordinate descent from the defaults, each candidate timed with ``glu_refactor_timed``
(CUDA events around every launch) on a sample of the caller's instances, best of ``repeats``.
The result is stored in a JSON cache keyed by a digest of the pattern (sym_c_ptr, sym_r_idx,
level sets) and the batch size, so a second call for the same pattern costs nothing.
"""
from __future__ import annotations

import hashlib
import json
import os
import time
from typing import Optional

import numpy as np

from . import glu

DEFAULT_CACHE = os.environ.get("GLU_TUNE_CACHE",
                               os.path.join(os.path.expanduser("~"), ".cache", "glu_b200",
                                            "tune.json"))

SPACE = {
    "dense_threshold": [0.9, 0.8, 0.95, 0.99],
    "gemm_variant": [12, 11, 13, 0, 6, 5],
    "panel": [64, 128],
    "update_depth": [2, 1, 4, 8],
    "hub_min_frac": [0.02, 0.005, 0.08],
    "sparse_warps_per_col": [0, 1, 2, 4, 8],
    "sparse_cols_per_warp": [1, 2, 4],
    "wide_level_cols": [592, 148, 2368],
    "sparse_block": [256, 128],
    "sparse_persistent": [2, 0],
    "sparse_col_lanes": [32, 0, 16, 8],
    "level_warps_per_sm": [64, 0, 24, 48],
}
DEFAULTS = {"dense_threshold": 0.9, "gemm_variant": 12, "panel": 64, "update_depth": 8,
            "hub_min_frac": 0.02, "sparse_warps_per_col": 0, "sparse_cols_per_warp": 1,
            "wide_level_cols": 592, "sparse_block": 256, "sparse_persistent": 2,
            "sparse_col_lanes": 32, "level_warps_per_sm": 64}


def pattern_key(sym: glu.SymbolicMatrix, count: int) -> str:
    h = hashlib.sha256()
    for a in (sym.sym_c_ptr, sym.sym_r_idx, sym.level_ptr, sym.level_idx):
        h.update(np.ascontiguousarray(a).tobytes())
    h.update(str(count).encode())
    return h.hexdigest()[:32]


def _time_options(sym, values_dev, lu_values: bool, opts: dict, repeats: int, nic=None,
                  indptr=None, indices=None) -> tuple[float, dict]:
    plan = glu.Plan(sym, **opts)
    if not lu_values:
        plan.set_ingest_from_nicslu(indptr, indices, nic)
    batch = glu.Batch(plan, values_dev.shape[0])
    best, phases = float("inf"), {}
    for _ in range(repeats):
        if lu_values:
            batch.load_lu_values(values_dev)
        else:
            batch.load_values(values_dev)
        ph = batch.refactor_timed(0.0)
        ms = sum(v[0] for v in ph.values())
        if ms < best:
            best, phases = ms, ph
    del batch, plan
    return best, phases


def autotune(sym: glu.SymbolicMatrix, values_dev, *, lu_values: bool = False, nic=None,
             indptr=None, indices=None, count_hint: Optional[int] = None, repeats: int = 2,
             cache: Optional[str] = DEFAULT_CACHE, verbose: bool = False) -> dict:
    """Returns the best plan options for this pattern (a dict for ``glu.Plan(sym, **opts)``).

    ``values_dev``: a float64 CUDA tensor with a sample of instances, either original-order
    values ([k, nnz_a], needs ``nic``, ``indptr``, ``indices``) or, with ``lu_values=True``,
    filled-pattern values ([k, nnz]).  ``count_hint``: the batch size the options are for
    (defaults to the sample size); it is part of the cache key.
    """
    count = count_hint or values_dev.shape[0]
    key = pattern_key(sym, count)
    table = {}
    if cache and os.path.exists(cache):
        try:
            table = json.load(open(cache))
        except (OSError, ValueError):
            table = {}
    if key in table:
        return dict(table[key]["options"])
    t0 = time.time()
    cur = dict(DEFAULTS)
    best, _ = _time_options(sym, values_dev, lu_values, cur, repeats, nic, indptr, indices)
    trials = [(dict(cur), best)]
    for knob, choices in SPACE.items():
        for v in choices:
            if v == cur[knob]:
                continue
            cand = dict(cur)
            cand[knob] = v
            try:
                ms, _ = _time_options(sym, values_dev, lu_values, cand, repeats, nic, indptr,
                                      indices)
            except glu.GluError as e:          # a candidate that does not fit: skip it
                if e.status != -3:
                    raise
                continue
            trials.append((dict(cand), ms))
            if verbose:
                print(f"autotune {knob}={v}: {ms:.3f} ms (best {best:.3f})", flush=True)
            if ms < best:
                best, cur = ms, cand
    entry = {"options": cur, "ms": best, "sample": int(values_dev.shape[0]), "count": count,
             "trials": [{"options": o, "ms": m} for o, m in trials],
             "seconds": time.time() - t0}
    if cache:
        os.makedirs(os.path.dirname(cache), exist_ok=True)
        table[key] = entry
        tmp = cache + ".tmp"
        with open(tmp, "w") as f:
            json.dump(table, f, indent=1)
        os.replace(tmp, cache)
    return dict(cur)
