"""Shared test helpers: problem construction through the reference pipeline (the checker) and
comparison metrics."""
from __future__ import annotations

import dataclasses
import functools
import os

import numpy as np

from glu_public_b200 import gen, glu
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
ADD32 = "/root/reference/src/add32.mtx"   # the reference's sample matrix (only in the build container)


@dataclasses.dataclass
class Case:
    name: str
    circuit: gen.Circuit
    ref: O.RefPipeline
    pre: O.Preprocessed
    sym_ref: O.RefSymbolic
    nic: glu.NicsluArrays
    sym: glu.SymbolicMatrix

    @property
    def n(self):
        return self.circuit.n

    def lu_val(self, data: np.ndarray) -> np.ndarray:
        """Symbolic_Matrix::val for new original-order values (predictLU after preprocess)."""
        ap, ai, ax = self.nic.preprocess(self.circuit.indptr, self.circuit.indices, data)
        pos = self.sym.positions(ai, ap)
        val = np.zeros(self.sym.nnz)
        ok = pos >= 0
        val[pos[ok]] = ax[ok]
        return val


def circuit_for(name: str) -> gen.Circuit:
    kind, _, rest = name.partition(":")
    if kind == "mna":
        n, seed = (int(x) for x in rest.split(","))
        return gen.mna_netlist(n, seed)
    if kind == "grid":
        side, seed = (int(x) for x in rest.split(","))
        return gen.power_grid(side, seed, pads=16 if side < 128 else 64,
                              hubs=4 if side < 128 else 16)
    if kind == "add32":
        return gen.circuit_from_csc(gen.read_mtx(ADD32), "add32")
    raise ValueError(name)


@functools.lru_cache(maxsize=None)
def case(name: str) -> Case:
    c = circuit_for(name)
    ref = O.RefPipeline.from_csc(c.n, c.indptr, c.indices, c.data)
    pre = ref.preprocessed()
    sym_ref = ref.symbolic()
    nic = glu.NicsluArrays(c.n, pre.row_perm, pre.row_perm_inv, pre.col_perm, pre.col_perm_inv,
                           pre.row_scale, pre.col_scale_perm, pre.mc64_scale)
    sym = glu.SymbolicMatrix(c.n).analyze(pre.ai, pre.ap, pre.ax)
    return Case(name, c, ref, pre, sym_ref, nic, sym)


def column_rel_err(sym, a: np.ndarray, b: np.ndarray) -> float:
    """max over columns of max|a-b| / max|b| within the column (max-norm per column)."""
    cp = np.asarray(sym.sym_c_ptr, np.int64)
    col = np.repeat(np.arange(sym.n), np.diff(cp))
    num = np.zeros(sym.n)
    den = np.zeros(sym.n)
    np.maximum.at(num, col, np.abs(a - b))
    np.maximum.at(den, col, np.abs(b))
    den[den == 0] = 1.0
    return float((num / den).max())


def have_add32() -> bool:
    return os.path.exists(ADD32)


def lu_tolerance(cs: Case, val: np.ndarray) -> float:
    """Per-column tolerance for comparing a factorization with the oracle's.

    1e-12, unless the matrix's trailing pivots lose digits to cancellation: then two valid
    rounding orders of the same algorithm (the oracle built with and without fused
    multiply-adds) already differ by more, and the bound is 8x that measured difference.
    """
    a, _ = O.factor(cs.sym_ref, val)
    b, _ = O.factor(cs.sym_ref, val, fma=True)
    return max(1e-12, 8.0 * column_rel_err(cs.sym, b, a))
