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
# the reference's sample matrix src/add32.mtx, as CSC (tests/golden/make_fixtures.py --add32)
ADD32 = os.path.join(GOLDEN, "add32.npz")


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
        return gen.circuit_from_csc(add32_matrix(), "add32")
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


def add32_matrix():
    import scipy.sparse as sp
    z = np.load(ADD32)
    n = int(z["n"])
    return sp.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=(n, n))


def order_sensitivity(sym, val: np.ndarray, expect: np.ndarray, pert: float = 0.0,
                      threads: int = 1) -> dict:
    """How much the oracle's own factors move under other valid rounding orders of the same
    algorithm: built with fused multiply-adds, and with the columns of every level taken in
    reverse order (the reference's atomic updates fix no order among a level's columns), alone
    and together.  Per-column relative differences from ``expect`` (max over columns, and the
    number of columns above 1e-12)."""
    out = {}
    for name, kw in (("fma", dict(fma=True)), ("reversed", dict(reverse_levels=True)),
                     ("reversed_fma", dict(fma=True, reverse_levels=True))):
        other, _ = O.factor(sym, val, pert=pert, threads=threads, **kw)
        e = column_errors(sym, other, expect)
        out[name] = (float(e.max()), int((e > 1e-12).sum()))
    return out


def lu_tolerance(cs: Case, val: np.ndarray, pert: float = 0.0) -> float:
    """Per-column tolerance for comparing a factorization with the oracle's.

    1e-12, unless the matrix's trailing pivots lose digits to cancellation: then other valid
    rounding orders of the same algorithm (order_sensitivity) already differ by more, and the
    bound is 8x the largest of those measured differences.
    """
    a, _ = O.factor(cs.sym_ref, val, pert=pert)
    sens = order_sensitivity(cs.sym_ref, val, a, pert=pert)
    return max(1e-12, 8.0 * max(v[0] for v in sens.values()))


@dataclasses.dataclass
class BenchCase:
    """A benchmark pattern: the generated matrix, the reference's NICSLU preprocessing of it (the
    committed fixture tests/golden/nicslu_<name>.npz, checked against the matrix's digest) and
    this package's symbolic analysis, which equals symbolic.cc's bit for bit (pinned by
    tests/golden/symbolic_golden.json where symbolic.cc finishes)."""
    name: str
    circuit: gen.Circuit
    nic: glu.NicsluArrays
    sym: glu.SymbolicMatrix

    @property
    def n(self):
        return self.circuit.n

    def lu_val(self, data: np.ndarray) -> np.ndarray:
        ap, ai, ax = self.nic.preprocess(self.circuit.indptr, self.circuit.indices, data)
        pos = self.sym.positions(ai, ap)
        val = np.zeros(self.sym.nnz)
        ok = pos >= 0
        val[pos[ok]] = ax[ok]
        return val


def circuit_digest(c: gen.Circuit) -> str:
    import hashlib
    h = hashlib.sha256()
    for a in (c.indptr.astype(np.int64), c.indices.astype(np.int32), c.data):
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


@functools.lru_cache(maxsize=None)
def bench_case(name: str) -> BenchCase:
    kind, seed = name.split("_s")
    if kind.startswith("mna"):
        c = gen.mna_netlist(int(kind[3:]), int(seed))
    else:
        c = gen.power_grid(int(kind[4:]), int(seed))
    path = os.path.join(GOLDEN, f"nicslu_{name}.npz")
    if str(np.load(path)["matrix_digest"]) != circuit_digest(c):
        raise RuntimeError(f"{path} does not belong to the generated pattern {name}")
    nic = glu.NicsluArrays.from_npz(path)
    ap, ai, _ = nic.preprocess(c.indptr, c.indices, c.data)
    sym = glu.SymbolicMatrix(c.n).analyze(ai, ap)
    return BenchCase(name, c, nic, sym)


def column_errors(sym, a: np.ndarray, b: np.ndarray) -> np.ndarray:
    """Per column: max|a-b| / max|b| within the column."""
    cp = np.asarray(sym.sym_c_ptr, np.int64)
    col = np.repeat(np.arange(sym.n), np.diff(cp))
    num = np.zeros(sym.n)
    den = np.zeros(sym.n)
    np.maximum.at(num, col, np.abs(a - b))
    np.maximum.at(den, col, np.abs(b))
    den[den == 0] = 1.0
    return num / den


def parity_report(record: dict) -> None:
    """Appends one JSON line to the file named by $GLU_PARITY_REPORT (if set), so a GPU run can
    keep the measured parity figures."""
    path = os.environ.get("GLU_PARITY_REPORT")
    if path:
        import json
        with open(path, "a") as f:
            f.write(json.dumps(record) + "\n")
