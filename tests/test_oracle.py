"""The oracle pinned against the reference's own code run here (oracle/_ref) and against
known answers.  CPU only.

* Symbolic_Matrix::solve (reference, REAL=double) and the oracle's solve agree bit for bit.
* The oracle's factors reproduce the preprocessed matrix: L*U == A_hat (the reference's own
  GLU_DEBUG check is a column checksum of the same identity, src/symbolic.cc:163-197).
* Known answer b = A*1 -> residual <= 1e-12 and x ~ 1.
* The oracle's L/U equal a dense no-pivot LU of A_hat (n = 200), since LU without pivoting is
  unique.
* The transposed solve equals a dense solve with A^T.
"""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle as O
from tests.common import case, column_rel_err, have_add32

CASES = ["mna:200,3", "mna:2000,5", "grid:24,4"] + (["add32"] if have_add32() else [])


def _lu_split(sym, val):
    n = sym.n
    cp = np.asarray(sym.sym_c_ptr, np.int64)
    ri = np.asarray(sym.sym_r_idx, np.int64)
    col = np.repeat(np.arange(n), np.diff(cp))
    low = ri > col
    L = sp.csc_matrix((val[low], (ri[low], col[low])), shape=(n, n)) + sp.identity(n, format="csc")
    up = ~low
    U = sp.csc_matrix((val[up], (ri[up], col[up])), shape=(n, n))
    return L, U


@pytest.mark.parametrize("name", CASES)
def test_oracle_solve_bit_exact_with_reference_solve(name):
    cs = case(name)
    lu, st = O.factor(cs.sym_ref, cs.sym_ref.val)
    assert st == 0
    c = cs.circuit
    b = c.to_scipy() @ np.ones(c.n)
    x_ref = cs.ref.solve(lu, b)
    x = O.solve(cs.sym_ref, lu, cs.pre, b)
    assert np.array_equal(x, x_ref)
    assert O.residual(c.n, c.indptr, c.indices, c.data, x, b) <= 1e-12


@pytest.mark.parametrize("name", CASES)
def test_oracle_factors_reproduce_preprocessed_matrix(name):
    cs = case(name)
    lu, _ = O.factor(cs.sym_ref, cs.sym_ref.val)
    L, U = _lu_split(cs.sym_ref, lu)
    Ahat = sp.csc_matrix((cs.pre.ax, cs.pre.ai, cs.pre.ap), shape=(cs.n, cs.n))
    R = (L @ U - Ahat).toarray() if cs.n <= 2000 else None
    if R is not None:
        scale = np.abs(L).toarray() @ np.abs(U).toarray()
        assert np.max(np.abs(R) / np.maximum(scale, 1e-300)) <= 1e-13
    # column checksums (the reference's ABFT identity): 1^T (L U) == 1^T A_hat
    cca = np.asarray(Ahat.sum(axis=0)).ravel()
    ccl = np.asarray((np.ones(cs.n) @ L) @ U).ravel()
    den = np.asarray(abs(L).sum(axis=0) @ abs(U)).ravel()
    assert np.max(np.abs(ccl - cca) / np.maximum(den, 1e-300)) <= 1e-12


@pytest.mark.parametrize("name", ["mna:2000,5", "grid:24,4"])
def test_oracle_other_orders_are_valid_factorizations(name):
    """The orders tests.common.order_sensitivity compares against -- each level's columns
    reversed (an order the reference's atomic updates allow), fused multiply-adds -- still give
    factors whose product is the preprocessed matrix; the threaded oracle is bit-identical."""
    cs = case(name)
    base, _ = O.factor(cs.sym_ref, cs.sym_ref.val)
    assert np.array_equal(base, O.factor(cs.sym_ref, cs.sym_ref.val, threads=4)[0])
    Ahat = sp.csc_matrix((cs.pre.ax, cs.pre.ai, cs.pre.ap), shape=(cs.n, cs.n)).toarray()
    for kw in (dict(reverse_levels=True), dict(reverse_levels=True, fma=True)):
        lu, st = O.factor(cs.sym_ref, cs.sym_ref.val, **kw)
        assert st == 0
        L, U = _lu_split(cs.sym_ref, lu)
        L, U = L.toarray(), U.toarray()
        scale = np.abs(L) @ np.abs(U)
        assert np.max(np.abs(L @ U - Ahat) / np.maximum(scale, 1e-300)) <= 1e-13
        assert column_rel_err(cs.sym, lu, base) <= 1e-9


def test_oracle_matches_dense_lu_without_pivoting():
    cs = case("mna:200,3")
    n = cs.n
    A = sp.csc_matrix((cs.pre.ax, cs.pre.ai, cs.pre.ap), shape=(n, n)).toarray()
    for k in range(n):                      # textbook right-looking LU, no pivoting
        A[k + 1:, k] /= A[k, k]
        A[k + 1:, k + 1:] -= np.outer(A[k + 1:, k], A[k, k + 1:])
    lu, _ = O.factor(cs.sym_ref, cs.sym_ref.val)
    cp = np.asarray(cs.sym_ref.sym_c_ptr, np.int64)
    col = np.repeat(np.arange(n), np.diff(cp))
    dense_at_pattern = A[np.asarray(cs.sym_ref.sym_r_idx, np.int64), col]
    assert column_rel_err(cs.sym, lu, dense_at_pattern) <= 1e-12
    # and the fill pattern holds every nonzero of the dense factors
    mask = np.zeros((n, n), bool)
    mask[np.asarray(cs.sym_ref.sym_r_idx, np.int64), col] = True
    assert np.all(np.abs(A[~mask]) == 0.0)


@pytest.mark.parametrize("name", ["mna:200,3", "grid:24,4"])
def test_oracle_transpose_solve_matches_dense(name):
    cs = case(name)
    c = cs.circuit
    lu, _ = O.factor(cs.sym_ref, cs.sym_ref.val)
    g = np.random.default_rng(1).standard_normal(c.n)
    lam = O.solve_transpose(cs.sym_ref, lu, cs.pre, g)
    ref = np.linalg.solve(c.to_scipy().toarray().T, g)
    assert np.max(np.abs(lam - ref)) <= 1e-8 * np.max(np.abs(ref))
    AT = c.to_scipy().T.tocsc()
    assert O.residual(c.n, AT.indptr.astype(np.int64), AT.indices, AT.data, lam, g) <= 1e-12


def test_oracle_perturbation_only_on_columns_with_l_part():
    from glu_public_b200 import glu
    cs = case("mna:200,3")
    val = cs.sym_ref.val
    pert = O.perturbation(cs.sym_ref, val)
    assert pert == pytest.approx(3.45e-4 * max(
        np.abs(val[cs.sym_ref.sym_c_ptr[j]:cs.sym_ref.sym_c_ptr[j + 1]]).sum() for j in range(cs.n)))
    # 2x2 known answer: [[1e-9, 0], [2, 1e-9]].  Column 0 has an L part and its tiny pivot is
    # clamped to pert; column 1 has none and, as numeric.cu clamps inside the L loop, is not.
    ap = np.array([0, 2, 3], np.uint32)
    ai = np.array([0, 1, 1], np.uint32)
    ax = np.array([1e-9, 2.0, 1e-9])
    s = glu.SymbolicMatrix(2).analyze(ai, ap, ax)
    lu, _ = O.factor(s, s.val, 1e-3)
    assert list(lu) == [1e-3, 2.0 / 1e-3, 1e-9]


def test_flop_count_matches_definition():
    cs = case("mna:200,3")
    s = cs.sym_ref
    f = 0.0
    for c in range(s.n):
        nl = s.sym_c_ptr[c + 1] - s.l_col_ptr[c] - 1
        nu = s.csr_r_ptr[c + 1] - s.csr_diag_ptr[c] - 1
        f += nl + 2.0 * nl * nu
    assert O.flops(s) == f


def _write(path, banner, size, rows):
    with open(path, "w") as f:
        f.write(banner + "\n% comment\n" + size + "\n" + "".join(r + "\n" for r in rows))


def test_matrixmarket_reader_variants(tmp_path):
    """Any entry order, duplicates summed, pattern / integer fields, symmetric and
    skew-symmetric storage mirrored; unsupported files rejected."""
    from glu_public_b200 import gen
    p = tmp_path / "g.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real general", "3 3 5",
           ["3 1 2.5", "1 1 4", "2 3 -1", "1 1 1", "2 2 7"])
    a = gen.read_mtx(p).toarray()
    assert np.array_equal(a, [[5, 0, 0], [0, 7, -1], [2.5, 0, 0]])
    p = tmp_path / "s.mtx"
    _write(p, "%%MatrixMarket matrix coordinate integer symmetric", "3 3 3",
           ["2 1 3", "1 1 1", "3 2 -2"])
    assert np.array_equal(gen.read_mtx(p).toarray(), [[1, 3, 0], [3, 0, -2], [0, -2, 0]])
    p = tmp_path / "k.mtx"
    _write(p, "%%MatrixMarket matrix coordinate real skew-symmetric", "2 2 1", ["2 1 4"])
    assert np.array_equal(gen.read_mtx(p).toarray(), [[0, -4], [4, 0]])
    p = tmp_path / "p.mtx"
    _write(p, "%%MatrixMarket matrix coordinate pattern general", "2 2 2", ["1 2", "2 1"])
    assert np.array_equal(gen.read_mtx(p).toarray(), [[0, 1], [1, 0]])
    for banner in ("%%MatrixMarket matrix coordinate complex general",
                   "%%MatrixMarket matrix array real general",
                   "%%MatrixMarket matrix coordinate real hermitian"):
        p = tmp_path / "bad.mtx"
        _write(p, banner, "1 1 1", ["1 1 1"])
        with pytest.raises(ValueError):
            gen.read_mtx(p)


def test_matrixmarket_round_trip_and_cache(tmp_path):
    from glu_public_b200 import gen
    c = gen.mna_netlist(300, 4)
    p = tmp_path / "c.mtx"
    gen.write_mtx(p, c)
    a = gen.read_mtx(p, cache=True)
    assert (a != c.to_scipy()).nnz == 0
    assert (tmp_path / "c.mtx.csc.npz").exists()
    b = gen.read_mtx(p, cache=True)               # now from the binary copy
    assert (b != a).nnz == 0 and np.array_equal(b.indptr, a.indptr)
