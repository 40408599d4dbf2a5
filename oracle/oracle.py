"""ctypes access to the oracle: the reference's own CPU pipeline (``_ref/libglu_ref.so``) and the
C restatement of the GLU numeric phase (``liboracle.so``).

TEST INFRASTRUCTURE ONLY.  Imported by ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py``, as the checker; the product package never imports it.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libglu_ref.so")
ORACLE_SO = os.path.join(HERE, "liboracle.so")
ORACLE_FMA_SO = os.path.join(HERE, "liboracle_fma.so")

_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")

_oracle = None
_oracle_fma = None
_ref = None


def have_ref() -> bool:
    return os.path.exists(REF_SO)


def oracle_lib(fma: bool = False):
    global _oracle, _oracle_fma
    if fma:
        if _oracle_fma is None:
            _oracle_fma = _bind(C.CDLL(ORACLE_FMA_SO))
        return _oracle_fma
    if _oracle is None:
        _oracle = _bind(C.CDLL(ORACLE_SO))
    return _oracle


def _bind(lib):
    lib.oracle_factor.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p,
                                  C.c_int, _i32p, _i32p, _f64p, C.c_double]
    lib.oracle_factor.restype = C.c_int
    lib.oracle_factor_mt.argtypes = lib.oracle_factor.argtypes + [C.c_int]
    lib.oracle_factor_mt.restype = C.c_int
    lib.oracle_perturbation.argtypes = [C.c_uint32, _u32p, _f64p]
    lib.oracle_perturbation.restype = C.c_double
    lib.oracle_solve.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _f64p, _u32p, _u32p,
                                 _f64p, _f64p, C.c_int, _f64p, _f64p]
    lib.oracle_solve.restype = None
    lib.oracle_solve_transpose.argtypes = lib.oracle_solve.argtypes
    lib.oracle_solve_transpose.restype = None
    lib.oracle_residual.argtypes = [C.c_uint32, _i64p, _i32p, _f64p, _f64p, _f64p]
    lib.oracle_residual.restype = C.c_double
    lib.oracle_flops.argtypes = [C.c_uint32, _u32p, _u32p, _u32p, _u32p]
    lib.oracle_flops.restype = C.c_double
    return lib


def ref_lib():
    global _ref
    if _ref is None:
        lib = C.CDLL(REF_SO)
        lib.ref_open.argtypes = [C.c_char_p, C.c_int]
        lib.ref_open.restype = C.c_void_p
        vp = C.c_void_p
        up = C.POINTER(C.c_uint32)
        lib.ref_dims.argtypes = [vp, up, up]
        lib.ref_get_preprocessed.argtypes = [vp, _f64p, _u32p, _u32p]
        lib.ref_get_perm.argtypes = [vp, _u32p, _u32p, _u32p, _u32p, _f64p, _f64p, up]
        lib.ref_symbolic.argtypes = [vp, up, C.POINTER(C.c_int)]
        lib.ref_sym_get.argtypes = [vp, _u32p, _u32p, _u32p, _u32p, _u32p, _u32p, _i32p, _i32p,
                                    _f64p]
        lib.ref_sym_set_val.argtypes = [vp, _f64p]
        lib.ref_solve.argtypes = [vp, _f64p, _f64p]
        lib.ref_nicslu_factorize.argtypes = [vp]
        lib.ref_nicslu_create_threads.argtypes = [vp, C.c_uint]
        lib.ref_nicslu_refactorize.argtypes = [vp, _f64p, C.c_int]
        lib.ref_nicslu_solve.argtypes = [vp, _f64p]
        lib.ref_nicslu_stat.argtypes = [vp, C.c_int]
        lib.ref_nicslu_stat.restype = C.c_double
        lib.ref_nicslu_lu_nnz.argtypes = [vp]
        lib.ref_nicslu_lu_nnz.restype = C.c_size_t
        lib.ref_close.argtypes = [vp]
        lib.ref_close.restype = None
        _ref = lib
    return _ref


@dataclasses.dataclass
class Preprocessed:
    """Output of the reference's ``preprocess()`` (NICSLU MC64 + AMD, then ``my_DumpA``)."""
    n: int
    ap: np.ndarray   # uint32 [n+1]
    ai: np.ndarray   # uint32 [nnz]
    ax: np.ndarray   # float64 [nnz]
    row_perm: np.ndarray
    row_perm_inv: np.ndarray
    col_perm: np.ndarray
    col_perm_inv: np.ndarray
    row_scale: np.ndarray
    col_scale_perm: np.ndarray
    mc64_scale: int


@dataclasses.dataclass
class RefSymbolic:
    """``Symbolic_Matrix`` members after fill_in/csr/predictLU/leveling (include/symbolic.h)."""
    n: int
    nnz: int
    num_lev: int
    sym_c_ptr: np.ndarray
    sym_r_idx: np.ndarray
    l_col_ptr: np.ndarray
    csr_r_ptr: np.ndarray
    csr_c_idx: np.ndarray
    csr_diag_ptr: np.ndarray
    level_ptr: np.ndarray
    level_idx: np.ndarray
    val: np.ndarray


class RefPipeline:
    """The reference's CPU pipeline on one MatrixMarket file (lu_cmd.cpp:64-111 minus the GPU)."""

    def __init__(self, mtx_path: str, quiet: bool = True):
        self.lib = ref_lib()
        self.h = self.lib.ref_open(mtx_path.encode(), 1 if quiet else 0)
        if not self.h:
            raise RuntimeError(f"reference preprocess() failed on {mtx_path}")
        n = C.c_uint32()
        nnz = C.c_uint32()
        self.lib.ref_dims(self.h, C.byref(n), C.byref(nnz))
        self.n, self.nnz_a = n.value, nnz.value
        self.sym: RefSymbolic | None = None

    @classmethod
    def from_csc(cls, n: int, indptr, indices, data, quiet: bool = True) -> "RefPipeline":
        """Writes a column-sorted MatrixMarket file and runs preprocess() on it."""
        fd, path = tempfile.mkstemp(suffix=".mtx")
        os.close(fd)
        try:
            write_mtx_arrays(path, n, indptr, indices, data)
            return cls(path, quiet)
        finally:
            os.unlink(path)

    def preprocessed(self) -> Preprocessed:
        n, nnz = self.n, self.nnz_a
        ax = np.empty(nnz, np.float64)
        ai = np.empty(nnz, np.uint32)
        ap = np.empty(n + 1, np.uint32)
        self.lib.ref_get_preprocessed(self.h, ax, ai, ap)
        arr = [np.empty(n, np.uint32) for _ in range(4)]
        rs = np.empty(n, np.float64)
        cs = np.empty(n, np.float64)
        mc = C.c_uint32()
        self.lib.ref_get_perm(self.h, arr[0], arr[1], arr[2], arr[3], rs, cs, C.byref(mc))
        return Preprocessed(n, ap, ai, ax, arr[0], arr[1], arr[2], arr[3], rs, cs, mc.value)

    def symbolic(self) -> RefSymbolic:
        nnz = C.c_uint32()
        nl = C.c_int()
        self.lib.ref_symbolic(self.h, C.byref(nnz), C.byref(nl))
        n, z, L = self.n, nnz.value, nl.value
        s = RefSymbolic(n, z, L, np.empty(n + 1, np.uint32), np.empty(z, np.uint32),
                        np.empty(n, np.uint32), np.empty(n + 1, np.uint32), np.empty(z, np.uint32),
                        np.empty(n, np.uint32), np.empty(L + 1, np.int32), np.empty(n, np.int32),
                        np.empty(z, np.float64))
        self.lib.ref_sym_get(self.h, s.sym_c_ptr, s.sym_r_idx, s.l_col_ptr, s.csr_r_ptr,
                             s.csr_c_idx, s.csr_diag_ptr, s.level_ptr, s.level_idx, s.val)
        self.sym = s
        return s

    def solve(self, lu_val: np.ndarray, rhs: np.ndarray) -> np.ndarray:
        """Symbolic_Matrix::solve on the given factored values."""
        self.lib.ref_sym_set_val(self.h, np.ascontiguousarray(lu_val, np.float64))
        x = np.empty(self.n, np.float64)
        self.lib.ref_solve(self.h, np.ascontiguousarray(rhs, np.float64), x)
        return x

    # NICSLU's CPU LU (baseline)
    def nicslu_factorize(self) -> int:
        return self.lib.ref_nicslu_factorize(self.h)

    def nicslu_create_threads(self, threads: int) -> int:
        return self.lib.ref_nicslu_create_threads(self.h, threads)

    def nicslu_refactorize(self, ax_orig: np.ndarray, multithreaded: bool) -> int:
        return self.lib.ref_nicslu_refactorize(self.h, np.ascontiguousarray(ax_orig, np.float64),
                                               1 if multithreaded else 0)

    def nicslu_solve(self, rhs: np.ndarray) -> np.ndarray:
        x = np.array(rhs, dtype=np.float64, copy=True)
        self.lib.ref_nicslu_solve(self.h, x)
        return x

    def close(self):
        if self.h:
            self.lib.ref_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def write_mtx_arrays(path: str, n: int, indptr, indices, data) -> None:
    indptr = np.asarray(indptr, np.int64)
    col = np.repeat(np.arange(n), np.diff(indptr))
    arr = np.empty(indptr[-1], dtype=[("r", np.int64), ("c", np.int64), ("v", np.float64)])
    arr["r"] = np.asarray(indices, np.int64) + 1
    arr["c"] = col + 1
    arr["v"] = data
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{n} {n} {int(indptr[-1])}\n")
        np.savetxt(f, arr, fmt="%d %d %.17g")


# ---- C restatement ----

def factor(sym, val: np.ndarray, pert: float = 0.0, fma: bool = False,
           threads: int = 1, reverse_levels: bool = False) -> tuple[np.ndarray, int]:
    """Right-looking level-ordered LU of ``val`` (copied) on the symbolic arrays of ``sym``.
    ``fma=True`` uses the build with fused multiply-adds (a second valid rounding order).
    ``reverse_levels=True`` takes the columns of every level in reverse order: another order the
    reference's own kernels can take (its updates into a shared target are atomicAdds,
    src/numeric.cu:78-83, so the order of a level's columns is not fixed), which changes the
    order in which a target sums its updates.  ``threads > 1`` updates the sub-columns of each
    pivot column concurrently (bit-identical result); ``threads=0`` uses every core."""
    if threads <= 0:
        threads = os.cpu_count() or 1
    level_idx = _i32(sym.level_idx)
    if reverse_levels:
        lp = np.asarray(sym.level_ptr, np.int64)
        level_idx = level_idx.copy()
        for lv in range(len(lp) - 1):
            level_idx[lp[lv]:lp[lv + 1]] = level_idx[lp[lv]:lp[lv + 1]][::-1].copy()
    v = np.array(val, dtype=np.float64, copy=True)
    st = oracle_lib(fma).oracle_factor_mt(sym.n, _u32(sym.sym_c_ptr), _u32(sym.sym_r_idx),
                                       _u32(sym.l_col_ptr), _u32(sym.csr_r_ptr),
                                       _u32(sym.csr_c_idx), _u32(sym.csr_diag_ptr),
                                       int(sym.num_lev), _i32(sym.level_ptr), level_idx,
                                       v, float(pert), int(threads))
    return v, st


def perturbation(sym, val: np.ndarray) -> float:
    return oracle_lib().oracle_perturbation(sym.n, _u32(sym.sym_c_ptr), _f64(val))


def solve(sym, lu_val, pre: Preprocessed, rhs) -> np.ndarray:
    x = np.empty(sym.n, np.float64)
    oracle_lib().oracle_solve(sym.n, _u32(sym.sym_c_ptr), _u32(sym.sym_r_idx),
                              _u32(sym.l_col_ptr), _f64(lu_val), _u32(pre.col_perm),
                              _u32(pre.row_perm_inv), _f64(pre.col_scale_perm),
                              _f64(pre.row_scale), int(pre.mc64_scale), _f64(rhs), x)
    return x


def solve_transpose(sym, lu_val, pre: Preprocessed, g) -> np.ndarray:
    lam = np.empty(sym.n, np.float64)
    oracle_lib().oracle_solve_transpose(sym.n, _u32(sym.sym_c_ptr), _u32(sym.sym_r_idx),
                                        _u32(sym.l_col_ptr), _f64(lu_val), _u32(pre.col_perm),
                                        _u32(pre.row_perm), _f64(pre.col_scale_perm),
                                        _f64(pre.row_scale), int(pre.mc64_scale), _f64(g), lam)
    return lam


def residual(n: int, indptr, indices, data, x, b) -> float:
    return oracle_lib().oracle_residual(n, np.ascontiguousarray(indptr, np.int64),
                                        np.ascontiguousarray(indices, np.int32), _f64(data),
                                        _f64(x), _f64(b))


def flops(sym) -> float:
    return oracle_lib().oracle_flops(sym.n, _u32(sym.sym_c_ptr), _u32(sym.l_col_ptr),
                                     _u32(sym.csr_r_ptr), _u32(sym.csr_diag_ptr))


def _u32(a):
    return np.ascontiguousarray(a, np.uint32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def _f64(a):
    return np.ascontiguousarray(a, np.float64)
