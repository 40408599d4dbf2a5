"""Host-side mirror of the reference's numeric-phase interface, backed by the CUDA library.

Reference interface (what a GLU user calls) and its counterpart here:

=====================================================  =============================================
reference                                              this package
=====================================================  =============================================
``Symbolic_Matrix`` (include/symbolic.h:9-51)           :class:`SymbolicMatrix` (same members)
``Symbolic_Matrix::fill_in/csr/leveling``               same methods; the analysis runs in C++
(src/symbolic.cc:11-151)                                (``glu_symbolic_create``), bit-exact
``Symbolic_Matrix::predictLU`` (symbolic.cc:82-103)     :meth:`SymbolicMatrix.predictLU`
``LUonDevice(A_sym, out, err, PERTURB)``                :func:`LUonDevice` / :func:`lu_on_device`
(include/numeric.h:6, src/numeric.cu:339-633)
``Symbolic_Matrix::solve(nicslu, rhs)``                 :meth:`SymbolicMatrix.solve` (GPU solve)
(src/symbolic.cc:200-248)
=====================================================  =============================================

Beyond the reference: :class:`Plan` / :class:`Batch` expose same-pattern batches of value sets,
device value ingest from the original matrix, transposed solves, the gradient over A's nonzeros
and CUDA-graph capture.  Device buffers are torch tensors (plumbing only); every computation runs
in ``libglu_b200.so``.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
from typing import Optional

import numpy as np

from . import _lib
from ._lib import GluError, check, lib  # noqa: F401  (GluError: re-exported)


def _torch():
    import torch
    return torch


def _stream_ptr(stream=None) -> int:
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


# ---------------------------------------------------------------------------------------------
# NICSLU analysis arrays (the part of SNicsLU that the solve and the value ingest read)
# ---------------------------------------------------------------------------------------------

@dataclasses.dataclass
class NicsluArrays:
    """Permutations and MC64 scalings of ``NicsLU_Analyze`` (include/nicslu.h:50-60).

    ``Symbolic_Matrix::solve`` reads ``col_perm``, ``row_perm_inv``, ``col_scale_perm``,
    ``row_scale`` and ``cfgi[1]`` (src/symbolic.cc:203-209); the value ingest also needs the
    inverse maps.
    """
    n: int
    row_perm: np.ndarray
    row_perm_inv: np.ndarray
    col_perm: np.ndarray
    col_perm_inv: np.ndarray
    row_scale: np.ndarray
    col_scale_perm: np.ndarray
    mc64_scale: int = 1

    @classmethod
    def from_npz(cls, path: str) -> "NicsluArrays":
        """Reads arrays saved by the fixture generator (col_perm stored as col_perm - row_perm;
        the inverse permutations are rebuilt)."""
        z = np.load(path)
        n = int(z["n"])
        row_perm = z["row_perm"].astype(np.int64)
        col_perm = row_perm + z["col_perm_delta"] if "col_perm_delta" in z else \
            z["col_perm"].astype(np.int64)
        rpi = np.empty(n, np.int64)
        rpi[row_perm] = np.arange(n)
        cpi = np.empty(n, np.int64)
        cpi[col_perm] = np.arange(n)
        return cls(n, row_perm.astype(np.uint32), rpi.astype(np.uint32), col_perm.astype(np.uint32),
                   cpi.astype(np.uint32), z["row_scale"].astype(np.float64),
                   z["col_scale_perm"].astype(np.float64), int(z["mc64_scale"]))

    def preprocess(self, indptr, indices, data):
        """The matrix NICSLU hands to GLU: ``my_DumpA`` output after MC64 scaling and permutation
        (src/preprocess/preprocess.c:66-79, src/nicslu/source/nicslu_mc64scale.c:38-46).

        Column i of the result is original column ``row_perm[i]``; an entry of original row r
        moves to row ``col_perm_inv[r]`` and is multiplied by
        ``row_scale[c] * col_scale_perm[col_perm_inv[r]]``.  Returns (ap, ai, ax) with uint32
        indices; rows inside a column keep the original entry order.
        """
        n = self.n
        indptr = np.asarray(indptr, np.int64)
        indices = np.asarray(indices, np.int64)
        data = np.asarray(data, np.float64)
        cnt = np.diff(indptr)
        src_col = self.row_perm.astype(np.int64)
        ap = np.zeros(n + 1, np.int64)
        ap[1:] = np.cumsum(cnt[src_col])
        take = np.concatenate([np.arange(indptr[c], indptr[c + 1]) for c in src_col]) \
            if n else np.zeros(0, np.int64)
        col_of = np.repeat(src_col, cnt[src_col])
        k = self.col_perm_inv.astype(np.int64)[indices[take]]
        if self.mc64_scale:
            scale = self.row_scale[col_of] * self.col_scale_perm[k]
            ax = data[take] * scale
        else:
            ax = data[take].copy()
        return ap.astype(np.uint32), k.astype(np.uint32), ax


# ---------------------------------------------------------------------------------------------
# Symbolic_Matrix mirror
# ---------------------------------------------------------------------------------------------

class SymbolicMatrix:
    """Same members as the reference's ``Symbolic_Matrix`` (include/symbolic.h:9-24).

    The analysis itself runs in C++ (``glu_symbolic_create``), whose output is bit-exact with
    ``src/symbolic.cc``; ``fill_in`` runs it, ``csr`` and ``leveling`` publish the CSR mirror and
    the level sets it computed.
    """

    def __init__(self, n: int):
        self.n = int(n)
        self.nnz = 0
        self.num_lev = 0
        self.sym_c_ptr = self.sym_r_idx = self.l_col_ptr = None
        self.csr_r_ptr = self.csr_c_idx = self.csr_diag_ptr = None
        self.level_ptr = self.level_idx = None
        self.val: Optional[np.ndarray] = None
        self._h = None
        self._all = None
        self._device = None     # (Plan, Batch) after LUonDevice

    def __del__(self):
        try:
            if self._h is not None:
                lib().glu_symbolic_destroy(self._h)
        except Exception:
            pass

    def fill_in(self, ai, ap) -> None:
        """Symbolic_Matrix::fill_in(ai, ap) (src/symbolic.cc:11-53)."""
        ai = np.ascontiguousarray(ai, np.uint32)
        ap = np.ascontiguousarray(ap, np.uint32)
        h = C.c_void_p()
        check(lib().glu_symbolic_create(self.n, ap, ai, C.byref(h)), "glu_symbolic_create")
        self._take(h)

    def _take(self, h) -> None:
        """Adopts an analysis handle and copies its arrays out."""
        self._h = h
        nnz = C.c_uint32()
        nl = C.c_int32()
        check(lib().glu_symbolic_sizes(h, C.byref(nnz), C.byref(nl)), "glu_symbolic_sizes")
        n, z, L = self.n, nnz.value, nl.value
        arr = dict(sym_c_ptr=np.empty(n + 1, np.uint32), sym_r_idx=np.empty(z, np.uint32),
                   l_col_ptr=np.empty(n, np.uint32), csr_r_ptr=np.empty(n + 1, np.uint32),
                   csr_c_idx=np.empty(z, np.uint32), csr_diag_ptr=np.empty(n, np.uint32),
                   level_ptr=np.empty(L + 1, np.int32), level_idx=np.empty(n, np.int32))
        check(lib().glu_symbolic_get(h, arr["sym_c_ptr"], arr["sym_r_idx"], arr["l_col_ptr"],
                                     arr["csr_r_ptr"], arr["csr_c_idx"], arr["csr_diag_ptr"],
                                     arr["level_ptr"], arr["level_idx"]), "glu_symbolic_get")
        self._all = (arr, L)
        self.nnz = z
        self.sym_c_ptr, self.sym_r_idx, self.l_col_ptr = (arr["sym_c_ptr"], arr["sym_r_idx"],
                                                          arr["l_col_ptr"])

    def csr(self) -> None:
        """Symbolic_Matrix::csr() (src/symbolic.cc:55-79)."""
        arr, _ = self._all
        self.csr_r_ptr, self.csr_c_idx, self.csr_diag_ptr = (arr["csr_r_ptr"], arr["csr_c_idx"],
                                                             arr["csr_diag_ptr"])

    def predictLU(self, ai, ap, ax) -> None:
        """Symbolic_Matrix::predictLU(ai, ap, ax) (src/symbolic.cc:82-103)."""
        pos = self.positions(ai, ap)
        val = np.zeros(self.nnz, np.float64)
        ok = pos >= 0
        val[pos[ok]] = np.asarray(ax, np.float64)[ok]
        self.val = val

    def positions(self, ai, ap) -> np.ndarray:
        ai = np.ascontiguousarray(ai, np.uint32)
        ap = np.ascontiguousarray(ap, np.uint32)
        pos = np.empty(int(ap[-1]), np.int64)
        check(lib().glu_symbolic_positions(self._h, ap, ai, pos), "glu_symbolic_positions")
        return pos

    def save(self, path: str) -> None:
        """Writes the analysis to a file (``glu_symbolic_save``) so a later run can skip it."""
        if self._h is None:
            raise RuntimeError("save() needs fill_in() first")
        check(lib().glu_symbolic_save(self._h, os.fsencode(path)), "glu_symbolic_save")

    @classmethod
    def load(cls, path: str, ai=None, ap=None, n: Optional[int] = None) -> "SymbolicMatrix":
        """Reads an analysis written by :meth:`save` (``glu_symbolic_load``), with ``csr`` and
        ``leveling`` applied.  Given the pattern (``ai``, ``ap``), checks that the file was made
        from it."""
        if ap is not None:
            ap = np.ascontiguousarray(ap, np.uint32)
            ai = np.ascontiguousarray(ai, np.uint32)
            n = ap.shape[0] - 1
        h = C.c_void_p()
        check(lib().glu_symbolic_load(os.fsencode(path), int(n or 0),
                                      None if ap is None else ap.ctypes.data_as(C.c_void_p),
                                      None if ai is None else ai.ctypes.data_as(C.c_void_p),
                                      C.byref(h)), "glu_symbolic_load")
        order = C.c_uint32()
        check(lib().glu_symbolic_order(h, C.byref(order)), "glu_symbolic_order")
        sm = cls(order.value)
        sm._take(h)
        sm.csr()
        sm.leveling()
        return sm

    def leveling(self) -> None:
        """Symbolic_Matrix::leveling() (src/symbolic.cc:106-151)."""
        arr, L = self._all
        self.num_lev = L
        self.level_ptr, self.level_idx = arr["level_ptr"], arr["level_idx"]

    def analyze(self, ai, ap, ax=None) -> "SymbolicMatrix":
        """fill_in + csr + (predictLU) + leveling, the sequence of lu_cmd.cpp:78-96."""
        self.fill_in(ai, ap)
        self.csr()
        if ax is not None:
            self.predictLU(ai, ap, ax)
        self.leveling()
        return self

    def flops(self) -> float:
        """Algorithmic flops of one refactorization, sum_c |L(:,c)| + 2 |L(:,c)| |U(c,:)|."""
        nl = (np.asarray(self.sym_c_ptr[1:], np.int64) - np.asarray(self.l_col_ptr, np.int64) - 1)
        nu = (np.asarray(self.csr_r_ptr[1:], np.int64) - np.asarray(self.csr_diag_ptr, np.int64)
              - 1)
        return float(np.sum(nl + 2.0 * nl * nu))

    def solve(self, nicslu: NicsluArrays, rhs) -> np.ndarray:
        """Symbolic_Matrix::solve(nicslu, rhs) (src/symbolic.cc:200-248), on the GPU factors left
        by :func:`LUonDevice`."""
        if self._device is None:
            raise RuntimeError("solve() needs LUonDevice() first")
        plan, batch = self._device
        if not plan.has_solve_maps:
            plan.set_solve_maps(nicslu)
        torch = _torch()
        b = torch.as_tensor(np.asarray(rhs, np.float64), device="cuda").reshape(1, 1, self.n)
        x = batch.solve(b)
        return x.reshape(self.n).cpu().numpy()


# ---------------------------------------------------------------------------------------------
# plan / batch
# ---------------------------------------------------------------------------------------------

STAT = dict(n=0, nnz=1, t=2, nt=3, sparse_levels=4, flops=5, plan_bytes=6, slots=7, map_entries=8,
            panel=9, ntp=10, flops_dense=11, lsolve_levels=12, usolve_levels=13, sparse_slots=14,
            hubs=15, dense_updates=16, hub_updates=17, pull_entries=18, fronts=19,
            front_updates=20, front_max=21, unit_levels=22, update_depth=23, gemm_variant=24,
            pull_chunks=25, front_w_max=26)


class Plan:
    """One sparsity pattern on the device (``glu_plan_create``)."""

    def __init__(self, sym: SymbolicMatrix, **options):
        self.sym = sym
        o = _lib.default_options(**options)
        h = C.c_void_p()
        check(lib().glu_plan_create(sym.n, sym.nnz, _u32(sym.sym_c_ptr), _u32(sym.sym_r_idx),
                                    _u32(sym.l_col_ptr), _u32(sym.csr_r_ptr), _u32(sym.csr_c_idx),
                                    _u32(sym.csr_diag_ptr), int(sym.num_lev), _i32(sym.level_ptr),
                                    _i32(sym.level_idx), C.byref(o), C.byref(h)), "glu_plan_create")
        self.h = h
        self.n = sym.n
        self.nnz_a = 0
        self.has_solve_maps = False
        self.grad_pattern = False

    def __del__(self):
        try:
            if self.h:
                lib().glu_plan_destroy(self.h)
                self.h = None
        except Exception:
            pass

    def stat(self, name: str) -> float:
        v = C.c_double()
        check(lib().glu_plan_stat(self.h, STAT[name], C.byref(v)), "glu_plan_stat")
        return v.value

    def stats(self) -> dict:
        return {k: self.stat(k) for k in STAT}

    def autotune(self, values, repeats: int = 1, start: Optional[dict] = None,
                 stream=None) -> tuple:
        """``glu_autotune``: the options (a dict for ``Plan(sym, **opts)``) that refactor the
        instances of ``values`` (float64 CUDA tensor [count, nnz_a], original entry order) fastest,
        and that time in ms.  The plan needs its ingest map."""
        _check_dev(values, (values.shape[0], self.nnz_a))
        o = _lib.default_options(**(start or {}))
        ms = C.c_double()
        check(lib().glu_autotune(self.h, values.shape[0], values.data_ptr(), int(repeats),
                                 C.byref(o), C.byref(ms), _stream_ptr(stream)), "glu_autotune")
        keys = ("dense_threshold", "gemm_variant", "panel", "update_depth", "hub_min_frac",
                "sparse_warps_per_col", "sparse_cols_per_warp", "wide_level_cols",
                "sparse_block", "sparse_persistent", "sparse_col_lanes", "level_warps_per_sm")
        return {k: getattr(o, k) for k in keys}, ms.value

    def set_ingest(self, lu_pos: np.ndarray, scale: Optional[np.ndarray] = None) -> None:
        lu_pos = np.ascontiguousarray(lu_pos, np.int64)
        sc = None if scale is None else np.ascontiguousarray(scale, np.float64)
        check(lib().glu_plan_set_ingest(self.h, lu_pos.shape[0], lu_pos,
                                        None if sc is None else sc.ctypes.data), "glu_plan_set_ingest")
        self._scale_keep = sc
        self.nnz_a = lu_pos.shape[0]

    def set_ingest_from_nicslu(self, indptr, indices, nic: NicsluArrays) -> None:
        ap = np.ascontiguousarray(indptr, np.uint32)
        ai = np.ascontiguousarray(indices, np.uint32)
        rs = np.ascontiguousarray(nic.row_scale, np.float64)
        cs = np.ascontiguousarray(nic.col_scale_perm, np.float64)
        check(lib().glu_plan_ingest_from_nicslu(
            self.h, self.n, ap, ai, _u32(nic.row_perm_inv), _u32(nic.col_perm_inv),
            rs.ctypes.data if nic.mc64_scale else None, cs.ctypes.data if nic.mc64_scale else None),
            "glu_plan_ingest_from_nicslu")
        self.nnz_a = int(ap[-1])

    def set_solve_maps(self, nic: NicsluArrays) -> None:
        cs = np.ascontiguousarray(nic.col_scale_perm, np.float64)
        rs = np.ascontiguousarray(nic.row_scale, np.float64)
        check(lib().glu_plan_set_solve_maps(self.h, _u32(nic.col_perm), _u32(nic.row_perm_inv),
                                            cs.ctypes.data if nic.mc64_scale else None,
                                            rs.ctypes.data if nic.mc64_scale else None),
              "glu_plan_set_solve_maps")
        self.has_solve_maps = True

    def set_original_pattern(self, rows, cols) -> None:
        """Pattern of the user's original matrix (entry e = A(rows[e], cols[e])), for residuals,
        refinement and the gradient over A's nonzeros."""
        r = np.ascontiguousarray(rows, np.uint32)
        c = np.ascontiguousarray(cols, np.uint32)
        check(lib().glu_plan_set_original_pattern(self.h, r.shape[0], r, c),
              "glu_plan_set_original_pattern")
        self.grad_pattern = True
        self._nnz_g = int(r.shape[0])

    def set_original_csc(self, indptr, indices) -> None:
        n = self.n
        cols = np.repeat(np.arange(n, dtype=np.uint32), np.diff(np.asarray(indptr, np.int64)))
        self.set_original_pattern(np.asarray(indices, np.uint32), cols)


class Batch:
    """``count`` value instances of one :class:`Plan`, factored in place on the device."""

    def __init__(self, plan: Plan, count: int, storage=None):
        self.plan = plan
        self.count = int(count)
        h = C.c_void_p()
        self._storage = storage
        if storage is None:
            check(lib().glu_batch_create(plan.h, self.count, C.byref(h)), "glu_batch_create")
        else:
            check(lib().glu_batch_create_external(plan.h, self.count, storage.data_ptr(),
                                                  C.byref(h)), "glu_batch_create_external")
        self.h = h
        self._graph_keep = None

    def __del__(self):
        try:
            if self.h:
                lib().glu_batch_destroy(self.h)
                self.h = None
        except Exception:
            pass

    @staticmethod
    def slots_per_instance(plan: Plan) -> int:
        v = C.c_uint64()
        check(lib().glu_batch_slots_per_instance(plan.h, C.byref(v)), "slots")
        return v.value

    def load_values(self, a, first: int = 0, stream=None) -> None:
        """a: float64 CUDA tensor [count, nnz_a] in the original entry order."""
        _check_dev(a, (a.shape[0], self.plan.nnz_a))
        check(lib().glu_load_values(self.h, first, a.shape[0], a.data_ptr(), _stream_ptr(stream)),
              "glu_load_values")

    def load_lu_values(self, val, first: int = 0, stream=None) -> None:
        """val: float64 CUDA tensor [count, nnz] in Symbolic_Matrix::val layout."""
        _check_dev(val, (val.shape[0], self.plan.sym.nnz))
        check(lib().glu_load_lu_values(self.h, first, val.shape[0], val.data_ptr(),
                                       _stream_ptr(stream)), "glu_load_lu_values")

    def refactor(self, pert: float = 0.0, stream=None) -> None:
        check(lib().glu_refactor(self.h, float(pert), _stream_ptr(stream)), "glu_refactor")

    def refactor_timed(self, pert: float = 0.0, stream=None) -> dict:
        """Refactor with per-launch CUDA events; returns device ms and launches per phase."""
        ms = np.zeros(7, np.float64)
        nl = np.zeros(7, np.int64)
        check(lib().glu_refactor_timed(self.h, float(pert), _stream_ptr(stream), ms, nl),
              "glu_refactor_timed")
        names = ("setup", "sparse", "panel", "update", "to_dense", "fronts", "strips")
        return {n: (float(ms[i]), int(nl[i])) for i, n in enumerate(names)}

    def status(self, stream=None) -> np.ndarray:
        out = np.zeros(self.count, np.int32)
        check(lib().glu_batch_status(self.h, out, _stream_ptr(stream)), "glu_batch_status")
        return out

    def solve(self, B, transpose: bool = False, out=None, stream=None):
        """B: float64 CUDA tensor [count, nrhs, n]; returns X of the same shape."""
        torch = _torch()
        n = self.plan.n
        if B.dim() != 3 or B.shape[0] != self.count or B.shape[2] != n:
            raise ValueError(f"B must be [count={self.count}, nrhs, n={n}]")
        _check_dev(B, tuple(B.shape))
        X = torch.empty_like(B) if out is None else out
        _check_dev(X, tuple(B.shape))
        check(lib().glu_solve(self.h, B.shape[1], B.data_ptr(), X.data_ptr(), 1 if transpose else 0,
                              _stream_ptr(stream)), "glu_solve")
        return X

    def residual(self, a, B, X, transpose: bool = False, stream=None):
        """Relative residuals ||b - op(A) x|| / (||A|| ||x|| + ||b||) per (instance, rhs)."""
        torch = _torch()
        r = torch.empty(B.shape[0] * B.shape[1], dtype=torch.float64, device=B.device)
        check(lib().glu_residual(self.h, B.shape[1], a.data_ptr(), B.data_ptr(), X.data_ptr(),
                                 1 if transpose else 0, r.data_ptr(), _stream_ptr(stream)),
              "glu_residual")
        return r.reshape(B.shape[0], B.shape[1])

    def refine(self, a, B, X, steps: int = 1, transpose: bool = False, with_residual=False,
               stream=None):
        """``steps`` rounds of iterative refinement of X in place; optionally returns the final
        relative residuals."""
        torch = _torch()
        r = torch.empty(B.shape[0] * B.shape[1], dtype=torch.float64, device=B.device) \
            if with_residual else None
        check(lib().glu_refine(self.h, B.shape[1], a.data_ptr(), B.data_ptr(), X.data_ptr(),
                               int(steps), 1 if transpose else 0,
                               r.data_ptr() if r is not None else None, _stream_ptr(stream)),
              "glu_refine")
        return None if r is None else r.reshape(B.shape[0], B.shape[1])

    def grad_a(self, lam, x, out=None, stream=None):
        """-lambda_r * x_c summed over right-hand sides, on the gradient pattern: [count, nnz_g]."""
        torch = _torch()
        nrhs = lam.shape[1]
        ga = out if out is not None else torch.empty((self.count, self._nnz_g()), dtype=torch.float64,
                                                      device=lam.device)
        check(lib().glu_grad_a(self.h, nrhs, lam.data_ptr(), x.data_ptr(), ga.data_ptr(),
                               _stream_ptr(stream)), "glu_grad_a")
        return ga

    def _nnz_g(self) -> int:
        return self.plan._nnz_g

    def get_lu(self, instance: int = 0, stream=None):
        torch = _torch()
        v = torch.empty(self.plan.sym.nnz, dtype=torch.float64, device="cuda")
        check(lib().glu_get_lu(self.h, instance, v.data_ptr(), _stream_ptr(stream)), "glu_get_lu")
        return v

    def capture(self, a, B=None, X=None, pert: float = 0.0, refine: int = 0, stream=None) -> None:
        """Captures load_values + refactor (+ solve, + ``refine`` refinement rounds) for the whole
        batch in one CUDA graph."""
        nrhs = 0 if B is None else B.shape[1]
        s = _stream_ptr(stream)
        check(lib().glu_graph_capture(self.h, a.data_ptr(), nrhs, 0 if B is None else B.data_ptr(),
                                      0 if X is None else X.data_ptr(), float(pert), int(refine),
                                      s), "glu_graph_capture")
        self._graph_keep = (a, B, X)

    def replay(self, stream=None) -> None:
        check(lib().glu_graph_launch(self.h, _stream_ptr(stream)), "glu_graph_launch")

    @property
    def launches(self) -> int:
        v = C.c_int64()
        check(lib().glu_batch_launch_count(self.h, C.byref(v)), "launch count")
        return v.value


class Group:
    """Batches of several patterns (uneven sizes) captured in ONE CUDA graph, one branch each."""

    def __init__(self, batches, values, Bs=None, Xs=None, pert: float = 0.0, refine: int = 0,
                 stream=None):
        nb = len(batches)
        VP = C.c_void_p * nb
        self.batches = list(batches)
        self._keep = (values, Bs, Xs)
        nrhs = (C.c_int32 * nb)(*[0 if Bs is None or Bs[i] is None else Bs[i].shape[1]
                                  for i in range(nb)])
        bp = VP(*[b.h.value if isinstance(b.h, C.c_void_p) else b.h for b in batches])
        ap = VP(*[v.data_ptr() for v in values])
        Bp = VP(*[0 if Bs is None or Bs[i] is None else Bs[i].data_ptr() for i in range(nb)])
        Xp = VP(*[0 if Xs is None or Xs[i] is None else Xs[i].data_ptr() for i in range(nb)])
        h = C.c_void_p()
        check(lib().glu_group_capture(nb, bp, ap, nrhs, Bp, Xp, float(pert), int(refine),
                                      _stream_ptr(stream), C.byref(h)), "glu_group_capture")
        self.h = h

    def launch(self, stream=None) -> None:
        check(lib().glu_group_launch(self.h, _stream_ptr(stream)), "glu_group_launch")

    @property
    def launches(self) -> int:
        v = C.c_int64()
        check(lib().glu_group_launch_count(self.h, C.byref(v)), "group launch count")
        return v.value

    def __del__(self):
        try:
            if self.h:
                lib().glu_group_destroy(self.h)
                self.h = None
        except Exception:
            pass


# ---------------------------------------------------------------------------------------------
# LUonDevice
# ---------------------------------------------------------------------------------------------

def lu_on_device(A_sym: SymbolicMatrix, perturb: bool = False, **options) -> None:
    """The work of ``LUonDevice(A_sym, out, err, PERTURB)`` (src/numeric.cu:339-633).

    Factors ``A_sym.val`` in place on the GPU: on return it holds L (unit, strictly below
    ``l_col_ptr``) and U (with the diagonal).  With ``perturb`` the static-pivot perturbation
    3.45e-4 * ||A||_1 is applied (src/numeric.cu:405-421).  The device factors stay attached to
    ``A_sym`` for :meth:`SymbolicMatrix.solve`.
    """
    torch = _torch()
    plan = Plan(A_sym, **options)
    batch = Batch(plan, 1)
    val = torch.as_tensor(np.asarray(A_sym.val, np.float64), device="cuda").reshape(1, -1)
    batch.load_lu_values(val)
    batch.refactor(-1.0 if perturb else 0.0)
    A_sym.val = batch.get_lu(0).cpu().numpy()
    A_sym._device = (plan, batch)
    return None


LUonDevice = lu_on_device


def _u32(a):
    return np.ascontiguousarray(a, np.uint32)


def _i32(a):
    return np.ascontiguousarray(a, np.int32)


def _check_dev(t, shape):
    torch = _torch()
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda" or t.dtype != torch.float64:
        raise TypeError("expected a float64 CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    if tuple(t.shape) != tuple(shape):
        raise ValueError(f"shape {tuple(t.shape)} != {tuple(shape)}")
