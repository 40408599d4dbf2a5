"""The C-ABI library loads and exports every entry point include/glu_b200.h declares; host-side
validation rejects malformed plans before any device work.  CPU only (no compute calls)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from glu_public_b200 import _lib, glu
from tests.common import ROOT, case


def _declared():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", fn)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(glu_[a-z0-9_]+)\s*\(", txt)
    return sorted(set(names))


def test_library_exports_every_declared_symbol(built_lib):
    lib = C.CDLL(_lib.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert sorted(_lib.EXPORTS) == sorted(n for n in declared if n in _lib.EXPORTS)
    assert set(_lib.EXPORTS) == set(declared)


def test_status_strings(built_lib):
    L = _lib.lib()
    assert L.glu_status_string(0) == b"ok"
    assert L.glu_status_string(-6) == b"numerically singular matrix"


def _plan_args(s):
    return [s.n, s.nnz, glu._u32(s.sym_c_ptr), glu._u32(s.sym_r_idx), glu._u32(s.l_col_ptr),
            glu._u32(s.csr_r_ptr), glu._u32(s.csr_c_idx), glu._u32(s.csr_diag_ptr),
            int(s.num_lev), glu._i32(s.level_ptr), glu._i32(s.level_idx)]


@pytest.mark.parametrize("corrupt,code", [
    ("level_order", -7), ("csr", -7), ("diag", -5), ("rows_unsorted", -7),
])
def test_plan_rejects_malformed_symbolic_arrays(built_lib, corrupt, code):
    cs = case("mna:200,3")
    args = _plan_args(cs.sym)
    args = [a.copy() if isinstance(a, np.ndarray) else a for a in args]
    if corrupt == "level_order":
        args[10] = args[10][::-1].copy()                  # dependencies now point forward
    elif corrupt == "csr":
        args[6][5] = (args[6][5] + 1) % cs.n
    elif corrupt == "diag":
        args[4][7] = args[4][7] + 1 if args[4][7] + 1 < args[2][8] else args[4][7] - 1
    elif corrupt == "rows_unsorted":
        j = int(np.argmax(np.diff(args[2]) > 2))
        p = int(args[2][j])
        args[3][p], args[3][p + 1] = args[3][p + 1], args[3][p]
    o = _lib.default_options()
    h = C.c_void_p()
    st = _lib.lib().glu_plan_create(*args, C.byref(o), C.byref(h))
    assert st == code, (_lib.lib().glu_last_error(), st)
    assert not h.value
