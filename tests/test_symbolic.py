"""The product's fast symbolic analysis is bit-exact with the reference's symbolic.cc.  CPU only.

Small and medium patterns are compared array by array with symbolic.cc run here (oracle/_ref);
the benchmark-size patterns are compared through the SHA-256 digests that
tests/golden/make_fixtures.py recorded from symbolic.cc (running symbolic.cc itself there takes
about a minute per pattern)."""
import json
import os

import numpy as np
import pytest

from glu_public_b200 import gen, glu
from tests.common import GOLDEN, case, have_add32

ARRAYS = ["sym_c_ptr", "sym_r_idx", "l_col_ptr", "csr_r_ptr", "csr_c_idx", "csr_diag_ptr",
          "level_ptr", "level_idx", "val"]


@pytest.mark.parametrize("name", ["mna:200,3", "mna:2000,5", "mna:4960,1", "mna:3000,9",
                                  "grid:24,4", "grid:48,2"] + (["add32"] if have_add32() else []))
def test_symbolic_bit_exact_with_reference(name):
    cs = case(name)
    assert cs.sym.nnz == cs.sym_ref.nnz
    assert cs.sym.num_lev == cs.sym_ref.num_lev
    for a in ARRAYS:
        mine, ref = getattr(cs.sym, a), getattr(cs.sym_ref, a)
        assert mine.shape == ref.shape and np.array_equal(mine, ref), a


def _digest(a):
    import hashlib
    h = hashlib.sha256()
    a = np.ascontiguousarray(a)
    h.update(str(a.dtype).encode())
    h.update(str(a.shape).encode())
    h.update(a.tobytes())
    return h.hexdigest()


GOLDEN_PATTERNS = {
    "mna2000_s3": lambda: gen.mna_netlist(2000, 3),
    "mna4960_s0": lambda: gen.mna_netlist(4960, 0),
    "mna20000_s2": lambda: gen.mna_netlist(20000, 2),
    "grid128_s1": lambda: gen.power_grid(128, 1),
    "grid512_s1": lambda: gen.power_grid(512, 1),
}


@pytest.mark.parametrize("name", list(GOLDEN_PATTERNS))
def test_symbolic_matches_golden_digests(name):
    golden = json.load(open(os.path.join(GOLDEN, "symbolic_golden.json")))
    npz = os.path.join(GOLDEN, f"nicslu_{name}.npz")
    if name not in golden or not os.path.exists(npz):
        pytest.skip("fixture not generated")
    g = golden[name]
    c = GOLDEN_PATTERNS[name]()
    nic = glu.NicsluArrays.from_npz(npz)
    ap, ai, ax = nic.preprocess(c.indptr, c.indices, c.data)
    s = glu.SymbolicMatrix(c.n).analyze(ai, ap, ax)
    assert s.nnz == g["nnz_lu"] and s.num_lev == g["num_lev"]
    for a in ARRAYS:
        assert _digest(getattr(s, a)) == g[a], a


def test_structurally_missing_diagonal_is_rejected():
    from glu_public_b200._lib import GluError
    n = 4
    ap = np.array([0, 1, 2, 3, 4], np.uint32)
    ai = np.array([1, 0, 2, 3], np.uint32)     # columns 0, 1 have no diagonal
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix(n).analyze(ai, ap)
    assert e.value.status == -5


def test_positions_follow_predictlu_first_match():
    n = 3
    ap = np.array([0, 3, 4, 5], np.uint32)
    ai = np.array([0, 2, 0, 1, 2], np.uint32)   # (0,0) appears twice in column 0
    s = glu.SymbolicMatrix(n).analyze(ai, ap)
    pos = s.positions(ai, ap)
    assert pos[0] >= 0 and pos[2] == -1 and pos[1] >= 0


def _pattern(name):
    cs = case(name)
    return cs, np.ascontiguousarray(cs.pre.ai, np.uint32), np.ascontiguousarray(cs.pre.ap, np.uint32)


@pytest.mark.parametrize("name", ["mna:2000,5", "grid:24,4"])
def test_symbolic_save_load_round_trip(name, tmp_path):
    """A saved analysis loads back array for array, checked against the pattern it came from,
    and gives the same entry positions (the ingest map)."""
    cs, ai, ap = _pattern(name)
    s = glu.SymbolicMatrix(cs.n).analyze(ai, ap)
    path = str(tmp_path / "sym.bin")
    s.save(path)
    t = glu.SymbolicMatrix.load(path, ai, ap)
    assert t.n == s.n and t.nnz == s.nnz and t.num_lev == s.num_lev
    for a in ARRAYS[:-1]:
        assert np.array_equal(getattr(t, a), getattr(s, a)), a
    assert np.array_equal(t.positions(ai, ap), s.positions(ai, ap))
    u = glu.SymbolicMatrix.load(path)              # without the pattern: no pattern check
    assert np.array_equal(u.sym_r_idx, s.sym_r_idx)


def test_symbolic_load_rejects_other_patterns_and_damaged_files(tmp_path):
    from glu_public_b200._lib import GluError
    cs, ai, ap = _pattern("mna:200,3")
    s = glu.SymbolicMatrix(cs.n).analyze(ai, ap)
    path = tmp_path / "sym.bin"
    s.save(str(path))
    other, ai2, ap2 = _pattern("mna:2000,5")
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix.load(str(path), ai2, ap2)
    assert e.value.status == -7
    # the same pattern with two entries of a column swapped is another entry order
    ai3 = ai.copy()
    j = int(np.argmax(np.diff(ap) > 1))
    ai3[ap[j]], ai3[ap[j] + 1] = ai3[ap[j] + 1], ai3[ap[j]]
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix.load(str(path), ai3, ap)
    assert e.value.status == -7
    raw = bytearray(path.read_bytes())
    damaged = tmp_path / "damaged.bin"
    raw[len(raw) // 2] ^= 0x40
    damaged.write_bytes(bytes(raw))
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix.load(str(damaged), ai, ap)
    assert e.value.status == -7
    short = tmp_path / "short.bin"
    short.write_bytes(path.read_bytes()[:-12])
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix.load(str(short), ai, ap)
    assert e.value.status == -7
    with pytest.raises(GluError) as e:
        glu.SymbolicMatrix.load(str(tmp_path / "missing.bin"), ai, ap)
    assert e.value.status == -4


_RLIMIT_SCRIPT = r"""
import ctypes as C, resource, sys
import numpy as np
sys.path.insert(0, sys.argv[1])
from glu_public_b200 import _lib, gen
c = gen.mna_netlist(20000, 2)
nic_ap = np.ascontiguousarray(c.indptr, np.uint32)
nic_ai = np.ascontiguousarray(c.indices, np.uint32)
L = _lib.lib()
vm = int(open('/proc/self/status').read().split('VmSize:')[1].split()[0]) * 1024
extra = int(sys.argv[2]) * 2 ** 20
resource.setrlimit(resource.RLIMIT_AS, (vm + extra, vm + extra))
h = C.c_void_p()
st = L.glu_symbolic_create(c.n, nic_ap, nic_ai, C.byref(h))
print("STATUS", st, L.glu_last_error().decode())
"""


@pytest.mark.parametrize("extra_mb", [16, 128, 512])
def test_host_allocation_failure_returns_memory_overflow(tmp_path, extra_mb):
    """Under an address-space limit (the host allocator's failure path, made on the host with
    RLIMIT_AS in a child process) the symbolic analysis returns GLU_MEMORY_OVERFLOW (-3) or
    succeeds -- it never aborts the process."""
    import subprocess
    import sys
    script = tmp_path / "rlimit.py"
    script.write_text(_RLIMIT_SCRIPT)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, str(script), root, str(extra_mb)], capture_output=True,
                         text=True, timeout=300)
    assert res.returncode == 0, res.stdout + res.stderr
    line = [x for x in res.stdout.splitlines() if x.startswith("STATUS")][0]
    st = int(line.split()[1])
    assert st in (0, -3), line
    if st == -3:
        assert "host allocation failed" in line
