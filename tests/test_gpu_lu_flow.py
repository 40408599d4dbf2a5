"""The drop-in boundary exercised in the reference's own flow.

oracle/_ref/lu_flow (source: tests/lu_flow.cpp) runs the reference's lu_cmd sequence --
preprocess (NICSLU MC64 + AMD), Symbolic_Matrix::fill_in / csr / predictLU / leveling, all the
reference's own code -- and replaces LUonDevice and Symbolic_Matrix::solve with this library's C
ABI exactly as the integration guide shows.  Checked here:
  * predictLU's values (LUonDevice's input) equal the oracle pipeline's, bit for bit;
  * the GPU factors left in A_sym.val match the oracle per column (1e-12, or 8x the oracle's own
    rounding-order sensitivity);
  * glu_solve's x (b = 1, as lu_cmd) matches Symbolic_Matrix::solve run on those factors, and
    its residual on the original matrix is <= 1e-12.
"""
import os
import subprocess

import numpy as np
import pytest

from glu_public_b200 import gen
from oracle import oracle as O
from tests.common import case, column_rel_err, lu_tolerance

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LU_FLOW = os.path.join(ROOT, "oracle", "_ref", "lu_flow")


@pytest.mark.parametrize("name,perturb", [("add32", False), ("mna:4960,0", False),
                                          ("mna:4960,0", True)])
def test_lu_cmd_flow_through_the_c_abi(built_lib, cuda, tmp_path, name, perturb):
    if not os.path.exists(LU_FLOW):
        pytest.skip("oracle/_ref/lu_flow not built (needs the reference tree at build time)")
    cs = case(name)
    c = cs.circuit
    mtx = str(tmp_path / "a.mtx")
    gen.write_mtx(mtx, c)
    prefix = str(tmp_path / "out")
    res = subprocess.run([LU_FLOW] + (["-p"] if perturb else []) + [mtx, prefix],
                         capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    line = [x for x in res.stdout.splitlines() if x.startswith("lu_flow ")][-1]
    flags = int(line.split("flags=")[1].split()[0])
    val = np.fromfile(prefix + ".val", np.float64)
    lu = np.fromfile(prefix + ".lu", np.float64)
    x_gpu = np.fromfile(prefix + ".x_gpu", np.float64)
    x_ref = np.fromfile(prefix + ".x_ref", np.float64)
    assert np.array_equal(val, cs.sym_ref.val)
    pert = O.perturbation(cs.sym_ref, val) if perturb else 0.0
    expect, st = O.factor(cs.sym_ref, val, pert=pert)
    assert st == 0
    assert (flags & ~4) == 0, line                 # perturbed pivots (4) are allowed with -p
    if perturb:
        other, _ = O.factor(cs.sym_ref, val, pert=pert, fma=True)
        tol = max(1e-12, 8.0 * column_rel_err(cs.sym_ref, other, expect))
    else:
        tol = lu_tolerance(cs, val)
    assert column_rel_err(cs.sym_ref, lu, expect) <= tol, line
    assert np.max(np.abs(x_gpu - x_ref)) <= 1e-9 * max(1.0, np.max(np.abs(x_ref))), line
    if not perturb:
        b = np.ones(c.n)
        assert O.residual(c.n, c.indptr, c.indices, c.data, x_gpu, b) <= 1e-12, line
