"""The C++ driver glu_cmd (glu_public_b200/cmd/glu_cmd.cpp): lu_cmd's flow through the C ABI."""
import os
import re
import subprocess

import numpy as np
import pytest

from glu_public_b200 import build, gen, glu


@pytest.fixture(scope="module")
def glu_cmd(built_lib):
    return build.build_cmd()


def _matrix(tmp_path, n=300, seed=4):
    c = gen.mna_netlist(n, seed)
    path = str(tmp_path / "m.mtx")
    gen.write_mtx(path, c)
    return c, path


def test_glu_cmd_usage(glu_cmd):
    res = subprocess.run([glu_cmd, "--help"], capture_output=True, text=True)
    assert res.returncode == 0 and "usage" in res.stdout


def test_glu_cmd_symbolic_and_saved_analysis_without_a_gpu(glu_cmd, tmp_path):
    """On a machine without a GPU the driver reads the matrix, runs (and saves) the symbolic
    analysis, then stops with a clear error at the first device call."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("covered by the GPU test")
    c, path = _matrix(tmp_path)
    sym_file = str(tmp_path / "m.glusym")
    res = subprocess.run([glu_cmd, "-s", sym_file, path], capture_output=True, text=True)
    assert res.returncode == 2, res.stdout + res.stderr
    a = gen.read_mtx(path)
    ap = a.indptr.astype(np.uint32)
    ai = a.indices.astype(np.uint32)
    s = glu.SymbolicMatrix(c.n).analyze(ai, ap)
    assert f"nnz(L+U) = {s.nnz}" in res.stdout
    assert "plan failed" in res.stderr
    t = glu.SymbolicMatrix.load(sym_file, ai, ap)
    assert np.array_equal(t.sym_r_idx, s.sym_r_idx)


@pytest.mark.gpu
def test_glu_cmd_factors_and_solves(glu_cmd, cuda, tmp_path):
    _, path = _matrix(tmp_path, n=2000, seed=5)
    sym_file = str(tmp_path / "m.glusym")
    for _ in range(2):                           # the second run loads the saved analysis
        res = subprocess.run([glu_cmd, "-s", sym_file, path], capture_output=True, text=True)
        assert res.returncode == 0, res.stdout + res.stderr
        m = re.search(r"residual .* = ([0-9.eE+-]+)", res.stdout)
        assert m and float(m.group(1)) <= 1e-12, res.stdout
    assert "loaded in" in res.stdout


_BANNERS = {
    "skew": ("%%MatrixMarket matrix coordinate real skew-symmetric",
             ["4 4 4", "2 1 1.5", "3 1 -2.25", "4 3 0.5", "4 2 7"]),
    "sym": ("%%MatrixMarket matrix coordinate real symmetric",
            ["3 3 4", "1 1 4", "2 1 -1", "3 2 -1", "3 3 4"]),
    "pattern": ("%%MatrixMarket matrix coordinate pattern general",
                ["3 3 3", "1 1", "2 2", "3 1"]),
    "integer_dup": ("%%MatrixMarket matrix coordinate integer general",
                    ["2 2 4", "1 1 3", "2 2 5", "1 1 4", "2 1 -6"]),
    "no_banner": (None, ["3 3 3", "1 1 1.0", "2 2 2.0", "3 3 3.0"]),
}


@pytest.mark.parametrize("kind", sorted(_BANNERS))
def test_glu_cmd_reader_agrees_with_read_mtx(glu_cmd, tmp_path, kind):
    """glu_cmd's own MatrixMarket reader (its -o mode writes the matrix as read) and
    gen.read_mtx give the same CSC for every accepted banner, skew-symmetric included."""
    banner, body = _BANNERS[kind]
    src = tmp_path / f"{kind}.mtx"
    src.write_text("\n".join(([banner] if banner else []) + ["% a comment"] * (banner is not None)
                             + body) + "\n")
    out = tmp_path / f"{kind}.out.mtx"
    res = subprocess.run([glu_cmd, "-o", str(out), str(src)], capture_output=True, text=True)
    assert res.returncode == 0, res.stdout + res.stderr
    a, b = gen.read_mtx(str(src)), gen.read_mtx(str(out))
    assert np.array_equal(a.indptr, b.indptr) and np.array_equal(a.indices, b.indices)
    assert np.array_equal(a.data, b.data)
    if kind == "skew":
        d = a.toarray()
        assert np.array_equal(d, -d.T) and d[0, 1] == -1.5


@pytest.mark.parametrize("banner", ["%%MatrixMarket matrix coordinate real hermitian",
                                    "%%MatrixMarket matrix coordinate complex general",
                                    "%%MatrixMarket matrix array real general",
                                    "%%MatrixMarket matrix coordinate real skew"])
def test_glu_cmd_reader_rejects_unknown_banners(glu_cmd, tmp_path, banner):
    src = tmp_path / "bad.mtx"
    src.write_text(banner + "\n2 2 1\n1 1 1.0\n")
    res = subprocess.run([glu_cmd, "-o", str(tmp_path / "o.mtx"), str(src)],
                         capture_output=True, text=True)
    assert res.returncode == 1 and "cannot read" in res.stderr
    with pytest.raises(ValueError):
        gen.read_mtx(str(src))
