"""Generates the committed golden fixtures from the reference's own CPU code (oracle/_ref).

Run in the build container, where the reference tree exists:
    python tests/golden/make_fixtures.py [--skip-slow]

Outputs (tests/golden/):
  nicslu_<pattern>.npz    NICSLU_Analyze's permutations and MC64 scalings of the nominal matrix of
                          a benchmark pattern (row_perm, col_perm as col_perm - row_perm,
                          row_scale, col_scale_perm, mc64_scale) plus a digest of the generated
                          matrix they belong to.  With them the preprocessed matrix the reference
                          hands to GLU is rebuilt exactly (glu.NicsluArrays.preprocess), on
                          machines without the reference.
  symbolic_golden.json    per pattern: n, nnz_A, nnz_LU, num_lev and SHA-256 digests of every
                          array symbolic.cc (fill_in/csr/leveling, REAL=double) produced, and of
                          predictLU's val.  Pins the bit-exact symbolic at sizes where running
                          symbolic.cc in a test would take minutes.
  add32.npz               the reference's one sample matrix (src/add32.mtx, n = 4,960) as CSC
                          (indptr, indices, data) plus a digest of the file, so the add32 cases
                          also run where the reference tree is absent (python
                          tests/golden/make_fixtures.py --add32 writes only this file).

The reference tree is found at $GLU_REFERENCE_DIR (default /root/reference).
"""
from __future__ import annotations

import hashlib
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from glu_public_b200 import gen  # noqa: E402
from oracle import oracle as O  # noqa: E402

# benchmark patterns: name -> generator call (seeds fixed here and in bench.py)
PATTERNS = {
    "mna2000_s3": lambda: gen.mna_netlist(2000, 3),      # multi-pattern batch, pattern A
    "mna4960_s0": lambda: gen.mna_netlist(4960, 0),      # plain pipeline, n = 4,960
    "mna20000_s2": lambda: gen.mna_netlist(20000, 2),    # batched same-pattern, n = 20,000
    "grid128_s1": lambda: gen.power_grid(128, 1),        # reduced power-grid mesh
}
SLOW = {
    "grid512_s1": lambda: gen.power_grid(512, 1),        # power-grid mesh, n = 524,352
}
# patterns whose symbolic.cc run would take from many minutes to hours: preprocessing only
NO_SYMBOLIC = {
    "mna50000_s4": lambda: gen.mna_netlist(50000, 4),    # multi-pattern batch, pattern B
    "mna100000_s6": lambda: gen.mna_netlist(100000, 6),  # adjoint, n = 100,000
}


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str(a.dtype).encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def circuit_digest(c: gen.Circuit) -> str:
    return digest(c.indptr.astype(np.int64), c.indices.astype(np.int32), c.data)


REFERENCE = os.environ.get("GLU_REFERENCE_DIR", "/root/reference")


def make_add32() -> None:
    """tests/golden/add32.npz from the reference's src/add32.mtx (read by gen.read_mtx: a file
    without a banner, real general, 1-based)."""
    src = os.path.join(REFERENCE, "src", "add32.mtx")
    a = gen.read_mtx(src)
    with open(src, "rb") as f:
        file_digest = hashlib.sha256(f.read()).hexdigest()
    np.savez_compressed(os.path.join(HERE, "add32.npz"), n=a.shape[0],
                        indptr=a.indptr.astype(np.int64), indices=a.indices.astype(np.int32),
                        data=a.data.astype(np.float64), file_sha256=file_digest)
    print(f"add32: n={a.shape[0]} nnz={a.nnz}", flush=True)


def main() -> None:
    if "--add32" in sys.argv:
        make_add32()
        return
    skip_slow = "--skip-slow" in sys.argv
    only = [a for a in sys.argv[1:] if not a.startswith("--")]
    pats = dict(PATTERNS)
    if not skip_slow:
        pats.update(SLOW)
        pats.update(NO_SYMBOLIC)
    if only:
        pats = {k: v for k, v in pats.items() if k in only}
    gpath = os.path.join(HERE, "symbolic_golden.json")
    golden = json.load(open(gpath)) if os.path.exists(gpath) else {}
    for name, mk in pats.items():
        t0 = time.time()
        c = mk()
        ref = O.RefPipeline.from_csc(c.n, c.indptr, c.indices, c.data)
        pre = ref.preprocessed()
        # compact: inverses are derived on load, col_perm is stored as its difference from
        # row_perm (NICSLU orders rows and columns alike, so the difference is mostly zero)
        np.savez_compressed(os.path.join(HERE, f"nicslu_{name}.npz"), n=c.n,
                            row_perm=pre.row_perm,
                            col_perm_delta=pre.col_perm.astype(np.int64) - pre.row_perm,
                            row_scale=pre.row_scale, col_scale_perm=pre.col_scale_perm,
                            mc64_scale=pre.mc64_scale, matrix_digest=circuit_digest(c))
        if name in NO_SYMBOLIC:
            ref.close()
            print(f"{name}: n={c.n} preprocessing only ({time.time() - t0:.1f}s)", flush=True)
            continue
        s = ref.symbolic()
        golden[name] = {
            "n": c.n, "nnz_a": c.nnz, "nnz_lu": s.nnz, "num_lev": s.num_lev,
            "matrix": circuit_digest(c),
            "sym_c_ptr": digest(s.sym_c_ptr), "sym_r_idx": digest(s.sym_r_idx),
            "l_col_ptr": digest(s.l_col_ptr), "csr_r_ptr": digest(s.csr_r_ptr),
            "csr_c_idx": digest(s.csr_c_idx), "csr_diag_ptr": digest(s.csr_diag_ptr),
            "level_ptr": digest(s.level_ptr), "level_idx": digest(s.level_idx),
            "val": digest(s.val), "flops": O.flops(s),
        }
        ref.close()
        json.dump(golden, open(gpath, "w"), indent=1, sort_keys=True)
        print(f"{name}: n={c.n} nnz_lu={s.nnz} levels={s.num_lev} ({time.time() - t0:.1f}s)",
              flush=True)


if __name__ == "__main__":
    main()
