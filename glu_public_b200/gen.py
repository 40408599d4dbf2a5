"""Seeded synthetic circuit matrices (modified nodal analysis) for the GLU numeric phase.

The reference ships one small matrix (``src/add32.mtx``) and quotes its timings on the UFL circuit
collection, which is not available here.  These generators stand in for it with the shapes,
sizes and value distributions of the benchmark configurations:

* :func:`mna_netlist` -- random netlist MNA matrix: every node links to 1-4 other nodes (70 % of
  the links inside a +-32 index window, 30 % uniform), log-uniform conductances in [1e-3, 1e2] S
  stamped as a +-g Laplacian, voltage-controlled current sources on 3 % of the nodes (one entry
  of magnitude U[0.1, 10] with a random sign) and a 1e-9 S ground shunt on every node.
* :func:`power_grid` -- two-layer 5-point power-grid mesh with lognormal(0, 0.5) conductances,
  10 S vias every 8th node in both directions, 16 rail hubs tied by 1 S to 0.5 % of the nodes,
  supply pads stamped as voltage sources (extra MNA rows/columns with +-1 entries) and 1e-9 S
  shunts.

A :class:`Circuit` keeps the element list, so Monte Carlo instances of the same pattern
(:meth:`Circuit.instance_values`) are produced by rescaling the elements and re-stamping.

Matrices are stored as CSC with sorted row indices (the layout ``NicsLU_ReadTripletColumnToSparse``
builds, ``src/nicslu/util/nicslu_readfile.c:197-224``) and are written as column-sorted, 1-based
MatrixMarket ``real general`` files, because that reader requires column order.

Link count per node: drawing the number of links a node *initiates* from {1, 2, 3, 4} with
probabilities (0.45, 0.30, 0.15, 0.10) (mean 1.9) gives a node degree of about 3.8 and, with the
diagonal, about 4.8 stored entries per row; drawing it uniformly would give about 5.9.
"""
from __future__ import annotations

import dataclasses
import os

import numpy as np
import scipy.sparse as sp

LINK_COUNT_P = (0.45, 0.30, 0.15, 0.10)
WINDOW = 32
P_WINDOW = 0.70
VCCS_FRACTION = 0.03
SHUNT = 1e-9

# element kinds
K_COND = 0      # conductance: +g at (i,i),(j,j); -g at (i,j),(j,i)
K_VCCS = 1      # controlled source: one entry
K_FIXED = 2     # fixed stamp (shunt, pad incidence): not perturbed across instances


@dataclasses.dataclass
class Circuit:
    """A circuit matrix in CSC form plus the element stamps that produced its values."""

    n: int
    indptr: np.ndarray          # int64 [n+1]
    indices: np.ndarray         # int32 [nnz], sorted inside each column
    data: np.ndarray            # float64 [nnz], nominal values
    stamp: sp.csr_matrix        # [nnz, n_elements]: data = stamp @ elem_value
    elem_value: np.ndarray      # float64 [n_elements]
    elem_kind: np.ndarray       # int8 [n_elements]
    name: str = ""

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])

    def to_scipy(self, data: np.ndarray | None = None) -> sp.csc_matrix:
        d = self.data if data is None else data
        return sp.csc_matrix((d, self.indices, self.indptr), shape=(self.n, self.n))

    def instance_values(self, count: int, seed: int, sigma: float = 0.1,
                        src_lo: float = 0.8, src_hi: float = 1.2) -> np.ndarray:
        """Monte Carlo value sets of the same pattern, shape ``[count, nnz]`` (float64).

        Every conductance is scaled by lognormal(0, sigma) and every controlled-source entry by
        U[src_lo, src_hi], independently per instance; fixed stamps keep their value.
        """
        rng = np.random.default_rng(seed)
        ne = self.elem_value.shape[0]
        f = np.ones((ne, count))
        cond = self.elem_kind == K_COND
        vccs = self.elem_kind == K_VCCS
        f[cond] = rng.lognormal(0.0, sigma, size=(int(cond.sum()), count))
        f[vccs] = rng.uniform(src_lo, src_hi, size=(int(vccs.sum()), count))
        vals = self.stamp @ (f * self.elem_value[:, None])
        return np.ascontiguousarray(np.asarray(vals).T)

    def instance_values_indexed(self, first: int, count: int, seed: int, sigma: float = 0.1,
                                src_lo: float = 0.8, src_hi: float = 1.2) -> np.ndarray:
        """Instances [first, first + count) of a batch whose instance i draws its factors from its
        own generator seeded with (seed, i): same distribution as :meth:`instance_values`, and an
        instance's values depend only on its global index, so shards of a batch made on
        different ranks together are exactly the batch.  Shape ``[count, nnz]``."""
        ne = self.elem_value.shape[0]
        f = np.ones((ne, count))
        cond = self.elem_kind == K_COND
        vccs = self.elem_kind == K_VCCS
        nc, nv = int(cond.sum()), int(vccs.sum())
        for k in range(count):
            rng = np.random.default_rng((seed, first + k))
            f[cond, k] = rng.lognormal(0.0, sigma, size=nc)
            f[vccs, k] = rng.uniform(src_lo, src_hi, size=nv)
        vals = self.stamp @ (f * self.elem_value[:, None])
        return np.ascontiguousarray(np.asarray(vals).T)

    def realised_nnz_per_row(self) -> float:
        return self.nnz / self.n


def _assemble(n: int, rows: list, cols: list, coef: list, elem: list,
              elem_value: np.ndarray, elem_kind: np.ndarray, name: str) -> Circuit:
    """Stamps (row, col, coef, element) -> CSC pattern + stamp matrix (duplicates summed)."""
    r = np.concatenate(rows).astype(np.int64)
    c = np.concatenate(cols).astype(np.int64)
    w = np.concatenate(coef).astype(np.float64)
    e = np.concatenate(elem).astype(np.int64)
    key = c * n + r                      # column-major order => CSC order after sorting
    uniq, inv = np.unique(key, return_inverse=True)
    nnz = uniq.shape[0]
    stamp = sp.csr_matrix((w, (inv, e)), shape=(nnz, elem_value.shape[0]))
    stamp.sum_duplicates()
    data = stamp @ elem_value
    ucol = uniq // n
    urow = (uniq % n).astype(np.int32)
    indptr = np.zeros(n + 1, dtype=np.int64)
    np.add.at(indptr, ucol + 1, 1)
    indptr = np.cumsum(indptr)
    return Circuit(n=n, indptr=indptr, indices=urow, data=np.asarray(data, dtype=np.float64),
                   stamp=stamp, elem_value=elem_value, elem_kind=elem_kind, name=name)


def _partner(rng: np.random.Generator, src: np.ndarray, n: int) -> np.ndarray:
    """Other end of a link: 70 % inside a +-32 window (reflected at the ends), 30 % uniform."""
    m = src.shape[0]
    near = rng.random(m) < P_WINDOW
    off = rng.integers(1, WINDOW + 1, size=m) * np.where(rng.random(m) < 0.5, -1, 1)
    dst_near = src + off
    dst_near = np.where(dst_near < 0, src - off, dst_near)
    dst_near = np.where(dst_near >= n, src - off, dst_near)
    dst_far = rng.integers(0, n - 1, size=m)
    dst_far = np.where(dst_far >= src, dst_far + 1, dst_far)   # uniform over the other nodes
    dst = np.where(near, dst_near, dst_far)
    return np.clip(dst, 0, n - 1)


def mna_netlist(n: int, seed: int) -> Circuit:
    """Random-netlist MNA matrix of order ``n`` (see the module docstring for the rules)."""
    if n < 2 * WINDOW + 2:
        raise ValueError("n too small for the link window")
    rng = np.random.default_rng(seed)
    k = rng.choice(np.arange(1, 5), size=n, p=LINK_COUNT_P)
    src = np.repeat(np.arange(n), k)
    dst = _partner(rng, src, n)
    keep = dst != src
    src, dst = src[keep], dst[keep]
    nl = src.shape[0]
    g = 10.0 ** rng.uniform(-3.0, 2.0, size=nl)

    nv = int(round(VCCS_FRACTION * n))
    vnode = rng.choice(n, size=nv, replace=False)
    vctl = _partner(rng, vnode, n)
    keepv = vctl != vnode
    vnode, vctl = vnode[keepv], vctl[keepv]
    nv = vnode.shape[0]
    gm = rng.uniform(0.1, 10.0, size=nv) * np.where(rng.random(nv) < 0.5, -1.0, 1.0)

    ne = nl + nv + n
    elem_value = np.concatenate([g, gm, np.full(n, SHUNT)])
    elem_kind = np.concatenate([np.full(nl, K_COND), np.full(nv, K_VCCS),
                                np.full(n, K_FIXED)]).astype(np.int8)
    le = np.arange(nl)
    ve = nl + np.arange(nv)
    se = nl + nv + np.arange(n)
    rows = [src, dst, src, dst, vnode, np.arange(n)]
    cols = [src, dst, dst, src, vctl, np.arange(n)]
    coef = [np.ones(nl), np.ones(nl), -np.ones(nl), -np.ones(nl), np.ones(nv), np.ones(n)]
    elem = [le, le, le, le, ve, se]
    assert ne == elem_value.shape[0]
    return _assemble(n, rows, cols, coef, elem, elem_value, elem_kind, f"mna{n}_s{seed}")


def power_grid(side: int, seed: int, layers: int = 2, pads: int = 64, hubs: int = 16,
               via_pitch: int = 8, hub_fraction: float = 0.005) -> Circuit:
    """Two-layer power-grid MNA matrix: ``layers*side*side`` nodes plus ``pads`` source rows."""
    rng = np.random.default_rng(seed)
    nn = layers * side * side
    n = nn + pads
    ids = np.arange(side * side).reshape(side, side)
    rows, cols, coef, elem, vals, kinds = [], [], [], [], [], []
    ecount = 0

    def add_links(a: np.ndarray, b: np.ndarray, gv: np.ndarray, kind: int):
        nonlocal ecount
        m = a.shape[0]
        e = ecount + np.arange(m)
        ecount += m
        rows.extend([a, b, a, b])
        cols.extend([a, b, b, a])
        coef.extend([np.ones(m), np.ones(m), -np.ones(m), -np.ones(m)])
        elem.extend([e, e, e, e])
        vals.append(gv)
        kinds.append(np.full(m, kind, dtype=np.int8))

    for layer in range(layers):
        base = layer * side * side
        h_a = (base + ids[:, :-1]).ravel()
        h_b = (base + ids[:, 1:]).ravel()
        v_a = (base + ids[:-1, :]).ravel()
        v_b = (base + ids[1:, :]).ravel()
        a = np.concatenate([h_a, v_a])
        b = np.concatenate([h_b, v_b])
        add_links(a, b, rng.lognormal(0.0, 0.5, size=a.shape[0]), K_COND)
    via = ids[::via_pitch, ::via_pitch].ravel()
    for layer in range(layers - 1):
        add_links(layer * side * side + via, (layer + 1) * side * side + via,
                  np.full(via.shape[0], 10.0), K_COND)
    hub_nodes = rng.choice(nn, size=hubs, replace=False)
    for h in hub_nodes:
        m = max(1, int(round(hub_fraction * nn)))
        tgt = rng.choice(nn, size=m, replace=False)
        tgt = tgt[tgt != h]
        add_links(np.full(tgt.shape[0], h), tgt, np.ones(tgt.shape[0]), K_COND)
    # supply pads on the top layer, on an evenly spaced sqrt(pads) x sqrt(pads) grid
    g = int(round(np.sqrt(pads)))
    if g * g != pads:
        raise ValueError("pads must be a perfect square")
    pos = (side // g) // 2 + (side // g) * np.arange(g)
    pad_nodes = ((layers - 1) * side * side + ids[np.ix_(pos, pos)]).ravel()
    pad_rows = nn + np.arange(pads)
    e = ecount + np.arange(pads)
    ecount += pads
    rows.extend([pad_nodes, pad_rows])
    cols.extend([pad_rows, pad_nodes])
    coef.extend([np.ones(pads), -np.ones(pads)])
    elem.extend([e, e])
    vals.append(np.ones(pads))
    kinds.append(np.full(pads, K_FIXED, dtype=np.int8))
    # shunts on the grid nodes
    e = ecount + np.arange(nn)
    ecount += nn
    rows.append(np.arange(nn))
    cols.append(np.arange(nn))
    coef.append(np.ones(nn))
    elem.append(e)
    vals.append(np.full(nn, SHUNT))
    kinds.append(np.full(nn, K_FIXED, dtype=np.int8))
    return _assemble(n, rows, cols, coef, elem, np.concatenate(vals), np.concatenate(kinds),
                     f"grid{layers}x{side}_s{seed}")


def write_mtx(path: str | os.PathLike, c: Circuit, data: np.ndarray | None = None) -> None:
    """Column-sorted, 1-based MatrixMarket ``coordinate real general`` with 17 significant digits."""
    d = c.data if data is None else data
    col = np.repeat(np.arange(c.n), np.diff(c.indptr))
    with open(path, "w") as f:
        f.write("%%MatrixMarket matrix coordinate real general\n")
        f.write(f"{c.n} {c.n} {c.nnz}\n")
        # numpy's text formatter is far faster than a Python loop for millions of lines
        arr = np.empty(c.nnz, dtype=[("r", np.int64), ("c", np.int64), ("v", np.float64)])
        arr["r"] = c.indices + 1
        arr["c"] = col + 1
        arr["v"] = d
        np.savetxt(f, arr, fmt="%d %d %.17g")


def read_mtx(path: str | os.PathLike, cache: bool = False) -> sp.csc_matrix:
    """Read a MatrixMarket ``coordinate`` file into CSC (rows sorted, duplicates summed).

    Entries may come in any order.  A file without the banner line is read as ``real general``.
    Fields ``real``, ``integer`` and ``pattern`` (values 1) are accepted, with symmetry ``general``, ``symmetric`` (the stored triangle is mirrored) or
    ``skew-symmetric`` (mirrored with the sign flipped); ``complex`` / ``hermitian`` and the
    ``array`` format are rejected.  (The reference's reader, nicslu_readfile.c:98-224, needs
    column-sorted ``real general`` triplets.)  With ``cache``, the matrix is also kept as
    ``<path>.csc.npz`` and read from there next time while the file is not newer than it.
    """
    path = os.fspath(path)
    cpath = path + ".csc.npz"
    if cache and os.path.exists(cpath) and os.path.getmtime(cpath) >= os.path.getmtime(path):
        z = np.load(cpath)
        return sp.csc_matrix((z["data"], z["indices"], z["indptr"]), shape=tuple(z["shape"]))
    with open(path) as f:
        first = f.readline()
        banner = first.split()
        if banner and banner[0].lower() == "%%matrixmarket":
            if len(banner) < 5 or banner[1].lower() != "matrix":
                raise ValueError(f"{path}: not a MatrixMarket matrix file")
            fmt, field, sym = (x.lower() for x in banner[2:5])
            line = f.readline()
        else:                     # no banner (like the reference's src/add32.mtx): real general
            fmt, field, sym = "coordinate", "real", "general"
            line = first
        if fmt != "coordinate":
            raise ValueError(f"{path}: only the coordinate format is supported (got {fmt})")
        if field not in ("real", "integer", "pattern"):
            raise ValueError(f"{path}: field {field} is not supported (real, integer, pattern)")
        if sym not in ("general", "symmetric", "skew-symmetric"):
            raise ValueError(f"{path}: symmetry {sym} is not supported")
        while line.startswith("%") or not line.strip():
            line = f.readline()
        m, n, nnz = (int(x) for x in line.split()[:3])
        cols = 2 if field == "pattern" else 3
        body = np.loadtxt(f, ndmin=2, usecols=range(cols)) if nnz else np.zeros((0, cols))
    if body.shape[0] != nnz:
        raise ValueError(f"{path}: {body.shape[0]} entries, the size line says {nnz}")
    r = body[:, 0].astype(np.int64) - 1
    c = body[:, 1].astype(np.int64) - 1
    if nnz and (r.min() < 0 or c.min() < 0 or r.max() >= m or c.max() >= n):
        raise ValueError(f"{path}: entry index out of range")
    v = np.ones(nnz) if field == "pattern" else body[:, 2].astype(np.float64)
    if sym != "general":
        off = r != c
        sign = -1.0 if sym == "skew-symmetric" else 1.0
        r, c, v = (np.concatenate([r, c[off]]), np.concatenate([c, r[off]]),
                   np.concatenate([v, sign * v[off]]))
    a = sp.coo_matrix((v, (r, c)), shape=(m, n)).tocsc()
    a.sum_duplicates()
    a.sort_indices()
    if cache:
        np.savez(cpath, data=a.data, indices=a.indices, indptr=a.indptr,
                 shape=np.asarray(a.shape))
    return a


def circuit_from_csc(a: sp.csc_matrix, name: str = "") -> Circuit:
    """Wrap an arbitrary CSC matrix (each entry its own fixed element)."""
    a = a.tocsc()
    a.sum_duplicates()
    a.sort_indices()
    nnz = a.nnz
    stamp = sp.identity(nnz, format="csr")
    return Circuit(n=a.shape[0], indptr=a.indptr.astype(np.int64),
                   indices=a.indices.astype(np.int32), data=a.data.astype(np.float64),
                   stamp=stamp, elem_value=a.data.astype(np.float64).copy(),
                   elem_kind=np.full(nnz, K_FIXED, dtype=np.int8), name=name)
