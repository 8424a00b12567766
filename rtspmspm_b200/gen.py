"""Deterministic synthetic sparse matrices for the SpGEMM workloads.

The reference benchmarks real SuiteSparse matrices that it downloads
(scripts/download_dataset.sh:4-21) and halves on failure
(scripts/AE_test.py:76-105).  No dataset is available offline, so every
workload here is a seeded synthetic matrix with the shape, density and value
distribution of the named configuration:

* ``erdos_renyi``  -- n x m, Poisson(mean) nonzeros per row, uniform columns,
  duplicates merged, values U(-1, 1).
* ``stencil27``    -- 27-point 3-D stencil on a g^3 grid, off-diagonal values
  N(0, 1), diagonal = 26 + sum of |off-diagonal| of the row, sorted columns.
* ``rmat``         -- R-MAT graph, 2^scale vertices, edge_factor * 2^scale
  edges, quadrant probabilities (a, b, c, d), duplicates merged, values
  U(0, 1).
* ``batch_uneven`` -- the 512 independent rectangular products of the batched
  workload.

Every generator returns a :class:`Csr` with int32 column indices, float32
values, rows sorted by column and no duplicate (row, col) pairs -- the
canonical form that both the CUDA engine and the CPU oracle expect.
All random draws come from ``numpy.random.default_rng(seed)`` (PCG64) in a
fixed order, so a (recipe, seed) pair names one matrix on every machine.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Csr:
    """Host CSR matrix: row_ptr (int64), col_idx (int32), val (float32)."""

    rows: int
    cols: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    val: np.ndarray

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def to_scipy(self):
        import scipy.sparse as sp

        return sp.csr_matrix((self.val, self.col_idx, self.row_ptr),
                             shape=(self.rows, self.cols))

    @staticmethod
    def from_scipy(m) -> "Csr":
        m = m.tocsr()
        m.sum_duplicates()
        m.sort_indices()
        return Csr(m.shape[0], m.shape[1], m.indptr.astype(np.int64),
                   m.indices.astype(np.int32), m.data.astype(np.float32))

    def row_block(self, r0: int, r1: int) -> "Csr":
        """Rows [r0, r1) as their own CSR (columns unchanged)."""
        p0, p1 = int(self.row_ptr[r0]), int(self.row_ptr[r1])
        return Csr(r1 - r0, self.cols, self.row_ptr[r0:r1 + 1] - p0,
                   self.col_idx[p0:p1], self.val[p0:p1])


def coo_to_csr(rows: int, cols: int, r: np.ndarray, c: np.ndarray,
               v: np.ndarray, merge: str = "first") -> Csr:
    """Sort COO by (row, col) and merge duplicates.

    ``merge="first"`` keeps the first occurrence (the generators assign values
    after de-duplication, so this only picks positions); ``merge="sum"`` adds
    duplicates as Matrix Market readers conventionally do.
    """
    r = np.asarray(r, dtype=np.int64)
    c = np.asarray(c, dtype=np.int64)
    v = np.asarray(v, dtype=np.float32)
    key = r * np.int64(cols) + c
    order = np.argsort(key, kind="stable")
    key = key[order]
    v = v[order]
    if key.size:
        first = np.empty(key.size, dtype=bool)
        first[0] = True
        np.not_equal(key[1:], key[:-1], out=first[1:])
        if merge == "sum":
            seg = np.cumsum(first) - 1
            vs = np.zeros(int(first.sum()), dtype=np.float64)
            np.add.at(vs, seg, v.astype(np.float64))
            v = vs.astype(np.float32)
        else:
            v = v[first]
        key = key[first]
    rr = (key // cols).astype(np.int64)
    cc = (key % cols).astype(np.int32)
    counts = np.bincount(rr, minlength=rows).astype(np.int64)
    row_ptr = np.zeros(rows + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    return Csr(rows, cols, row_ptr, cc, v.astype(np.float32))


def erdos_renyi(n: int, m: int | None = None, mean: float = 8.0, seed: int = 0,
                lo: float = -1.0, hi: float = 1.0) -> Csr:
    """n x m matrix, Poisson(mean) draws per row, uniform columns, merged.

    Draw order: per-row counts, then all column positions, then the values of
    the merged entries.
    """
    m = n if m is None else m
    rng = np.random.default_rng(seed)
    counts = rng.poisson(mean, size=n).astype(np.int64)
    total = int(counts.sum())
    r = np.repeat(np.arange(n, dtype=np.int64), counts)
    c = rng.integers(0, m, size=total, dtype=np.int64)
    csr = coo_to_csr(n, m, r, c, np.zeros(total, dtype=np.float32))
    csr.val = rng.uniform(lo, hi, size=csr.nnz).astype(np.float32)
    return csr


def stencil27(g: int, seed: int = 0) -> Csr:
    """27-point stencil on a g x g x g grid; row = x + g*y + g*g*z.

    Off-diagonal values N(0,1) drawn in CSR order; the diagonal is
    26 + sum_{j != i} |a_ij| (strictly diagonally dominant).
    """
    rng = np.random.default_rng(seed)
    n = g * g * g
    idx = np.arange(n, dtype=np.int64)
    x = idx % g
    y = (idx // g) % g
    z = idx // (g * g)
    # offsets in increasing column order: dz major, then dy, then dx
    offs = [(dx, dy, dz) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    valid = np.empty((n, 27), dtype=bool)
    colm = np.empty((n, 27), dtype=np.int64)
    for t, (dx, dy, dz) in enumerate(offs):
        valid[:, t] = ((x + dx >= 0) & (x + dx < g) & (y + dy >= 0) & (y + dy < g)
                       & (z + dz >= 0) & (z + dz < g))
        colm[:, t] = idx + dx + g * dy + g * g * dz
    counts = valid.sum(axis=1).astype(np.int64)
    row_ptr = np.zeros(n + 1, dtype=np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    col = colm[valid].astype(np.int32)
    nnz = int(row_ptr[-1])
    val = rng.standard_normal(nnz).astype(np.float32)
    rows_of = np.repeat(idx, counts)
    diag = col.astype(np.int64) == rows_of
    absv = np.abs(val).astype(np.float64)
    absv[diag] = 0.0
    rowsum = np.add.reduceat(absv, row_ptr[:-1]) if nnz else np.zeros(n)
    val[diag] = (26.0 + rowsum).astype(np.float32)
    return Csr(n, n, row_ptr, col, val)


def rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19,
         c: float = 0.19, seed: int = 0) -> Csr:
    """R-MAT (Chakrabarti et al. 2004) without noise, duplicates merged.

    For each of the edge_factor * 2^scale edges and each of the ``scale``
    levels (most significant bit first) one uniform draw picks the quadrant:
    [0,a) -> (0,0), [a,a+b) -> (0,1), [a+b,a+b+c) -> (1,0), else (1,1).
    Values U(0,1) are drawn for the merged entries in CSR order.
    """
    rng = np.random.default_rng(seed)
    n = 1 << scale
    ne = edge_factor * n
    r = np.zeros(ne, dtype=np.int64)
    cc = np.zeros(ne, dtype=np.int64)
    ab = a + b
    abc = a + b + c
    chunk = 1 << 22
    for lvl in range(scale):
        bit = np.int64(1) << np.int64(scale - 1 - lvl)
        for s in range(0, ne, chunk):
            u = rng.random(min(chunk, ne - s))
            rb = u >= ab
            cb = ((u >= a) & (u < ab)) | (u >= abc)
            r[s:s + u.size] |= rb * bit
            cc[s:s + u.size] |= cb * bit
    csr = coo_to_csr(n, n, r, cc, np.zeros(ne, dtype=np.float32))
    csr.val = rng.random(csr.nnz).astype(np.float32)
    return csr


def log_uniform_int(rng, lo: int, hi: int) -> int:
    return int(round(math.exp(rng.uniform(math.log(lo), math.log(hi)))))


def batch_uneven(count: int = 512, seed: int = 1, lo: int = 1024,
                 hi: int = 65536, mean_lo: float = 2.0, mean_hi: float = 32.0):
    """``count`` independent (A_i, B_i) pairs of uneven rectangular shapes.

    Per pair, in this order: rows, inner, cols ~ log-uniform[lo, hi]; then
    mean_A, mean_B ~ U(mean_lo, mean_hi); then A_i and B_i are Erdos-Renyi
    matrices with sub-seeds drawn from the same stream.
    """
    rng = np.random.default_rng(seed)
    pairs = []
    for _ in range(count):
        rows = log_uniform_int(rng, lo, hi)
        inner = log_uniform_int(rng, lo, hi)
        cols = log_uniform_int(rng, lo, hi)
        mu_a = float(rng.uniform(mean_lo, mean_hi))
        mu_b = float(rng.uniform(mean_lo, mean_hi))
        sa = int(rng.integers(0, 2**31 - 1))
        sb = int(rng.integers(0, 2**31 - 1))
        A = erdos_renyi(rows, inner, mu_a, sa)
        B = erdos_renyi(inner, cols, mu_b, sb)
        pairs.append((A, B))
    return pairs


def row_products(A: Csr, B: Csr) -> np.ndarray:
    """Intermediate products per row of A*B: sum of |B_k| over k in A_i."""
    bl = B.row_lengths()
    per = bl[A.col_idx]
    out = np.zeros(A.rows, dtype=np.int64)
    if A.nnz:
        nz = A.row_lengths() > 0
        out[nz] = np.add.reduceat(per, A.row_ptr[:-1][nz])
    return out


def by_name(name: str) -> Csr:
    """Named workloads used by the CLI, tests and benchmark."""
    table = {
        "er4096": lambda: erdos_renyi(4096, 4096, 8.0, 0),
        "stencil96": lambda: stencil27(96, 0),
        "rmat20": lambda: rmat(20, 16, seed=0),
    }
    if name in table:
        return table[name]()
    if name.startswith("stencil"):
        return stencil27(int(name[len("stencil"):]))
    if name.startswith("rmat"):
        return rmat(int(name[len("rmat"):]))
    if name.startswith("er"):
        return erdos_renyi(int(name[2:]))
    raise KeyError(name)
