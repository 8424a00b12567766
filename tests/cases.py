"""Small seeded inputs with known answers or oracle-checkable sizes."""
import numpy as np

from rtspmspm_b200 import gen
from rtspmspm_b200.gen import Csr, coo_to_csr


def identity(n):
    return Csr(n, n, np.arange(n + 1, dtype=np.int64), np.arange(n, dtype=np.int32), np.ones(n, np.float32))


def permutation(n, seed=0):
    p = np.random.default_rng(seed).permutation(n)
    return coo_to_csr(n, n, np.arange(n), p, np.ones(n, np.float32))


def dense_ones(n):
    r, c = np.divmod(np.arange(n * n), n)
    return coo_to_csr(n, n, r, c, np.ones(n * n, np.float32))


def with_empty_rows_cols(n=64, seed=3):
    A = gen.erdos_renyi(n, n, 4.0, seed)
    keep = np.ones(n, bool)
    keep[::5] = False   # empty rows
    r = np.repeat(np.arange(n), A.row_lengths())
    m = keep[r] & (A.col_idx % 7 != 0)  # empty columns too
    return coo_to_csr(n, n, r[m], A.col_idx[m], A.val[m])


def heavy_row(n=3000, seed=4):
    """Row 0 touches every column; the rest are sparse."""
    A = gen.erdos_renyi(n, n, 3.0, seed)
    r = np.concatenate([np.zeros(n, np.int64), np.repeat(np.arange(n), A.row_lengths())])
    c = np.concatenate([np.arange(n), A.col_idx])
    v = np.concatenate([np.linspace(-1, 1, n, dtype=np.float32), A.val])
    return coo_to_csr(n, n, r, c, v, merge="first")


def cancelling():
    """C[0,0] = 1*1 + 1*(-1) = 0 exactly: a structural entry with value 0."""
    A = coo_to_csr(2, 2, [0, 0], [0, 1], np.array([1.0, 1.0], np.float32))
    B = coo_to_csr(2, 2, [0, 1], [0, 0], np.array([1.0, -1.0], np.float32))
    return A, B


def empty(rows=10, cols=10):
    return Csr(rows, cols, np.zeros(rows + 1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32))


def named_pairs():
    """(name, A, B) pairs used by the parity tests."""
    out = []
    out.append(("identity", identity(100), gen.erdos_renyi(100, 100, 5.0, 1)))
    out.append(("permutation", permutation(200), gen.erdos_renyi(200, 300, 6.0, 2)))
    out.append(("ones16", dense_ones(16), dense_ones(16)))
    E = with_empty_rows_cols()
    out.append(("empty_rows_cols", E, E))
    H = heavy_row()
    out.append(("heavy_row", H, H))
    a, b = cancelling()
    out.append(("cancelling", a, b))
    out.append(("empty", empty(10, 12), empty(12, 7)))
    out.append(("zero_rows", empty(0, 5), gen.erdos_renyi(5, 5, 2.0, 3)))
    out.append(("rect", gen.erdos_renyi(300, 500, 7.0, 5), gen.erdos_renyi(500, 200, 9.0, 6)))
    out.append(("er4096", gen.erdos_renyi(4096, 4096, 8.0, 0), None))
    out.append(("wide_cols", gen.erdos_renyi(2000, 2000, 6.0, 7), gen.erdos_renyi(2000, 40000, 30.0, 8)))
    out.append(("stencil12", gen.stencil27(12), None))
    out.append(("rmat12", gen.rmat(12, 16, seed=1), None))
    # ~289 products per row, nearly all distinct: expand-sort-fold rows by default
    out.append(("er_mid", gen.erdos_renyi(3000, 3000, 17.0, 9), None))
    # the same rows over 2^22 columns: spans too wide for the fold's words, hashed instead
    out.append(("esc_wide_span", gen.erdos_renyi(1500, 1500, 17.0, 10), gen.erdos_renyi(1500, 1 << 22, 17.0, 11)))
    return [(n, a, a if b is None else b) for n, a, b in out]
