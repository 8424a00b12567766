"""Loads the golden fixtures made by tests/golden/make_golden.py."""
import glob
import os

import numpy as np

from rtspmspm_b200.gen import Csr

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
# the reference prints values with 6 significant digits
PRINT_REL = 5e-6


def cases():
    out = []
    for path in sorted(glob.glob(os.path.join(HERE, "*.npz"))):
        z = np.load(path)
        A = Csr(int(z["a_shape"][0]), int(z["a_shape"][1]), z["a_rp"], z["a_col"], z["a_val"])
        B = Csr(int(z["b_shape"][0]), int(z["b_shape"][1]), z["b_rp"], z["b_col"], z["b_val"])
        C = Csr(A.rows, B.cols, z["c_rp"], z["c_col"], z["c_val"])
        out.append((os.path.basename(path)[:-4], A, B, C))
    return out


def assert_matches_reference(got, ref, bound):
    """Structure exact; values within the 1e-5 * sum|a*b| contract plus the
    reference's print rounding."""
    np.testing.assert_array_equal(np.asarray(got.row_ptr, np.int64), np.asarray(ref.row_ptr, np.int64))
    np.testing.assert_array_equal(np.asarray(got.col_idx, np.int32), np.asarray(ref.col_idx, np.int32))
    g = np.asarray(got.val, np.float64)
    r = np.asarray(ref.val, np.float64)
    tol = 1e-5 * bound + PRINT_REL * np.abs(r) + 1e-30
    bad = np.flatnonzero(np.abs(g - r) > tol)
    assert bad.size == 0, f"{bad.size} values off, first {bad[:5]}: {g[bad[:5]]} vs {r[bad[:5]]}"
