"""Comparison helpers shared by the parity tests (oracle = checker only)."""
import numpy as np

# Values: FP32 in the canonical order, so the engine must match the FP32
# oracle bit for bit; the contract's bound is |c - c_oracle| <= 1e-5 * sum|a*b|.
REL_TOL = 1e-5


def assert_same_structure(C, R):
    assert C.rows == R.rows and C.cols == R.cols
    np.testing.assert_array_equal(np.asarray(C.row_ptr, dtype=np.int64), np.asarray(R.row_ptr, dtype=np.int64))
    np.testing.assert_array_equal(np.asarray(C.col_idx, dtype=np.int32), np.asarray(R.col_idx, dtype=np.int32))


def value_errors(C, R):
    """(max rel err vs FP32 oracle / bound, max and mean abs err vs FP64)."""
    c = np.asarray(C.val, dtype=np.float64)
    bound = np.maximum(R.bound, np.finfo(np.float64).tiny)
    rel = np.abs(c - R.val.astype(np.float64)) / bound
    e64 = np.abs(c - R.val64)
    return (float(rel.max()) if rel.size else 0.0, float(e64.max()) if e64.size else 0.0,
            float(e64.mean()) if e64.size else 0.0)


def assert_parity(C, R, bit_exact=True):
    assert_same_structure(C, R)
    rel, _, _ = value_errors(C, R)
    assert rel <= REL_TOL, f"relative error {rel} > {REL_TOL}"
    if bit_exact:
        mism = np.flatnonzero(np.asarray(C.val, np.float32).view(np.uint32) != R.val.view(np.uint32))
        assert mism.size == 0, f"{mism.size} values differ from the FP32 oracle (first at {mism[:5]})"
