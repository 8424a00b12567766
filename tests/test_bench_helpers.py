"""bench.py's host-side helpers (no GPU): the CPU baseline repeats whole
passes when the workload is shorter than its sample time, the parity sample
flags a changed value and a changed structure, and the scipy reference
reports a positive rate."""
import numpy as np

import bench
from oracle import oracle
from rtspmspm_b200 import gen


def test_cpu_sample_repeats_short_workloads():
    A = gen.stencil27(12, seed=0)
    v, info = bench.cpu_sample(A, 0.3)
    assert v > 0 and info["rows"] == A.rows and info["passes"] > 1 and info["seconds"] >= 0.3
    assert info["products"] == int(gen.row_products(A, A).sum()) * info["passes"]
    assert bench.sample_text(info, "x").startswith(f"{info['passes']} passes over all {A.rows} rows")


def test_cpu_sample_takes_leading_rows_of_long_workloads():
    A = gen.rmat(13, 16, seed=2)
    v, info = bench.cpu_sample(A, 0.01)
    assert v > 0 and info["passes"] == 1 and info["rows"] <= A.rows
    assert bench.sample_text(info, "x").startswith("leading")


def test_parity_sample_flags_changes():
    A = gen.stencil27(14, seed=1)
    R = oracle.spgemm(A, A)
    rp = R.row_ptr.astype(np.int32)
    ok = bench.parity_sample(A, rp, R.col_idx, R.val, 1000, 1200)
    assert ok["structure_exact"] and ok["bit_exact_fp32"] and ok["max_rel_err_vs_sum_abs"] == 0.0
    assert ok["nnz"] == int(R.row_ptr[1200] - R.row_ptr[1000])
    # one value moved by one ulp (planted in the oracle's own output)
    val = R.val.copy()
    i = int(R.row_ptr[1100])
    val[i] = np.nextafter(val[i], np.float32(np.inf))
    off = bench.parity_sample(A, rp, R.col_idx, val, 1000, 1200)
    assert off["structure_exact"] and not off["bit_exact_fp32"]
    assert 0.0 < off["max_rel_err_vs_sum_abs"] < 1e-5
    # one column changed: the structure check fails
    col = R.col_idx.copy()
    col[i] = col[i] + 1 if col[i] + 1 < A.cols else col[i] - 1
    bad = bench.parity_sample(A, rp, col, R.val, 1000, 1200)
    assert not bad["structure_exact"] and "bit_exact_fp32" not in bad


def test_scipy_sample():
    A = gen.erdos_renyi(3000, 3000, 8.0, 3)
    out = bench.scipy_sample(A, 0.05)
    assert out is not None
    rate, rows, secs = out
    assert rate > 0 and 1 <= rows <= A.rows and secs > 0
