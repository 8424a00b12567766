"""The spgemm CLI: same flags and contract as the reference executables
(-m1 -m2 -o -l; one ms number in the log; exit 1 on failure)."""
import json
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import gen, read_mtx, write_mtx

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "rtspmspm_b200", "spgemm")


def test_help_and_bad_flags_exit_1():
    r = subprocess.run([CLI, "-h"], capture_output=True, text=True)
    assert r.returncode == 1 and "--mat1" in r.stderr
    r = subprocess.run([CLI, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1


def test_missing_input_exit_1(tmp_path):
    r = subprocess.run([CLI, "-m1", str(tmp_path / "none.mtx")], capture_output=True, text=True)
    assert r.returncode == 1


@pytest.mark.gpu
@pytest.mark.parametrize("algo", ["plain", "learned", "cusparse"])
def test_cli_end_to_end(tmp_path, algo):
    A = gen.erdos_renyi(700, 500, 6.0, 8)
    B = gen.erdos_renyi(500, 400, 5.0, 9)
    pa, pb, pc, pl, pj = (str(tmp_path / n) for n in ("a.mtx", "b.mtx", "c.mtx", "log.txt", "r.json"))
    write_mtx(pa, A)
    write_mtx(pb, B)
    r = subprocess.run([CLI, "-m1", pa, "-m2", pb, "-o", pc, "-l", pl, "--algo", algo, "--json", pj, "--check"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    ms = float(open(pl).read())
    assert ms > 0
    rep = json.load(open(pj))
    assert rep["products"] == int(gen.row_products(A, B).sum())
    # the per-result error report of --check (FP64 recomputation on the GPU)
    chk = rep["check"]
    assert chk["missing"] == 0 and chk["extra"] == 0 and chk["max_rel_err"] <= 1e-5
    assert "check vs FP64" in r.stderr
    C = read_mtx(pc)
    R = oracle.spgemm(A, B)
    np.testing.assert_array_equal(C.row_ptr, R.row_ptr)
    np.testing.assert_array_equal(C.col_idx, R.col_idx)
    if algo != "cusparse":
        np.testing.assert_array_equal(C.val, R.val)  # shortest round-trip decimals


@pytest.mark.gpu
def test_cli_transpose_m2(tmp_path):
    """C = A * A^T for a rectangular A read once (--transpose-m2)."""
    from rtspmspm_b200 import transpose

    A = gen.erdos_renyi(600, 900, 5.0, 12)
    pa, pc, pl = (str(tmp_path / n) for n in ("a.mtx", "c.mtx", "log.txt"))
    write_mtx(pa, A)
    r = subprocess.run([CLI, "-m1", pa, "-m2", pa, "--transpose-m2", "-o", pc, "-l", pl, "--algo", "plain"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    C = read_mtx(pc)
    R = oracle.spgemm(A, transpose(A))
    assert (C.rows, C.cols) == (600, 600)
    np.testing.assert_array_equal(C.row_ptr, R.row_ptr)
    np.testing.assert_array_equal(C.col_idx, R.col_idx)
    np.testing.assert_array_equal(C.val, R.val)


@pytest.mark.gpu
def test_ae_harness_with_the_cli(tmp_path):
    """The AE_test-compatible harness driving the real CLI (cuSPARSE vs the
    learned method): CSV files written, square and rectangular datasets."""
    import csv

    from rtspmspm_b200 import ae_harness

    d = tmp_path / "data"
    (d / "sq").mkdir(parents=True)
    write_mtx(str(d / "sq" / "sq.mtx"), gen.erdos_renyi(1200, 1200, 5.0, 3))
    write_mtx(str(d / "rect.mtx"), gen.erdos_renyi(1500, 900, 4.0, 4))
    out = tmp_path / "result"
    used, failed = ae_harness.profile(str(d), str(out), ae_harness.default_programs(), runs=2, log=lambda *a: None)
    assert failed == [] and set(used) == {"sq", "rect"}
    rows = list(csv.reader(open(out / "final_result.csv")))
    assert rows[0] == ["DataSet", "cuSparse", "spgemm", "Speedup (cuSparse / spgemm)"]
    assert all(float(r[3]) > 0 for r in rows[1:])
    # the rectangular product ran against the transpose and matches the oracle
    from rtspmspm_b200 import transpose

    R = read_mtx(str(d / "rect.mtx"))
    C = read_mtx(str(out / "rect" / "result" / "spgemm.mtx"))
    want = oracle.spgemm(R, transpose(R))
    np.testing.assert_array_equal(C.row_ptr, want.row_ptr)
    np.testing.assert_array_equal(C.col_idx, want.col_idx)
