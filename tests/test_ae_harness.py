"""The AE_test-compatible profiling harness: dataset discovery, the three CSV
files, rectangular inputs run against their transpose, and the
top-left-quarter reduction after a failure (fake programs, no GPU)."""
import csv
import os
import sys

import numpy as np
import pytest

from rtspmspm_b200 import ae_harness, gen, read_mtx, write_mtx

FAKE = r'''
import sys
a = dict(zip(sys.argv[1::2], sys.argv[2::2]))
with open(a["-m1"]) as f:
    for line in f:
        if not line.startswith("%"):
            rows, cols, nnz = map(int, line.split())
            break
limit = int(sys.argv[0].rsplit("_", 1)[1].split(".")[0])
if rows > limit:
    sys.exit(1)
open(a["-o"], "w").write("%%MatrixMarket matrix coordinate real general\n0 0 0\n")
open(a["-l"], "w").write(str(0.5 + rows / 1000.0))
'''


def fake_program(tmp_path, limit):
    p = tmp_path / f"fake_{limit}.py"
    p.write_text(FAKE)
    return [sys.executable, str(p)]


@pytest.fixture
def data_dir(tmp_path):
    d = tmp_path / "data"
    (d / "sq").mkdir(parents=True)
    write_mtx(str(d / "sq" / "sq.mtx"), gen.erdos_renyi(1500, 1500, 3.0, 1))
    write_mtx(str(d / "rect.mtx"), gen.erdos_renyi(1200, 900, 3.0, 2))
    write_mtx(str(d / "big.mtx"), gen.erdos_renyi(5000, 5000, 2.0, 3))
    return d


def rows_of(path):
    with open(path) as f:
        return list(csv.reader(f))


def test_discovery_prefers_nested_files(data_dir):
    found = ae_harness.discover(str(data_dir))
    assert set(found) == {"sq", "rect", "big"}
    assert found["sq"].endswith(os.path.join("sq", "sq.mtx"))


def test_csv_contract_transpose_and_reduction(tmp_path, data_dir):
    out = tmp_path / "result"
    progs = {"cuSparse": fake_program(tmp_path, 10 ** 9), "ours": fake_program(tmp_path, 3000)}
    used, failed = ae_harness.profile(str(data_dir), str(out), progs, runs=3, log=lambda *a: None)
    assert failed == []
    # "big" (5000 rows) failed for `ours` and ran reduced to 2500 x 2500
    assert used["big"].endswith("big_small.mtx")
    small = read_mtx(used["big"])
    assert (small.rows, small.cols) == (2500, 2500)
    B = read_mtx(str(data_dir / "big.mtx"))
    r = np.repeat(np.arange(B.rows), np.diff(B.row_ptr))
    assert small.nnz == int(((r < 2500) & (B.col_idx < 2500)).sum())
    # the rectangular dataset ran against its transpose
    T = read_mtx(str(out / "rect" / "result" / "rect_transpose.mtx"))
    R = read_mtx(str(data_dir / "rect.mtx"))
    assert (T.rows, T.cols, T.nnz) == (R.cols, R.rows, R.nnz)
    allr = rows_of(out / "all_result.csv")
    assert allr[0] == ["Software", "DataSet", "Scenario", "Runtime(ms)"]
    body = [r for r in allr[1:] if r]
    assert len(body) == 3 * 2 * 3
    assert {r[2].strip() for r in body} == {"run0", "run1", "run2"}
    avg = rows_of(out / "avg_result.csv")
    assert avg[0] == ["Software", "DataSet", "Runtime(ms)"] and len(avg) == 1 + 6
    fin = rows_of(out / "final_result.csv")
    assert fin[0] == ["DataSet", "cuSparse", "ours", "Speedup (cuSparse / ours)"]
    by = {r[0]: r for r in fin[1:]}
    assert float(by["big"][3]) == pytest.approx(1.0)
    assert float(by["sq"][1]) == pytest.approx(0.5 + 1.5)


def test_unreducible_failure_is_reported(tmp_path, data_dir):
    out = tmp_path / "result2"
    progs = {"base": fake_program(tmp_path, 10 ** 9), "tiny": fake_program(tmp_path, 10)}
    used, failed = ae_harness.profile(str(data_dir), str(out), progs, runs=1, log=lambda *a: None)
    assert sorted(failed) == ["big", "rect", "sq"] and not used


def test_cli_arguments(tmp_path, data_dir):
    out = tmp_path / "r3"
    prog = " ".join(fake_program(tmp_path, 10 ** 9))
    rc = ae_harness.main(["--data-dir", str(data_dir), "--out-dir", str(out), "--runs", "1",
                          "--program", f"a={prog}", "--program", f"b={prog}", "--baseline", "b"])
    assert rc == 0
    assert rows_of(out / "final_result.csv")[0] == ["DataSet", "b", "a", "Speedup (b / a)"]
