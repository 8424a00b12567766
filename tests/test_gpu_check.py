"""The FP64 check entry point (spg_check) against the oracle's own error
figures, and on a C with a planted structure error (the error planted on the
host copy of C, not in any kernel)."""
import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import Engine, gen
from rtspmspm_b200.gen import Csr

from helpers import value_errors

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algo", ["plain", "learned", "cusparse"])
@pytest.mark.parametrize("name", ["er", "stencil", "rmat"])
def test_check_matches_the_oracle_errors(name, algo):
    A = {"er": gen.erdos_renyi(3000, 3000, 8.0, 31), "stencil": gen.stencil27(16, seed=2),
         "rmat": gen.rmat(11, 16, seed=4)}[name]
    with Engine(0) as eng:
        C, _ = eng.multiply(A, A, algo=algo)
        chk = eng.check(A, A, C)
        H = C.to_host()
    R = oracle.spgemm(A, A)
    rel, mx64, mean64 = value_errors(H, R)
    assert chk["entries"] == R.nnz and chk["missing"] == 0 and chk["extra"] == 0
    # the GPU's FP64 sums differ from the oracle's FP64 twin by FP64 rounding only
    assert chk["max_abs_err_fp64"] == pytest.approx(mx64, rel=1e-6, abs=1e-12)
    assert chk["mean_abs_err_fp64"] == pytest.approx(mean64, rel=1e-6, abs=1e-12)
    assert chk["max_rel_err"] <= 1e-5


def test_check_counts_a_planted_missing_and_extra_entry():
    A = gen.erdos_renyi(500, 500, 6.0, 8)
    R = oracle.spgemm(A, A)
    rp, col, val = R.row_ptr.copy(), R.col_idx.copy(), R.val.copy()
    r = int(np.argmax(np.diff(rp)))
    s, e = int(rp[r]), int(rp[r + 1])
    # row r: its first column replaced by a column no product of the row reaches
    hit = set(col[s:e].tolist())
    free = next(j for j in range(A.cols) if j not in hit)
    cols = np.concatenate([col[s + 1:e], [free]]).astype(np.int32)
    vals = np.concatenate([val[s + 1:e], [np.float32(1.0)]]).astype(np.float32)
    order = np.argsort(cols, kind="stable")
    col[s:e], val[s:e] = cols[order], vals[order]
    bad = Csr(R.rows, R.cols, rp, col, val)
    with Engine(0) as eng:
        chk = eng.check(A, A, bad)
    assert chk["extra"] == 1
    assert chk["missing"] >= 1
