"""Full-size workloads: the stencil 96^3 product compared whole with the
oracle, and the R-MAT scale-20 product (about 7e9 output entries, too large
for host memory) checked on sampled rows -- the heaviest ones included --
plus size-independent properties."""
import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import DeviceCsr, Engine, gen

from helpers import assert_parity

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_stencil96_full(eng, algo):
    A = gen.stencil27(96, seed=0)
    dA = DeviceCsr.from_host(A)
    C, rep = eng.multiply(dA, dA, algo=algo)
    assert rep["nnz_c"] == (5 * 96 - 6) ** 3 and rep["products"] == (9 * 96 - 10) ** 3
    R = oracle.spgemm(A, A, twin=False)
    H = C.to_host()
    C.free()
    np.testing.assert_array_equal(H.row_ptr, R.row_ptr)
    np.testing.assert_array_equal(H.col_idx, R.col_idx)
    np.testing.assert_array_equal(H.val.view(np.uint32), R.val.view(np.uint32))


def test_rmat20_sampled_rows(eng):
    A = gen.rmat(20, 16, seed=0)
    prod = gen.row_products(A, A)
    rng = np.random.default_rng(0)
    sel = np.unique(np.concatenate([np.argsort(prod)[-64:], rng.choice(A.rows, 1500, replace=False)]))
    R = oracle.rows(A, A, sel)
    dA = DeviceCsr.from_host(A)
    for algo in ("plain", "learned"):
        C, rep = eng.multiply(dA, dA, algo=algo)
        assert rep["device_flags"] == 0 and rep["products"] == int(prod.sum())
        assert C.s.index_bits == 64 and rep["nnz_c"] > 2 ** 31   # needs 64-bit row pointers
        got = C.rows_to_host(sel)
        C.free()
        assert_parity(got, R)
