"""C = A*B delivered into caller host buffers with the download overlapped
with the product (spg_multiply_into_host): bit-exact against the oracle for
every block count and index width, capacity errors report the size needed,
and A = B given once is uploaded once."""
import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import SpgError, gen

from cases import heavy_row
from helpers import assert_parity
from rtspmspm_b200.gen import Csr

pytestmark = pytest.mark.gpu


def host_buffers(rows, cap, bits, pinned):
    import torch

    rp = torch.zeros(rows + 1, dtype=torch.int32 if bits == 32 else torch.int64)
    col = torch.zeros(cap, dtype=torch.int32)
    val = torch.zeros(cap, dtype=torch.float32)
    if pinned:
        rp, col, val = rp.pin_memory(), col.pin_memory(), val.pin_memory()
    return rp, col, val


def as_csr(rows, cols, rp, col, val, nnz):
    return Csr(rows, cols, rp.numpy().astype(np.int64), col.numpy()[:nnz].copy(), val.numpy()[:nnz].copy())


@pytest.mark.parametrize("algo", ["plain", "learned"])
@pytest.mark.parametrize("blocks", [1, 3, 8])
@pytest.mark.parametrize("bits", [32, 64])
def test_into_host_matches_oracle(engine, algo, blocks, bits):
    A = gen.stencil27(14, seed=2)
    R = oracle.spgemm(A, A)
    rp, col, val = host_buffers(A.rows, R.nnz + 5, bits, pinned=blocks != 3)
    nnz, rep = engine.multiply_into_host(A, A, rp, col, val, blocks=blocks, index_bits=bits, algo=algo)
    assert nnz == R.nnz and rep["nnz_c"] == R.nnz
    assert rep["products"] == int(gen.row_products(A, A).sum())
    assert_parity(as_csr(A.rows, A.cols, rp, col, val, nnz), R)


def test_into_host_rectangular_and_heavy(engine):
    for A, B in ((gen.erdos_renyi(700, 400, 6.0, 3), gen.erdos_renyi(400, 900, 5.0, 4)), (heavy_row(), None)):
        B = A if B is None else B
        R = oracle.spgemm(A, B)
        rp, col, val = host_buffers(A.rows, R.nnz, 64, pinned=True)
        nnz, _ = engine.multiply_into_host(A, B, rp, col, val, blocks=5, algo="plain")
        assert_parity(as_csr(A.rows, B.cols, rp, col, val, nnz), R)


def test_into_host_capacity_too_small(engine):
    A = gen.erdos_renyi(500, 500, 6.0, 7)
    R = oracle.spgemm(A, A)
    rp, col, val = host_buffers(A.rows, R.nnz - 1, 64, pinned=False)
    with pytest.raises(SpgError) as e:
        engine.multiply_into_host(A, A, rp, col, val, blocks=4, algo="plain")
    assert e.value.status == 1
    assert "needs room for %d" % R.nnz in str(e.value)
    # the engine stays usable
    rp, col, val = host_buffers(A.rows, R.nnz, 64, pinned=False)
    nnz, _ = engine.multiply_into_host(A, A, rp, col, val, blocks=4, algo="plain")
    assert_parity(as_csr(A.rows, A.cols, rp, col, val, nnz), R)


def test_into_host_empty_rows_and_more_blocks_than_rows(engine):
    A = gen.erdos_renyi(5, 5, 2.0, 1)
    R = oracle.spgemm(A, A)
    rp, col, val = host_buffers(A.rows, max(R.nnz, 1), 64, pinned=False)
    nnz, _ = engine.multiply_into_host(A, A, rp, col, val, blocks=64, algo="plain")
    assert_parity(as_csr(A.rows, A.cols, rp, col, val, nnz), R)


@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_into_host_chunked_upload(engine, algo):
    """A = B from host memory with validation off goes up in row chunks
    beside the compute: a banded matrix (each block waits for the next chunk
    or two), a product with heavy rows whose blocked index reads every row of
    B (it waits for the whole upload), and a random matrix (every block
    reaches the last chunk) all match the oracle."""
    cases = [(gen.stencil27(16, seed=4), {}), (gen.erdos_renyi(3000, 3000, 6.0, 13), {}),
             (heavy_row(), {"warp_table_max": 64, "block_table_max": 1024, "block_min_nnz": -1, "small_rows": -1})]
    for A, tune in cases:
        saved = engine.get_tuning()
        if tune:
            engine.set_tuning(**tune)
        try:
            R = oracle.spgemm(A, A)
            for pinned in (True, False):
                rp, col, val = host_buffers(A.rows, R.nnz, 64, pinned=pinned)
                nnz, rep = engine.multiply_into_host(A, A, rp, col, val, blocks=7, algo=algo, skip_validation=True,
                                                     use_tuning=bool(tune))
                assert nnz == R.nnz
                assert_parity(as_csr(A.rows, A.cols, rp, col, val, nnz), R)
            if tune:
                assert rep["rows_heavy"] > 0
        finally:
            engine.set_tuning(**saved)
