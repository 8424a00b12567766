"""CPU oracle pinned against the reference's own outputs and known answers."""
import numpy as np
import pytest
import scipy.sparse as sp

from oracle import oracle
from rtspmspm_b200 import gen

from cases import cancelling, dense_ones, empty, heavy_row, identity, permutation, with_empty_rows_cols
from golden_util import assert_matches_reference, cases as golden_cases

GOLDEN = golden_cases()


def test_golden_fixtures_present():
    assert len(GOLDEN) >= 5


@pytest.mark.parametrize("name,A,B,C", GOLDEN, ids=[g[0] for g in GOLDEN])
def test_oracle_matches_reference_cusparse_driver(name, A, B, C):
    R = oracle.spgemm(A, B)
    assert_matches_reference(R, C, R.bound)


def test_identity_and_permutation():
    B = gen.erdos_renyi(100, 80, 5.0, 1)
    R = oracle.spgemm(identity(100), B)
    np.testing.assert_array_equal(R.row_ptr, B.row_ptr)
    np.testing.assert_array_equal(R.col_idx, B.col_idx)
    np.testing.assert_array_equal(R.val, B.val)
    P = permutation(100, 3)
    R = oracle.spgemm(P, B)
    perm = P.col_idx  # row i of P selects row perm[i] of B
    for i in range(100):
        s, e = B.row_ptr[perm[i]], B.row_ptr[perm[i] + 1]
        np.testing.assert_array_equal(R.col_idx[R.row_ptr[i]:R.row_ptr[i + 1]], B.col_idx[s:e])


def test_dense_ones():
    R = oracle.spgemm(dense_ones(4), dense_ones(4))
    assert R.nnz == 16 and np.all(R.val == 4.0)


def test_cancellation_keeps_structure():
    A, B = cancelling()
    R = oracle.spgemm(A, B)
    assert R.nnz == 1 and R.val[0] == 0.0 and R.bound[0] == 2.0


def test_empty_and_zero_rows():
    R = oracle.spgemm(empty(10, 12), empty(12, 7))
    assert R.nnz == 0 and R.row_ptr.size == 11
    E = with_empty_rows_cols()
    R = oracle.spgemm(E, E)
    S = (E.to_scipy().astype(np.float64) @ E.to_scipy().astype(np.float64)).tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(R.row_ptr, S.indptr)


@pytest.mark.parametrize("make", [lambda: gen.erdos_renyi(800, 600, 7.0, 9),
                                  lambda: gen.stencil27(10, seed=2), lambda: gen.rmat(10, 16, seed=3),
                                  heavy_row])
def test_structure_and_fp64_twin_vs_scipy(make):
    A = make()
    B = A if A.rows == A.cols else gen.erdos_renyi(A.cols, 300, 4.0, 5)
    R = oracle.spgemm(A, B)
    # boolean structure equals the structure of |A| |B|
    S = (abs(A.to_scipy()).astype(np.float64) @ abs(B.to_scipy()).astype(np.float64)).tocsr()
    S.sort_indices()
    np.testing.assert_array_equal(R.row_ptr, S.indptr)
    np.testing.assert_array_equal(R.col_idx, S.indices)
    np.testing.assert_allclose(R.bound, S.data, rtol=1e-12)
    # FP64 twin equals the FP64 product; FP32 within the contract of it
    D = (A.to_scipy().astype(np.float64) @ B.to_scipy().astype(np.float64)).tocsr()
    D.sort_indices()
    dense = np.zeros(R.nnz)
    # D may drop exact-zero cancellations; align by (row, col)
    keyR = np.repeat(np.arange(A.rows), np.diff(R.row_ptr)) * B.cols + R.col_idx
    keyD = np.repeat(np.arange(A.rows), np.diff(D.indptr)) * B.cols + D.indices
    pos = np.searchsorted(keyR, keyD)
    dense[pos] = D.data
    np.testing.assert_allclose(R.val64, dense, rtol=1e-12, atol=1e-12)
    assert np.all(np.abs(R.val - R.val64) <= 1e-5 * R.bound + 1e-30)


def test_row_sums_match_A_times_B_ones():
    A = gen.rmat(11, 16, seed=4)
    R = oracle.spgemm(A, A)
    rs = np.bincount(np.repeat(np.arange(A.rows), np.diff(R.row_ptr)), weights=R.val64, minlength=A.rows)
    Bs = A.to_scipy().astype(np.float64)
    np.testing.assert_allclose(rs, Bs @ (Bs @ np.ones(A.cols)), rtol=1e-10, atol=1e-12)


def test_rows_subset_matches_full():
    A = gen.erdos_renyi(2000, 2000, 10.0, 6)
    full = oracle.spgemm(A, A)
    sel = np.array([0, 5, 1999, 1000, 5])
    sub = oracle.rows(A, A, sel)
    for t, r in enumerate(sel):
        a, b = full.row_ptr[r], full.row_ptr[r + 1]
        c, d = sub.row_ptr[t], sub.row_ptr[t + 1]
        np.testing.assert_array_equal(sub.col_idx[c:d], full.col_idx[a:b])
        np.testing.assert_array_equal(sub.val[c:d].view(np.uint32), full.val[a:b].view(np.uint32))


def test_baseline_rows_counts():
    A = gen.stencil27(12)
    n, _ = oracle.baseline_rows(A, A, 0, A.rows)
    assert n == oracle.spgemm(A, A, twin=False).nnz
