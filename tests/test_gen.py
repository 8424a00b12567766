"""Synthetic workload generators: shapes, known sizes, determinism."""
import numpy as np

from rtspmspm_b200 import gen


def test_stencil_sizes():
    # per dimension: sum of squared neighbour counts 9g-10, distance-2 counts 5g-6
    from oracle import oracle

    for g in (4, 8, 17):
        A = gen.stencil27(g)
        assert A.rows == g ** 3 and A.nnz == (3 * g - 2) ** 3
        assert int(gen.row_products(A, A).sum()) == (9 * g - 10) ** 3
        assert oracle.spgemm(A, A, twin=False).nnz == (5 * g - 6) ** 3
    A = gen.stencil27(8, seed=0)
    d = A.to_scipy().diagonal()
    off = np.abs(A.to_scipy()).sum(1).A1 - np.abs(d)
    np.testing.assert_allclose(d, 26 + off, rtol=1e-6)


def test_stencil96_headline_sizes():
    # sizes quoted for the benchmark workload, from the closed forms
    g = 96
    assert (3 * g - 2) ** 3 == 23393656
    assert (9 * g - 10) ** 3 == 622835864
    assert (5 * g - 6) ** 3 == 106496424


def test_er_poisson_mean_and_determinism():
    A = gen.erdos_renyi(4096, 4096, 8.0, 0)
    B = gen.erdos_renyi(4096, 4096, 8.0, 0)
    assert np.array_equal(A.col_idx, B.col_idx) and np.array_equal(A.val, B.val)
    assert 7.8 < A.nnz / A.rows < 8.1
    assert A.val.min() >= -1 and A.val.max() <= 1
    for r in range(0, 4096, 97):
        c = A.col_idx[A.row_ptr[r]:A.row_ptr[r + 1]]
        assert np.all(np.diff(c) > 0)


def test_rmat_skew_and_dedup():
    A = gen.rmat(12, 16, seed=0)
    assert A.rows == 4096 and A.nnz <= 16 * 4096
    lens = A.row_lengths()
    assert lens[:16].mean() > 10 * lens.mean()   # low ids are the heavy ones
    key = np.repeat(np.arange(A.rows), lens) * A.cols + A.col_idx
    assert np.unique(key).size == key.size
    assert A.val.min() >= 0 and A.val.max() < 1


def test_batch_recipe():
    pairs = gen.batch_uneven(count=6, seed=1)
    assert len(pairs) == 6
    for A, B in pairs:
        assert A.cols == B.rows
        for d in (A.rows, A.cols, B.cols):
            assert 1024 <= d <= 65536
    again = gen.batch_uneven(count=6, seed=1)
    assert all(np.array_equal(a.col_idx, b.col_idx) for (a, _), (b, _) in zip(pairs, again))
