"""Matrix Market reader/writer of the C ABI, checked against the reference's
own reader/writer (cuSparse/src/util.cpp, built into oracle/_ref/) where
available, and on tricky inputs."""
import ctypes
import glob
import os

import numpy as np
import pytest

from rtspmspm_b200 import SpgError, gen, read_mtx, write_mtx
from rtspmspm_b200.gen import coo_to_csr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_UTIL = os.path.join(ROOT, "oracle", "_ref", "libref_util.so")
from oracle import reference_root

REF_DATA = os.path.join(reference_root() or "", "optixSpMSpM", "src", "data")


def ref_util():
    if not os.path.exists(REF_UTIL):
        pytest.skip("reference util not built (make -C oracle ref)")
    L = ctypes.CDLL(REF_UTIL)
    L.ref_read_coo.restype = ctypes.c_int64
    L.ref_read_coo.argtypes = [ctypes.c_char_p] + [ctypes.c_void_p] * 5
    L.ref_free.argtypes = [ctypes.c_void_p] * 3
    L.ref_write_coo.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                ctypes.c_int, ctypes.c_int, ctypes.c_int64]
    return L


def ref_read(path):
    L = ref_util()
    r, c, v = ctypes.POINTER(ctypes.c_int)(), ctypes.POINTER(ctypes.c_int)(), ctypes.POINTER(ctypes.c_float)()
    nr, nc = ctypes.c_int(), ctypes.c_int()
    n = L.ref_read_coo(path.encode(), ctypes.byref(r), ctypes.byref(c), ctypes.byref(v), ctypes.byref(nr),
                       ctypes.byref(nc))
    assert n >= 0
    rr = np.ctypeslib.as_array(r, (n,)).copy() if n else np.zeros(0, np.int32)
    cc = np.ctypeslib.as_array(c, (n,)).copy() if n else np.zeros(0, np.int32)
    vv = np.ctypeslib.as_array(v, (n,)).copy() if n else np.zeros(0, np.float32)
    L.ref_free(r, c, v)
    return nr.value, nc.value, rr, cc, vv


def test_roundtrip(tmp_path):
    A = gen.erdos_renyi(300, 200, 5.0, 3)
    p = str(tmp_path / "a.mtx")
    write_mtx(p, A)
    B = read_mtx(p)
    assert (B.rows, B.cols) == (A.rows, A.cols)
    np.testing.assert_array_equal(B.row_ptr, A.row_ptr)
    np.testing.assert_array_equal(B.col_idx, A.col_idx)
    np.testing.assert_array_equal(B.val, A.val)  # shortest round-trip decimal


def test_writer_matches_reference_reader(tmp_path):
    A = gen.rmat(9, 8, seed=1)
    p = str(tmp_path / "a.mtx")
    write_mtx(p, A)
    nr, nc, r, c, v = ref_read(p)
    assert (nr, nc) == (A.rows, A.cols)
    B = coo_to_csr(nr, nc, r - 1, c - 1, v)
    np.testing.assert_array_equal(B.row_ptr, A.row_ptr)
    np.testing.assert_array_equal(B.col_idx, A.col_idx)
    np.testing.assert_array_equal(B.val, A.val)


def test_reader_matches_reference_on_reference_writer_output(tmp_path):
    L = ref_util()
    rng = np.random.default_rng(5)
    r = rng.integers(1, 51, 400).astype(np.int32)
    c = rng.integers(1, 41, 400).astype(np.int32)
    keep = np.unique(r.astype(np.int64) * 100 + c, return_index=True)[1]
    r, c = r[keep], c[keep]
    v = rng.standard_normal(r.size).astype(np.float32)
    p = str(tmp_path / "ref.mtx")
    L.ref_write_coo(p.encode(), r.ctypes.data, c.ctypes.data, v.ctypes.data, 50, 40, r.size)
    ours = read_mtx(p)
    nr, nc, rr, cc, vv = ref_read(p)
    ref = coo_to_csr(nr, nc, rr - 1, cc - 1, vv)
    np.testing.assert_array_equal(ours.row_ptr, ref.row_ptr)
    np.testing.assert_array_equal(ours.col_idx, ref.col_idx)
    np.testing.assert_array_equal(ours.val, ref.val)


@pytest.mark.skipif(not os.path.isdir(REF_DATA), reason="reference fixtures not present")
@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(REF_DATA, "*", "*_small.mtx"))))
def test_reads_reference_fixtures_like_reference(path):
    """Column-major, 1-based SuiteSparse subsets: same entries as the reference reader."""
    ours = read_mtx(path)
    nr, nc, r, c, v = ref_read(path)
    ref = coo_to_csr(nr, nc, r - 1, c - 1, v, merge="sum")
    assert (ours.rows, ours.cols) == (ref.rows, ref.cols)
    np.testing.assert_array_equal(ours.row_ptr, ref.row_ptr)
    np.testing.assert_array_equal(ours.col_idx, ref.col_idx)
    np.testing.assert_allclose(ours.val, ref.val, rtol=1e-6)


def test_symmetric_pattern_comments_duplicates(tmp_path):
    p = tmp_path / "s.mtx"
    p.write_text("%%MatrixMarket matrix coordinate pattern symmetric\n% comment\n\n4 4 4\n1 1\n3 1\n4 2\n3 1\n")
    m = read_mtx(str(p))
    d = m.to_scipy().toarray()
    want = np.zeros((4, 4))
    want[0, 0] = 1
    want[2, 0] = want[0, 2] = 2  # the duplicate (3,1) is summed, then mirrored
    want[3, 1] = want[1, 3] = 1
    np.testing.assert_array_equal(d, want)


def test_unsorted_real_general_sorted_on_read(tmp_path):
    p = tmp_path / "u.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n3 3 4\n3 3 1.5\n1 2 -2\n1 1 +3e0\n2 3 .25\n")
    m = read_mtx(str(p))
    np.testing.assert_array_equal(m.row_ptr, [0, 2, 3, 4])
    np.testing.assert_array_equal(m.col_idx, [0, 1, 2, 2])
    np.testing.assert_array_equal(m.val, np.array([3, -2, 0.25, 1.5], np.float32))


@pytest.mark.parametrize("text,status", [
    ("%%MatrixMarket matrix array real general\n2 2\n1\n2\n3\n4\n", 5),
    ("%%MatrixMarket matrix coordinate real general\n2 2 3\n1 1 1\n2 2 2\n", 5),   # truncated
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n3 1 1\n", 5),          # out of range
    ("%%MatrixMarket matrix coordinate real general\n2 2 1\n1 x 1\n", 5),          # garbage
])
def test_malformed_files_rejected(tmp_path, text, status):
    p = tmp_path / "bad.mtx"
    p.write_text(text)
    with pytest.raises(SpgError) as e:
        read_mtx(str(p))
    assert e.value.status == status


def test_missing_file():
    with pytest.raises(SpgError) as e:
        read_mtx("/nonexistent/x.mtx")
    assert e.value.status == 4


def test_drop_zeros_writer(tmp_path):
    m = coo_to_csr(2, 3, [0, 0, 1], [0, 2, 1], np.array([0.0, 1.0, 0.0], np.float32))
    p = str(tmp_path / "z.mtx")
    write_mtx(p, m, drop_zeros=True)
    lines = open(p).read().split("\n")
    assert lines[1] == "2 3 1" and lines[2] == "1 3 1"
    write_mtx(p, m)
    assert open(p).read().split("\n")[1] == "2 3 3"


def _lines(r, c, v):
    return "".join(f"{i + 1} {j + 1} {x:g}\n" for i, j, x in zip(r, c, v))


def test_large_shuffled_file_parsed_in_slices(tmp_path):
    """A body of several MB is parsed in newline-aligned slices on all host
    threads: shuffled order, duplicates summed in file order, comment and
    blank lines inside the body, extra lines past the header's count."""
    rng = np.random.default_rng(5)
    n, m = 3000, 900_000
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    v = rng.integers(-8, 9, m).astype(np.float32)  # small integers: every FP32 sum is exact
    body = _lines(r, c, v)
    cut = len(body) // 2
    cut = body.index("\n", cut) + 1
    text = ("%%MatrixMarket matrix coordinate real general\n% head comment\n"
            f"{n} {n} {m}\n" + body[:cut] + "% mid comment\n\n" + body[cut:] + "1 1 99\n2 2 99\n")
    p = tmp_path / "big.mtx"
    p.write_text(text)
    assert p.stat().st_size > 2 * (4 << 20)  # at least two 4 MB slices
    got = read_mtx(str(p))
    want = coo_to_csr(n, n, r, c, v, merge="sum")
    np.testing.assert_array_equal(got.row_ptr, want.row_ptr)
    np.testing.assert_array_equal(got.col_idx, want.col_idx)
    np.testing.assert_array_equal(got.val, want.val)


def test_symmetric_file_in_slices_and_truncated_body(tmp_path):
    rng = np.random.default_rng(6)
    n, m = 2000, 400_000
    r = rng.integers(0, n, m)
    c = rng.integers(0, n, m)
    lo, hi = np.minimum(r, c), np.maximum(r, c)
    v = rng.integers(1, 5, m).astype(np.float32)
    p = tmp_path / "sym.mtx"
    p.write_text(f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {m}\n" + _lines(hi, lo, v))
    got = read_mtx(str(p))
    off = hi != lo
    want = coo_to_csr(n, n, np.concatenate([hi, lo[off]]), np.concatenate([lo, hi[off]]),
                      np.concatenate([v, v[off]]), merge="sum")
    np.testing.assert_array_equal(got.row_ptr, want.row_ptr)
    np.testing.assert_array_equal(got.col_idx, want.col_idx)
    np.testing.assert_array_equal(got.val, want.val)
    # a header promising more entries than the body holds is an error
    p.write_text(f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {m + 1}\n" + _lines(hi, lo, v))
    with pytest.raises(SpgError) as e:
        read_mtx(str(p))
    assert e.value.status == 5


def test_transpose_matches_numpy():
    from rtspmspm_b200 import transpose

    for m in (gen.erdos_renyi(300, 170, 5.0, 3), gen.rmat(9, 8, seed=4), coo_to_csr(4, 6, [], [], [])):
        t = transpose(m)
        want = m.to_scipy().T.tocsr()
        want.sort_indices()
        assert (t.rows, t.cols, t.nnz) == (m.cols, m.rows, m.nnz)
        np.testing.assert_array_equal(t.row_ptr, want.indptr)
        np.testing.assert_array_equal(t.col_idx, want.indices)
        np.testing.assert_array_equal(t.val, want.data.astype(np.float32))
        assert t.to_scipy().T.toarray().tolist() == m.to_scipy().toarray().tolist()


def test_reader_faster_than_the_reference_reader(tmp_path, capsys):
    """spg_mtx_read (newline-aligned slices parsed on all host threads, rows
    sorted in parallel) against the reference's per-line istringstream
    reader (cuSparse/src/util.cpp:9-44, built from the reference sources) on
    a ~100 MB Matrix Market file and on the reference's own fixtures.  Times
    are printed; ours must be faster."""
    import time

    ref_util()  # skips when the reference reader is not built
    A = gen.erdos_renyi(200_000, 200_000, 20.0, 17)
    big = str(tmp_path / "big.mtx")
    write_mtx(big, A)
    size_mb = os.path.getsize(big) / 1e6
    paths = [big] + sorted(glob.glob(os.path.join(REF_DATA, "*", "*_small.mtx")))
    t_ours = t_ref = 0.0
    for p in paths:
        t = time.perf_counter()
        ours = read_mtx(p)
        d_ours = time.perf_counter() - t
        t = time.perf_counter()
        nr, nc, r, c, v = ref_read(p)
        d_ref = time.perf_counter() - t
        assert ours.nnz <= r.size and (ours.rows, ours.cols) == (nr, nc)
        if p == big:
            big_ours, big_ref = d_ours, d_ref
        t_ours += d_ours
        t_ref += d_ref
    with capsys.disabled():
        print(f"\n.mtx read: {size_mb:.0f} MB file {big_ours:.2f} s (ours, {os.cpu_count()} threads) vs "
              f"{big_ref:.2f} s (reference reader); {len(paths)} files {t_ours:.2f} s vs {t_ref:.2f} s")
    assert big_ours < big_ref
