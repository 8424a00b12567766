"""COO -> CSR on the GPU (spg_coo_to_csr) and the Matrix Market reader that
builds its CSR there (spg_mtx_read_device): sorted columns, duplicates
summed in the order given, bit for bit against a numpy restatement and
against the host reader."""
import numpy as np
import pytest

from rtspmspm_b200 import Engine, SpgError
from rtspmspm_b200.engine import read_mtx

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = Engine(0)
    yield e
    e.close()


def coo_reference(rows, r, c, v):
    """CSR of COO entries: stable order by (row, column), each run of equal
    pairs folded left to right in FP32."""
    order = np.lexsort((c, r))  # stable: equal pairs keep their input order
    r, c, v = r[order], c[order], v[order]
    head = np.ones(len(r), bool)
    head[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
    starts = np.flatnonzero(head)
    ends = np.append(starts[1:], len(r))
    out_v = v[starts].copy()
    for i in np.flatnonzero(ends - starts > 1):
        s = v[starts[i]]
        for q in range(starts[i] + 1, ends[i]):
            s = np.float32(s + v[q])
        out_v[i] = s
    rp = np.zeros(rows + 1, np.int64)
    np.add.at(rp, r[starts] + 1, 1)
    return np.cumsum(rp), c[starts].astype(np.int32), out_v


def check(H, rows, r, c, v):
    rp, col, val = coo_reference(rows, r, c, v)
    assert np.array_equal(H.row_ptr, rp)
    assert np.array_equal(H.col_idx, col)
    assert np.array_equal(H.val.view(np.uint32), val.view(np.uint32))


def random_coo(rows, cols, n, dup, seed):
    g = np.random.default_rng(seed)
    r = g.integers(0, rows, n).astype(np.int32)
    c = g.integers(0, cols, n).astype(np.int32)
    k = int(n * dup)
    pick = g.integers(0, n, k)  # repeated pairs with new values, placed anywhere
    r = np.concatenate([r, r[pick]])
    c = np.concatenate([c, c[pick]])
    perm = g.permutation(len(r))
    v = g.uniform(-1, 1, len(r)).astype(np.float32)
    return r[perm], c[perm], v


@pytest.mark.parametrize("rows,cols,n,dup", [(1000, 1500, 20000, 0.3), (7, 3, 200, 2.0), (1, 1, 50, 1.0),
                                             (300, 70000, 5000, 0.1)])
def test_coo_to_csr_matches_reference(eng, rows, cols, n, dup):
    r, c, v = random_coo(rows, cols, n, dup, seed=rows + n)
    C = eng.coo_to_csr(rows, cols, r, c, v)
    check(C.to_host(), rows, r, c, v)


def test_coo_to_csr_large(eng):
    """2^21 entries over 2^20 x 2^20 (three row and three column passes),
    each repeated pair at most twice."""
    g = np.random.default_rng(5)
    n = 1 << 21
    key = np.unique(g.integers(0, 1 << 40, n))
    r = (key >> 20).astype(np.int32)
    c = (key & ((1 << 20) - 1)).astype(np.int32)
    pick = g.choice(len(r), len(r) // 4, replace=False)
    r = np.concatenate([r, r[pick]])
    c = np.concatenate([c, c[pick]])
    perm = g.permutation(len(r))
    r, c = r[perm], c[perm]
    v = g.standard_normal(len(r)).astype(np.float32)
    C = eng.coo_to_csr(1 << 20, 1 << 20, r, c, v)
    check(C.to_host(), 1 << 20, r, c, v)


def test_coo_to_csr_device_inputs_and_edges(eng):
    import torch

    r, c, v = random_coo(500, 400, 8000, 0.5, seed=9)
    tr, tc, tv = (torch.from_numpy(x).cuda() for x in (r, c, v))
    C = eng.coo_to_csr(500, 400, tr, tc, tv)
    check(C.to_host(), 500, r, c, v)
    # no entries; no rows
    E = eng.coo_to_csr(12, 5, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)).to_host()
    assert E.nnz == 0 and np.array_equal(E.row_ptr, np.zeros(13, np.int64))
    Z = eng.coo_to_csr(0, 5, np.zeros(0, np.int32), np.zeros(0, np.int32), np.zeros(0, np.float32)).to_host()
    assert Z.rows == 0 and Z.nnz == 0
    # an entry outside the shape is rejected and the context stays usable
    with pytest.raises(SpgError) as e:
        eng.coo_to_csr(10, 10, np.array([3, 10], np.int32), np.array([1, 1], np.int32), np.ones(2, np.float32))
    assert e.value.status == 1
    with pytest.raises(SpgError):
        eng.coo_to_csr(10, 10, np.array([3, 2], np.int32), np.array([1, -1], np.int32), np.ones(2, np.float32))
    C = eng.coo_to_csr(500, 400, r, c, v)
    check(C.to_host(), 500, r, c, v)


def write_mtx(path, rows, cols, r, c, v, kind="real general"):
    with open(path, "w") as f:
        f.write(f"%%MatrixMarket matrix coordinate {kind}\n% generated\n{rows} {cols} {len(r)}\n")
        if "pattern" in kind:
            f.writelines(f"{a + 1} {b + 1}\n" for a, b in zip(r, c))
        else:
            f.writelines(f"{a + 1} {b + 1} {x!r}\n" for a, b, x in zip(r, c, v.tolist()))


@pytest.mark.parametrize("kind", ["real general", "real symmetric", "pattern general", "integer general"])
def test_read_mtx_device_matches_host_reader(eng, tmp_path, kind):
    g = np.random.default_rng(11)
    r, c, v = random_coo(3000, 3000, 60000, 0.2, seed=12)
    if "symmetric" in kind:  # lower triangle only, as symmetric files store it
        keep = r >= c
        r, c, v = r[keep], c[keep], v[keep]
    if "integer" in kind:
        v = g.integers(-50, 50, len(r)).astype(np.float32)
    # column-major file order, as the reference's fixtures come
    order = np.lexsort((r, c))
    r, c, v = r[order], c[order], v[order]
    p = str(tmp_path / "m.mtx")
    write_mtx(p, 3000, 3000, r, c, v, kind)
    H = read_mtx(p)
    D = eng.read_mtx_device(p).to_host()
    assert np.array_equal(D.row_ptr, H.row_ptr)
    assert np.array_equal(D.col_idx, H.col_idx)
    assert np.array_equal(D.val.view(np.uint32), H.val.view(np.uint32))
