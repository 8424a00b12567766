"""Parity of the CUDA engine with the CPU oracle, through the C ABI.

Structure (row_ptr, sorted col_idx) must be bit-exact; values are
accumulated in FP32 in the canonical order and must equal the FP32 oracle
bit for bit (which implies the contract bound |err| <= 1e-5 * sum|a*b|).
"""
import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import DeviceCsr, SpgError, gen

from cases import named_pairs
from helpers import assert_parity, assert_same_structure, value_errors, REL_TOL

pytestmark = pytest.mark.gpu

PAIRS = named_pairs()
_ORACLE = {}


def ref(name, A, B):
    if name not in _ORACLE:
        _ORACLE[name] = oracle.spgemm(A, B)
    return _ORACLE[name]


# tunings that push rows onto every accumulator kind
TUNINGS = {
    "default": {},
    # CTA hash bins off: rows beyond 32 entries go to the heavy-row tiles
    "tiny_tables": {"warp_table_max": 64, "block_table_max": 1024, "max_load": 0.5, "block_min_nnz": -1},
    # rows beyond 100 entries in the CTA hash bins
    "mid_tables": {"warp_table_max": 256, "block_table_max": 2048, "max_load": 0.65, "warps_per_block": 4,
                   "block_min_nnz": 100},
    # heavy rows through the staged per-tile buckets instead of the rescanning tile kernel
    "tiny_staged": {"warp_table_max": 64, "block_table_max": 1024, "max_load": 0.5, "heavy_path": 1,
                    "block_min_nnz": -1},
    # every row of more than 8 entries in a CTA hash bin
    "cta_bins": {"block_min_nnz": 8},
    # heavy rows with long B-row segments staged in shared memory by bulk copies
    "tiny_bulk": {"warp_table_max": 64, "block_table_max": 1024, "max_load": 0.5, "heavy_path": 2,
                  "block_min_nnz": -1},
    # every warp-bin row that fits its warp's memory with half or more of its products distinct
    # expanded, sorted and folded instead of hashed
    "esc_all": {"esc_min_prod": 1},
    # the same with learned capacities below the prediction: rows overflow out of the fold
    "esc_tight_caps": {"esc_min_prod": 1, "predict_margin": 0.6, "predict_slack": 0},
    # hashing only
    "esc_off": {"esc_min_prod": -1},
    # the small-product path for every case it takes (heavy_row and rmat12 fall back to the bins)
    "small": {"small_rows": 65536},
}


@pytest.mark.parametrize("tuning", list(TUNINGS))
@pytest.mark.parametrize("algo", ["plain", "learned"])
@pytest.mark.parametrize("name,A,B", PAIRS, ids=[p[0] for p in PAIRS])
def test_parity(engine, name, A, B, algo, tuning):
    engine.set_tuning(**{**{"warp_table_max": 4096, "block_table_max": 16384, "max_load": 0.5,
                            "warps_per_block": 8, "heavy_path": 0, "block_min_nnz": 0, "esc_min_prod": 0,
                            "predict_margin": 1.25, "predict_slack": 8, "small_rows": -1}, **TUNINGS[tuning]})
    C, rep = engine.multiply(A, B, algo=algo, use_tuning=True, stage_timing=True)
    R = ref(name, A, B)
    assert_parity(C.to_host(), R)
    assert rep["nnz_c"] == R.nnz
    assert rep["products"] == int(gen.row_products(A, B).sum())
    assert rep["device_flags"] == 0


@pytest.mark.parametrize("wpb", [0, 1, 3, 6])
@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_cta_sizes(engine, algo, wpb):
    """Per-kernel CTA sizes (0) and odd explicit ones give the same C."""
    engine.set_tuning(warps_per_block=wpb)
    for name, A, B in PAIRS:
        if name in ("stencil12", "rmat12", "er4096", "rect"):
            C, rep = engine.multiply(A, B, algo=algo, use_tuning=True)
            assert_parity(C.to_host(), ref(name, A, B))
    for bad in (-1, 17):
        with pytest.raises(SpgError):
            engine.set_tuning(warps_per_block=bad)


@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_small_path_and_fallback(engine, algo):
    """Products of at most small_rows rows take the small-product path (one
    counting launch, a one-CTA scan, one numeric launch); a row of more than
    2048 products sends the call to the binned pipeline; both match the
    oracle bit for bit, in both index widths of C."""
    engine.set_tuning(small_rows=0)
    for name, A, B in PAIRS:
        if name not in ("er4096", "stencil12", "wide_cols", "heavy_row", "empty", "zero_rows"):
            continue
        for bits in (0, 64):
            C, rep = engine.multiply(A, B, algo=algo, use_tuning=True, out_index_bits=bits)
            R = ref(name, A, B)
            assert_parity(C.to_host(), R)
            assert rep["nnz_c"] == R.nnz and rep["device_flags"] == 0
            assert rep["products"] == int(gen.row_products(A, B).sum())
            # heavy_row's first row has about 12,000 products; a product with no rows has nothing to do
            assert rep["small_path"] == (0 if name in ("heavy_row", "zero_rows") else 1), (name, rep)
            if rep["small_path"]:
                assert rep["rows_predicted"] == 0
    A = gen.erdos_renyi(4096, 4096, 8.0, 0)
    engine.set_tuning(small_rows=4095)
    C, rep = engine.multiply(A, A, algo=algo, use_tuning=True)
    assert rep["small_path"] == 0
    assert_parity(C.to_host(), ref("er4096", A, A))
    engine.set_tuning(small_rows=-1)
    C, rep = engine.multiply(A, A, algo=algo, use_tuning=True)
    assert rep["small_path"] == 0
    engine.set_tuning(small_rows=0)
    for bad in (-2, 65537):
        with pytest.raises(SpgError):
            engine.set_tuning(small_rows=bad)


@pytest.mark.parametrize("name,A,B", PAIRS[:9], ids=[p[0] for p in PAIRS[:9]])
def test_learned_forced_overflow(engine, name, A, B):
    """Every row mispredicted (capacity 1): all rows go through the exact re-run."""
    C, rep = engine.multiply(A, B, algo="learned", force_overflow=True)
    assert_parity(C.to_host(), ref(name, A, B))


@pytest.mark.parametrize("index_bits", [32, 64])
@pytest.mark.parametrize("out_bits", [0, 32, 64])
def test_device_inputs_and_index_widths(engine, index_bits, out_bits):
    A = gen.erdos_renyi(1500, 1500, 10.0, 11)
    dA = DeviceCsr.from_host(A, index_bits=index_bits)
    C, rep = engine.multiply(dA, dA, algo="plain", out_index_bits=out_bits)
    if out_bits:
        assert C.s.index_bits == out_bits
    assert_parity(C.to_host(), oracle.spgemm(A, A))


def test_host_output(engine):
    A = gen.erdos_renyi(800, 800, 6.0, 12)
    C, rep = engine.multiply(A, A, algo="learned", out="host")
    assert C.location == 0
    assert_parity(C.to_host(), oracle.spgemm(A, A))


def test_deterministic_runs(engine):
    A = gen.rmat(11, 16, seed=3)
    outs = []
    for _ in range(3):
        C, _ = engine.multiply(A, A, algo="plain")
        outs.append(C.to_host())
    for o in outs[1:]:
        assert np.array_equal(o.col_idx, outs[0].col_idx)
        assert np.array_equal(o.val.view(np.uint32), outs[0].val.view(np.uint32))


def test_cusparse_reference_point(engine):
    """cuSPARSE (reported reference point): same structure, values within tolerance."""
    A = gen.erdos_renyi(4096, 4096, 8.0, 0)
    C, rep = engine.multiply(A, A, algo="cusparse")
    H = C.to_host()
    R = oracle.spgemm(A, A)
    assert_same_structure(H, R)
    rel, _, _ = value_errors(H, R)
    assert rel <= REL_TOL


def test_invalid_inputs_rejected(engine):
    from rtspmspm_b200 import SpgError
    from rtspmspm_b200.gen import Csr

    A = gen.erdos_renyi(50, 50, 4.0, 1)
    bad = Csr(A.rows, A.cols, A.row_ptr.copy(), A.col_idx.copy(), A.val.copy())
    bad.col_idx[3] = 10_000  # out of range
    with pytest.raises(SpgError) as e:
        engine.multiply(bad, A, algo="plain")
    assert e.value.status == 1
    uns = Csr(A.rows, A.cols, A.row_ptr.copy(), A.col_idx.copy(), A.val.copy())
    r = int(np.argmax(A.row_lengths()))
    s = int(A.row_ptr[r])
    uns.col_idx[s], uns.col_idx[s + 1] = uns.col_idx[s + 1], uns.col_idx[s]  # unsorted row
    with pytest.raises(SpgError):
        engine.multiply(uns, A, algo="learned")
    with pytest.raises(SpgError):
        engine.multiply(A, gen.erdos_renyi(49, 50, 4.0, 1))  # inner dims differ
    # the context stays usable after rejected calls
    C, _ = engine.multiply(A, A, algo="plain")
    assert_parity(C.to_host(), oracle.spgemm(A, A))
