"""Value-only recompute (spg_multiply_reuse): C keeps the structure of A*B
from a first multiply; new values of A and B give C's new values in place,
bit-exact against the oracle on the new values.  Mirrors the reference's
cuSPARSE reuse flow (structure once, compute twice with updated values)."""
import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import DeviceCsr, Engine, SpgError, gen
from rtspmspm_b200.gen import Csr

from cases import heavy_row, named_pairs
from helpers import assert_parity

pytestmark = pytest.mark.gpu


def revalue(m: Csr, seed: int) -> Csr:
    """Same structure, new values (signs and magnitudes both change)."""
    v = np.random.default_rng(seed).uniform(-2.0, 2.0, m.nnz).astype(np.float32)
    return Csr(m.rows, m.cols, m.row_ptr.copy(), m.col_idx.copy(), v)


PAIRS = {n: (a, b) for n, a, b in named_pairs() if n in
         ("identity", "rect", "er4096", "wide_cols", "stencil12", "rmat12", "cancelling", "empty_rows_cols")}


@pytest.mark.parametrize("name", sorted(PAIRS))
@pytest.mark.parametrize("bits", [32, 64])
def test_reuse_matches_oracle_on_new_values(engine, name, bits):
    A, B = PAIRS[name]
    C, _ = engine.multiply(A, B, algo="plain", out_index_bits=bits)
    try:
        for seed in (1, 2):
            A2, B2 = revalue(A, 10 * seed), revalue(B, 10 * seed + 1)
            rep = engine.multiply_reuse(A2, B2, C)
            assert rep["device_flags"] == 0
            assert_parity(C.to_host(), oracle.spgemm(A2, B2))
    finally:
        C.free()


@pytest.mark.parametrize("tuning,heavy", [
    ({"warp_table_max": 64, "block_table_max": 1024, "max_load": 0.5, "block_min_nnz": -1}, True),
    ({"warp_table_max": 4096, "block_min_nnz": -1}, True),
    ({"warp_table_max": 4096, "block_min_nnz": 8}, False)])
def test_reuse_heavy_rows(tuning, heavy):
    """Rows beyond the warp tables take the column-tile path (tile counts
    read from C's columns) or, with the CTA hash bins on, the CTA tables."""
    eng = Engine(0)
    try:
        eng.set_tuning(**tuning)
        for A in (heavy_row(), gen.rmat(13, 16, seed=3)):
            dA = DeviceCsr.from_host(A)
            C, rep = eng.multiply(dA, dA, algo="plain", use_tuning=True)
            assert (rep["rows_heavy"] > 0) == heavy
            if not heavy:
                assert rep["bin_rows"][8] + rep["bin_rows"][9] > 0
            A2 = revalue(A, 5)
            eng.multiply_reuse(A2, A2, C, use_tuning=True)
            assert_parity(C.to_host(), oracle.spgemm(A2, A2))
            C.free()
    finally:
        eng.close()


def test_reuse_after_learned_and_device_inputs(engine):
    A = gen.stencil27(16, seed=4)
    dA = DeviceCsr.from_host(A)
    C, _ = engine.multiply(dA, dA, algo="learned")
    A2 = revalue(A, 7)
    dA.val.copy_(__import__("torch").from_numpy(A2.val).cuda())
    engine.multiply_reuse(dA, dA, C, skip_validation=True)
    assert_parity(C.to_host(), oracle.spgemm(A2, A2))
    C.free()


def test_reuse_rejects_a_different_structure(engine):
    A = gen.erdos_renyi(500, 500, 6.0, 1)
    C, _ = engine.multiply(A, A, algo="plain")
    other = gen.erdos_renyi(500, 500, 9.0, 2)
    with pytest.raises(SpgError) as e:
        engine.multiply_reuse(other, other, C)
    assert e.value.status == 1
    # the engine stays usable
    engine.multiply_reuse(A, A, C)
    assert_parity(C.to_host(), oracle.spgemm(A, A))
    C.free()


def test_reuse_rejects_bad_shapes(engine):
    A = gen.erdos_renyi(100, 120, 4.0, 1)
    B = gen.erdos_renyi(120, 90, 4.0, 2)
    C, _ = engine.multiply(A, B, algo="plain")
    with pytest.raises(SpgError):
        engine.multiply_reuse(B, A, C)
    C.free()
