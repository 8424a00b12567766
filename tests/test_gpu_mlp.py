"""Learned row-size predictor: kernels vs the FP64 CPU reference, training,
and what the trained network gains over the method without it."""
import numpy as np
import pytest

from oracle import mlp_oracle, oracle
from rtspmspm_b200 import DeviceCsr, Engine, HostCsr, gen

from helpers import assert_parity

pytestmark = pytest.mark.gpu


def _batch(rows=3000, seed=0):
    rng = np.random.default_rng(seed)
    x = rng.uniform(0.0, 1.2, size=(rows, 8)).astype(np.float32)
    t = np.stack([rng.uniform(0, 12, rows), rng.integers(5, 14, rows)], 1).astype(np.float32)
    return x, t


def test_backward_matches_fp64_reference(engine):
    import torch

    engine.mlp_init(7)
    p = engine.mlp_params()
    x, t = _batch()
    loss, g = engine.mlp_grad(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    rl, rg = mlp_oracle.loss_and_grad(p, x, t)
    assert abs(loss - rl) <= 1e-4 * max(1.0, abs(rl))
    # FP32 accumulation over 3000 rows: relative error well under 1e-3
    err = np.abs(g - rg).max() / max(np.abs(rg).max(), 1e-12)
    assert err < 1e-3, err


def test_tensor_core_inference_matches_reference(engine):
    import torch

    engine.mlp_init(3)
    p = engine.mlp_params()
    x, _ = _batch(1000, 1)
    y = engine.mlp_predict(torch.from_numpy(x).cuda()).cpu().numpy()
    ry, _ = mlp_oracle.forward(p, x, bf16_weights=True, bf16_acts=True)
    np.testing.assert_allclose(y, ry, rtol=2e-2, atol=2e-2)


@pytest.mark.parametrize("bits", [32, 64])
def test_features_match_oracle(engine, bits):
    """The feature kernel's integer statistics and features equal the CPU
    restatement: short and long rows (> 32 entries, sampled by stride),
    empty rows and columns, a heavy row, rectangular shapes, a ragged last
    tile, and both row-pointer widths."""
    from cases import heavy_row, with_empty_rows_cols

    mats = [(gen.stencil27(10, seed=1), None), (gen.rmat(12, 16, seed=5), None),
            (gen.erdos_renyi(333, 250, 7.0, 2), gen.erdos_renyi(250, 517, 40.0, 3)),
            (with_empty_rows_cols(), None), (heavy_row(), None), (gen.erdos_renyi(17, 17, 0.5, 4), None)]
    for A, B in mats:
        B = A if B is None else B
        dA, dB = DeviceCsr.from_host(A, index_bits=bits), DeviceCsr.from_host(B, index_bits=bits)
        got = engine.features(dA, dB).cpu().numpy()
        ref, _ = mlp_oracle.row_features(A, B)
        # integer features exactly (up to log2f's rounding), float ones to 2 ulp
        np.testing.assert_allclose(got, ref, rtol=0, atol=5e-7)


def test_training_reduces_loss_and_roundtrips(tmp_path):
    eng = Engine(0)
    try:
        eng.mlp_init(11)
        mats = [gen.erdos_renyi(3000, 3000, m, s) for s, m in enumerate([4.0, 9.0, 16.0, 25.0])]
        mats += [gen.stencil27(14), gen.rmat(12, 16, seed=5)]
        hs = [HostCsr(m) for m in mats]
        r0 = eng.mlp_train(hs, hs, epochs=1, lr=1e-5, max_rows_per_matrix=3000)
        r1 = eng.mlp_train(hs, hs, epochs=15, lr=3e-3, max_rows_per_matrix=3000)
        assert r1["final_loss"] < 0.5 * r0["final_loss"]
        path = str(tmp_path / "w.bin")
        eng.mlp_save(path)
        p = eng.mlp_params()
        eng.mlp_init(0)
        eng.mlp_load(path)
        np.testing.assert_array_equal(eng.mlp_params(), p)
    finally:
        eng.close()


@pytest.mark.parametrize("name", ["stencil48", "er", "rmat14"])
def test_trained_network_gain(name):
    """With the shipped weights most rows skip the symbolic pass (and the
    result stays exact); with a fresh untrained network nearly all rows
    overflow and fall back."""
    A = {"stencil48": lambda: gen.stencil27(48, seed=9),
         "er": lambda: gen.erdos_renyi(50000, 50000, 12.0, 77),
         "rmat14": lambda: gen.rmat(14, 16, seed=41)}[name]()
    R = oracle.spgemm(A, A)
    eng = Engine(0)
    try:
        dA = DeviceCsr.from_host(A)
        C, rep = eng.multiply(dA, dA, algo="learned")
        assert_parity(C.to_host(), R)
        rows_nonempty = int((gen.row_products(A, A) > 0).sum())
        skipped = rep["rows_predicted"] - rep["rows_overflow"]
        mis = rep["rows_overflow"] / max(1, rep["rows_predicted"])
        assert mis < 0.05, rep
        # predicted-heavy rows go to the exact path by design; the rest skip symbolic
        assert skipped + rep["rows_heavy"] >= 0.9 * rows_nonempty or skipped >= 0.9 * rows_nonempty, rep
        eng.mlp_init(123)  # untrained network
        C2, rep2 = eng.multiply(dA, dA, algo="learned")
        assert_parity(C2.to_host(), R)
        assert rep2["rows_predicted"] - rep2["rows_overflow"] < skipped
    finally:
        eng.close()
