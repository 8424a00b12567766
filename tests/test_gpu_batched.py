"""Batched uneven products in one persistent launch per stage, captured as a
CUDA graph and replayed; and the autotuner with its JSON cache."""
import json

import numpy as np
import pytest

from oracle import oracle
from rtspmspm_b200 import DeviceCsr, Engine, gen

from helpers import assert_parity

pytestmark = pytest.mark.gpu


def small_batch(count=24, seed=5):
    return gen.batch_uneven(count=count, seed=seed, lo=64, hi=4096)


@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_matches_oracle(use_graph):
    pairs = small_batch()
    eng = Engine(0)
    try:
        dA = [DeviceCsr.from_host(a) for a, _ in pairs]
        dB = [DeviceCsr.from_host(b) for _, b in pairs]
        for _ in range(2):  # second call replays the cached plan / graph
            res, rep = eng.multiply_batched(dA, dB, use_graph=use_graph)
            assert rep["device_flags"] == 0
            tot = 0
            for (A, B), C in zip(pairs, res):
                R = oracle.spgemm(A, B)
                assert_parity(C.to_host(), R)
                tot += R.nnz
            assert rep["nnz_c"] == tot
            assert rep["products"] == sum(int(gen.row_products(a, b).sum()) for a, b in pairs)
    finally:
        eng.close()


@pytest.mark.parametrize("force_overflow", [False, True])
@pytest.mark.parametrize("use_graph", [False, True])
def test_batched_learned_matches_oracle(use_graph, force_overflow):
    """Learned batch: rows sized by the predictor in one numeric pass into a
    slab, then copied into C; with every row mispredicted (capacity 1) all
    rows take the exact symbolic + numeric queues instead.  Two calls (the
    second replays the graph) give the oracle's C."""
    pairs = small_batch(16, 21) + gen.batch_uneven(count=4, seed=11, lo=2048, hi=8192, mean_lo=40.0, mean_hi=64.0)
    eng = Engine(0)
    try:
        dA = [DeviceCsr.from_host(a) for a, _ in pairs]
        dB = [DeviceCsr.from_host(b) for _, b in pairs]
        for _ in range(2):
            res, rep = eng.multiply_batched(dA, dB, use_graph=use_graph, algo="learned",
                                            force_overflow=force_overflow)
            assert rep["device_flags"] == 0
            if force_overflow:  # every row with products overflows its capacity of 1
                assert 0 < rep["rows_overflow"] <= rep["rows_predicted"]
            for (A, B), C in zip(pairs, res):
                assert_parity(C.to_host(), oracle.spgemm(A, B))
    finally:
        eng.close()


@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_batched_fold_rows_match_hashed_rows(algo):
    """Rows of mostly distinct products go through the expand-sort-fold path
    in the queue kernels (by default above 128 products, every eligible row
    with esc_min_prod 1) or are hashed (-1): the same bits as the oracle
    either way, over a capture and a replay each."""
    pairs = gen.batch_uneven(count=12, seed=31, lo=256, hi=4096, mean_lo=8.0, mean_hi=28.0)
    eng = Engine(0)
    try:
        dA = [DeviceCsr.from_host(a) for a, _ in pairs]
        dB = [DeviceCsr.from_host(b) for _, b in pairs]
        refs = [oracle.spgemm(a, b) for a, b in pairs]
        for esc in (0, 1, -1):
            eng.set_tuning(esc_min_prod=esc, max_load=0.8, learned_load=0.8)
            for _ in range(2):
                res, rep = eng.multiply_batched(dA, dB, use_graph=True, use_tuning=True, algo=algo)
                assert rep["device_flags"] == 0
                for R, C in zip(refs, res):
                    assert_parity(C.to_host(), R)
    finally:
        eng.close()


def test_graph_replay_reads_new_values():
    import torch

    pairs = small_batch(8, 9)
    eng = Engine(0)
    try:
        dA = [DeviceCsr.from_host(a) for a, _ in pairs]
        dB = [DeviceCsr.from_host(b) for _, b in pairs]
        eng.multiply_batched(dA, dB, use_graph=True)
        for d in dA:
            d.val.mul_(2.0)
        torch.cuda.synchronize()
        res, _ = eng.multiply_batched(dA, dB, use_graph=True)
        for (A, B), C in zip(pairs, res):
            A2 = gen.Csr(A.rows, A.cols, A.row_ptr, A.col_idx, (A.val * 2).astype(np.float32))
            assert_parity(C.to_host(), oracle.spgemm(A2, B))
    finally:
        eng.close()


def test_batched_rows_in_the_cta_tables():
    """Denser products: rows of 1,000-4,096 products take the CTA-wide tables
    of the queue (symbolic and numeric), beside rows in the warp tables."""
    pairs = gen.batch_uneven(count=8, seed=11, lo=2048, hi=8192, mean_lo=40.0, mean_hi=64.0)
    bounds = [int(np.minimum(gen.row_products(a, b), b.cols).max()) for a, b in pairs]
    assert max(bounds) > 1500 and max(bounds) <= 4096
    eng = Engine(0)
    try:
        for graph in (False, True):
            res, rep = eng.multiply_batched([DeviceCsr.from_host(a) for a, _ in pairs],
                                            [DeviceCsr.from_host(b) for _, b in pairs], use_graph=graph)
            assert rep["device_flags"] == 0 and rep["rows_heavy"] == 0
            for (A, B), C in zip(pairs, res):
                assert_parity(C.to_host(), oracle.spgemm(A, B))
    finally:
        eng.close()


def test_batch_with_a_heavy_product_falls_back_per_product():
    H = gen.rmat(13, 16, seed=2)  # rows beyond the queue's tables (more than 4,096 products, capped at the columns)
    assert int(np.minimum(gen.row_products(H, H), H.cols).max()) > 4096
    pairs = small_batch(6, 3) + [(H, H)]
    eng = Engine(0)
    try:
        res, rep = eng.multiply_batched([DeviceCsr.from_host(a) for a, _ in pairs],
                                        [DeviceCsr.from_host(b) for _, b in pairs], use_graph=True)
        assert rep["rows_heavy"] == 1
        for (A, B), C in zip(pairs, res):
            assert_parity(C.to_host(), oracle.spgemm(A, B))
    finally:
        eng.close()


def _digest(H):
    """Order-sensitive digest of a host CSR (row pointers, columns, value bits)."""
    rp = np.asarray(H.row_ptr, np.int64)
    col = np.asarray(H.col_idx, np.int64)
    bits = np.asarray(H.val, np.float32).view(np.uint32).astype(np.uint64)
    w = np.arange(1, col.size + 1, dtype=np.uint64)
    return (int(rp.sum()), int(col.sum()), int((col.astype(np.uint64) * w).sum()), int(bits.sum()),
            int((bits * w).sum()))


@pytest.mark.parametrize("algo", ["plain", "learned"])
def test_batch512_full_size_capture_then_replay(algo):
    """The 512 uneven products (seed 1; rows, inner and column dimensions
    log-uniform on [1k, 64k], Poisson nnz/row with means U(2, 32)) through one
    batched call captured as a CUDA graph, then replayed: every product of
    the replay is checked whole against the oracle, and the captured call's
    output is bit-identical to the replay's."""
    pairs = gen.batch_uneven(count=512, seed=1)
    eng = Engine(0)
    try:
        dA = [DeviceCsr.from_host(a) for a, _ in pairs]
        dB = [DeviceCsr.from_host(b) for _, b in pairs]
        res, rep = eng.multiply_batched(dA, dB, use_graph=True, algo=algo)
        assert rep["device_flags"] == 0
        first = [_digest(C.to_host()) for C in res]
        res, rep = eng.multiply_batched(dA, dB, use_graph=True, algo=algo)
        assert rep["device_flags"] == 0
        assert rep["products"] == sum(int(gen.row_products(a, b).sum()) for a, b in pairs)
        tot = 0
        for i, ((A, B), C) in enumerate(zip(pairs, res)):
            H = C.to_host()
            assert _digest(H) == first[i], f"product {i}: replay differs from the captured call"
            R = oracle.spgemm(A, B)
            assert_parity(H, R)
            tot += R.nnz
            del H, R
        assert rep["nnz_c"] == tot
    finally:
        eng.close()


def test_autotuner_cache(tmp_path):
    A = gen.stencil27(20)
    eng = Engine(0)
    try:
        dA = DeviceCsr.from_host(A)
        path = str(tmp_path / "tune.json")
        best = eng.tune([dA], [dA], path)
        entries = json.load(open(path))["entries"]
        assert len(entries) == 1 and entries[0]["warp_table_max"] == best["warp_table_max"]
        # a second call is answered from the cache
        best2 = eng.tune([dA], [dA], path)
        assert best2["warp_table_max"] == best["warp_table_max"]
        assert len(json.load(open(path))["entries"]) == 1
        C, _ = eng.multiply(dA, dA, algo="plain", use_tuning=True)
        assert_parity(C.to_host(), oracle.spgemm(A, A))
    finally:
        eng.close()
