"""The allocation-free entry point (spg_multiply_noalloc) gives the same C as
spg_multiply, through the C ABI, on two calls in a row.

It exists for callers that cannot let a library call cudaMalloc -- a process
whose device memory is owned by its own arena or budget, or a hot path that
must not risk an allocation's latency or an out-of-memory failure -- so its
scratch is a fixed device array inside the library and C goes into buffers
the caller allocates (here with torch).  This file is collected last so
that a failure here does not stop the rest of a run at the first failure.
"""
import ctypes

import numpy as np
import pytest

from rtspmspm_b200 import DeviceCsr, Engine, _lib, gen

pytestmark = pytest.mark.gpu


def _call(L, stream, sa, sb, c):
    buf = ctypes.create_string_buffer(512)
    st = L.spg_multiply_noalloc(ctypes.c_void_p(stream), ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                buf, 512)
    return st, buf.value.decode()


def test_noalloc_matches_spg_multiply_on_two_calls_in_a_row():
    import torch

    L = _lib.load()
    eng = Engine(0)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        inputs = [(gen.erdos_renyi(3000, 2500, 6.0, 41), gen.erdos_renyi(2500, 2000, 7.0, 42), 64),
                  (gen.stencil27(24, seed=3), None, 32)]
        for A, B, bits in inputs:
            B = A if B is None else B
            dA, dB = DeviceCsr.from_host(A, index_bits=32), DeviceCsr.from_host(B, index_bits=64)
            want, _ = eng.multiply(dA, dB, algo="plain")
            W = want.to_host()
            cap = W.nnz + 7
            rp = torch.full((A.rows + 1,), -1, dtype=torch.int64 if bits == 64 else torch.int32, device="cuda")
            col = torch.full((cap,), -1, dtype=torch.int32, device="cuda")
            val = torch.full((cap,), float("nan"), dtype=torch.float32, device="cuda")
            c = _lib.SpgCsr(rows=A.rows, cols=B.cols, nnz=0, index_bits=bits, location=_lib.SPG_DEVICE,
                            row_ptr=rp.data_ptr(), col_idx=col.data_ptr(), val=val.data_ptr(), capacity=cap)
            st, msg = _call(L, stream, dA.struct(), dB.struct(), c)
            assert st == _lib.SPG_OK, msg
            torch.cuda.synchronize()
            assert c.nnz == W.nnz
            np.testing.assert_array_equal(rp.cpu().numpy().astype(np.int64), W.row_ptr)
            np.testing.assert_array_equal(col[:W.nnz].cpu().numpy(), W.col_idx)
            np.testing.assert_array_equal(val[:W.nnz].cpu().numpy().view(np.uint32), W.val.view(np.uint32))
    finally:
        eng.close()


def test_noalloc_rejects_out_of_limit_inputs_with_a_message():
    import torch

    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    A = gen.erdos_renyi(1000, 1000, 4.0, 1)
    dA = DeviceCsr.from_host(A)
    too_tall = dA.struct()
    too_tall.rows = (1 << 18) + 1  # rejected on the host before any device work
    c = _lib.SpgCsr(rows=0, cols=0, index_bits=64, location=_lib.SPG_DEVICE, row_ptr=dA.row_ptr.data_ptr(),
                    capacity=0)
    st, msg = _call(L, stream, too_tall, dA.struct(), c)
    assert st == _lib.SPG_ERR_INVALID_ARG and "at most 262144" in msg
    # capacity too small: fails cleanly and reports the size needed
    rp = torch.empty(A.rows + 1, dtype=torch.int64, device="cuda")
    col = torch.empty(8, dtype=torch.int32, device="cuda")
    val = torch.empty(8, dtype=torch.float32, device="cuda")
    c = _lib.SpgCsr(rows=A.rows, cols=A.cols, index_bits=64, location=_lib.SPG_DEVICE, row_ptr=rp.data_ptr(),
                    col_idx=col.data_ptr(), val=val.data_ptr(), capacity=8)
    st, msg = _call(L, stream, dA.struct(), dA.struct(), c)
    assert st == _lib.SPG_ERR_INVALID_ARG and c.nnz > 8 and "capacity" in msg


def _device_out(rows, cap, bits=64):
    import torch

    rp = torch.full((rows + 1,), -1, dtype=torch.int64 if bits == 64 else torch.int32, device="cuda")
    col = torch.full((max(cap, 1),), -1, dtype=torch.int32, device="cuda")
    val = torch.full((max(cap, 1),), float("nan"), dtype=torch.float32, device="cuda")
    c = _lib.SpgCsr(rows=rows, cols=0, nnz=0, index_bits=bits, location=_lib.SPG_DEVICE, row_ptr=rp.data_ptr(),
                    col_idx=col.data_ptr(), val=val.data_ptr(), capacity=cap)
    return c, (rp, col, val)


def test_noalloc_rejects_rows_beyond_the_warp_tables_and_bad_input():
    import torch

    from rtspmspm_b200.gen import Csr, coo_to_csr

    L = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    # row 0 of A touches 100 rows of B with 40 entries each: 4,000 products
    # over 3,000 columns, beyond the 2,048-product limit of the warp tables
    n = 3000
    B = gen.erdos_renyi(n, n, 40.0, 5)
    r = np.concatenate([np.zeros(100, np.int64), np.arange(1, 50)])
    cc = np.concatenate([np.arange(100), np.arange(1, 50)])
    A = coo_to_csr(n, n, r, cc, np.ones(r.size, np.float32))
    dA, dB = DeviceCsr.from_host(A), DeviceCsr.from_host(B)
    c, keep = _device_out(n, 1 << 20)
    st, msg = _call(L, stream, dA.struct(), dB.struct(), c)
    assert st == _lib.SPG_ERR_UNSUPPORTED and "warp hash tables" in msg
    # an unsorted row is rejected by the validation kernel
    E = gen.erdos_renyi(500, 500, 6.0, 9)
    bad = Csr(E.rows, E.cols, E.row_ptr.copy(), E.col_idx.copy(), E.val.copy())
    rr = int(np.argmax(E.row_lengths()))
    s = int(E.row_ptr[rr])
    bad.col_idx[s], bad.col_idx[s + 1] = bad.col_idx[s + 1], bad.col_idx[s]
    dbad, dE = DeviceCsr.from_host(bad), DeviceCsr.from_host(E)
    c, keep = _device_out(E.rows, 1 << 16)
    st, msg = _call(L, stream, dbad.struct(), dE.struct(), c)
    assert st == _lib.SPG_ERR_INVALID_ARG and "validation" in msg


def test_noalloc_empty_rows_match_spg_multiply():
    """Empty rows and rows whose B rows are all empty go to the empty bin and
    rely on the per-call reset of the counts: bit-exact against
    spg_multiply, twice in a row."""
    import torch

    from rtspmspm_b200.gen import coo_to_csr

    L = _lib.load()
    eng = Engine(0)
    stream = torch.cuda.current_stream().cuda_stream
    try:
        n = 2000
        E = gen.erdos_renyi(n, n, 5.0, 13)
        rows_of = np.repeat(np.arange(n), E.row_lengths())
        keep_e = (rows_of % 3 != 0) & (E.col_idx % 4 != 1)  # every third row empty, B rows 1 mod 4 empty
        A = coo_to_csr(n, n, rows_of[keep_e], E.col_idx[keep_e], E.val[keep_e])
        dA = DeviceCsr.from_host(A)
        W = eng.multiply(dA, dA, algo="plain")[0].to_host()
        assert (np.diff(W.row_ptr) == 0).sum() > n // 3
        for _ in range(2):
            c, (rp, col, val) = _device_out(n, W.nnz + 3)
            st, msg = _call(L, stream, dA.struct(), dA.struct(), c)
            assert st == _lib.SPG_OK, msg
            torch.cuda.synchronize()
            assert c.nnz == W.nnz
            np.testing.assert_array_equal(rp.cpu().numpy(), W.row_ptr)
            np.testing.assert_array_equal(col[:W.nnz].cpu().numpy(), W.col_idx)
            np.testing.assert_array_equal(val[:W.nnz].cpu().numpy().view(np.uint32), W.val.view(np.uint32))
    finally:
        eng.close()
