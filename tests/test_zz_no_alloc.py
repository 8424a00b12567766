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
