"""ctypes binding of the C oracle (spgemm_oracle.c) -- TEST INFRASTRUCTURE.

The oracle is the checker, never the thing measured or shipped: only tests/,
``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import it.

Canonical order and arithmetic (restated from the reference's any-hit
accumulate, optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cu:246-258): for each
row i, k ascending through A_i, then j ascending through B_k,
``acc[j] = fl32(acc[j] + fl32(a_ik * b_kj))``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


class _Csr(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int64), ("cols", ctypes.c_int64),
                ("row_ptr", ctypes.c_void_p), ("col_idx", ctypes.c_void_p),
                ("val", ctypes.c_void_p)]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    return os.path.join(HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "spgemm_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(_Csr)
        vp = ctypes.c_void_p
        L.orc_row_products.argtypes = [P, P, vp]
        L.orc_row_nnz.argtypes = [P, P, vp]
        L.orc_row_nnz.restype = ctypes.c_int
        L.orc_spgemm.argtypes = [P, P, vp, vp, vp, vp, vp]
        L.orc_spgemm.restype = ctypes.c_int
        L.orc_rows_nnz.argtypes = [P, P, vp, ctypes.c_int64, vp]
        L.orc_rows_nnz.restype = ctypes.c_int
        L.orc_rows.argtypes = [P, P, vp, ctypes.c_int64, vp, vp, vp, vp, vp]
        L.orc_rows.restype = ctypes.c_int
        L.orc_baseline_rows.argtypes = [P, P, ctypes.c_int64, ctypes.c_int64,
                                        ctypes.POINTER(ctypes.c_double)]
        L.orc_baseline_rows.restype = ctypes.c_int64
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def _wrap(M):
    rp = np.ascontiguousarray(M.row_ptr, dtype=np.int64)
    ci = np.ascontiguousarray(M.col_idx, dtype=np.int32)
    va = np.ascontiguousarray(M.val, dtype=np.float32)
    s = _Csr(M.rows, M.cols, _ptr(rp), _ptr(ci), _ptr(va))
    return s, (rp, ci, va)


class OracleResult:
    """C = A*B from the oracle: FP32 canonical values, FP64 twin, |a*b| bound."""

    def __init__(self, rows, cols, row_ptr, col_idx, val, val64, bound):
        self.rows, self.cols = rows, cols
        self.row_ptr, self.col_idx, self.val = row_ptr, col_idx, val
        self.val64, self.bound = val64, bound

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1])


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def row_products(A, B) -> np.ndarray:
    a, ka = _wrap(A)
    b, kb = _wrap(B)
    out = np.zeros(A.rows, dtype=np.int64)
    lib().orc_row_products(ctypes.byref(a), ctypes.byref(b), _ptr(out))
    return out


def row_nnz(A, B) -> np.ndarray:
    a, ka = _wrap(A)
    b, kb = _wrap(B)
    out = np.zeros(A.rows, dtype=np.int64)
    if lib().orc_row_nnz(ctypes.byref(a), ctypes.byref(b), _ptr(out)):
        raise MemoryError("oracle: accumulator allocation failed")
    return out


def spgemm(A, B, twin: bool = True) -> OracleResult:
    """Full product in canonical order (all rows)."""
    if A.cols != B.rows:
        raise ValueError("inner dimensions differ")
    a, ka = _wrap(A)
    b, kb = _wrap(B)
    nnz = row_nnz(A, B)
    rp = np.zeros(A.rows + 1, dtype=np.int64)
    np.cumsum(nnz, out=rp[1:])
    n = int(rp[-1])
    col = np.empty(n, dtype=np.int32)
    val = np.empty(n, dtype=np.float32)
    v64 = np.empty(n, dtype=np.float64) if twin else None
    bnd = np.empty(n, dtype=np.float64) if twin else None
    rc = lib().orc_spgemm(ctypes.byref(a), ctypes.byref(b), _ptr(rp), _ptr(col), _ptr(val),
                          _ptr(v64) if twin else None, _ptr(bnd) if twin else None)
    if rc:
        raise RuntimeError(f"oracle spgemm failed ({rc})")
    return OracleResult(A.rows, B.cols, rp, col, val, v64, bnd)


def rows(A, B, sel) -> OracleResult:
    """Only the rows in ``sel`` (packed in that order)."""
    sel = np.ascontiguousarray(sel, dtype=np.int64)
    a, ka = _wrap(A)
    b, kb = _wrap(B)
    cnt = np.zeros(sel.size, dtype=np.int64)
    if lib().orc_rows_nnz(ctypes.byref(a), ctypes.byref(b), _ptr(sel), sel.size, _ptr(cnt)):
        raise MemoryError("oracle: accumulator allocation failed")
    rp = np.zeros(sel.size + 1, dtype=np.int64)
    np.cumsum(cnt, out=rp[1:])
    n = int(rp[-1])
    col = np.empty(n, dtype=np.int32)
    val = np.empty(n, dtype=np.float32)
    v64 = np.empty(n, dtype=np.float64)
    bnd = np.empty(n, dtype=np.float64)
    rc = lib().orc_rows(ctypes.byref(a), ctypes.byref(b), _ptr(sel), sel.size, _ptr(rp),
                        _ptr(col), _ptr(val), _ptr(v64), _ptr(bnd))
    if rc:
        raise RuntimeError(f"oracle rows failed ({rc})")
    return OracleResult(sel.size, B.cols, rp, col, val, v64, bnd)


def baseline_rows(A, B, r0: int, r1: int):
    """Timed CPU baseline body: FP32 canonical product of rows [r0, r1).

    Returns (nnz of those rows, value checksum)."""
    a, ka = _wrap(A)
    b, kb = _wrap(B)
    cs = ctypes.c_double(0.0)
    n = lib().orc_baseline_rows(ctypes.byref(a), ctypes.byref(b), r0, r1, ctypes.byref(cs))
    return int(n), float(cs.value)
