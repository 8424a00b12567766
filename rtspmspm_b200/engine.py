"""Python host API over the C ABI (librtspmspm.so).

Mirrors the reference's operator surface -- "matrix files in, C = A*B out,
latency in ms" (optixSpMSpM/src/optixSpMSpM/optixSpMSpM.cpp:496-660,
cuSparse/src/main.cpp:365-591) -- as calls:

    eng = Engine(device=0)
    C, rep = eng.multiply(A, B, algo="learned")     # A, B: Csr (host) or DeviceCsr
    host_c = C.to_host()                            # Csr with numpy arrays

Every call goes through the C ABI; there is no Python or CPU fallback.
Errors raise SpgError carrying the library status and message.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from .gen import Csr

ALGOS = {"plain": _lib.SPG_ALGO_PLAIN, "learned": _lib.SPG_ALGO_LEARNED, "cusparse": _lib.SPG_ALGO_CUSPARSE}


class SpgError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_lib.load().spg_status_string(status).decode()} ({status}): {message}")
        self.status = status


def _np_ptr(a: np.ndarray) -> int:
    return a.ctypes.data if a.size else 0


class DeviceCsr:
    """CSR matrix resident on the GPU (torch tensors own the memory)."""

    def __init__(self, rows, cols, row_ptr, col_idx, val):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr, self.col_idx, self.val = row_ptr, col_idx, val

    @property
    def nnz(self) -> int:
        return int(self.col_idx.numel())

    @staticmethod
    def from_host(m: Csr, device: int = 0, index_bits: int = 32) -> "DeviceCsr":
        import torch

        dev = torch.device("cuda", device)
        rp_dtype = torch.int32 if index_bits == 32 else torch.int64
        rp = torch.from_numpy(np.ascontiguousarray(m.row_ptr)).to(dev, dtype=rp_dtype)
        ci = torch.from_numpy(np.ascontiguousarray(m.col_idx, dtype=np.int32)).to(dev)
        va = torch.from_numpy(np.ascontiguousarray(m.val, dtype=np.float32)).to(dev)
        return DeviceCsr(m.rows, m.cols, rp, ci, va)

    def struct(self) -> _lib.SpgCsr:
        s = _lib.SpgCsr()
        s.rows, s.cols, s.nnz = self.rows, self.cols, self.nnz
        s.index_bits = 32 if self.row_ptr.element_size() == 4 else 64
        s.location = _lib.SPG_DEVICE
        s.row_ptr = self.row_ptr.data_ptr()
        s.col_idx = self.col_idx.data_ptr() if self.nnz else 0
        s.val = self.val.data_ptr() if self.nnz else 0
        s.capacity = self.nnz
        s.owner = 0
        return s


class HostCsr:
    """Host CSR whose arrays the library reads directly (numpy or pinned torch)."""

    def __init__(self, m: Csr, index_bits: int = 64, pinned: bool = False):
        self.rows, self.cols = m.rows, m.cols
        rp = np.ascontiguousarray(m.row_ptr, dtype=np.int32 if index_bits == 32 else np.int64)
        ci = np.ascontiguousarray(m.col_idx, dtype=np.int32)
        va = np.ascontiguousarray(m.val, dtype=np.float32)
        if pinned:
            import torch

            self._t = [torch.from_numpy(x).pin_memory() for x in (rp, ci, va)]
            self._ptrs = [t.data_ptr() if t.numel() else 0 for t in self._t]
        else:
            self._arrs = (rp, ci, va)
            self._ptrs = [_np_ptr(x) for x in (rp, ci, va)]
        self.index_bits = index_bits
        self.nnz = int(ci.size)

    def struct(self) -> _lib.SpgCsr:
        s = _lib.SpgCsr()
        s.rows, s.cols, s.nnz = self.rows, self.cols, self.nnz
        s.index_bits = self.index_bits
        s.location = _lib.SPG_HOST
        s.row_ptr, s.col_idx, s.val = self._ptrs
        s.capacity = self.nnz
        return s


class Result:
    """C owned by the library (device or host); freed with the engine or free()."""

    def __init__(self, engine: "Engine", s: _lib.SpgCsr):
        self.engine = engine
        self.s = s

    @property
    def rows(self) -> int:
        return int(self.s.rows)

    @property
    def cols(self) -> int:
        return int(self.s.cols)

    @property
    def nnz(self) -> int:
        return int(self.s.nnz)

    @property
    def location(self) -> int:
        return int(self.s.location)

    def to_host(self) -> Csr:
        """Copies C into numpy arrays (int64 row_ptr)."""
        L = _lib.load()
        s = self.s
        if s.location == _lib.SPG_DEVICE:
            h = _lib.SpgCsr()
            self.engine._check(L.spg_csr_copy(self.engine.ctx, ctypes.byref(s), _lib.SPG_HOST, ctypes.byref(h)))
        else:
            h = s
        rp_t = ctypes.c_int32 if h.index_bits == 32 else ctypes.c_int64
        rp = np.ctypeslib.as_array(ctypes.cast(h.row_ptr, ctypes.POINTER(rp_t)), shape=(h.rows + 1,)).astype(np.int64)
        if h.nnz:
            col = np.ctypeslib.as_array(ctypes.cast(h.col_idx, ctypes.POINTER(ctypes.c_int32)), shape=(h.nnz,)).copy()
            val = np.ctypeslib.as_array(ctypes.cast(h.val, ctypes.POINTER(ctypes.c_float)), shape=(h.nnz,)).copy()
        else:
            col = np.zeros(0, np.int32)
            val = np.zeros(0, np.float32)
        if h is not s:
            L.spg_csr_free(self.engine.ctx, ctypes.byref(h))
        return Csr(int(h.rows), int(h.cols), rp, col, val)

    def rows_to_host(self, rows) -> Csr:
        """Copies only the given rows (a device C) into a host Csr."""
        L = _lib.load()
        sel = np.ascontiguousarray(rows, dtype=np.int64)
        h = _lib.SpgCsr()
        self.engine._check(L.spg_csr_extract_rows(self.engine.ctx, ctypes.byref(self.s), sel.ctypes.data,
                                                  sel.size, ctypes.byref(h)))
        try:
            rp = np.ctypeslib.as_array(ctypes.cast(h.row_ptr, ctypes.POINTER(ctypes.c_int64)),
                                       shape=(h.rows + 1,)).copy()
            n = int(h.nnz)
            col = np.ctypeslib.as_array(ctypes.cast(h.col_idx, ctypes.POINTER(ctypes.c_int32)), shape=(n,)).copy() \
                if n else np.zeros(0, np.int32)
            val = np.ctypeslib.as_array(ctypes.cast(h.val, ctypes.POINTER(ctypes.c_float)), shape=(n,)).copy() \
                if n else np.zeros(0, np.float32)
        finally:
            L.spg_csr_free(self.engine.ctx, ctypes.byref(h))
        return Csr(int(h.rows), int(h.cols), rp, col, val)

    def free(self) -> None:
        if self.s.owner and self.engine.ctx:
            _lib.load().spg_csr_free(self.engine.ctx, ctypes.byref(self.s))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Engine:
    """One library context on one GPU (its own stream, or torch's current one)."""

    def __init__(self, device: int = 0, use_torch_stream: bool = False):
        self.L = _lib.load()
        ctx = ctypes.c_void_p()
        st = self.L.spg_create(ctypes.byref(ctx), device)
        if st != _lib.SPG_OK:
            raise SpgError(st, "spg_create")
        self.ctx = ctx
        self.device = device
        if use_torch_stream:
            import torch

            self.L.spg_set_stream(self.ctx, ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream))

    def close(self) -> None:
        if self.ctx:
            self.L.spg_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int) -> None:
        if st != _lib.SPG_OK:
            raise SpgError(st, self.L.spg_last_error(self.ctx).decode(errors="replace"))

    @staticmethod
    def _as_struct(m, device: int):
        if isinstance(m, (DeviceCsr, HostCsr)):
            return m.struct(), m
        if isinstance(m, Csr):
            h = HostCsr(m)
            return h.struct(), h
        raise TypeError(f"unsupported matrix type {type(m)}")

    def opts(self, algo="learned", out="device", out_index_bits=0, stage_timing=False, force_overflow=False,
             use_tuning=False, use_graph=False, skip_validation=False, cusparse_alg=0) -> _lib.SpgOpts:
        o = _lib.SpgOpts()
        o.algo = ALGOS[algo] if isinstance(algo, str) else int(algo)
        o.out_location = _lib.SPG_HOST if out == "host" else _lib.SPG_DEVICE
        o.out_index_bits = out_index_bits
        o.stage_timing = int(stage_timing)
        o.force_overflow = int(force_overflow)
        o.use_tuning = int(use_tuning)
        o.use_graph = int(use_graph)
        o.skip_validation = int(skip_validation)
        o.reserved[0] = cusparse_alg
        return o

    def multiply(self, A, B, **kw):
        """C = A*B. Returns (Result, report dict)."""
        sa, ka = self._as_struct(A, self.device)
        sb, kb = self._as_struct(B, self.device)
        o = self.opts(**kw)
        c = _lib.SpgCsr()
        rep = _lib.SpgReport()
        self._check(self.L.spg_multiply(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                        ctypes.byref(o), ctypes.byref(rep)))
        return Result(self, c), rep.as_dict()

    def multiply_into_host(self, A, B, row_ptr, col_idx, val, blocks: int = 8, index_bits: int = 64, **kw):
        """C = A*B written into caller host arrays (numpy or pinned torch tensors,
        len(col_idx) = capacity), the download overlapped with the product in
        `blocks` row blocks. Returns (nnz, report dict)."""
        sa, ka = self._as_struct(A, self.device)
        sb, kb = self._as_struct(B, self.device) if B is not A else (sa, ka)
        c = self._host_out(row_ptr, col_idx, val, index_bits)
        o = self.opts(**kw)
        rep = _lib.SpgReport()
        self._check(self.L.spg_multiply_into_host(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                                  int(blocks), ctypes.byref(o), ctypes.byref(rep)))
        return int(c.nnz), rep.as_dict()

    def multiply_into_host_raw(self, sa: _lib.SpgCsr, sb: _lib.SpgCsr, c: _lib.SpgCsr, blocks: int,
                               o: _lib.SpgOpts, rep: _lib.SpgReport) -> None:
        """Low-overhead call on prepared structs (benchmark loops)."""
        self._check(self.L.spg_multiply_into_host(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                                  int(blocks), ctypes.byref(o), ctypes.byref(rep)))

    @staticmethod
    def _host_out(row_ptr, col_idx, val, index_bits: int) -> _lib.SpgCsr:
        def ptr(x):
            return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data

        c = _lib.SpgCsr()
        c.index_bits = index_bits
        c.location = _lib.SPG_HOST
        c.row_ptr = ptr(row_ptr)
        c.col_idx = ptr(col_idx) if len(col_idx) else 0
        c.val = ptr(val) if len(val) else 0
        c.capacity = len(col_idx)
        return c

    def multiply_reuse(self, A, B, C: "Result", **kw):
        """Recomputes the values of C = A*B in place; C (a device Result of an
        earlier multiply) holds the structure of A*B. Returns the report dict."""
        sa, ka = self._as_struct(A, self.device)
        sb, kb = self._as_struct(B, self.device)
        o = self.opts(**kw)
        rep = _lib.SpgReport()
        self._check(self.L.spg_multiply_reuse(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(C.s),
                                              ctypes.byref(o), ctypes.byref(rep)))
        return rep.as_dict()

    def multiply_reuse_raw(self, sa: _lib.SpgCsr, sb: _lib.SpgCsr, o: _lib.SpgOpts, c: _lib.SpgCsr,
                           rep: _lib.SpgReport) -> None:
        """Low-overhead value-only recompute on prepared structs (benchmark loops)."""
        self._check(self.L.spg_multiply_reuse(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                              ctypes.byref(o), ctypes.byref(rep)))

    def multiply_raw(self, sa: _lib.SpgCsr, sb: _lib.SpgCsr, o: _lib.SpgOpts, c: _lib.SpgCsr,
                     rep: _lib.SpgReport) -> None:
        """Low-overhead call on prepared structs (benchmark loops)."""
        self._check(self.L.spg_multiply(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(c),
                                        ctypes.byref(o), ctypes.byref(rep)))

    def download_raw(self, c: _lib.SpgCsr, row_ptr: int, col_idx: int, val: int) -> None:
        """Copies a device C into caller host buffers (raw pointers) and waits."""
        self._check(self.L.spg_csr_download(self.ctx, ctypes.byref(c), row_ptr, col_idx, val))

    def free_raw(self, c: _lib.SpgCsr) -> None:
        self.L.spg_csr_free(self.ctx, ctypes.byref(c))

    def check(self, A, B, C) -> dict:
        """FP64 check of C = A*B on the GPU (spg_check): max / mean |c - c64|,
        max |c - c64| / sum|a*b|, missing and extra entries."""
        sa, ka = self._as_struct(A, self.device)
        sb, kb = self._as_struct(B, self.device)
        sc, kc = (C.s, C) if isinstance(C, Result) else self._as_struct(C, self.device)
        rep = _lib.SpgCheckReport()
        self._check(self.L.spg_check(self.ctx, ctypes.byref(sa), ctypes.byref(sb), ctypes.byref(sc),
                                     ctypes.byref(rep)))
        return rep.as_dict()

    def multiply_batched(self, As, Bs, use_graph=True, use_tuning=False, skip_validation=False, algo="plain",
                         force_overflow=False):
        """Independent products C_i = A_i*B_i (device inputs). Returns (results, report).

        Results of the persistent batched path live in the engine's batch
        buffers until the next batched call with other inputs."""
        n = len(As)
        sa = (_lib.SpgCsr * n)(*[a.struct() for a in As])
        sb = (_lib.SpgCsr * n)(*[b.struct() for b in Bs])
        sc = (_lib.SpgCsr * n)()
        o = self.opts(algo=algo, use_graph=use_graph, use_tuning=use_tuning, skip_validation=skip_validation,
                      force_overflow=force_overflow)
        rep = _lib.SpgReport()
        self._check(self.L.spg_multiply_batched(self.ctx, n, sa, sb, sc, ctypes.byref(o), ctypes.byref(rep)))
        return [Result(self, sc[i]) for i in range(n)], rep.as_dict()

    # ---- predictor -------------------------------------------------------
    def features(self, A: DeviceCsr, B: DeviceCsr):
        import torch

        out = torch.empty((A.rows, 8), dtype=torch.float32, device=A.col_idx.device)
        sa, sb = A.struct(), B.struct()
        self._check(self.L.spg_features(self.ctx, ctypes.byref(sa), ctypes.byref(sb), out.data_ptr()))
        return out

    def row_nnz(self, A: DeviceCsr, B: DeviceCsr):
        import torch

        out = torch.empty((A.rows,), dtype=torch.int64, device=A.col_idx.device)
        sa, sb = A.struct(), B.struct()
        self._check(self.L.spg_row_nnz(self.ctx, ctypes.byref(sa), ctypes.byref(sb), out.data_ptr()))
        return out

    def mlp_predict(self, feats):
        import torch

        out = torch.empty((feats.shape[0], 2), dtype=torch.float32, device=feats.device)
        self._check(self.L.spg_mlp_predict(self.ctx, feats.data_ptr(), feats.shape[0], out.data_ptr()))
        return out

    def mlp_grad(self, feats, targets):
        g = (ctypes.c_float * _lib.SPG_MLP_PARAMS)()
        loss = ctypes.c_float()
        self._check(self.L.spg_mlp_grad(self.ctx, feats.data_ptr(), targets.data_ptr(), feats.shape[0],
                                        ctypes.byref(loss), g))
        return float(loss.value), np.ctypeslib.as_array(g).copy()

    def mlp_init(self, seed: int = 0) -> None:
        self._check(self.L.spg_mlp_init(self.ctx, seed))

    def mlp_load(self, path: str) -> None:
        self._check(self.L.spg_mlp_load(self.ctx, path.encode()))

    def mlp_save(self, path: str) -> None:
        self._check(self.L.spg_mlp_save(self.ctx, path.encode()))

    def mlp_params(self) -> np.ndarray:
        p = np.zeros(_lib.SPG_MLP_PARAMS, dtype=np.float32)
        self._check(self.L.spg_mlp_get_params(self.ctx, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))
        return p

    def mlp_set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.L.spg_mlp_set_params(self.ctx, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), p.size))

    def mlp_train(self, As, Bs, epochs=20, batch=4096, lr=2e-3, weight_decay=1e-5, max_rows_per_matrix=20000,
                  seed=1) -> dict:
        n = len(As)
        sa = (_lib.SpgCsr * n)(*[a.struct() for a in As])
        sb = (_lib.SpgCsr * n)(*[b.struct() for b in Bs])
        o = _lib.SpgTrainOpts()
        o.epochs, o.batch, o.lr, o.weight_decay = epochs, batch, lr, weight_decay
        o.max_rows_per_matrix, o.seed = max_rows_per_matrix, seed
        r = _lib.SpgTrainReport()
        self._check(self.L.spg_mlp_train(self.ctx, n, sa, sb, ctypes.byref(o), ctypes.byref(r)))
        return {"final_loss": r.final_loss, "ms_train": r.ms_train, "rows_used": r.rows_used, "steps": r.steps}

    # ---- tuning ------------------------------------------------------------
    def get_tuning(self) -> dict:
        t = _lib.SpgTuning()
        self._check(self.L.spg_get_tuning(self.ctx, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw) -> None:
        t = _lib.SpgTuning()
        self._check(self.L.spg_get_tuning(self.ctx, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        self._check(self.L.spg_set_tuning(self.ctx, ctypes.byref(t)))

    def tune(self, As, Bs, cache_path: str | None = None) -> dict:
        n = len(As)
        sa = (_lib.SpgCsr * n)(*[a.struct() for a in As])
        sb = (_lib.SpgCsr * n)(*[b.struct() for b in Bs])
        t = _lib.SpgTuning()
        self._check(self.L.spg_tune(self.ctx, n, sa, sb, cache_path.encode() if cache_path else None,
                                    ctypes.byref(t)))
        return t.as_dict()

    def coo_to_csr(self, rows: int, cols: int, row_idx, col_idx, val) -> Result:
        """Device CSR from 0-based COO arrays in any order (numpy: uploaded,
        or torch CUDA tensors: used in place), built on the GPU; duplicates
        are summed in the order given."""
        def ptr(x):
            return x.data_ptr() if hasattr(x, "data_ptr") else x.ctypes.data

        r = np.ascontiguousarray(row_idx, np.int32) if not hasattr(row_idx, "data_ptr") else row_idx
        c = np.ascontiguousarray(col_idx, np.int32) if not hasattr(col_idx, "data_ptr") else col_idx
        v = np.ascontiguousarray(val, np.float32) if not hasattr(val, "data_ptr") else val
        loc = _lib.SPG_DEVICE if hasattr(row_idx, "data_ptr") and row_idx.is_cuda else _lib.SPG_HOST
        n = len(r)
        out = _lib.SpgCsr()
        self._check(self.L.spg_coo_to_csr(self.ctx, int(rows), int(cols), int(n), ptr(r) if n else None,
                                          ptr(c) if n else None, ptr(v) if n else None, loc, ctypes.byref(out)))
        return Result(self, out)

    def read_mtx_device(self, path: str) -> Result:
        """Matrix Market file -> device CSR: parsed on the host threads, the
        CSR built on the GPU from the file's COO."""
        out = _lib.SpgCsr()
        self._check(self.L.spg_mtx_read_device(self.ctx, os.fsencode(path), ctypes.byref(out)))
        return Result(self, out)

    def write_mtx(self, path: str, C, drop_zeros: bool = False) -> None:
        s = C.s if isinstance(C, Result) else self._as_struct(C, self.device)[0]
        self._check(self.L.spg_mtx_write(self.ctx, path.encode(), ctypes.byref(s), int(drop_zeros)))


def read_mtx(path: str) -> Csr:
    """Reads a Matrix Market file with the library's reader."""
    L = _lib.load()
    s = _lib.SpgCsr()
    st = L.spg_mtx_read(os.fsencode(path), ctypes.byref(s))
    if st != _lib.SPG_OK:
        raise SpgError(st, path)
    try:
        rp = np.ctypeslib.as_array(ctypes.cast(s.row_ptr, ctypes.POINTER(ctypes.c_int64)), shape=(s.rows + 1,)).copy()
        if s.nnz:
            col = np.ctypeslib.as_array(ctypes.cast(s.col_idx, ctypes.POINTER(ctypes.c_int32)), shape=(s.nnz,)).copy()
            val = np.ctypeslib.as_array(ctypes.cast(s.val, ctypes.POINTER(ctypes.c_float)), shape=(s.nnz,)).copy()
        else:
            col, val = np.zeros(0, np.int32), np.zeros(0, np.float32)
    finally:
        L.spg_csr_free(None, ctypes.byref(s))
    return Csr(int(s.rows), int(s.cols), rp, col, val)


def transpose(m: Csr) -> Csr:
    """Transpose of a host Csr with the library's host routine (no GPU needed)."""
    L = _lib.load()
    h = HostCsr(m)
    src = h.struct()
    t = _lib.SpgCsr()
    st = L.spg_csr_transpose(ctypes.byref(src), ctypes.byref(t))
    if st != _lib.SPG_OK:
        raise SpgError(st, "spg_csr_transpose")
    try:
        rp = np.ctypeslib.as_array(ctypes.cast(t.row_ptr, ctypes.POINTER(ctypes.c_int64)), shape=(t.rows + 1,)).copy()
        n = int(t.nnz)
        col = np.ctypeslib.as_array(ctypes.cast(t.col_idx, ctypes.POINTER(ctypes.c_int32)), shape=(n,)).copy() \
            if n else np.zeros(0, np.int32)
        val = np.ctypeslib.as_array(ctypes.cast(t.val, ctypes.POINTER(ctypes.c_float)), shape=(n,)).copy() \
            if n else np.zeros(0, np.float32)
    finally:
        L.spg_csr_free(None, ctypes.byref(t))
    return Csr(int(t.rows), int(t.cols), rp, col, val)


def write_mtx(path: str, m: Csr, drop_zeros: bool = False) -> None:
    """Writes a host Csr with the library's writer (no GPU needed)."""
    L = _lib.load()
    h = HostCsr(m)
    s = h.struct()
    st = L.spg_mtx_write(None, os.fsencode(path), ctypes.byref(s), int(drop_zeros))
    if st != _lib.SPG_OK:
        raise SpgError(st, path)
