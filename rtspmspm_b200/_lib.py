"""ctypes declarations of the C ABI in include/rtspmspm.h.

Structure layouts and constants here must match the header; the CPU test
suite checks that every symbol the header declares is exported.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librtspmspm.so")

SPG_OK = 0
SPG_ERR_INVALID_ARG = 1
SPG_ERR_CUDA = 2
SPG_ERR_OUT_OF_MEMORY = 3
SPG_ERR_IO = 4
SPG_ERR_FORMAT = 5
SPG_ERR_TIMEOUT = 6
SPG_ERR_UNSUPPORTED = 7
SPG_ERR_INTERNAL = 8

SPG_HOST = 0
SPG_DEVICE = 1

SPG_ALGO_PLAIN = 0
SPG_ALGO_LEARNED = 1
SPG_ALGO_CUSPARSE = 2

SPG_STAGE_COUNT = 12
SPG_NUM_BINS = 16
SPG_MLP_PARAMS = 8 * 64 + 64 + 64 * 64 + 64 + 64 * 2 + 2

STAGES = ["upload", "products", "binning", "symbolic", "scan", "numeric", "features",
          "mlp", "fixup", "compact", "download", "other"]


class SpgCsr(ctypes.Structure):
    _fields_ = [("rows", ctypes.c_int64), ("cols", ctypes.c_int64), ("nnz", ctypes.c_int64),
                ("index_bits", ctypes.c_int32), ("location", ctypes.c_int32),
                ("row_ptr", ctypes.c_void_p), ("col_idx", ctypes.c_void_p), ("val", ctypes.c_void_p),
                ("capacity", ctypes.c_int64), ("owner", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class SpgOpts(ctypes.Structure):
    _fields_ = [("algo", ctypes.c_int32), ("out_location", ctypes.c_int32),
                ("out_index_bits", ctypes.c_int32), ("stage_timing", ctypes.c_int32),
                ("force_overflow", ctypes.c_int32), ("use_tuning", ctypes.c_int32),
                ("use_graph", ctypes.c_int32), ("skip_validation", ctypes.c_int32),
                ("reserved", ctypes.c_int32 * 4)]


class SpgReport(ctypes.Structure):
    _fields_ = [("ms_total", ctypes.c_double), ("ms_stage", ctypes.c_double * SPG_STAGE_COUNT),
                ("products", ctypes.c_int64), ("nnz_c", ctypes.c_int64), ("rows", ctypes.c_int64),
                ("rows_predicted", ctypes.c_int64), ("rows_overflow", ctypes.c_int64),
                ("rows_heavy", ctypes.c_int64), ("bin_rows", ctypes.c_int64 * SPG_NUM_BINS),
                ("algo", ctypes.c_int32), ("device_flags", ctypes.c_int32),
                ("kernel_launches", ctypes.c_int32), ("small_path", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {
            "ms_total": self.ms_total,
            "stages_ms": {STAGES[i]: self.ms_stage[i] for i in range(SPG_STAGE_COUNT) if self.ms_stage[i]},
            "products": self.products, "nnz_c": self.nnz_c, "rows": self.rows,
            "rows_predicted": self.rows_predicted, "rows_overflow": self.rows_overflow,
            "rows_heavy": self.rows_heavy, "bin_rows": list(self.bin_rows),
            "device_flags": self.device_flags, "kernel_launches": self.kernel_launches,
            "small_path": self.small_path,
        }


class SpgTrainOpts(ctypes.Structure):
    _fields_ = [("epochs", ctypes.c_int32), ("batch", ctypes.c_int32), ("lr", ctypes.c_float),
                ("weight_decay", ctypes.c_float), ("max_rows_per_matrix", ctypes.c_int64),
                ("seed", ctypes.c_uint64), ("reserved", ctypes.c_int32 * 4)]


class SpgTrainReport(ctypes.Structure):
    _fields_ = [("final_loss", ctypes.c_double), ("ms_train", ctypes.c_double),
                ("rows_used", ctypes.c_int64), ("steps", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class SpgTuning(ctypes.Structure):
    _fields_ = [("warp_table_max", ctypes.c_int32), ("warps_per_block", ctypes.c_int32),
                ("max_load", ctypes.c_float), ("tile_cols", ctypes.c_int32),
                ("block_table_max", ctypes.c_int32), ("predict_margin", ctypes.c_float),
                ("predict_slack", ctypes.c_int32), ("learned_load", ctypes.c_float),
                ("heavy_path", ctypes.c_int32), ("block_min_nnz", ctypes.c_int32), ("esc_min_prod", ctypes.c_int32),
                ("small_rows", ctypes.c_int32)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


class SpgCheckReport(ctypes.Structure):
    _fields_ = [("entries", ctypes.c_int64), ("missing", ctypes.c_int64), ("extra", ctypes.c_int64),
                ("max_abs_err_fp64", ctypes.c_double), ("mean_abs_err_fp64", ctypes.c_double),
                ("max_rel_err", ctypes.c_double), ("reserved", ctypes.c_int32 * 4)]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


# (name, restype, argtypes) of every exported entry point
_P = ctypes.POINTER
_vp = ctypes.c_void_p
SIGNATURES = [
    ("spg_version", ctypes.c_int32, []),
    ("spg_status_string", ctypes.c_char_p, [ctypes.c_int32]),
    ("spg_create", ctypes.c_int32, [_P(_vp), ctypes.c_int32]),
    ("spg_destroy", ctypes.c_int32, [_vp]),
    ("spg_last_error", ctypes.c_char_p, [_vp]),
    ("spg_set_stream", ctypes.c_int32, [_vp, _vp]),
    ("spg_get_stream", _vp, [_vp]),
    ("spg_multiply", ctypes.c_int32, [_vp, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), _P(SpgOpts), _P(SpgReport)]),
    ("spg_csr_transpose", ctypes.c_int32, [_P(SpgCsr), _P(SpgCsr)]),
    ("spg_multiply_into_host", ctypes.c_int32,
     [_vp, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), ctypes.c_int32, _P(SpgOpts), _P(SpgReport)]),
    ("spg_multiply_reuse", ctypes.c_int32, [_vp, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), _P(SpgOpts), _P(SpgReport)]),
    ("spg_multiply_batched", ctypes.c_int32,
     [_vp, ctypes.c_int32, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), _P(SpgOpts), _P(SpgReport)]),
    ("spg_multiply_noalloc", ctypes.c_int32,
     [_vp, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), ctypes.c_char_p, ctypes.c_int32]),
    ("spg_check", ctypes.c_int32, [_vp, _P(SpgCsr), _P(SpgCsr), _P(SpgCsr), _P(SpgCheckReport)]),
    ("spg_csr_free", ctypes.c_int32, [_vp, _P(SpgCsr)]),
    ("spg_csr_copy", ctypes.c_int32, [_vp, _P(SpgCsr), ctypes.c_int32, _P(SpgCsr)]),
    ("spg_csr_download", ctypes.c_int32, [_vp, _P(SpgCsr), _vp, _vp, _vp]),
    ("spg_csr_extract_rows", ctypes.c_int32, [_vp, _P(SpgCsr), _vp, ctypes.c_int64, _P(SpgCsr)]),
    ("spg_mtx_read", ctypes.c_int32, [ctypes.c_char_p, _P(SpgCsr)]),
    ("spg_mtx_read_device", ctypes.c_int32, [_vp, ctypes.c_char_p, _P(SpgCsr)]),
    ("spg_coo_to_csr", ctypes.c_int32, [_vp, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64, _vp, _vp, _vp,
                                        ctypes.c_int32, _P(SpgCsr)]),
    ("spg_mtx_write", ctypes.c_int32, [_vp, ctypes.c_char_p, _P(SpgCsr), ctypes.c_int32]),
    ("spg_mlp_load", ctypes.c_int32, [_vp, ctypes.c_char_p]),
    ("spg_mlp_save", ctypes.c_int32, [_vp, ctypes.c_char_p]),
    ("spg_mlp_init", ctypes.c_int32, [_vp, ctypes.c_uint64]),
    ("spg_mlp_get_params", ctypes.c_int32, [_vp, _P(ctypes.c_float), ctypes.c_int64]),
    ("spg_mlp_set_params", ctypes.c_int32, [_vp, _P(ctypes.c_float), ctypes.c_int64]),
    ("spg_mlp_train", ctypes.c_int32,
     [_vp, ctypes.c_int32, _P(SpgCsr), _P(SpgCsr), _P(SpgTrainOpts), _P(SpgTrainReport)]),
    ("spg_features", ctypes.c_int32, [_vp, _P(SpgCsr), _P(SpgCsr), _vp]),
    ("spg_row_nnz", ctypes.c_int32, [_vp, _P(SpgCsr), _P(SpgCsr), _vp]),
    ("spg_mlp_predict", ctypes.c_int32, [_vp, _vp, ctypes.c_int64, _vp]),
    ("spg_mlp_grad", ctypes.c_int32, [_vp, _vp, _vp, ctypes.c_int64, _P(ctypes.c_float), _P(ctypes.c_float)]),
    ("spg_get_tuning", ctypes.c_int32, [_vp, _P(SpgTuning)]),
    ("spg_set_tuning", ctypes.c_int32, [_vp, _P(SpgTuning)]),
    ("spg_tune", ctypes.c_int32, [_vp, ctypes.c_int32, _P(SpgCsr), _P(SpgCsr), ctypes.c_char_p, _P(SpgTuning)]),
]

_LIB = None


def load(path: str | None = None):
    """Loads librtspmspm.so (building it first if it is missing)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = path or LIB_PATH
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = ctypes.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib
