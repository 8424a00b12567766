"""B200-native SpGEMM engine (C = A*B on CSR matrices).

The compute path is librtspmspm.so (hand-written sm_100a CUDA behind the C
ABI of include/rtspmspm.h); this package is the host-side binding, the
synthetic workload generators and the build script.
"""
from . import gen
from .engine import DeviceCsr, Engine, HostCsr, Result, SpgError, read_mtx, transpose, write_mtx
from .gen import Csr

__all__ = ["gen", "Csr", "DeviceCsr", "Engine", "HostCsr", "Result", "SpgError", "read_mtx", "transpose",
           "write_mtx"]
