"""The C ABI library loads and exports every entry point include/rtspmspm.h
declares, and the ctypes layouts match the C structs (no GPU needed)."""
import ctypes
import os
import re
import subprocess

import pytest

from rtspmspm_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rtspmspm.h")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(spg_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    names = declared()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound


def test_status_strings_and_version():
    L = _lib.load()
    assert L.spg_version() >= 10000
    for st in range(9):
        assert L.spg_status_string(st)
    assert L.spg_last_error(None) == b"null context"


def test_struct_layouts_match_c(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text(f'''
#include <stdio.h>
#include <stddef.h>
#include "{HEADER}"
int main(void) {{
  printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(spg_csr), sizeof(spg_opts), sizeof(spg_report),
         sizeof(spg_tuning), sizeof(spg_train_opts), sizeof(spg_train_report));
  printf("%zu %zu %zu\\n", offsetof(spg_csr, val), offsetof(spg_report, products), offsetof(spg_opts, skip_validation));
  printf("%zu %zu\\n", sizeof(spg_check_report), offsetof(spg_check_report, max_rel_err));
  return 0;
}}''')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()
    got = [int(x) for x in out]
    want = [ctypes.sizeof(_lib.SpgCsr), ctypes.sizeof(_lib.SpgOpts), ctypes.sizeof(_lib.SpgReport),
            ctypes.sizeof(_lib.SpgTuning), ctypes.sizeof(_lib.SpgTrainOpts), ctypes.sizeof(_lib.SpgTrainReport),
            _lib.SpgCsr.val.offset, _lib.SpgReport.products.offset, _lib.SpgOpts.skip_validation.offset,
            ctypes.sizeof(_lib.SpgCheckReport), _lib.SpgCheckReport.max_rel_err.offset]
    assert got == want


def test_create_without_gpu_fails_cleanly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    L = _lib.load()
    ctx = ctypes.c_void_p()
    st = L.spg_create(ctypes.byref(ctx), 0)
    assert st == _lib.SPG_ERR_CUDA and not ctx.value
