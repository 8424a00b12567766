"""Builds the engine in-tree for sm_100a.

Outputs (next to this file):
  librtspmspm.so  -- the C-ABI library (include/rtspmspm.h)
  spgemm          -- the drop-in CLI (-m1 -m2 -o -l)
Objects go to rtspmspm_b200/_build/.  Compilation is incremental (by mtime
of the source and of every header) and runs nvcc jobs in parallel.

    python -m rtspmspm_b200.build [--force]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")
LIB = os.path.join(HERE, "librtspmspm.so")
CLI = os.path.join(HERE, "spgemm")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC",
                     "-Xcompiler", "-Wall", "--expt-relaxed-constexpr", "-I" + INCLUDE]
LIB_SOURCES = ["kernels.cu", "mlp.cu", "api.cu", "mlp_api.cu", "batched.cu",
               "cusparse_ref.cu", "mtx_io.cpp", "tune.cpp", "noalloc.cu", "heavy.cu", "check.cu", "coo.cu"]


def nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _headers():
    return [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".hpp", ".cuh", ".h"))] + \
        [os.path.join(INCLUDE, "rtspmspm.h")]


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        lang = ["-x", "cu"] if src.endswith(".cpp") and not src.endswith("cli.cpp") else []
        cmd = [nvcc()] + NVCC_FLAGS + lang + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(SRC, s) for s in LIB_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
        cli_obj = ex.submit(_compile, os.path.join(SRC, "cli.cpp"), force).result()
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcusparse", "-ldl"]
        subprocess.run(cmd, check=True, capture_output=not verbose)
    if force or _stale(CLI, [cli_obj, LIB]):
        cmd = [nvcc()] + ARCH + ["-o", CLI, cli_obj, "-L" + HERE, "-lrtspmspm",
                                 "-Xlinker", "-rpath,$ORIGIN"]
        subprocess.run(cmd, check=True, capture_output=not verbose)
    return LIB


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args(argv)
    path = build(force=args.force, verbose=True)
    print(path)
    return 0


if __name__ == "__main__":
    sys.exit(main())
