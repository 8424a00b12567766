"""Generates the golden fixtures: outputs of the reference's own program.

The reference ships no expected outputs, so this script runs the reference's
cuSPARSE driver -- cuSparse/src/main.cpp built with -DREUSE (the variant that
writes C as a full 1-based COO) by oracle/Makefile into oracle/_ref/ -- on
small seeded inputs and stores inputs and output together:

    tests/golden/<case>.npz : a_rp a_col a_val b_rp b_col b_val c_rp c_col c_val
                              (0-based CSR; c_val parsed from the reference's
                              text output, which prints 6 significant digits)

It needs a GPU (cuSPARSE) and the built reference binary:

    make -C oracle ref          # where the reference sources are present
    python tests/golden/make_golden.py [--out tests/golden]

Inputs are written row-major with sorted columns because the driver's
COO->CSR conversion (cuSparse/src/main.cpp:186-190) assumes row-sorted COO.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from rtspmspm_b200 import gen  # noqa: E402
from rtspmspm_b200.gen import coo_to_csr  # noqa: E402

REF_BIN = os.path.join(ROOT, "oracle", "_ref", "cusparse_ref")


def cases():
    """Seeded (name, A, B) inputs, small enough to commit."""
    return [
        ("er256_p8", gen.erdos_renyi(256, 256, 8.0, 0), None),
        ("er1024_p8", gen.erdos_renyi(1024, 1024, 8.0, 0), None),
        ("rect_300x500x150", gen.erdos_renyi(300, 500, 6.0, 3), gen.erdos_renyi(500, 150, 7.0, 4)),
        ("stencil8", gen.stencil27(8, seed=1), None),
        ("rmat9", gen.rmat(9, 16, seed=2), None),
        ("ones12", coo_to_csr(12, 12, np.repeat(np.arange(12), 12), np.tile(np.arange(12), 12),
                              np.ones(144, np.float32)), None),
    ]


def write_mtx(path: str, m) -> None:
    from rtspmspm_b200 import write_mtx as w

    w(path, m)


def read_ref_output(path: str, rows: int, cols: int):
    with open(path) as f:
        lines = f.read().split("\n")
    body = [ln for ln in lines[2:] if ln.strip()]
    if not body:
        return coo_to_csr(rows, cols, [], [], np.zeros(0, np.float32))
    arr = np.array([ln.split() for ln in body])
    r = arr[:, 0].astype(np.int64) - 1
    c = arr[:, 1].astype(np.int64) - 1
    v = arr[:, 2].astype(np.float64).astype(np.float32)
    key = r * cols + c
    if np.unique(key).size != key.size:
        raise RuntimeError("reference output has duplicate entries")
    return coo_to_csr(rows, cols, r, c, v)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(ROOT, "tests", "golden"))
    args = ap.parse_args(argv)
    if not os.path.exists(REF_BIN):
        print(f"reference driver not built: {REF_BIN} (make -C oracle ref)", file=sys.stderr)
        return 2
    os.makedirs(args.out, exist_ok=True)
    with tempfile.TemporaryDirectory() as td:
        for name, A, B in cases():
            B = A if B is None else B
            pa, pb, pc, pl = (os.path.join(td, f"{name}_{x}") for x in ("a.mtx", "b.mtx", "c.mtx", "log.txt"))
            write_mtx(pa, A)
            write_mtx(pb, B)
            subprocess.run([REF_BIN, "-m1", pa, "-m2", pb, "-o", pc, "-l", pl], check=True,
                           stdout=subprocess.DEVNULL)
            C = read_ref_output(pc, A.rows, B.cols)
            np.savez_compressed(os.path.join(args.out, f"{name}.npz"),
                                a_rp=A.row_ptr, a_col=A.col_idx, a_val=A.val, a_shape=np.array([A.rows, A.cols]),
                                b_rp=B.row_ptr, b_col=B.col_idx, b_val=B.val, b_shape=np.array([B.rows, B.cols]),
                                c_rp=C.row_ptr, c_col=C.col_idx, c_val=C.val)
            print(f"{name}: nnz(C)={C.nnz}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
