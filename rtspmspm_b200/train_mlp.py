"""Trains the row-size predictor on the GPU and writes its weight file.

Training set: 200 generated products C = A*A --
  * 90 Erdos-Renyi matrices, 4k-256k rows, mean 4-32 nonzeros per row,
  * 55 27-point stencils, grids 32^3 .. 96^3,
  * 55 R-MAT graphs, scales 16 .. 20 (a=0.57, b=c=0.19),
with seeds disjoint from the evaluation workloads (R-MAT-20 seed 0 and the
stencil-96 of the benchmark).  Labels are the exact per-row nnz of the
engine's own symbolic pass; features come from its feature kernel; the
forward, backward and Adam kernels are the engine's own (spg_mlp_train).

    python -m rtspmspm_b200.train_mlp [--out rtspmspm_b200/data/mlp_default.bin]
"""
from __future__ import annotations

import argparse
import json
import multiprocessing as mp
import os
import time

import numpy as np

from . import gen

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_OUT = os.path.join(HERE, "data", "mlp_default.bin")


def recipe(count: int = 200, seed: int = 1234):
    """(kind, args) of every training matrix, drawn from one seeded stream."""
    rng = np.random.default_rng(seed)
    out = []
    n_er = int(round(count * 0.45))
    n_st = (count - n_er) // 2
    n_rm = count - n_er - n_st
    for i in range(n_er):
        n = int(round(np.exp(rng.uniform(np.log(4096), np.log(262144)))))
        mean = float(rng.uniform(4, 32))
        out.append(("er", (n, n, mean, 1000 + i)))
    grids = np.linspace(32, 96, n_st).round().astype(int)
    for i, g in enumerate(grids):
        out.append(("stencil", (int(g), 2000 + i)))
    # scales 16..20, weighted toward the cheaper ones
    scales = rng.choice([16, 17, 18, 19, 20], size=n_rm, p=[0.3, 0.25, 0.2, 0.15, 0.1])
    for i, s in enumerate(scales):
        out.append(("rmat", (int(s), 3000 + i)))
    return out


def make(item):
    kind, a = item
    if kind == "er":
        return gen.erdos_renyi(a[0], a[1], a[2], a[3])
    if kind == "stencil":
        return gen.stencil27(a[0], seed=a[1])
    return gen.rmat(a[0], 16, seed=a[1])


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--count", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--rows-per-matrix", type=int, default=20000)
    ap.add_argument("--workers", type=int, default=min(8, os.cpu_count() or 1))
    ap.add_argument("--report", default=None)
    args = ap.parse_args(argv)

    items = recipe(args.count)
    t0 = time.time()
    # generate on the host with a spawn pool before the first GPU call
    ctx = mp.get_context("spawn")
    with ctx.Pool(args.workers) as pool:
        mats = pool.map(make, items, chunksize=1)
    t_gen = time.time() - t0

    from .engine import Engine, HostCsr

    eng = Engine(0)
    eng.mlp_init(0)
    hosts = [HostCsr(m) for m in mats]
    t1 = time.time()
    rep = eng.mlp_train(hosts, hosts, epochs=args.epochs, batch=4096, lr=3e-3,
                        max_rows_per_matrix=args.rows_per_matrix, seed=7)
    t_train = time.time() - t1
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    eng.mlp_save(args.out)
    summary = {"matrices": len(mats), "kinds": {k: sum(1 for i in items if i[0] == k) for k in ("er", "stencil", "rmat")},
               "rows_used": rep["rows_used"], "steps": rep["steps"], "final_loss": rep["final_loss"],
               "ms_train_device": rep["ms_train"], "s_generate": round(t_gen, 1), "s_train_wall": round(t_train, 1),
               "out": os.path.relpath(args.out)}
    print(json.dumps(summary))
    if args.report:
        with open(args.report, "w") as f:
            json.dump(summary, f, indent=1)
    eng.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
