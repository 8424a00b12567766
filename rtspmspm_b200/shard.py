"""Row-block sharding of C = A*B over ranks (one process per GPU).

Rows of C are independent, so the product shards by row blocks of A with B
replicated: rank r computes C[r0:r1) = A[r0:r1) * B with no data-path
collective.  Blocks are balanced by intermediate products (the work), not
by rows.  Gathering the blocks into one CSR on a single rank is optional and
is the only exchange (sizes, then entries).  The reference runs one product
per process on one GPU; this module only adds the row partition.
"""
from __future__ import annotations

import numpy as np

from .gen import Csr, row_products


def partition_rows(A: Csr, B: Csr, world: int) -> np.ndarray:
    """Row boundaries (world+1 entries) splitting the products evenly."""
    if world < 1:
        raise ValueError("world must be >= 1")
    prod = row_products(A, B)
    cum = np.concatenate([[0], np.cumsum(prod, dtype=np.int64)])
    total = int(cum[-1])
    bounds = [0]
    for r in range(1, world):
        target = total * r // world
        bounds.append(int(np.searchsorted(cum, target, side="left")))
    bounds.append(A.rows)
    b = np.maximum.accumulate(np.array(bounds, dtype=np.int64))
    b[-1] = A.rows
    return b


def local_block(A: Csr, bounds: np.ndarray, rank: int) -> Csr:
    return A.row_block(int(bounds[rank]), int(bounds[rank + 1]))


def gather_blocks(parts, rows: int, cols: int) -> Csr:
    """Concatenates per-rank row blocks (in rank order) into one CSR."""
    rp = [np.zeros(1, np.int64)]
    base = 0
    cols_l, vals_l = [], []
    for p in parts:
        rp.append(np.asarray(p.row_ptr[1:], np.int64) + base)
        base += int(p.row_ptr[-1])
        cols_l.append(np.asarray(p.col_idx, np.int32))
        vals_l.append(np.asarray(p.val, np.float32))
    row_ptr = np.concatenate(rp)
    if row_ptr.size != rows + 1:
        raise ValueError("blocks do not cover the rows")
    return Csr(rows, cols, row_ptr, np.concatenate(cols_l) if cols_l else np.zeros(0, np.int32),
               np.concatenate(vals_l) if vals_l else np.zeros(0, np.float32))


def gather_to_rank0(dist, part: Csr, rows: int, cols: int):
    """All ranks send their block to rank 0 over torch.distributed (any
    backend); rank 0 returns the full C, the others None."""
    import torch

    world = dist.get_world_size()
    rank = dist.get_rank()
    meta = torch.tensor([part.rows, part.nnz], dtype=torch.int64)
    metas = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(metas, meta)
    if rank == 0:
        parts = [part]
        for src in range(1, world):
            pr, pn = (int(x) for x in metas[src])
            rp = torch.zeros(pr + 1, dtype=torch.int64)
            ci = torch.zeros(pn, dtype=torch.int32)
            va = torch.zeros(pn, dtype=torch.float32)
            for t in (rp, ci, va):
                dist.recv(t, src=src)
            parts.append(Csr(pr, cols, rp.numpy(), ci.numpy(), va.numpy()))
        return gather_blocks(parts, rows, cols)
    for t in (torch.from_numpy(np.asarray(part.row_ptr, np.int64)),
              torch.from_numpy(np.asarray(part.col_idx, np.int32)),
              torch.from_numpy(np.asarray(part.val, np.float32))):
        dist.send(t.contiguous(), dst=0)
    return None
