"""N > 1: row-block sharding with world_size 2 over gloo on CPU.  Each rank
computes its block (with the oracle standing in for the GPU) and rank 0
gathers; the result must equal the single-rank product exactly."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from oracle import oracle
from rtspmspm_b200 import gen, shard


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = gen.rmat(11, 16, seed=7)
        bounds = shard.partition_rows(A, A, world)
        part = shard.local_block(A, bounds, rank)
        Cp = oracle.spgemm(part, A, twin=False)
        full = shard.gather_to_rank0(dist, Cp, A.rows, A.cols)
        # the timing rule of the benchmark: the slowest rank counts
        import torch

        t = torch.tensor([float(rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        if rank == 0:
            q.put((full.row_ptr, full.col_idx, full.val, float(t.item())))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_partition_balances_products():
    A = gen.rmat(12, 16, seed=1)
    for world in (1, 2, 3, 8):
        b = shard.partition_rows(A, A, world)
        assert b[0] == 0 and b[-1] == A.rows and np.all(np.diff(b) >= 0)
        prod = gen.row_products(A, A)
        per = [prod[b[r]:b[r + 1]].sum() for r in range(world)]
        assert max(per) <= prod.sum() / world + prod.max()


def test_gloo_world2_sharded_product_matches_single():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    rp, ci, va, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    A = gen.rmat(11, 16, seed=7)
    R = oracle.spgemm(A, A, twin=False)
    np.testing.assert_array_equal(rp, R.row_ptr)
    np.testing.assert_array_equal(ci, R.col_idx)
    np.testing.assert_array_equal(va.view(np.uint32), R.val.view(np.uint32))
    assert tmax == 2.0
