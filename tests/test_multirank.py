"""The block driver's multi-rank path on CPU: gloo ranks, the oracle as block handler.

Each rank runs MPIComputeLowerTriangularBlocked.Compute over its blocks, the transposed blocks
are exchanged (Scatter) and rank 0 assembles the matrix; the result must equal the reference's
own multi-rank run (golden mpi_p3 / mpi_p4).  A second test covers the byte all-reduce that
merges the ranks' disjoint entries in the one-process-per-GPU path.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from conftest import load_npz


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, name, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import oracle
        from conftest import load_npz as ld
        from csharp_b200 import ScoringMatrix
        from csharp_b200.driver import MPIComputeLowerTriangularBlocked
        z = ld(name)
        sc = ScoringMatrix.Load(z["matrix"].tobytes().decode()).Scores[:127, :127].astype(np.float32)
        N = len(z["offsets"]) - 1

        def handler(block, pm, is_diag):
            rs, re_ = block.RowRange.StartIndex, block.RowRange.EndIndex
            cs, ce = block.ColumnRange.StartIndex, block.ColumnRange.EndIndex
            blk, n = oracle.block(z["concat"], z["offsets"], rs, re_, cs, ce, is_diag, 0, sc,
                                  float(z["o"]), float(z["e"]), int(z["alignment_type"]))
            view = pm.block_view(block)
            if is_diag:
                view[...] = np.where(np.eye(len(blk), dtype=bool), view, blk)
            else:
                view[...] = blk
            return n

        drv = MPIComputeLowerTriangularBlocked(N, handler, rank, world)
        drv.Compute()
        drv.Scatter()
        full = drv.FullMatrixOnRank0()
        if rank == 0:
            q.put(("full", full))
    except Exception as e:  # report instead of leaving the parent waiting
        q.put(("error", repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world", [("mpi_p3.npz", 3), ("mpi_p4.npz", 4)])
def test_block_driver_gloo_matches_reference_multirank(name, world):
    z = load_npz(name)
    assert int(z["ranks"]) == world
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, q)) for r in range(world)]
    for p in procs:
        p.start()
    kind, full = q.get(timeout=300)
    assert kind == "full", full
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    np.testing.assert_array_equal(full, z["distances"])


def _reduce_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        N = 9
        full = (np.arange(N * N, dtype=np.int64).reshape(N, N) * 977 % 65536 - 32768).astype(np.int16)
        own = np.zeros((N, N), dtype=np.int16)
        mask = (np.add.outer(np.arange(N), np.arange(N)) % world) == rank
        own[mask] = full[mask]
        t = torch.from_numpy(own.copy())
        dist.all_reduce(t.view(torch.uint8).view(-1), op=dist.ReduceOp.SUM)
        q.put((rank, np.array_equal(t.numpy(), full)))
    finally:
        dist.destroy_process_group()


def test_disjoint_int16_entries_merge_by_byte_sum():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_reduce_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok in res)
