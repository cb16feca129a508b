"""The block driver's multi-rank path on CPU: gloo ranks, the oracle as block handler.

Each rank runs MPIComputeLowerTriangularBlocked.Compute over its blocks, the transposed blocks
are exchanged (Scatter) and rank 0 assembles the matrix; the result must equal the reference's
own multi-rank run (golden mpi_p3 / mpi_p4).  A second test covers the byte all-reduce that
merges the ranks' row slabs in the one-process-per-GPU path.
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


def _share_worker(rank, world, port, name, scheme, dst, q):
    """One rank of distributed_all_pairs with the oracle standing in for the engine's share: it
    writes this rank's pairs and, as the engine does, their mirrored entries too."""
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        import oracle
        from conftest import load_npz as ld
        from csharp_b200 import ScoringMatrix, block_is_computed
        from csharp_b200.driver import distributed_all_pairs
        z = ld(name)
        sc = ScoringMatrix.Load(z["matrix"].tobytes().decode()).Scores[:127, :127].astype(np.float32)
        concat, off = z["concat"], z["offsets"]
        N = len(off) - 1

        def share(r, w, out, ranges):
            lo, hi = ranges[r]
            if scheme == "balanced":
                qi = [(a, b) for a in range(lo, hi + 1) for b in range(a)]
            else:
                qi = []
                for c, (cs, ce) in enumerate(ranges):
                    if c == r:
                        qi += [(a, b) for a in range(lo, hi + 1) for b in range(cs, a)]
                    elif block_is_computed(r, c):
                        qi += [(a, b) for a in range(lo, hi + 1) for b in range(cs, ce + 1)]
            if not qi:
                return 0
            rr = np.array([x[0] for x in qi]); cc = np.array([x[1] for x in qi])
            d = oracle.pairs(concat, off, rr, cc, sc, float(z["o"]), float(z["e"]), int(z["alignment_type"]))
            t = torch.from_numpy(d)
            out[torch.from_numpy(rr), torch.from_numpy(cc)] = t
            out[torch.from_numpy(cc), torch.from_numpy(rr)] = t  # mirrors, some in other ranks' rows
            return len(qi)
        share.lengths = np.diff(off)
        out = torch.zeros((N, N), dtype=torch.int16)
        n = distributed_all_pairs(None, out, rank, world, scheme=scheme, dst=dst, share=share)
        if dst is None or rank == dst:
            q.put((rank, n, np.array_equal(out.numpy(), z["distances"])))
        else:
            q.put((rank, n, None))
    except Exception as e:
        q.put((rank, -1, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world,scheme,dst", [("mpi_p3.npz", 3, "checkerboard", None),
                                                   ("mpi_p4.npz", 4, "checkerboard", 0),
                                                   ("mpi_p1.npz", 2, "balanced", None),
                                                   ("mpi_p1.npz", 3, "balanced", 1)])
def test_row_slab_merge_matches_reference_runs(name, world, scheme, dst):
    """distributed_all_pairs' partition and merge over gloo ranks: the reference's 3- and 4-rank
    matrices (checkerboard orientation) and its 1-rank matrix (cost-balanced rows)."""
    z = load_npz(name)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_share_worker, args=(r, world, port, name, scheme, dst, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(n >= 0 for _, n, _ in res), res
    assert sum(n for _, n, _ in res) == int(z["pairs"])
    for r, _, ok in res:
        assert ok is (None if (dst is not None and r != dst) else True), (r, ok)


def test_balanced_ranges_cover_rows_with_equal_cells():
    from csharp_b200.driver import balanced_row_ranges
    rng = np.random.default_rng(2)
    lens = rng.integers(1, 2000, 3000)
    for w in (1, 2, 5, 8):
        r = balanced_row_ranges(lens, w)
        assert r[0][0] == 0 and r[-1][1] == len(lens) - 1
        assert all(r[k][1] + 1 == r[k + 1][0] for k in range(w - 1))
        before = np.concatenate([[0], np.cumsum(lens)[:-1]]).astype(np.float64)
        cost = lens * before
        share = [cost[a:b + 1].sum() / cost.sum() for a, b in r]
        assert max(share) - min(share) < 0.01
    assert balanced_row_ranges([5, 7], 4)[-1][1] == 1  # more ranks than rows: some ranks get none
