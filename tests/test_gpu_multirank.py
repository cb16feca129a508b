"""The one-process-per-GPU path with the engine: ranks as processes (here all on cuda:0, each
with its own context and engine; their kernels do not wait on one another), gloo collectives on
the host, distributed_all_pairs' partition and row-slab merge.  The merged matrix must equal the
reference's: its one-rank run for the cost-balanced scheme, its P-rank run for the checkerboard
(tolerance: exact Int16)."""
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, name, scheme, dst, mode, q):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parent.parent
    sys.path.insert(0, str(root))
    sys.path.insert(0, str(root / "tests"))
    from datetime import timedelta
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        import csharp_b200 as cs
        from conftest import load_npz
        from csharp_b200.driver import distributed_all_pairs
        z = load_npz(name)
        eng = cs.Engine(cs.ScoringMatrix.Load(z["matrix"].tobytes().decode()), float(z["o"]), float(z["e"]),
                        mode=mode, alignment_type=int(z["alignment_type"]), device=0)
        eng.upload(concat=z["concat"], offsets=z["offsets"])
        N = len(z["offsets"]) - 1
        out = torch.zeros((N, N), dtype=torch.int16, device="cuda:0")
        pairs = distributed_all_pairs(eng, out, rank, world, scheme=scheme, dst=dst)
        want = z["distances"].copy()
        if mode == 2:
            np.fill_diagonal(want, 0)
        ok = None if (dst is not None and rank != dst) else bool(np.array_equal(out.cpu().numpy(), want))
        q.put((rank, int(pairs), ok))
        eng.close()
    except Exception as e:  # reported to the parent, which fails the test
        q.put((rank, -1, repr(e)))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("name,world,scheme,dst,mode", [("mpi_p1.npz", 2, "balanced", None, 0),
                                                        ("mpi_p1.npz", 3, "balanced", 1, 0),
                                                        ("mpi_p3.npz", 3, "checkerboard", None, 0),
                                                        ("mpi_p4.npz", 4, "checkerboard", 0, 0),
                                                        ("nw_restated.npz", 2, "balanced", None, 2)])
def test_distributed_all_pairs_with_the_engine(name, world, scheme, dst, mode):
    from conftest import load_npz
    z = load_npz(name)
    N = len(z["offsets"]) - 1
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, name, scheme, dst, mode, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert all(n >= 0 for _, n, _ in res), res
    assert sum(n for _, n, _ in res) == N * (N - 1) // 2
    for r, _, ok in res:
        assert ok is (None if (dst is not None and r != dst) else True), (r, ok)
