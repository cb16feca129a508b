"""SWG-MS block driver on the CPU: block files every BlockWriteFrequency blocks, done files, and a
restart after a worker died and left a block file cut short.

The block handler here is a stand-in: the oracle's SWG-MS block (the driver logic under test does
not depend on which handler fills the blocks; the GPU engine's handler is tested against the same
oracle elsewhere).  Tolerance: block files byte-identical to a run without failures.
"""
import multiprocessing as mp
import os

import numpy as np
import pytest

N, WORLD = 60, 6


def _set():
    from csharp_b200 import synth
    rng = np.random.default_rng(8)
    seqs = [s.tobytes() for s in synth.dna_family(N, 4, rng.integers(1, 120, N), seed=9)]
    return seqs, [f"seq{k}" for k in range(N)]


def _handler():
    import oracle
    import csharp_b200 as cs
    seqs, _ = _set()
    concat, off = cs.pack_sequences(seqs)
    sc = cs.ScoringMatrix.Load("EDNAFULL").Scores[:127, :127].astype(np.float32)

    def handler(block, pm, is_diagonal, rank):
        rr, cr = block.RowRange, block.ColumnRange
        vals, n = oracle.block(concat, off, rr.StartIndex, rr.EndIndex, cr.StartIndex, cr.EndIndex, is_diagonal, 1,
                               sc, 16.0, 4.0)
        pm.block_view(block)[...] = vals
        return n
    return handler


def _run(rank, block_dir, freq, last=-1, die_after=None):
    from csharp_b200.msdriver import MSBlockRun
    _, ids = _set()
    inner = _handler()
    done = [0]

    def handler(block, pm, diag, r):
        n = inner(block, pm, diag, r)
        done[0] += 1
        if die_after is not None and done[0] > die_after:
            os._exit(17)  # the worker dies without any clean-up
        return n
    run = MSBlockRun(N, handler, rank, WORLD, str(block_dir), freq, ids)
    run.Compute(last)
    return run


def _killed_worker(rank, block_dir, freq, die_after):
    _run(rank, block_dir, freq, die_after=die_after)


def _files(d):
    return {f: open(os.path.join(d, f), "rb").read() for f in sorted(os.listdir(d))}


def test_block_files_every_frequency_and_done_files(tmp_path, oracle_mod):
    from csharp_b200.formats import read_ms_block
    from csharp_b200.msdriver import DONE_MSG, computes
    for freq in (1, 2, 0):
        d = tmp_path / f"f{freq}"
        d.mkdir()
        for r in range(WORLD):
            run = _run(r, d, freq)
            run.WriteDone(str(d))
            assert open(d / f"{r}.txt").read().strip() == DONE_MSG.format(r)
        names = {f for f in os.listdir(d) if f.endswith(".bin")}
        want = {f"{r}-{j}.bin" for r in range(WORLD) for j in range(WORLD) if computes(r, j)}
        assert names == (want if freq else set())
    # the files hold the handler's values with the block's header
    h, v = read_ms_block(str(tmp_path / "f1" / "2-0.bin"))
    assert (h["rank"], h["row_block"], h["col_block"]) == (2, 2, 0)
    assert v.shape == (h["row_end"] - h["row_start"] + 1, h["col_end"] - h["col_start"] + 1)


@pytest.mark.parametrize("freq,die_after", [(1, 1), (1, 2), (2, 2)])
def test_resume_after_a_killed_worker_and_a_cut_file(tmp_path, freq, die_after):
    from csharp_b200.msdriver import read_restart_entry, restart_point, write_restart_file, block_file
    clean = tmp_path / "clean"
    crash = tmp_path / "crash"
    clean.mkdir()
    crash.mkdir()
    for r in range(WORLD):
        _run(r, clean, freq)
    # rank 0 and rank 5's workers die part-way through (a spawned process that exits at once)
    ctx = mp.get_context("spawn")
    for r in (0, 5):
        p = ctx.Process(target=_killed_worker, args=(r, str(crash), freq, die_after))
        p.start()
        p.join(120)
        assert p.exitcode == 17
    for r in (1, 2, 3, 4):
        _run(r, crash, freq)
    # the last file rank 0 wrote is cut short, as by a crash in the middle of a write
    written = sorted(int(f.split("-")[1].split(".")[0]) for f in os.listdir(crash) if f.startswith("0-"))
    assert written
    path = block_file(str(crash), 0, written[-1])
    data = open(path, "rb").read()
    open(path, "wb").write(data[: len(data) // 2])
    # restart: the ranks to complete, with their last completely saved block
    entries = [(r, restart_point(str(crash), r, N, WORLD)) for r in (0, 5)]
    assert entries[0][1] < written[-1]
    rf = tmp_path / "restart.txt"
    write_restart_file(str(rf), WORLD, entries)
    for proc in range(len(entries)):
        world, rank, last = read_restart_entry(str(rf), proc)
        assert world == WORLD and (rank, last) == entries[proc]
        run = _run(rank, crash, freq, last=last)
        assert all(j > last for j in run.BlocksComputed)
    assert _files(crash) == _files(clean)
