"""The SWG-MS block driver: block files, checkpoints every few blocks, restart and done files.

Mirrors Salsa.SmithWatermanMS (Program.cs): each rank computes the blocks of its row slab that
the checkerboard gives it (MPIComputeLowerTriangularBlocked.Compute(lastSavedBlock), :1164-1227),
writes them as block files {BlockDir}/{rank}-{cb}.bin every BlockWriteFrequency computed blocks,
highest block first (WriteBlocks, :1081-1114; the format is the C ABI's sw_write_ms_block), skips
the blocks up to lastSavedBlock when it restarts from a restart file (ReadRestartFile, :245-262:
the world size, then one "rank lastSavedBlock" line per rank to be completed) and writes
"Done: Rank r done." to {DoneStatusDir}/{rank}.txt when its blocks are done (:187-201).

The reference's operators wrote the restart file by hand after a failure.  ``restart_point``
derives a rank's lastSavedBlock from its block files instead: the highest block such that every
block the rank computes up to it has a complete file (a file cut short by a crash does not count),
and ``write_restart_file`` writes the reference's format.
"""
import os

from .core import block_partition
from .driver import PartialMatrix
from .formats import read_ms_block, write_ms_block

DONE_MSG = "Done: Rank {0} done."


def computes(rank, j):
    """Rank `rank` computes block (rank, j): the diagonal, or the checkerboard half."""
    return rank == j or (rank > j and (rank + j) % 2 == 0) or (rank < j and (rank + j) % 2 == 1)


def block_file(block_dir, rank, j):
    return os.path.join(block_dir, f"{rank}-{j}.bin")


class MSBlockRun:
    """One rank of an SWG-MS run.  handler(block, partial_matrix, is_diagonal, rank) fills the
    block's values into the partial matrix and returns the pairs it aligned (the MS
    ComputeBlockHandler, Program.cs:1018)."""

    def __init__(self, size, handler, rank, world_size, block_dir, block_write_frequency, ids,
                 project="swg", system="b200", fasta="input.fasta"):
        self._size, self._handler = size, handler
        self._rank, self._world = rank, world_size
        self._blocks = block_partition(size, size, world_size, world_size)[rank]
        rr = self._blocks[0].RowRange
        self.PartialMatrix = PartialMatrix(rr.StartIndex, rr.EndIndex, 0, size - 1)
        self._dir, self._freq = block_dir, block_write_frequency
        self._ids, self._meta = ids, dict(project=project, system=system, fasta=fasta)
        self.CellsComputed = 0
        self.BlocksComputed = []

    def Compute(self, last_saved_block=-1):
        unsaved = 0
        for j in range(last_saved_block + 1, self._world):
            if not computes(self._rank, j):
                continue
            blk = self._blocks[j]
            self.CellsComputed += self._handler(blk, self.PartialMatrix, self._rank == j, self._rank)
            self.BlocksComputed.append(j)
            unsaved += 1
            if self._freq > 0 and unsaved == self._freq:
                self.WriteBlocks(last_saved_block, j)
                unsaved = 0
                last_saved_block = j
        if self._freq > 0 and unsaved > 0:  # the remaining unsaved blocks
            self.WriteBlocks(last_saved_block, self._world - 1)

    def WriteBlocks(self, last_saved_block, last_unsaved_block):
        for j in range(last_unsaved_block, last_saved_block, -1):
            if not computes(self._rank, j):
                continue
            blk = self._blocks[j]
            rr, cr = blk.RowRange, blk.ColumnRange
            write_ms_block(block_file(self._dir, self._rank, j), self.PartialMatrix.block_view(blk), self._rank,
                           self._rank, j, (rr.StartIndex, rr.EndIndex), (cr.StartIndex, cr.EndIndex), self._ids,
                           **self._meta)

    def WriteDone(self, done_dir):
        with open(os.path.join(done_dir, f"{self._rank}.txt"), "w") as f:
            f.write(DONE_MSG.format(self._rank) + "\n")


def engine_handler(engine):
    """The MS ComputeBlockHandler backed by the engine's block handler (sw_compute_block)."""

    def handler(block, pm, is_diagonal, rank):
        view = pm.block_view(block)
        out = view.copy()
        _, n = engine.compute_block(block.RowRange.StartIndex, block.RowRange.EndIndex, block.ColumnRange.StartIndex,
                                    block.ColumnRange.EndIndex, is_diagonal, out=out)
        view[...] = out
        return n
    return handler


def complete_block_file(block_dir, rank, j, size, world_size):
    """The block file exists, reads back whole, and covers block (rank, j) of this job."""
    path = block_file(block_dir, rank, j)
    if not os.path.exists(path):
        return False
    try:
        h, _ = read_ms_block(path)
    except Exception:
        return False
    blk = block_partition(size, size, world_size, world_size)[rank][j]
    return (h["rank"], h["row_block"], h["col_block"], h["row_start"], h["row_end"], h["col_start"], h["col_end"]) == \
        (rank, rank, j, blk.RowRange.StartIndex, blk.RowRange.EndIndex, blk.ColumnRange.StartIndex, blk.ColumnRange.EndIndex)


def restart_point(block_dir, rank, size, world_size):
    """lastSavedBlock of a rank: the highest block j such that every block the rank computes up to
    j has a complete file (-1: start from the beginning)."""
    last = -1
    for j in range(world_size):
        if not computes(rank, j):
            continue
        if not complete_block_file(block_dir, rank, j, size, world_size):
            break
        last = j
    return last


def write_restart_file(path, world_size, entries):
    """The reference's restart file: the world size, then one 'rank<TAB>lastSavedBlock' line per
    rank to be completed (the n-th line is read by the n-th restarted process)."""
    with open(path, "w") as f:
        f.write(f"{world_size}\n")
        for r, last in entries:
            f.write(f"{r}\t{last}\n")


def read_restart_entry(path, process_rank):
    """ReadRestartFile (Program.cs:245-262) for the process of rank `process_rank` of the
    restarted job: (world size, the rank it stands in for, its lastSavedBlock)."""
    with open(path) as f:
        world = int(f.readline().strip())
        for _ in range(process_rank):
            f.readline()
        a, b = f.readline().strip().replace("\t", " ").split()[:2]
    return world, int(a), int(b)
