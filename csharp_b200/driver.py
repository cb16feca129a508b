"""The block driver of Salsa.SmithWatermanMPI / Salsa.NeedlemanWunschTPL over torch.distributed.

``MPIComputeLowerTriangularBlocked`` mirrors the reference class of the same name
(Salsa.SmithWatermanMPI/Program.cs:559-889): rank r of P owns row block r, computes its diagonal
block and the checkerboard half of its off-diagonal blocks through a block handler (``Compute``,
:618-642), then the transposed blocks are exchanged so every rank holds its full row slab
(``Scatter``, :645-677) and rank 0 assembles the N x N matrix (``WriteFullMatrixOnRank0``,
:786-888).  MPI.NET is replaced by a torch.distributed process group (gloo on CPU, NCCL over
NVLink between GPUs); the handler is the engine's ``compute_block`` or any callable with the
reference's signature.

``distributed_all_pairs`` is the one-process-per-GPU path: each rank runs the engine over the
pairs its rank aligns (sw_compute_rank_blocks), the ranks' disjoint entries are summed with one
all-reduce (bytes, so Int16 needs no NCCL type), and every rank ends with the full matrix.
"""
import numpy as np

from .core import Block, block_is_computed, block_partition, range_partition


class PartialMatrix:
    """Rows [row_start, row_end] x columns [0, size) of the distance matrix (PartialMatrix.cs)."""

    def __init__(self, row_start, row_end, col_start, col_end, dtype=np.int16):
        self.GlobalRowStartIndex, self.GlobalColumnStartIndex = row_start, col_start
        self.values = np.zeros((row_end - row_start + 1, col_end - col_start + 1), dtype=dtype)

    def __getitem__(self, ij):
        i, j = ij
        return self.values[i - self.GlobalRowStartIndex, j - self.GlobalColumnStartIndex]

    def __setitem__(self, ij, v):
        i, j = ij
        self.values[i - self.GlobalRowStartIndex, j - self.GlobalColumnStartIndex] = v

    def block_view(self, block: Block):
        r0, c0 = self.GlobalRowStartIndex, self.GlobalColumnStartIndex
        return self.values[block.RowRange.StartIndex - r0: block.RowRange.EndIndex - r0 + 1,
                           block.ColumnRange.StartIndex - c0: block.ColumnRange.EndIndex - c0 + 1]


def engine_block_handler(engine):
    """ComputeBlockHandler backed by the engine's drop-in block kernel."""

    def handler(block: Block, matrix: PartialMatrix, is_diagonal: bool) -> int:
        view = matrix.block_view(block)
        out = np.ascontiguousarray(view)
        _, n = engine.compute_block(block.RowRange.StartIndex, block.RowRange.EndIndex,
                                    block.ColumnRange.StartIndex, block.ColumnRange.EndIndex,
                                    is_diagonal, out=out)
        view[...] = out
        return n

    return handler


class MPIComputeLowerTriangularBlocked:
    def __init__(self, size, block_handler, rank=0, world_size=1, group=None):
        self._size = size
        self._handler = block_handler
        self._rank, self._world = rank, world_size
        self._group = group
        self._blocks = block_partition(size, size, world_size, world_size)
        self._row_ranges = range_partition(size, world_size)
        rr = self._row_ranges[rank]
        self.PartialMatrix = PartialMatrix(rr.StartIndex, rr.EndIndex, 0, size - 1)
        self.CellsComputed = 0

    def Compute(self):
        for j, blk in enumerate(self._blocks[self._rank]):
            if blk.RowRange.Length <= 0 or blk.ColumnRange.Length <= 0:
                continue
            if self._rank == j:
                self.CellsComputed += self._handler(blk, self.PartialMatrix, True)
            elif block_is_computed(self._rank, j):
                self.CellsComputed += self._handler(blk, self.PartialMatrix, False)

    def Scatter(self):
        """Every rank receives the transposes of the blocks other ranks computed in its row slab."""
        import torch
        import torch.distributed as dist
        if self._world == 1:
            return
        mine = torch.from_numpy(self.PartialMatrix.values.copy())
        rr = self._row_ranges
        maxrows = max(r.Length for r in rr)
        padded = torch.zeros((maxrows, self._size), dtype=torch.int16)
        padded[: mine.shape[0]] = mine
        gathered = [torch.zeros_like(padded) for _ in range(self._world)]
        # bytes: neither gloo nor NCCL has an Int16 type
        dist.all_gather([g.view(torch.uint8) for g in gathered], padded.view(torch.uint8), group=self._group)
        me = self._rank
        for src in range(self._world):
            if src == me or not block_is_computed(src, me):
                continue
            # block (src, me) computed by src lands transposed in block (me, src)
            blk = self._blocks[src][me]
            sr = blk.RowRange
            vals = gathered[src][: sr.Length, blk.ColumnRange.StartIndex: blk.ColumnRange.EndIndex + 1]
            tgt = self.PartialMatrix.block_view(self._blocks[me][src])
            tgt[...] = vals.numpy().T

    def FullMatrixOnRank0(self):
        """The N x N matrix on rank 0 (None elsewhere), rows gathered in rank order."""
        import torch
        import torch.distributed as dist
        if self._world == 1:
            return self.PartialMatrix.values.copy()
        maxrows = max(r.Length for r in self._row_ranges)
        padded = torch.zeros((maxrows, self._size), dtype=torch.int16)
        padded[: self.PartialMatrix.values.shape[0]] = torch.from_numpy(self.PartialMatrix.values)
        gathered = [torch.zeros_like(padded) for _ in range(self._world)] if self._rank == 0 else None
        dist.gather(padded.view(torch.uint8), [g.view(torch.uint8) for g in gathered] if gathered else None,
                    dst=0, group=self._group)
        if self._rank != 0:
            return None
        return np.concatenate([g[: r.Length].numpy() for g, r in zip(gathered, self._row_ranges)], axis=0)

    def WriteFullMatrixOnRank0(self, path):
        full = self.FullMatrixOnRank0()
        if full is not None:
            from .formats import write_full_matrix
            write_full_matrix(path, full)
        return full


def distributed_all_pairs(engine, out, rank, world_size, group=None):
    """One process per GPU: this rank's pairs into `out` (a zeroed N x N int16 CUDA tensor),
    then one byte all-reduce so every rank holds the full matrix.  Returns this rank's pairs."""
    import torch
    import torch.distributed as dist
    n = out.shape[0]
    pairs = engine.rank_blocks_device(rank, world_size, out.data_ptr(), out.stride(0))
    engine.synchronize()
    if world_size > 1:
        dist.all_reduce(out.view(torch.uint8).view(-1), op=dist.ReduceOp.SUM, group=group)
    del n
    return pairs
