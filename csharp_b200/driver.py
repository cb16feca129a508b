"""The block driver of Salsa.SmithWatermanMPI / Salsa.NeedlemanWunschTPL over torch.distributed.

``MPIComputeLowerTriangularBlocked`` mirrors the reference class of the same name
(Salsa.SmithWatermanMPI/Program.cs:559-889): rank r of P owns row block r, computes its diagonal
block and the checkerboard half of its off-diagonal blocks through a block handler (``Compute``,
:618-642), then the transposed blocks are exchanged so every rank holds its full row slab
(``Scatter``, :645-677) and rank 0 assembles the N x N matrix (``WriteFullMatrixOnRank0``,
:786-888).  MPI.NET is replaced by a torch.distributed process group (gloo on CPU, NCCL over
NVLink between GPUs); the handler is the engine's ``compute_block`` or any callable with the
reference's signature.

``distributed_all_pairs`` is the one-process-per-GPU path: each rank runs the engine over its
share -- contiguous rows cut at equal DP cells (``balanced_row_ranges``), or the reference's
checkerboard -- and the ranks' row slabs are merged by one all-gather or one gather to a writer
(``merge_row_slabs``), the entries nobody sent following from who computed which pair.
"""
import numpy as np

from .core import SWG_MS, Block, block_is_computed, block_partition, range_partition


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


def balanced_row_ranges(lengths, world):
    """Contiguous query-row ranges of about equal DP cells, one per rank: with s1 = the larger
    index (a 1-rank run's orientation), row q aligns every d < q and costs m_q * sum of n_d over
    d < q.  Rank r takes the rows whose cumulative cost ends in (r / world, (r + 1) / world] of
    the total (inclusive (start, end); end < start: no rows)."""
    lens = np.asarray(lengths, dtype=np.float64)
    n = len(lens)
    before = np.concatenate([[0.0], np.cumsum(lens)[:-1]]) if n else np.zeros(0)
    cum = np.cumsum(lens * before)
    total = float(cum[-1]) if n else 0.0
    cuts = [0]
    for r in range(1, world):
        cuts.append(max(cuts[-1], int(np.searchsorted(cum, total * r / world, side="left")) + 1 if n else 0))
    cuts.append(n)
    cuts = [min(c, n) for c in cuts]
    return [(cuts[r], cuts[r + 1] - 1) for r in range(world)]


def checkerboard_row_ranges(n, world):
    return [(r.StartIndex, r.EndIndex) for r in range_partition(n, world)]


def merge_row_slabs(out, rank, world, row_ranges, scheme, group=None, dst=None):
    """Merges the ranks' row slabs of an N x N Int16 tensor into the full matrix on every rank (dst
    None: one all-gather) or on rank dst (one gather; the writer of WriteFullMatrixOnRank0).

    Rank r contributes only its rows row_ranges[r]: each rank sends 1/world of the matrix instead
    of the whole matrix a byte all-reduce moves.  The other entries follow from who computed what:
    "checkerboard" (the reference's P-rank run, Program.cs:618-677): a block (r, c) that rank r did
    not compute is the transpose of block (c, r) (Scatter); "balanced" (balanced_row_ranges): each
    pair sits below the diagonal in its s1 row and the upper triangle is its transpose.  Returns
    True where the full matrix is now in `out`."""
    import torch
    import torch.distributed as dist
    N = out.shape[0]
    rows = [max(0, hi - lo + 1) for lo, hi in row_ranges]
    maxrows = max(max(rows), 1)
    lo, hi = row_ranges[rank]
    dev = out.device
    if world > 1 and out.is_cuda and dist.get_backend(group) == "gloo":
        dev = torch.device("cpu")  # gloo's collectives take host tensors
    buf = torch.zeros((maxrows, N), dtype=torch.int16, device=dev)
    if rows[rank]:
        buf[:rows[rank]] = out[lo:hi + 1].to(dev)
    if world > 1:
        if dst is None:
            parts = [torch.empty_like(buf) for _ in range(world)]
            dist.all_gather([g.view(torch.uint8) for g in parts], buf.view(torch.uint8), group=group)
        else:  # bytes: neither gloo nor NCCL has an Int16 type
            parts = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
            dist.gather(buf.view(torch.uint8), [g.view(torch.uint8) for g in parts] if parts else None, dst=dst,
                        group=group)
            if rank != dst:
                return False
    else:
        parts = [buf]
    full = torch.zeros((N, N), dtype=torch.int16, device=dev)
    for r, (a, b) in enumerate(row_ranges):
        if rows[r]:
            full[a:b + 1] = parts[r][:rows[r]]
    if scheme == "balanced":
        low = torch.tril(full, -1)
        full = low + low.T
    else:
        for r, (a, b) in enumerate(row_ranges):
            for c, (cs, ce) in enumerate(row_ranges):
                if r != c and not block_is_computed(r, c) and rows[r] and rows[c]:
                    full[a:b + 1, cs:ce + 1] = full[cs:ce + 1, a:b + 1].T
    out.copy_(full)
    return True


def distributed_all_pairs(engine, out, rank, world_size, scheme="balanced", group=None, dst=None, share=None):
    """One process per GPU: this rank's pairs into `out` (a zeroed N x N int16 tensor), then the
    row-slab merge (merge_row_slabs) so that every rank (dst None) or rank dst holds the full matrix.
    scheme "balanced": rows cut at equal DP cells, pairs oriented s1 = the larger index (the
    distances of a 1-rank run); "checkerboard": the reference's world_size-rank run, its
    orientation included (sw_compute_rank_blocks).  share(rank, world, out) computes this rank's
    entries (default: the engine; a stand-in for tests).  Returns this rank's pairs."""
    n = out.shape[0]
    if scheme not in ("balanced", "checkerboard"):
        raise ValueError(f"distributed_all_pairs: unknown scheme {scheme!r}")
    if scheme == "balanced" and engine is not None and engine.mode == SWG_MS:
        raise ValueError("distributed_all_pairs: SWG-MS runs the checkerboard scheme")
    if scheme == "balanced":
        ranges = balanced_row_ranges(engine.lengths if engine is not None else share.lengths, world_size)
    else:
        ranges = checkerboard_row_ranges(n, world_size)
    if share is not None:
        pairs = share(rank, world_size, out, ranges)
    elif scheme == "balanced":
        lo, hi = ranges[rank]
        pairs = engine.rows_device(lo, hi, out.data_ptr(), out.stride(0)) if hi >= lo else 0
        engine.synchronize()
    else:
        pairs = engine.rank_blocks_device(rank, world_size, out.data_ptr(), out.stride(0))
        engine.synchronize()
    merge_row_slabs(out, rank, world_size, ranges, scheme, group=group, dst=dst)
    return pairs
