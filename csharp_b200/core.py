"""Host-side mirror of the reference's aligner and block-handler API over the C ABI.

Names follow the reference (DSC-SPIDAL/csharp, SalsaTPL/):

* :class:`ScoringMatrix`       Salsa.CoreTPL/Bio/Algorithms/ScoringMatrix.cs (``Load``, ``Scores``)
* :class:`SmithWatermanGotoh`  Salsa.CoreTPL/Bio/Algorithms/SmithWaterman/SmithWatermanGotoh.cs
  (``Align`` returning a :class:`PairwiseAlignment`, Alignment.cs)
* :class:`Range`, :class:`Block`, :func:`range_partition`, :func:`block_partition`
  Salsa.CoreTPL/Range.cs, Block.cs, RangePartitioner.cs, BlockPartitioner.cs
* :class:`Engine`              the block handler ``ComputeBlock`` of the three applications and the
  whole-job driver, on one CUDA device
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import lib as L

PROTEIN, NUCLEIC = L.SW_PROTEIN, L.SW_NUCLEIC
PERCENT_IDENTITY, KIMURA2, JUKES_CANTOR, MIN_MAX_NORM_SCORE = (L.SW_DIST_PERCENT_IDENTITY, L.SW_DIST_KIMURA2,
                                                          L.SW_DIST_JUKES_CANTOR, L.SW_DIST_MIN_MAX_NORM_SCORE)
SWG_MPI, SWG_MS, NW = L.SW_MODE_SWG_MPI, L.SW_MODE_SWG_MS, L.SW_MODE_NW


class ScoringMatrix:
    """A substitution table indexed by residue bytes (``Scores[c1, c2]``)."""

    BUILTIN = ("EDNAFULL", "BLOSUM62", "IDENTITY", "MATCH")

    def __init__(self, name, scores: np.ndarray):
        self.Name = name
        self.Scores = np.ascontiguousarray(scores, dtype=np.int16).reshape(128, 128)

    @staticmethod
    def Load(name: str) -> "ScoringMatrix":
        """A built-in matrix by the reference's resource name."""
        out = np.zeros((128, 128), dtype=np.int16)
        L.check(L.load().sw_builtin_scoring_matrix(name.encode(), L.ptr(out)))
        return ScoringMatrix(name, out)

    @staticmethod
    def Parse(text, name="custom") -> "ScoringMatrix":
        """ScoringMatrix.Load's parser over matrix text in the reference's format."""
        if isinstance(text, str):
            text = text.encode()
        out = np.zeros((128, 128), dtype=np.int16)
        L.check(L.load().sw_parse_scoring_matrix(text, len(text), L.ptr(out)))
        return ScoringMatrix(name, out)

    def GetScore(self, a, b):
        return int(self.Scores[ord(a) if isinstance(a, str) else a, ord(b) if isinstance(b, str) else b])


@dataclass
class PairwiseAlignment:
    """The PairwiseAlignment fields the distance path reads (Alignment.cs:29-195)."""
    Score: float
    Start1: int
    Start2: int
    End1: int
    End2: int
    Identity: int
    Similarity: int
    Gaps: int
    Length: int
    Distance: int

    @property
    def PercentIdentity(self):
        return np.float32(self.Identity) / np.float32(self.Length) if self.Length else np.float32("nan")

    @property
    def PercentSimilarity(self):
        return np.float32(self.Similarity) / np.float32(self.Length) if self.Length else np.float32("nan")


@dataclass
class Range:
    """Inclusive index range (Range.cs:9-89)."""
    StartIndex: int
    EndIndex: int

    @property
    def Length(self):
        return self.EndIndex - self.StartIndex + 1

    def Contains(self, i):
        return self.StartIndex <= i <= self.EndIndex


@dataclass
class Block:
    """A rectangle of the pair matrix (Block.cs:9-61)."""
    RowRange: Range
    ColumnRange: Range
    RowBlockNumber: int = 0
    ColumnBlockNumber: int = 0

    def Transpose(self):
        return Block(self.ColumnRange, self.RowRange, self.ColumnBlockNumber, self.RowBlockNumber)


def range_partition(length, parts, start=0):
    """RangePartitioner.Partition (RangePartitioner.cs:17-55)."""
    if parts < 1:
        raise ValueError("Partitioning requires numPartitions to be greater than zero.")
    s = np.zeros(parts, dtype=np.int32)
    e = np.zeros(parts, dtype=np.int32)
    L.check(L.load().sw_partition_ranges(start, length, parts, L.ptr(s), L.ptr(e)))
    return [Range(int(a), int(b)) for a, b in zip(s, e)]


def block_partition(rows, cols, row_blocks, col_blocks):
    """BlockPartitioner.Partition (BlockPartitioner.cs:10-28)."""
    rr, cc = range_partition(rows, row_blocks), range_partition(cols, col_blocks)
    return [[Block(r, c, i, j) for j, c in enumerate(cc)] for i, r in enumerate(rr)]


def block_is_computed(r, c):
    """Does rank r compute block (r, c) under the SWG-MPI checkerboard (Program.cs:628-639)?"""
    return bool(L.load().sw_block_is_computed(r, c))


def pack_sequences(seqs):
    """Concatenated residues + offsets from a list of byte strings / str / uint8 arrays."""
    parts = []
    for s in seqs:
        if isinstance(s, str):
            s = s.encode()
        parts.append(np.frombuffer(bytes(s), dtype=np.uint8) if not isinstance(s, np.ndarray) else s.astype(np.uint8))
    lens = np.array([len(p) for p in parts], dtype=np.int64)
    off = np.zeros(len(parts) + 1, dtype=np.int64)
    np.cumsum(lens, out=off[1:])
    concat = np.concatenate(parts) if parts else np.zeros(0, dtype=np.uint8)
    return np.ascontiguousarray(concat, dtype=np.uint8), off


class Engine:
    """One device context: configuration, resident sequences, block handler and job driver."""

    def __init__(self, matrix: ScoringMatrix, gap_open=14, gap_extension=4, mode=SWG_MPI,
                 alignment_type=NUCLEIC, distance_fn=PERCENT_IDENTITY, device=0, lanes=0):
        cfg = L.sw_config()
        cfg.mode, cfg.alignment_type, cfg.distance_fn = mode, alignment_type, distance_fn
        cfg.gap_open, cfg.gap_extension = float(gap_open), float(gap_extension)
        C.memmove(cfg.scores, matrix.Scores.ctypes.data, 128 * 128 * 2)
        cfg.device, cfg.lanes = device, lanes
        h = C.c_void_p()
        L.check(L.load().sw_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self.mode = mode
        self.nseq = 0
        self.lengths = np.zeros(0, dtype=np.int64)

    def close(self):
        if self._h:
            L.load().sw_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, status):
        L.check(status, self._h)

    def upload(self, seqs=None, concat=None, offsets=None):
        if seqs is not None:
            concat, offsets = pack_sequences(seqs)
        concat = np.ascontiguousarray(concat, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        self._ck(L.load().sw_upload_sequences(self._h, L.ptr(concat), L.ptr(offsets), len(offsets) - 1))
        self.nseq = len(offsets) - 1
        self.lengths = np.diff(offsets)
        return self

    def set_option(self, key, value):
        self._ck(L.load().sw_set_option(self._h, key.encode(), int(value)))

    def query(self, key):
        v = C.c_int64()
        self._ck(L.load().sw_query(self._h, key.encode(), C.byref(v)))
        return v.value

    def use_stream(self, stream_handle):
        """Order later calls on a caller's CUDA stream (an integer cudaStream_t, 0 = own)."""
        self.set_option("stream", int(stream_handle))

    def compute_block(self, row_start, row_end, col_start, col_end, is_diagonal, out=None):
        """The block handler: returns (Int16 block array, pairs computed)."""
        R, Cc = row_end - row_start + 1, col_end - col_start + 1
        if out is None:
            out = np.zeros((R, Cc), dtype=np.int16)
        n = C.c_int64()
        self._ck(L.load().sw_compute_block(self._h, row_start, row_end, col_start, col_end,
                                           int(is_diagonal), L.ptr(out), out.strides[0] // 2, C.byref(n)))
        return out, n.value

    def compute_block_device(self, row_start, row_end, col_start, col_end, is_diagonal, d_out_ptr, ld):
        n = C.c_int64()
        self._ck(L.load().sw_compute_block_device(self._h, row_start, row_end, col_start, col_end,
                                                  int(is_diagonal), C.c_void_p(d_out_ptr), ld, C.byref(n)))
        return n.value

    def rows_device(self, row_start, row_end, d_out_ptr, ld):
        """Rows row_start..row_end of a one-rank run -- every pair (i, j) with j < i, s1 = sequence
        i, written at (i, j) and (j, i) -- into the N x N device matrix at d_out_ptr (leading
        dimension ld), one engine job (sw_compute_rows).  SWG-MPI and NW modes; returns the pairs
        aligned."""
        if self.mode == SWG_MS:
            raise ValueError("rows_device: SWG-MS aligns both orientations; use its blocks")
        lo, hi = int(row_start), int(row_end)
        if hi < lo:
            return 0
        p = C.c_int64()
        self._ck(L.load().sw_compute_rows(self._h, lo, hi, C.c_void_p(d_out_ptr), ld, C.byref(p)))
        return p.value

    def align(self, s1, s2) -> PairwiseAlignment:
        a = np.frombuffer(s1.encode() if isinstance(s1, str) else bytes(s1), dtype=np.uint8)
        b = np.frombuffer(s2.encode() if isinstance(s2, str) else bytes(s2), dtype=np.uint8)
        a = np.ascontiguousarray(a)
        b = np.ascontiguousarray(b)
        r = L.sw_pair_result()
        self._ck(L.load().sw_align_pair(self._h, L.ptr(a), len(a), L.ptr(b), len(b), C.byref(r)))
        return PairwiseAlignment(r.score, r.start1, r.start2, r.end1, r.end2, r.identity, r.similarity,
                                 r.gaps, r.length, r.distance)

    def align_strings(self, pairs):
        """Alignment strings of explicit pairs (s1 index, s2 index) of the uploaded set, as the
        applications print them with WriteAlignments: a list of (aligned s1, aligned s2,
        PairwiseAlignment) with '-' for gaps."""
        pairs = np.asarray(pairs, dtype=np.int32).reshape(-1, 2)
        rows, cols = np.ascontiguousarray(pairs[:, 0]), np.ascontiguousarray(pairs[:, 1])
        n = len(pairs)
        if n and (rows.min() < 0 or cols.min() < 0 or rows.max() >= self.nseq or cols.max() >= self.nseq):
            raise L.SwError(L.SW_E_ARG, "pair outside the uploaded sequences")
        off = np.zeros(n + 1, dtype=np.int64)
        if n:
            np.cumsum(self.lengths[rows] + self.lengths[cols], out=off[1:])
        a = np.zeros(max(int(off[-1]), 1), dtype=np.uint8)
        b = np.zeros_like(a)
        res = (L.sw_pair_result * max(n, 1))()
        self._ck(L.load().sw_align_strings(self._h, L.ptr(rows), L.ptr(cols), n, L.ptr(a), L.ptr(b), L.ptr(off), res))
        out = []
        for k in range(n):
            r = res[k]
            s1 = a[off[k]:off[k] + r.length].tobytes()
            s2 = b[off[k]:off[k] + r.length].tobytes()
            out.append((s1, s2, PairwiseAlignment(r.score, r.start1, r.start2, r.end1, r.end2, r.identity,
                                                  r.similarity, r.gaps, r.length, r.distance)))
        return out

    def all_pairs(self, ranks=1):
        """Whole job to a host N x N Int16 matrix; returns (matrix, pairs, cells)."""
        out = np.zeros((self.nseq, self.nseq), dtype=np.int16)
        p, c = C.c_int64(), C.c_int64()
        self._ck(L.load().sw_all_pairs(self._h, ranks, L.ptr(out), self.nseq, C.byref(p), C.byref(c)))
        return out, p.value, c.value

    def all_pairs_device(self, d_out_ptr, ld, ranks=1):
        p, c = C.c_int64(), C.c_int64()
        self._ck(L.load().sw_all_pairs_device(self._h, ranks, C.c_void_p(d_out_ptr), ld, C.byref(p), C.byref(c)))
        return p.value, c.value

    def rank_blocks_device(self, rank, world, d_out_ptr, ld):
        p = C.c_int64()
        self._ck(L.load().sw_compute_rank_blocks(self._h, rank, world, C.c_void_p(d_out_ptr), ld, C.byref(p)))
        return p.value

    def autotune(self, d_out_ptr, ld):
        """Measures the rows-per-lane costs on this device and job (writing sample distances
        into the N x N device matrix at d_out_ptr); returns {rows per lane: weight}."""
        w = np.zeros(7, dtype=np.int32)
        self._ck(L.load().sw_autotune(self._h, C.c_void_p(d_out_ptr), ld, L.ptr(w)))
        return {k: int(v) for k, v in zip((4, 6, 8, 10, 12, 14, 16), w)}

    def rerun_count(self):
        n = C.c_int64()
        self._ck(L.load().sw_last_rerun_count(self._h, C.byref(n)))
        return n.value

    def synchronize(self):
        self._ck(L.load().sw_synchronize(self._h))

    # ---- serving: query batches against the uploaded sequences (the database) --------------
    def submit(self, queries, out=None):
        """Queues a batch of queries (byte strings) against the database; returns a ticket.
        The result (len(queries) x database Int16, query i = s1 of row i) is ``job_result``."""
        concat, off = pack_sequences(queries)
        nq = len(off) - 1
        if out is None:
            out = np.empty((nq, self.nseq), dtype=np.int16)
        t = C.c_int64()
        self._ck(L.load().sw_submit_job(self._h, L.ptr(concat), L.ptr(off), nq, L.ptr(out),
                                        out.strides[0] // 2, C.byref(t)))
        if not hasattr(self, "_jobs"):
            self._jobs = {}
        self._jobs[t.value] = out  # the library writes into it until the job is done
        return t.value

    def poll(self, ticket, timeout_ms=0):
        """None while the job runs; else a dict of its sw_job_info with the result under "out"."""
        done, info = C.c_int32(), L.sw_job_info()
        self._ck(L.load().sw_poll(self._h, ticket, int(timeout_ms), C.byref(done), C.byref(info)))
        if not done.value:
            return None
        r = {f: getattr(info, f) for f, _ in L.sw_job_info._fields_ if f != "reserved"}
        r["out"] = self._jobs.pop(ticket)
        return r

    def wait(self, ticket, timeout_s=600.0):
        """Polls until the job is done (raises TimeoutError after timeout_s)."""
        import time
        t_end = time.monotonic() + timeout_s
        while True:
            r = self.poll(ticket, 200)
            if r is not None:
                return r
            if time.monotonic() > t_end:
                raise TimeoutError(f"job {ticket} not done after {timeout_s} s")

    def serve_stats(self):
        s = L.sw_serve_counters()
        self._ck(L.load().sw_serve_stats(self._h, C.byref(s)))
        return {f: getattr(s, f) for f, _ in L.sw_serve_counters._fields_ if f != "reserved"}

    def serve_drain(self):
        self._ck(L.load().sw_serve_drain(self._h))


class SmithWatermanGotoh:
    """The reference's aligner object: ``Align(s1, s2, matrix, o, e)`` on the device."""

    def __init__(self, alignment_type=NUCLEIC):
        self._type = alignment_type
        self._engines = {}

    def Align(self, s1, s2, matrix: ScoringMatrix, gap_open_penalty, gap_extension_penalty):
        if s1 is None:
            raise ValueError("S1 is null")
        if s2 is None:
            raise ValueError("S2 is null")
        key = (matrix.Name, id(matrix), float(gap_open_penalty), float(gap_extension_penalty))
        eng = self._engines.get(key)
        if eng is None:
            eng = Engine(matrix, gap_open_penalty, gap_extension_penalty, alignment_type=self._type)
            self._engines[key] = eng
        return eng.align(s1, s2)


def measure_int_peak(device=0):
    """Integer-pipe peak of this device: (max lane-ops/s, add lane-ops/s)."""
    a, b = C.c_double(), C.c_double()
    L.check(L.load().sw_measure_int_peak(device, C.byref(a), C.byref(b)))
    return a.value, b.value
