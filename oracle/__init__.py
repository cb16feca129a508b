"""ORACLE - test infrastructure only.

Python handles onto the CPU checkers.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg import this package, and only as the checker or the timed CPU
reference; the product (``csharp_b200``) never does.

* ``liboracle.so``  - the plain-C restatement in ``swg_oracle.c`` (see its header for the
  reference file:line each function follows).
* ``_ref/libref_swg.so`` - the reference's own C# (SmithWatermanGotoh.cs, Alignment.cs,
  ScoringMatrix.cs, SWG-MPI Program.cs ComputeBlock/ComputeDistance) rewritten to C++ by
  ``cs2cpp.py`` and compiled here; present only when it was built in a container that holds the
  reference sources.  It pins the restatement: the tests require both to agree on every case.
"""
import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
SIZE = 127
ALN_PROTEIN, ALN_NUCLEIC = 0, 1
DF_PERCENT_IDENTITY, DF_KIMURA2, DF_JUKES_CANTOR = 0, 1, 2


class Result(C.Structure):
    _fields_ = [("score", C.c_float), ("end1", C.c_int), ("end2", C.c_int), ("start1", C.c_int),
                ("start2", C.c_int), ("identity", C.c_int), ("similarity", C.c_int),
                ("gaps", C.c_int), ("length", C.c_int)]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None
_ref = None
P = C.c_void_p


def build():
    """Compile liboracle.so (and oracle/_ref when the reference sources are present)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    from . import cs2cpp  # the recipe owns where the reference sources are read from
    if cs2cpp.DEFAULT_REF.exists():
        subprocess.run(["python3", str(HERE / "cs2cpp.py"), "--out", str(HERE / "_ref")],
                       check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        so = HERE / "liboracle.so"
        if not so.exists():
            build()
        L = C.CDLL(str(so))
        L.swo_parse_matrix.argtypes = [C.c_char_p, C.c_long, P]
        L.swo_align.argtypes = [P, C.c_int, P, C.c_int, P, C.c_float, C.c_float, C.POINTER(Result), P, P]
        L.swo_indp_align.argtypes = [P, C.c_int, P, C.c_int, P, C.c_int, C.c_int, C.POINTER(Result)]
        L.swo_distance_i16.argtypes = [C.POINTER(Result), P, P, C.c_int, C.c_int, C.POINTER(C.c_int16)]
        L.swo_ms_distance_i16.argtypes = [P, P, C.c_int, P, C.c_int, C.c_int, C.POINTER(C.c_int16)]
        L.swo_block.argtypes = [P, P, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P,
                                C.c_float, C.c_float, C.c_int, C.c_int, P, C.c_long]
        L.swo_block.restype = C.c_long
        L.nwo_align.argtypes = [P, C.c_int, P, C.c_int, P, C.c_float, C.c_float,
                                C.POINTER(C.c_float), P, P, C.POINTER(C.c_int)]
        L.nwo_distance_i16.argtypes = [P, P, C.c_int, P, C.c_int, C.POINTER(C.c_int16)]
        L.swo_pairs.argtypes = [P, P, P, P, C.c_long, P, C.c_float, C.c_float, C.c_int, P, C.c_int]
        L.swo_pairs.restype = C.c_long
        L.nwo_pairs.argtypes = [P, P, P, P, C.c_long, P, C.c_float, C.c_float, C.c_int, P, C.c_int]
        L.nwo_pairs.restype = C.c_long
        L.swo_indp_pairs.argtypes = [P, P, P, P, C.c_long, P, C.c_int, C.c_int, C.c_int, P, C.c_int]
        L.swo_indp_pairs.restype = C.c_long
        L.swo_count_pairs.argtypes = [P, P, P, P, C.c_long, P, C.c_int, C.c_int, C.c_int, P, C.c_int]
        L.swo_count_pairs.restype = C.c_long
        _lib = L
    return _lib


def ref_available():
    return (HERE / "_ref" / "libref_swg.so").exists()


def ref():
    """The transliterated reference (None when it was not built)."""
    global _ref
    if _ref is None:
        so = HERE / "_ref" / "libref_swg.so"
        if not so.exists():
            return None
        L = C.CDLL(str(so))
        L.ref_set_matrix_dir.argtypes = [C.c_char_p]
        L.ref_align.argtypes = [C.c_char_p, P, C.c_int, P, C.c_int, C.c_float, C.c_float] + [P] * 9
        L.ref_compute_block.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_float, C.c_float, P, P,
                                        C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, P]
        L.ref_compute_block.restype = C.c_long
        L.ref_distances.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_float, C.c_float, P, P, P, P, C.c_long, P]
        L.ref_distances.restype = C.c_long
        L.ref_set_matrix_dir(str(HERE / "_ref" / "Matrices").encode())
        _ref = L
    return _ref


def matrix_text(name):
    """Text of a named scoring matrix from the reference's matrix set (copied into oracle/_ref)."""
    return (HERE / "_ref" / "Matrices" / name).read_bytes()


def parse_matrix(text: bytes) -> np.ndarray:
    out = np.zeros(SIZE * SIZE, dtype=np.float32)
    rc = lib().swo_parse_matrix(text, len(text), out.ctypes.data)
    if rc:
        raise ValueError(f"matrix parse failed ({rc})")
    return out.reshape(SIZE, SIZE)


def _bytes(s):
    a = np.frombuffer(bytes(s), dtype=np.uint8) if not isinstance(s, np.ndarray) else s.astype(np.uint8)
    return np.ascontiguousarray(a)


def align(s1, s2, scores, o, e, with_strings=False):
    a, b = _bytes(s1), _bytes(s2)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    r = Result()
    cap = len(a) + len(b) + 1
    x = C.create_string_buffer(cap)
    y = C.create_string_buffer(cap)
    rc = lib().swo_align(a.ctypes.data, len(a), b.ctypes.data, len(b), sc.ctypes.data, o, e, C.byref(r), x, y)
    if rc:
        raise MemoryError
    d = r.asdict()
    if with_strings:
        d["aln1"], d["aln2"] = x.raw[: r.length], y.raw[: r.length]
    return d


def indp_align(s1, s2, iscores, o, e):
    a, b = _bytes(s1), _bytes(s2)
    sc = np.ascontiguousarray(iscores, dtype=np.int32)
    r = Result()
    rc = lib().swo_indp_align(a.ctypes.data, len(a), b.ctypes.data, len(b), sc.ctypes.data, int(o), int(e), C.byref(r))
    if rc:
        raise MemoryError
    return r.asdict()


def distance_i16(res, alignment_type=ALN_NUCLEIC, dist_fn=DF_PERCENT_IDENTITY, aln1=None, aln2=None):
    r = Result(**{k: res[k] for k, _ in Result._fields_})
    out = C.c_int16()
    rc = lib().swo_distance_i16(C.byref(r), aln1, aln2, alignment_type, dist_fn, C.byref(out))
    if rc:
        raise ArithmeticError("reference throws for this alignment")
    return out.value


def ms_distance_i16(aln1, aln2, scores, protein=False, dist_fn=DF_PERCENT_IDENTITY):
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    out = C.c_int16()
    rc = lib().swo_ms_distance_i16(aln1, aln2, len(aln1), sc.ctypes.data, int(protein), dist_fn, C.byref(out))
    if rc:
        raise ValueError("unsupported")
    return out.value


def block(seqs, offsets, row_start, row_end, col_start, col_end, is_diagonal, mode, scores, o, e,
          alignment_type=ALN_NUCLEIC, dist_fn=DF_PERCENT_IDENTITY):
    """Oracle block handler; returns (Int16 block [rows x cols], pairs computed)."""
    rows, cols = row_end - row_start + 1, col_end - col_start + 1
    out = np.zeros((rows, cols), dtype=np.int16)
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    n = lib().swo_block(sq.ctypes.data, of.ctypes.data, row_start, row_end, col_start, col_end,
                        int(is_diagonal), mode, sc.ctypes.data, o, e, alignment_type, dist_fn,
                        out.ctypes.data, cols)
    if n < 0:
        raise RuntimeError(f"oracle block failed ({n})")
    return out, n


def nw_align(s1, s2, scores, o, e):
    a, b = _bytes(s1), _bytes(s2)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    cap = len(a) + len(b) + 1
    x = C.create_string_buffer(cap)
    y = C.create_string_buffer(cap)
    score, ln = C.c_float(), C.c_int()
    rc = lib().nwo_align(a.ctypes.data, len(a), b.ctypes.data, len(b), sc.ctypes.data, o, e,
                         C.byref(score), x, y, C.byref(ln))
    if rc:
        raise MemoryError
    return {"score": score.value, "aln1": x.raw[: ln.value], "aln2": y.raw[: ln.value], "length": ln.value}


def nw_distance_i16(aln1, aln2, scores, protein=False):
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    out = C.c_int16()
    lib().nwo_distance_i16(aln1, aln2, len(aln1), sc.ctypes.data, int(protein), C.byref(out))
    return out.value


def pairs(seqs, offsets, rows, cols, scores, o, e, alignment_type=ALN_NUCLEIC, threads=None):
    """SWG-MPI distances of many pairs with the traceback aligner, OpenMP over host cores."""
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    out = np.zeros(len(r), dtype=np.int16)
    bad = lib().swo_pairs(sq.ctypes.data, of.ctypes.data, r.ctypes.data, c.ctypes.data, len(r),
                          sc.ctypes.data, o, e, alignment_type, out.ctypes.data, threads or os.cpu_count())
    if bad:
        raise MemoryError
    return out


def indp_pairs(seqs, offsets, rows, cols, iscores, o, e, alignment_type=ALN_NUCLEIC, threads=None, fast=False):
    """SWG-MPI distances of many pairs with the in-DP integer formulation, OpenMP over host
    cores (integer scores and penalties); fast: one packed counter word per state."""
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    sc = np.ascontiguousarray(iscores, dtype=np.int32)
    out = np.zeros(len(r), dtype=np.int16)
    fn = lib().swo_count_pairs if fast else lib().swo_indp_pairs
    bad = fn(sq.ctypes.data, of.ctypes.data, r.ctypes.data, c.ctypes.data, len(r), sc.ctypes.data, int(o), int(e),
             alignment_type, out.ctypes.data, threads or os.cpu_count())
    if bad:
        raise MemoryError
    return out


def nw_pairs(seqs, offsets, rows, cols, scores, o, e, protein=False, threads=None):
    """NW distances of many pairs with the traceback restatement, OpenMP over host cores."""
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    sc = np.ascontiguousarray(scores, dtype=np.float32)
    out = np.zeros(len(r), dtype=np.int16)
    bad = lib().nwo_pairs(sq.ctypes.data, of.ctypes.data, r.ctypes.data, c.ctypes.data, len(r),
                          sc.ctypes.data, o, e, int(protein), out.ctypes.data, threads or os.cpu_count())
    if bad:
        raise MemoryError
    return out


def ref_align(matrix_name, s1, s2, o, e, with_strings=False):
    L = ref()
    if L is None:
        raise FileNotFoundError("oracle/_ref not built")
    a, b = _bytes(s1), _bytes(s2)
    vals = [C.c_float()] + [C.c_int() for _ in range(6)]
    cap = len(a) + len(b) + 1
    x = C.create_string_buffer(cap)
    y = C.create_string_buffer(cap)
    rc = L.ref_align(matrix_name.encode(), a.ctypes.data, len(a), b.ctypes.data, len(b), o, e,
                     *[C.byref(v) for v in vals], x, y)
    if rc:
        raise RuntimeError("reference aligner raised")
    keys = ["score", "identity", "similarity", "length", "start1", "start2", "gaps"]
    d = {k: v.value for k, v in zip(keys, vals)}
    if with_strings:
        d["aln1"], d["aln2"] = x.raw[: d["length"]], y.raw[: d["length"]]
    return d


def ref_compute_block(matrix_name, alignment_type, dist_fn, o, e, seqs, offsets, rs, re, cs, ce, is_diag):
    """The reference's ComputeBlock; returns (N x N Int16 matrix with the block filled, count)."""
    L = ref()
    if L is None:
        raise FileNotFoundError("oracle/_ref not built")
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    nseq = len(of) - 1
    out = np.zeros((nseq, nseq), dtype=np.int16)
    n = L.ref_compute_block(matrix_name.encode(), alignment_type, dist_fn, o, e, sq.ctypes.data,
                            of.ctypes.data, nseq, rs, re, cs, ce, int(is_diag), out.ctypes.data)
    if n < 0:
        raise RuntimeError("reference ComputeBlock raised")
    return out, n


def ref_distances(matrix_name, alignment_type, dist_fn, o, e, seqs, offsets, rows, cols):
    """The reference's aligner + ComputeDistance over explicit pairs (one matrix load)."""
    L = ref()
    if L is None:
        raise FileNotFoundError("oracle/_ref not built")
    sq = np.ascontiguousarray(seqs, dtype=np.uint8)
    of = np.ascontiguousarray(offsets, dtype=np.int64)
    r = np.ascontiguousarray(rows, dtype=np.int32)
    c = np.ascontiguousarray(cols, dtype=np.int32)
    out = np.zeros(len(r), dtype=np.int16)
    n = L.ref_distances(matrix_name.encode(), alignment_type, dist_fn, o, e, sq.ctypes.data, of.ctypes.data,
                        r.ctypes.data, c.ctypes.data, len(r), out.ctypes.data)
    if n < 0:
        raise RuntimeError("reference aligner raised")
    return out


def _conv_i2_double(v):
    """.NET x64 conv.i2 of a double: truncate through int32 (NaN and out-of-range give 0x80000000),
    then the low 16 bits."""
    if not (-2147483649.0 < v < 2147483648.0):
        return 0
    return int(np.array(int(v) & 0xFFFF, dtype=np.uint16).view(np.int16))


def minmax_distance_i16(score, self1, self2, m, n, o, e, mode):
    """MinMaxNormScore's Int16 distance: (1 - (s - minS) / (maxS - minS)) * 32767 in binary64 with
    maxS = max of the self scores, minS = 0 (SWG-MS, Program.cs:544-553) or 2 open + (m + n)
    extend (NW, Program.cs:573-581); SWG-MPI's ComputeDistance has no case for it: 0."""
    if mode == 0:
        return 0
    mx = max(self1, self2)
    mn = 2 * o + (m + n) * e if mode == 2 else 0
    with np.errstate(all="ignore"):
        x = np.float64(score - mn) * 1.0 / np.float64(mx - mn)
        v = (np.float64(1.0) - x) * np.float64(32767.0)
    return _conv_i2_double(float(v))
