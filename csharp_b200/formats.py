"""File formats around the distance path, through the C ABI's host library.

* FASTA input            Salsa.CoreTPL/Bio/IO/Parser.cs:123-180 (residues trimmed, upper-cased)
* full Int16 matrix      Salsa.SmithWatermanMPI/Program.cs:786-888 (raw little-endian, no header)
* SWG-MS block files     Salsa.SmithWatermanMS/Program.cs:1081-1160 ({rank}-{cb}.bin)
"""
import ctypes as C
import os

import numpy as np

from . import lib as L


def parse_fasta(text):
    """Returns (labels, concatenated residues uint8, offsets int64)."""
    if isinstance(text, str):
        text = text.encode()
    cnt, res = C.c_int32(), C.c_int64()
    L.check(L.load().sw_parse_fasta(text, len(text), None, None, C.byref(cnt), C.byref(res)))
    concat = np.zeros(max(res.value, 1), dtype=np.uint8)
    off = np.zeros(cnt.value + 1, dtype=np.int64)
    L.check(L.load().sw_parse_fasta(text, len(text), L.ptr(concat), L.ptr(off), C.byref(cnt), C.byref(res)))
    labels = [ln[1:].strip() for ln in text.decode(errors="replace").splitlines() if ln.strip().startswith(">")]
    return labels, concat[: res.value], off


def read_fasta(path):
    with open(path, "rb") as f:
        return parse_fasta(f.read())


def write_fasta(path, labels, seqs):
    with open(path, "w") as f:
        for lab, s in zip(labels, seqs):
            f.write(f">{lab}\n")
            s = s.decode() if isinstance(s, (bytes, bytearray)) else (s.tobytes().decode() if isinstance(s, np.ndarray) else s)
            for k in range(0, len(s), 80):
                f.write(s[k:k + 80] + "\n")


def write_full_matrix(path, m: np.ndarray):
    m = np.ascontiguousarray(m, dtype=np.int16)
    L.check(L.load().sw_write_full_matrix(os.fsencode(path), L.ptr(m), m.shape[0], m.shape[1], m.shape[1]))


def read_full_matrix(path, n):
    return np.fromfile(path, dtype="<i2").reshape(n, n)


def write_ms_block(path, values: np.ndarray, rank, row_block, col_block, row_range, col_range,
                   ids, project="swg", system="b200", fasta="input.fasta"):
    """One SWG-MS block file; ids[k] is the label of sequence k (Range.StartSeqName etc.)."""
    v = np.ascontiguousarray(values, dtype=np.int16)
    h = L.sw_ms_block_header(project.encode(), system.encode(), fasta.encode(), rank, row_block,
                             col_block, row_range[0], row_range[1], col_range[0], col_range[1],
                             ids[row_range[0]].encode(), ids[row_range[1]].encode(),
                             ids[col_range[0]].encode(), ids[col_range[1]].encode())
    L.check(L.load().sw_write_ms_block(os.fsencode(path), C.byref(h), L.ptr(v), v.shape[1]))


def read_ms_block(path):
    """Returns (dict of header numbers, values)."""
    vals = [C.c_int32() for _ in range(7)]
    L.check(L.load().sw_read_ms_block_dims(os.fsencode(path), *[C.byref(x) for x in vals]))
    rank, rb, cb, rs, re, cs, ce = (x.value for x in vals)
    out = np.zeros((re - rs + 1, ce - cs + 1), dtype=np.int16)
    L.check(L.load().sw_read_ms_block_values(os.fsencode(path), L.ptr(out), out.shape[1]))
    return dict(rank=rank, row_block=rb, col_block=cb, row_start=rs, row_end=re, col_start=cs, col_end=ce), out


def read_restart_file(path):
    """SWG-MS restart file (Program.cs:245-262): world size, then 'rank lastSavedBlock' lines."""
    with open(path) as f:
        world = int(f.readline().strip())
        entries = []
        for ln in f:
            ln = ln.strip()
            if ln:
                a, b = ln.replace("\t", " ").split()[:2]
                entries.append((int(a), int(b)))
    return world, entries


def write_row_files(directory, prefix, ext, rows_of, size, parts):
    """The partial-matrix files the pairwise-clustering loader reads (PWCParallelism.cs:107-150,
    MatrixBinaryReader.cs:191-217): the size points are split into `parts` ranges (RangePartitioner;
    parts = processes x threads of the reader), and file {prefix}_{i}{ext} holds the rows of range i
    over all size columns, raw little-endian Int16.  rows_of(start, end) returns those rows (a host
    array, or a device tensor, which is copied to the host one range at a time)."""
    from .core import range_partition
    paths = []
    for i, r in enumerate(range_partition(size, parts)):
        if r.Length <= 0:
            continue
        rows = rows_of(r.StartIndex, r.EndIndex)
        if hasattr(rows, "cpu"):
            rows = rows.cpu().numpy()
        path = os.path.join(directory, f"{prefix}_{i}{ext}")
        write_full_matrix(path, rows)
        paths.append(path)
    return paths


def read_row_files(directory, prefix, ext, start, end, size, parts):
    """MatrixBinaryReader.ReadInt16(path, prefix, ext, startIndex, endIndex, ranges): the rows of
    files start..end stacked, size columns each."""
    from .core import range_partition
    rr = range_partition(size, parts)
    out = []
    for i in range(start, end + 1):
        out.append(np.fromfile(os.path.join(directory, f"{prefix}_{i}{ext}"), dtype="<i2").reshape(rr[i].Length, size))
    return np.concatenate(out, axis=0)


def _kimura2(a, b):
    """Alignment.ComputeKimuraDistance (Salsa.CoreTPL/Bio/Algorithms/Alignment.cs:254-302) over
    aligned strings."""
    import math
    length = gaps = ts = tv = 0.0
    for x, y in zip(a, b):
        length += 1
        if x != y:
            if x == 45 or y == 45:
                gaps += 1
            elif (x, y) in ((65, 71), (71, 65), (67, 84), (84, 67)):
                ts += 1
            else:
                tv += 1
    with np.errstate(all="ignore"):
        P = np.float64(ts) / np.float64(length - gaps)
        Q = np.float64(tv) / np.float64(length - gaps)
    eps = 4.9406564584124654e-324
    if 1.0 - (2.0 * P + Q) <= eps or 1.0 - 2.0 * Q <= eps:
        return 10.0
    return float(-0.5 * math.log(1.0 - 2.0 * P - Q) - 0.25 * math.log(1.0 - 2.0 * Q))


def _jukes_cantor(a, b):
    """Alignment.ComputeJukesCantorDistance (Alignment.cs:314-348); the reference throws for
    Log(Zero)."""
    import math
    length = gaps = diff = 0.0
    for x, y in zip(a, b):
        length += 1
        if x != y:
            if x == 45 or y == 45:
                gaps += 1
            else:
                diff += 1
    with np.errstate(all="ignore"):
        d = 1.0 - (4.0 / 3.0) * (np.float64(diff) / np.float64(length - gaps))
    if not d > 4.9406564584124654e-324:
        raise ValueError("JukesCantor: Log(Zero)")
    return -0.75 * math.log(d)


def write_alignments(path, alignments, names1, names2):
    """WriteAlignment (Salsa.SmithWatermanMPI/Program.cs:545-556) for each (aligned s1, aligned s2,
    PairwiseAlignment) of Engine.align_strings: the two names with the Kimura2, JukesCantor and
    PercentIdentity values (five decimals), the aligned strings, and an empty line."""
    with open(path, "w") as f:
        for (a, b, aln), n1, n2 in zip(alignments, names1, names2):
            k = _kimura2(a, b)
            jc = _jukes_cantor(a, b)
            pi = float(np.float32(aln.PercentIdentity))
            f.write(f">{n1} Kimera: {k:.5f}, JukesCantor: {jc:.5f}, PercentIdentity: {pi:.5f}\n")
            f.write(a.decode() + "\n")
            f.write(f">{n2} Kimera: {k:.5f}, JukesCantor: {jc:.5f}, PercentIdentity: {pi:.5f}\n")
            f.write(b.decode() + "\n")
            f.write("\n")
