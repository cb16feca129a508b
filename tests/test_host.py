"""Host-side library and the C ABI without a GPU: exports, formats, partitioning, validation."""
import ctypes as C
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT


def test_library_builds_and_exports_every_declared_symbol():
    from csharp_b200 import build, lib
    build.build()
    header = (ROOT / "include" / "swgb200.h").read_text()
    declared = set(re.findall(r"^\s*(?:int|const char\*)\s+(sw_\w+)\s*\(", header, re.M))
    assert declared, "no declarations parsed"
    nm = subprocess.run(["nm", "-D", "--defined-only", str(lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (sw_\w+)$", nm, re.M))
    assert declared <= exported, declared - exported
    assert set(lib.EXPORTS) == declared
    L = lib.load()
    for name in declared:
        assert getattr(L, name)
    assert L.sw_version().decode().startswith("swgb200")


def test_range_partitioner_matches_reference_rule():
    from csharp_b200 import range_partition
    # RangePartitioner.cs:36-52: the first length % parts ranges take one extra element
    for length in range(0, 40):
        for parts in range(1, 9):
            rs = range_partition(length, parts)
            chunk, rem = divmod(length, parts)
            s = 0
            for i, r in enumerate(rs):
                ln = chunk + (1 if i < rem else 0)
                assert (r.StartIndex, r.EndIndex) == (s, s + ln - 1)
                s += ln
    with pytest.raises(Exception):
        range_partition(10, 0)


def test_checkerboard_covers_each_unordered_block_once():
    from csharp_b200 import block_is_computed
    for P in range(1, 12):
        for r in range(P):
            assert block_is_computed(r, r)
            for c in range(P):
                if r != c:
                    assert block_is_computed(r, c) != block_is_computed(c, r)


def test_fasta_parser_uppercases_and_concatenates(tmp_path):
    from csharp_b200.formats import parse_fasta
    text = b">seq1 first\nacgt\n  ACGT  \n\n>seq2\nNNnn\r\n>empty\n>s4\nA C\n"
    labels, concat, off = parse_fasta(text)
    assert labels == ["seq1 first", "seq2", "empty", "s4"]
    seqs = [concat[off[k]:off[k + 1]].tobytes() for k in range(len(off) - 1)]
    assert seqs == [b"ACGTACGT", b"NNNN", b"", b"A C"]


def test_full_matrix_file_is_raw_little_endian(tmp_path):
    from csharp_b200.formats import read_full_matrix, write_full_matrix
    m = np.arange(-12, 13, dtype=np.int16).reshape(5, 5) * 1000
    p = tmp_path / "d.bin"
    write_full_matrix(p, m)
    raw = p.read_bytes()
    assert len(raw) == 50
    assert raw[:2] == int(m[0, 0]).to_bytes(2, "little", signed=True)
    np.testing.assert_array_equal(read_full_matrix(p, 5), m)


def test_ms_block_file_layout(tmp_path):
    from csharp_b200.formats import read_ms_block, write_ms_block
    ids = [f"s{k}" for k in range(10)]
    vals = np.arange(12, dtype=np.int16).reshape(3, 4) - 5
    p = tmp_path / "2-1.bin"
    write_ms_block(p, vals, rank=2, row_block=2, col_block=1, row_range=(6, 8), col_range=(2, 5),
                   ids=ids, project="proj", system="host", fasta="in.fa")
    raw = p.read_bytes()
    # u16 len + "proj", u16 rank, u16 len + "host", u16 len + "in.fa", u16 rb, u16 cb, 4 x u32
    assert raw[:6] == b"\x04\x00proj" and raw[6:8] == b"\x02\x00"
    assert raw[8:14] == b"\x04\x00host" and raw[14:21] == b"\x05\x00in.fa"
    assert raw[21:25] == b"\x02\x00\x01\x00"
    assert raw[25:41] == (6).to_bytes(4, "little") + (8).to_bytes(4, "little") + (2).to_bytes(4, "little") + (5).to_bytes(4, "little")
    assert raw[41:45] == b"\x02\x00s6"
    hdr, back = read_ms_block(p)
    assert hdr == dict(rank=2, row_block=2, col_block=1, row_start=6, row_end=8, col_start=2, col_end=5)
    np.testing.assert_array_equal(back, vals)
    assert raw[-2:] == int(vals[-1, -1]).to_bytes(2, "little", signed=True)


def test_matrix_parser_matches_reference_rules():
    from csharp_b200 import ScoringMatrix
    from csharp_b200.lib import SwError
    text = "# comment\n#another\n   A  B  C\nA 1 -2 3\nB -2 5 0\nC 3 0 7\nZ 9 9 9\n"
    m = ScoringMatrix.Parse(text)
    assert m.GetScore("A", "C") == 3 and m.GetScore("C", "C") == 7 and m.GetScore("Z", "B") == 9
    assert m.GetScore("A", "Q") == 0  # letters outside the header score 0
    with pytest.raises(SwError):
        ScoringMatrix.Parse("   A B\nA 1.5 2\nB 2 1\n")  # non-integer: the float DP is not reproduced


def _cfg(**kw):
    from csharp_b200 import lib
    cfg = lib.sw_config()
    cfg.mode, cfg.alignment_type, cfg.distance_fn = 0, 1, 0
    cfg.gap_open, cfg.gap_extension = 16.0, 4.0
    cfg.device, cfg.lanes = 0, 0
    for k, v in kw.items():
        setattr(cfg, k, v)
    return cfg


@pytest.mark.parametrize("kw,status", [
    (dict(mode=7), 1), (dict(alignment_type=3), 1), (dict(lanes=8), 1),
    (dict(gap_open=14.5), 5), (dict(gap_extension=0.25), 5), (dict(gap_open=0.0), 5),
    (dict(gap_extension=-1.0), 5), (dict(mode=2, gap_open=4.0, gap_extension=4.0), 5),
    (dict(distance_fn=4), 1), (dict(distance_fn=-1), 1),
])
def test_create_rejects_configs_before_touching_a_device(kw, status):
    from csharp_b200 import lib
    h = C.c_void_p()
    assert lib.load().sw_create(C.byref(_cfg(**kw)), C.byref(h)) == status
    assert not h.value


def test_synthetic_generator_is_seeded():
    from csharp_b200 import synth
    a = synth.dna_family(30, 3, np.full(30, 120), seed=5)
    b = synth.dna_family(30, 3, np.full(30, 120), seed=5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert all(len(x) == 120 for x in a)
    assert set(np.concatenate(a).tobytes()) <= set(b"ACGT")


def test_row_files_for_the_clustering_loader(tmp_path):
    """Row files {prefix}_{i}{ext} over RangePartitioner ranges (MatrixBinaryReader.cs:191-217): a
    reader with the same parallelism gets back exactly its rows of the matrix."""
    from csharp_b200.formats import read_row_files, write_row_files
    rng = np.random.default_rng(4)
    n, procs, threads = 37, 3, 2
    m = rng.integers(-32768, 32767, (n, n)).astype(np.int16)
    paths = write_row_files(str(tmp_path), "dist", ".bin", lambda a, b: m[a:b + 1], n, procs * threads)
    assert len(paths) == procs * threads
    from csharp_b200 import range_partition
    tr = range_partition(n, procs * threads)
    for p in range(procs):  # process p reads its threads' files
        got = read_row_files(str(tmp_path), "dist", ".bin", p * threads, p * threads + threads - 1, n, procs * threads)
        np.testing.assert_array_equal(got, m[tr[p * threads].StartIndex:tr[p * threads + threads - 1].EndIndex + 1])
    assert (tmp_path / "dist_0.bin").stat().st_size == tr[0].Length * n * 2
