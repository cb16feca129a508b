"""The two-pass box step on the CPU: the source of the GPU box kernels (swg_box_reg.cuh),
compiled for the host, against the oracle.

The score pass hands the box step each pair's best score S, first-maximum cell (ie, je) and the
bounds of the rows above it; here a plain forward DP supplies them (with the bounds exact, or
loosened at random: any bound at least the row's maximum must give the same result).  Every pair
the box step solves must carry exactly the traceback's aligned columns and identity (similarity
for protein) -- tolerance: exact -- on uneven DNA family sets at several gap settings, tie-heavy
two-letter sequences and BLOSUM62 protein; pairs it hands on are the GPU path's to redo (the warp
box kernel, then the int32 DP).
"""
import ctypes as C
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
CUDA_INC = Path("/usr/local/cuda/include")


@pytest.fixture(scope="module")
def box_reg(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not (CUDA_INC / "vector_types.h").exists():
        pytest.skip("g++ or the CUDA headers are missing")
    so = tmp_path_factory.mktemp("box_reg") / "libbox_reg.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{CUDA_INC}", "-o", str(so),
                    str(HERE / "box_reg_host.cpp")], check=True)
    lib = C.CDLL(str(so))
    lib.box_reg_run.restype = C.c_int
    return lib


def _run(lib, oracle_mod, cs, seqs, pairs, matrix, o, e, protein=False, threads=7, slack=0):
    concat, off = cs.pack_sequences(seqs)
    sc = cs.ScoringMatrix.Load(matrix).Scores.astype(np.int32)
    x = np.arange(128)
    fl = ((x[:, None] == x[None, :]) | ((sc > 0) if protein else False)).astype(np.uint32)
    pairs = np.asarray(pairs, dtype=np.int32)
    n = len(pairs)
    q, d = np.ascontiguousarray(pairs[:, 0]), np.ascontiguousarray(pairs[:, 1])
    S, ie, je, outcome, bw = (np.zeros(n, np.int32) for _ in range(5))
    counters = np.zeros(n, np.uint32)
    P = C.c_void_p
    rc = lib.box_reg_run(P(concat.ctypes.data), P(off.ctypes.data), P(q.ctypes.data), P(d.ctypes.data), C.c_long(n),
                         P(np.ascontiguousarray(sc).ctypes.data), P(np.ascontiguousarray(fl).ctypes.data), int(o), int(e),
                         int(threads), int(slack), *[P(a.ctypes.data) for a in (S, ie, je, outcome, counters, bw)])
    assert rc == 0, "a pair's outcome came twice or never"
    isc = np.ascontiguousarray(sc[:127, :127])
    for k in range(n):
        r = oracle_mod.indp_align(seqs[q[k]], seqs[d[k]], isc, o, e)
        if outcome[k] == 5:
            assert not (np.isfinite(r["score"]) and r["score"] > 0)
            continue
        assert (S[k], ie[k], je[k]) == (int(r["score"]), r["end1"], r["end2"])
        if outcome[k] == 0:
            want = r["similarity"] if protein else r["identity"]
            assert (int(counters[k] >> 16), int(counters[k] & 0xFFFF)) == (r["length"], want), k
    assert not (outcome == 4).any(), "a band DP missed the best score"
    assert not (outcome == 2).any(), "a scan found no first pair"
    return outcome, bw


@pytest.mark.parametrize("o,e", [(16, 4), (20, 8), (10, 3), (4, 2)])
def test_box_reg_uneven_dna_matches_oracle(box_reg, oracle_mod, o, e):
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(o * 31 + e)
    lens = synth.lognormal_lengths(160, 400, 0.6, 50, 1500, rng)
    seqs = [s.tobytes() for s in synth.dna_family(160, 40, lens, seed=o + e)]
    pairs = [(int(i), int(j)) for i, j in rng.integers(0, 160, (900, 2)) if i != j]
    outcome, _ = _run(box_reg, oracle_mod, cs, seqs, pairs, "EDNAFULL", o, e)
    if (o, e) in ((16, 4), (20, 8)):
        assert (outcome == 0).mean() > 0.97  # the headline gap settings: nearly all solved here


def test_box_reg_loose_bounds_give_the_same_counters(box_reg, oracle_mod):
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(5)
    lens = synth.lognormal_lengths(120, 400, 0.6, 50, 1500, rng)
    seqs = [s.tobytes() for s in synth.dna_family(120, 30, lens, seed=9)]
    pairs = [(int(i), int(j)) for i, j in rng.integers(0, 120, (600, 2)) if i != j]
    for slack in (3, 40, 1000):
        _run(box_reg, oracle_mod, cs, seqs, pairs, "EDNAFULL", 16, 4, slack=slack, threads=5)


@pytest.mark.parametrize("o,e", [(4, 2), (2, 2), (6, 2), (3, 1)])
def test_box_reg_ties_match_oracle(box_reg, oracle_mod, o, e):
    """{A, C} sequences: many equal scores, equal maxima and extend-versus-open ties."""
    import csharp_b200 as cs
    rng = np.random.default_rng(100 + o)
    seqs = [bytes(rng.choice([65, 67], int(rng.integers(1, 70))).astype(np.uint8)) for _ in range(90)]
    pairs = [(i, j) for i in range(90) for j in range(90) if i != j][::5]
    outcome, _ = _run(box_reg, oracle_mod, cs, seqs, pairs, "EDNAFULL", o, e, threads=32)
    assert (outcome == 0).mean() > 0.5


def test_box_reg_protein(box_reg, oracle_mod):
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(7)
    bl = cs.ScoringMatrix.Load("BLOSUM62").Scores
    seqs = [s.tobytes() for s in synth.protein_family(90, 15, rng.integers(40, 300, 90), 8, bl)]
    pairs = [(i, j) for i in range(90) for j in range(90) if i != j][::6]
    for o, e in ((11, 3), (10, 1)):
        _run(box_reg, oracle_mod, cs, seqs, pairs, "BLOSUM62", o, e, protein=True)


def test_box_reg_short_and_edge_sequences(box_reg, oracle_mod):
    """One-residue sequences, alignments touching row 0 / column 0, identical sequences."""
    import csharp_b200 as cs
    rng = np.random.default_rng(3)
    base = bytes(rng.choice(list(b"ACGT"), 300).astype(np.uint8))
    seqs = [b"A", b"C", b"AC", base, base[:40], base[100:200], base[250:], base + base[:50], b"T" * 30 + base[:60]]
    pairs = [(i, j) for i in range(len(seqs)) for j in range(len(seqs)) if i != j]
    for o, e in ((16, 4), (5, 2)):
        _run(box_reg, oracle_mod, cs, seqs, pairs, "EDNAFULL", o, e, threads=4)
