"""The two-pass box step on the CPU: the source of the lane box kernel (swg_box_lane.cuh),
compiled for the host, against the oracle.

The score pass hands the box step each pair's best score S and first-maximum cell (ie, je); here
the oracle's in-DP aligner supplies them.  Every pair the box step solves must carry exactly the
traceback's aligned columns and identity (similarity for protein) — tolerance: exact — on
uneven DNA family sets at several gap settings, tie-heavy two-letter sequences and BLOSUM62
protein; pairs it gives up on are the GPU path's to redo (the warp box kernel or the int32 DP).
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
def box_step(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not (CUDA_INC / "vector_types.h").exists():
        pytest.skip("g++ or the CUDA headers are missing")
    so = tmp_path_factory.mktemp("box_step") / "libbox_step.so"
    subprocess.run([gxx, "-O2", "-std=c++17", "-shared", "-fPIC", f"-I{CUDA_INC}", "-o", str(so),
                    str(HERE / "box_step_host.cpp")], check=True)
    lib = C.CDLL(str(so))
    lib.box_step_run.restype = C.c_int
    return lib


def _run(lib, oracle_mod, cs, seqs, pairs, matrix, o, e, protein=False, threads=7, max_score=1 << 30):
    concat, off = cs.pack_sequences(seqs)
    sc = cs.ScoringMatrix.Load(matrix).Scores.astype(np.int32)
    x = np.arange(128)
    fl = ((x[:, None] == x[None, :]) | ((sc > 0) if protein else False)).astype(np.uint32)
    isc = np.ascontiguousarray(sc[:127, :127])
    rows = []
    for qi, di in pairs:
        r = oracle_mod.indp_align(seqs[qi], seqs[di], isc, o, e)
        if np.isfinite(r["score"]) and r["score"] > 0:
            rows.append((qi, di, int(r["score"]), r["end1"], r["end2"], r["length"],
                         r["similarity"] if protein else r["identity"]))
    a = np.array(rows, dtype=np.int64)
    cols = [np.ascontiguousarray(a[:, k].astype(np.int32)) for k in range(5)]
    n = len(a)
    outcome = np.zeros(n, np.int32)
    counters = np.zeros(n, np.uint32)
    P = C.c_void_p
    rc = lib.box_step_run(P(concat.ctypes.data), P(off.ctypes.data), *[P(c.ctypes.data) for c in cols], C.c_long(n),
                          P(np.ascontiguousarray(sc).ctypes.data), P(np.ascontiguousarray(fl).ctypes.data), 128,
                          int(o), int(e), int(max_score), int(threads), P(outcome.ctypes.data), P(counters.ctypes.data))
    assert rc == 0
    assert (outcome >= 0).all() and (outcome <= 5).all()
    ok = outcome == 0
    got = np.stack([(counters[ok] >> 8).astype(np.int64), (counters[ok] & 0xFF).astype(np.int64)], 1)
    np.testing.assert_array_equal(got, a[ok][:, 5:7])
    return outcome, a[:, 2]


@pytest.mark.parametrize("o,e", [(16, 4), (20, 8), (10, 3), (4, 2)])
def test_box_step_uneven_dna_matches_oracle(box_step, oracle_mod, o, e):
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(o * 31 + e)
    lens = synth.lognormal_lengths(160, 400, 0.6, 50, 1500, rng)
    seqs = [s.tobytes() for s in synth.dna_family(160, 40, lens, seed=o + e)]
    pairs = [(int(i), int(j)) for i, j in rng.integers(0, 160, (900, 2)) if i != j]
    outcome, _ = _run(box_step, oracle_mod, cs, seqs, pairs, "EDNAFULL", o, e)
    if (o, e) in ((16, 4), (20, 8)):
        assert (outcome == 0).mean() > 0.9  # the headline gap settings: nearly all solved here


@pytest.mark.parametrize("o,e", [(4, 2), (2, 2), (6, 2)])
def test_box_step_ties_match_oracle(box_step, oracle_mod, o, e):
    """{A, C} sequences: many equal scores, equal maxima and extend-versus-open ties."""
    import csharp_b200 as cs
    rng = np.random.default_rng(100 + o)
    seqs = [bytes(rng.choice([65, 67], int(rng.integers(1, 70))).astype(np.uint8)) for _ in range(90)]
    pairs = [(i, j) for i in range(90) for j in range(90) if i != j][::5]
    outcome, _ = _run(box_step, oracle_mod, cs, seqs, pairs, "EDNAFULL", o, e, threads=32)
    assert (outcome == 0).mean() > 0.5


def test_box_step_protein_and_score_cap(box_step, oracle_mod):
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(7)
    bl = cs.ScoringMatrix.Load("BLOSUM62").Scores
    seqs = [s.tobytes() for s in synth.protein_family(90, 15, rng.integers(40, 300, 90), 8, bl)]
    pairs = [(i, j) for i in range(90) for j in range(90) if i != j][::6]
    _run(box_step, oracle_mod, cs, seqs, pairs, "BLOSUM62", 11, 3, protein=True)
    # pairs above the score cap are handed on untouched (reason 4)
    outcome, S = _run(box_step, oracle_mod, cs, seqs, pairs, "BLOSUM62", 11, 3, protein=True, threads=3, max_score=60)
    assert (outcome[S > 60] == 4).all()
