"""The oracle (CPU restatement) against the golden vectors of the reference itself.

The golden vectors were produced by the reference's own C# aligner and block handler, rewritten
mechanically to C++ (oracle/cs2cpp.py) and run by tests/golden/make_golden.py.  When that build
(oracle/_ref) is present the restatement is also compared with it on fresh random inputs.
"""
import numpy as np
import pytest

from conftest import load_npz, unpack

FIELDS = ["identity", "similarity", "length", "start1", "start2", "gaps"]


def _scores(oracle, name, cache={}):
    if name not in cache:
        cache[name] = oracle.parse_matrix(oracle.matrix_text(name)) if oracle.ref_available() else None
    return cache[name]


def _matrix(name):
    from csharp_b200 import ScoringMatrix
    return ScoringMatrix.Load(name).Scores[:127, :127].astype(np.float32)


def test_restatement_matches_reference_kats(kats, oracle_mod):
    for k in kats:
        sc = _matrix(k["matrix"])
        a = oracle_mod.align(k["s1"].encode(), k["s2"].encode(), sc, k["o"], k["e"], with_strings=True)
        for f in FIELDS:
            assert a[f] == k[f], (f, k)
        if k["score"] is None:
            assert np.isinf(a["score"]) and a["score"] < 0
        else:
            assert a["score"] == k["score"]
        assert a["aln1"].decode() == k["aln1"] and a["aln2"].decode() == k["aln2"]
        d = oracle_mod.distance_i16(a, alignment_type=k["alignment_type"])
        assert d == k["distance"], k
        if k.get("kimura2") is not None:
            kd = oracle_mod.distance_i16(a, 1, 1, a["aln1"], a["aln2"])
            assert kd == k["kimura2"], k


def test_indp_formulation_matches_reference_kats(kats, oracle_mod):
    """The in-DP integer formulation the kernels use equals the traceback on every KAT."""
    for k in kats:
        sc = _matrix(k["matrix"]).astype(np.int32)
        a = oracle_mod.indp_align(k["s1"].encode(), k["s2"].encode(), sc, k["o"], k["e"])
        for f in FIELDS:
            assert a[f] == k[f], (f, k)


@pytest.mark.parametrize("name", ["mpi_p1.npz", "mpi_p3.npz", "mpi_p4.npz", "protein_mpi.npz",
                                  "identity_mpi.npz", "mpi_kimura_p3.npz", "mpi_jc_p1.npz"])
def test_restatement_block_driver_matches_reference(name, oracle_mod):
    z = load_npz(name)
    seqs = unpack(z)
    N, P = len(seqs), int(z["ranks"])
    sc = _matrix(z["matrix"].tobytes().decode())
    bounds, s = [], 0
    for r in range(P):
        ln = N // P + (1 if r < N % P else 0)
        bounds.append((s, s + ln - 1))
        s += ln
    full = np.zeros((N, N), dtype=np.int16)
    for r in range(P):
        for c in range(P):
            diag = r == c
            if not (diag or (r > c and (r + c) % 2 == 0) or (r < c and (r + c) % 2 == 1)):
                continue
            (rs, re_), (cs, ce) = bounds[r], bounds[c]
            blk, _ = oracle_mod.block(z["concat"], z["offsets"], rs, re_, cs, ce, diag, 0, sc,
                                      float(z["o"]), float(z["e"]), int(z["alignment_type"]),
                                      int(z.get("dist_fn", 0)))
            if diag:
                full[rs:re_ + 1, cs:ce + 1] = blk
            else:
                full[rs:re_ + 1, cs:ce + 1] = blk
                full[cs:ce + 1, rs:re_ + 1] = blk.T
    np.testing.assert_array_equal(full, z["distances"])


@pytest.mark.parametrize("name,mode", [("nw_restated.npz", 2), ("ms_restated.npz", 1),
                                       ("ms_protein_restated.npz", 1), ("nw_protein_restated.npz", 2)])
def test_restated_modes_regression(name, mode, oracle_mod):
    """NW / SWG-MS fixtures are the restatement's own output (their aligner is closed Bio.dll):
    this guards the restatement against drift."""
    z = load_npz(name)
    seqs = unpack(z)
    sc = _matrix(z["matrix"].tobytes().decode())
    protein = int(z["alignment_type"]) == 0
    N = len(seqs)
    for i in range(N):
        for j in range(N):
            if mode == 2:
                if j >= i:
                    continue
                r = oracle_mod.nw_align(seqs[i], seqs[j], sc, float(z["o"]), float(z["e"]))
                d = oracle_mod.nw_distance_i16(r["aln1"], r["aln2"], sc, protein)
            else:
                r = oracle_mod.align(seqs[i], seqs[j], sc, float(z["o"]), float(z["e"]), with_strings=True)
                d = oracle_mod.ms_distance_i16(r["aln1"], r["aln2"], sc, protein)
            assert d == z["distances"][i, j], (i, j)


def test_restatement_matches_transliterated_reference_fuzz(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref (transliterated reference) not built on this host")
    rng = np.random.default_rng(99)
    sc = _matrix("EDNAFULL")
    for _ in range(150):
        m, n = rng.integers(0, 60, 2)
        alph = np.frombuffer(b"ACGT" if rng.random() < 0.5 else b"AC", np.uint8)
        s1, s2 = rng.choice(alph, m).tobytes(), rng.choice(alph, n).tobytes()
        o, e = int(rng.integers(1, 20)), int(rng.integers(0, 8))
        a = oracle_mod.align(s1, s2, sc, o, e)
        r = oracle_mod.ref_align("EDNAFULL", s1, s2, o, e)
        for f in FIELDS:
            assert a[f] == r[f], (f, s1, s2, o, e)


def test_builtin_matrices_equal_reference_files(oracle_mod):
    """The engine's built-in tables equal the reference's embedded matrix resources."""
    from csharp_b200 import ScoringMatrix
    if not oracle_mod.ref_available():
        pytest.skip("reference matrix files not available on this host")
    for name in ScoringMatrix.BUILTIN:
        ref = oracle_mod.parse_matrix(oracle_mod.matrix_text(name))
        mine = ScoringMatrix.Load(name).Scores[:127, :127]
        np.testing.assert_array_equal(mine.astype(np.float32), ref, err_msg=name)
        parsed = ScoringMatrix.Parse(oracle_mod.matrix_text(name)).Scores[:127, :127]
        np.testing.assert_array_equal(parsed, mine, err_msg=name)


def test_batched_integer_checkers_equal_traceback_restatement(kats, oracle_mod):
    """The two batched in-DP checkers (cnt5 counters; one packed counter word) used for whole
    configurations give the traceback restatement's distances: the KAT pairs, uneven DNA
    families, tie-heavy {A, C} sequences and BLOSUM62 protein (exact Int16)."""
    import csharp_b200 as cs
    from csharp_b200 import synth
    rng = np.random.default_rng(17)
    kat = [k for k in kats if float(k["o"]).is_integer() and float(k["e"]).is_integer() and k["matrix"] != "IDENTITY"]
    cases = []
    for k in kat[:120]:
        cases.append(([k["s1"].encode(), k["s2"].encode()], [(0, 1)], k["matrix"], int(k["o"]), int(k["e"]), k["alignment_type"]))
    dna = [s.tobytes() for s in synth.dna_family(60, 6, synth.lognormal_lengths(60, 200, 0.6, 1, 600, rng), seed=3)]
    cases.append((dna, [(i, j) for i in range(60) for j in range(i)][::3], "EDNAFULL", 16, 4, 1))
    ac = [bytes(rng.choice([65, 67], int(rng.integers(1, 50))).astype(np.uint8)) for _ in range(50)]
    cases.append((ac, [(i, j) for i in range(50) for j in range(50) if i != j][::4], "EDNAFULL", 4, 2, 1))
    prot = [s.tobytes() for s in synth.protein_family(40, 5, rng.integers(20, 200, 40), 9, cs.ScoringMatrix.Load("BLOSUM62").Scores)]
    cases.append((prot, [(i, j) for i in range(40) for j in range(40) if i != j][::3], "BLOSUM62", 10, 1, 0))
    for seqs, pairs, matrix, o, e, atype in cases:
        concat, off = cs.pack_sequences(seqs)
        r = np.array([p[0] for p in pairs]); c = np.array([p[1] for p in pairs])
        m = cs.ScoringMatrix.Load(matrix).Scores[:127, :127]
        want = oracle_mod.pairs(concat, off, r, c, m.astype(np.float32), float(o), float(e), alignment_type=atype)
        for fast in (False, True):
            got = oracle_mod.indp_pairs(concat, off, r, c, m.astype(np.int32), o, e, alignment_type=atype, fast=fast)
            np.testing.assert_array_equal(got, want)
