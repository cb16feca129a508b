"""Generates the golden fixtures in tests/golden from the reference itself.

Run in a container that holds the reference sources (it builds oracle/_ref first):

    python tests/golden/make_golden.py

SWG-MPI fixtures (``kat_pairs.json``, ``mpi_*.npz``, ``protein_mpi.npz``, ``identity_mpi.npz``)
are outputs of the reference's own C# aligner and ComputeBlock/ComputeDistance
(SmithWatermanGotoh.cs, Alignment.cs, Salsa.SmithWatermanMPI/Program.cs), transliterated to C++
by oracle/cs2cpp.py and run here.  The NW and SWG-MS fixtures come from the oracle's
restatement (their aligner lives in the closed Bio.dll; parity with it is unpinned).
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))

import oracle  # noqa: E402
from csharp_b200 import synth  # noqa: E402


def pack(seqs):
    parts = [np.frombuffer(bytes(s), dtype=np.uint8) for s in seqs]
    off = np.zeros(len(parts) + 1, dtype=np.int64)
    np.cumsum([len(p) for p in parts], out=off[1:])
    return (np.concatenate(parts) if parts else np.zeros(0, np.uint8)), off


def ref_pair_distance(matrix, atype, s1, s2, o, e, dist_fn=0):
    """matrix[1, 0] of ComputeBlock over the two-sequence set (s1 = sequence 1, s2 = sequence 0)."""
    seqs, off = pack([s2, s1])
    full, n = oracle.ref_compute_block(matrix, atype, dist_fn, o, e, seqs, off, 1, 1, 0, 0, False)
    assert n == 1
    return int(full[1, 0])


def draw(rng, letters, k):
    return rng.choice(np.frombuffer(letters, dtype=np.uint8), int(k)).tobytes()


def kat_pairs():
    rng = np.random.default_rng(20240601)
    cases = []
    designed = [
        ("ACGTACGT", "ACGTACGT", 16, 4), ("ACGTACGT", "ACGAACGT", 16, 4), ("AAAA", "CCCC", 16, 4),
        ("", "ACGT", 16, 4), ("ACGT", "", 16, 4), ("", "", 16, 4), ("A", "A", 16, 4), ("A", "C", 16, 4),
        ("ACGTTGCA", "ACGTGCA", 16, 4), ("ACGTTTTTGCA", "ACGTGCA", 16, 4), ("ACAC", "CACA", 5, 5),
        ("AACCAACC", "AACC", 4, 4), ("ACGT", "ACGTACGT", 16, 4), ("ACGTACGT", "ACGT", 16, 4),
        ("GATTACA", "GCATGCT", 8, 4), ("ACGTNACGT", "ACGTXACGT", 16, 4), ("XXXX", "XXXX", 16, 4),
        ("TTTTUUUU", "UUUUTTTT", 16, 4), ("ACGTACGTAC", "TGCATGCATG", 16, 4),
        ("AAAAAAAAAA", "AAAAACAAAAA", 9, 0), ("ACACACACAC", "ACACCACACAC", 1, 1),
    ]
    for s1, s2, o, e in designed:
        cases.append(("EDNAFULL", 1, s1.encode(), s2.encode(), o, e))
    # tie hunting: two-letter alphabet, small penalties (extend/open ties, equal maxima)
    for _ in range(240):
        m, n = rng.integers(1, 41, 2)
        o = int(rng.integers(1, 17))
        e = int(rng.integers(0, 9))
        s1, s2 = draw(rng, b"AC", m), draw(rng, b"AC", n)
        cases.append(("EDNAFULL", 1, s1, s2, o, e))
    for _ in range(120):
        m, n = rng.integers(0, 90, 2)
        s1, s2 = draw(rng, b"ACGT", m), draw(rng, b"ACGT", n)
        cases.append(("EDNAFULL", 1, s1, s2, 16, 4))
    aa = b"ARNDCQEGHILKMFPSTWYVBZX"
    for _ in range(80):
        m, n = rng.integers(1, 70, 2)
        cases.append(("BLOSUM62", 0, draw(rng, aa, m), draw(rng, aa, n), 10, 1))
    for _ in range(40):
        m, n = rng.integers(1, 50, 2)
        cases.append(("IDENTITY", 0, draw(rng, aa[:6], m), draw(rng, aa[:6], n), 10, 1))
    out = []
    for matrix, atype, s1, s2, o, e in cases:
        r = oracle.ref_align(matrix, s1, s2, o, e, with_strings=True)
        d = ref_pair_distance(matrix, atype, s1, s2, o, e)
        rec = dict(matrix=matrix, alignment_type=atype, s1=s1.decode(), s2=s2.decode(), o=o, e=e,
                   score=(None if np.isinf(r["score"]) else r["score"]), identity=r["identity"],
                   similarity=r["similarity"], length=r["length"], start1=r["start1"],
                   start2=r["start2"], gaps=r["gaps"], distance=d,
                   aln1=r["aln1"].decode(), aln2=r["aln2"].decode())
        if atype == 1 and r["length"] > 0:
            try:
                rec["kimura2"] = ref_pair_distance(matrix, atype, s1, s2, o, e, dist_fn=1)
            except RuntimeError:
                rec["kimura2"] = None
        out.append(rec)
    (HERE / "kat_pairs.json").write_text(json.dumps(out, separators=(",", ":")).replace("},{", "},\n{"))
    return len(out)


def mpi_job(name, seqs, matrix, atype, o, e, ranks, dist_fn=0):
    """The reference's block driver for `ranks` ranks: every rank's ComputeBlock calls plus the
    Scatter mirror, assembled into the full N x N matrix."""
    concat, off = pack(seqs)
    N = len(seqs)
    a, b = N // ranks, N % ranks
    bounds, s = [], 0
    for r in range(ranks):
        ln = a + (1 if r < b else 0)
        bounds.append((s, s + ln - 1))
        s += ln
    full = np.zeros((N, N), dtype=np.int16)
    pairs = 0
    for r in range(ranks):
        for c in range(ranks):
            diag = r == c
            computed = diag or (r > c and (r + c) % 2 == 0) or (r < c and (r + c) % 2 == 1)
            if not computed or bounds[r][0] > bounds[r][1] or bounds[c][0] > bounds[c][1]:
                continue
            got, n = oracle.ref_compute_block(matrix, atype, dist_fn, o, e, concat, off, bounds[r][0],
                                              bounds[r][1], bounds[c][0], bounds[c][1], diag)
            pairs += n
            rs, re_ = bounds[r]
            cs, ce = bounds[c]
            full[rs:re_ + 1, cs:ce + 1] = got[rs:re_ + 1, cs:ce + 1]
            if not diag:  # Scatter: the transposed block lands in rank c's rows
                full[cs:ce + 1, rs:re_ + 1] = got[rs:re_ + 1, cs:ce + 1].T
    np.savez_compressed(HERE / name, concat=concat, offsets=off, matrix=np.frombuffer(matrix.encode(), np.uint8),
                        alignment_type=atype, o=o, e=e, ranks=ranks, distances=full, pairs=pairs,
                        dist_fn=dist_fn)
    return pairs


def restated_job(name, seqs, matrix, mode, atype, o, e, dist_fn=0):
    """NW (mode 2) and SWG-MS (mode 1) from the oracle restatement (unpinned)."""
    concat, off = pack(seqs)
    N = len(seqs)
    sc = oracle.parse_matrix(oracle.matrix_text(matrix))
    full = np.zeros((N, N), dtype=np.int16)
    for i in range(N):
        for j in range(N):
            if mode == 2 and j >= i:
                continue
            s1, s2 = seqs[i], seqs[j]
            if mode == 2:
                r = oracle.nw_align(s1, s2, sc, o, e)
                d = oracle.nw_distance_i16(r["aln1"], r["aln2"], sc, protein=(atype == 0))
                full[i, j] = full[j, i] = d
            else:
                r = oracle.align(s1, s2, sc, o, e, with_strings=True)
                full[i, j] = oracle.ms_distance_i16(r["aln1"], r["aln2"], sc, protein=(atype == 0),
                                                    dist_fn=dist_fn)
    np.savez_compressed(HERE / name, concat=concat, offsets=off, matrix=np.frombuffer(matrix.encode(), np.uint8),
                        alignment_type=atype, o=o, e=e, mode=mode, distances=full, dist_fn=dist_fn)


def distance_function_jobs(dna):
    """Kimura2 / JukesCantor (Alignment.cs:254-348): SWG-MPI from the reference's own driver,
    SWG-MS from the restatement."""
    print("mpi kimura p3", mpi_job("mpi_kimura_p3.npz", dna, "EDNAFULL", 1, 16, 4, 3, dist_fn=1))
    print("mpi jukes-cantor p1", mpi_job("mpi_jc_p1.npz", dna, "EDNAFULL", 1, 16, 4, 1, dist_fn=2))
    restated_job("ms_kimura_restated.npz", dna[:24], "EDNAFULL", 1, 1, 16, 4, dist_fn=1)
    restated_job("ms_jc_restated.npz", dna[:24], "EDNAFULL", 1, 1, 16, 4, dist_fn=2)


def main():
    oracle.build()
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref could not be built (reference sources missing)")
    rng = np.random.default_rng(7)
    dna = [s.tobytes() for s in synth.dna_family(46, 4, rng.integers(20, 160, 46), seed=11)]
    dna = dna[:20] + [b"", b"A", b"ACGTNNACGT"] + dna[20:]
    if "--distance-functions" in sys.argv:  # only the Kimura2 / JukesCantor fixtures
        distance_function_jobs(dna)
        return
    print("kat pairs", kat_pairs())
    print("mpi p1", mpi_job("mpi_p1.npz", dna, "EDNAFULL", 1, 16, 4, 1))
    print("mpi p3", mpi_job("mpi_p3.npz", dna, "EDNAFULL", 1, 16, 4, 3))
    print("mpi p4", mpi_job("mpi_p4.npz", dna, "EDNAFULL", 1, 14, 4, 4))
    from csharp_b200 import ScoringMatrix  # noqa: E402  (built-in table equals the reference's)
    bl = oracle.parse_matrix(oracle.matrix_text("BLOSUM62")).astype(np.int16)
    pro = [s.tobytes() for s in synth.protein_family(36, 3, rng.integers(10, 140, 36), 12, np.pad(bl, ((0, 1), (0, 1))))]
    print("protein", mpi_job("protein_mpi.npz", pro, "BLOSUM62", 0, 10, 1, 1))
    idn = [draw(rng, b"ARNDCQ", k) for k in rng.integers(1, 90, 30)]
    print("identity", mpi_job("identity_mpi.npz", idn, "IDENTITY", 0, 10, 1, 1))
    restated_job("nw_restated.npz", dna[:30], "EDNAFULL", 2, 1, 16, 4)
    restated_job("ms_restated.npz", dna[:24], "EDNAFULL", 1, 1, 16, 4)
    restated_job("ms_protein_restated.npz", pro[:20], "BLOSUM62", 1, 0, 10, 1)
    restated_job("nw_protein_restated.npz", pro[:20], "BLOSUM62", 2, 0, 10, 1)
    distance_function_jobs(dna)
    del ScoringMatrix


if __name__ == "__main__":
    main()
