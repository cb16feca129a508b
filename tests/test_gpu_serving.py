"""Serving on the GPU through the C ABI: query batches against a device-resident database.

Each query is aligned (query = s1, database entry = s2) against every entry, as the MS block
handler aligns a row sequence against a column range (Salsa.SmithWatermanMS/Program.cs:341-375).
Distances are checked bit-exact (Int16 equality) against the oracle.  A job's result must not
depend on what else is on the GPU: jobs submitted together, admitted at once and sharing waves,
equal the same jobs run one at a time.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cs():
    from csharp_b200 import build
    build.build()
    import csharp_b200
    return csharp_b200


def _dna(n, seed, lo, hi, roots=6):
    from csharp_b200 import synth
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, n)
    return [s.tobytes() for s in synth.dna_family(n, roots, lens, seed=seed)]


def _expected(cs, oracle_mod, queries, db, matrix, o, e, atype=1):
    concat, off = cs.pack_sequences(list(queries) + list(db))
    nq, nd = len(queries), len(db)
    ii = np.repeat(np.arange(nq), nd)
    jj = np.tile(np.arange(nq, nq + nd), nq)
    sc = cs.ScoringMatrix.Load(matrix).Scores[:127, :127].astype(np.float32)
    d = oracle_mod.pairs(concat, off, ii, jj, sc, float(o), float(e), alignment_type=atype,
                         threads=os.cpu_count())
    return d.reshape(nq, nd)


def _engine(cs, db, matrix="EDNAFULL", o=16, e=4, atype=1, **opts):
    eng = cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, alignment_type=atype)
    eng.upload(db)
    for k, v in opts.items():
        eng.set_option(k, v)
    return eng


@pytest.mark.parametrize("opts", [{}, {"third_pass": 0}, {"two_pass": 0}, {"two_pass": 2}])
def test_query_batch_matches_oracle(cs, oracle_mod, opts):
    """Two passes with the third pass (the default at 16/4), without it, one pass, and two passes
    forced at 3/2 gap costs (most pairs given up by the box step)."""
    db = _dna(300, 11, 1, 700)
    queries = _dna(9, 12, 30, 600) + [b"", b"A", _dna(1, 13, 1500, 1500)[0]]
    o, e = (3, 2) if opts.get("two_pass") == 2 else (16, 4)
    eng = _engine(cs, db, o=o, e=e, **opts)
    t = eng.submit(queries)
    r = eng.wait(t)
    assert r["status"] == 0 and r["queries"] == len(queries) and r["pairs"] == len(queries) * len(db)
    np.testing.assert_array_equal(r["out"], _expected(cs, oracle_mod, queries, db, "EDNAFULL", o, e))
    assert r["submit_s"] <= r["admit_s"] <= r["done_s"]


@pytest.mark.parametrize("dist_fn,mode", [(1, 0), (2, 1), (1, 1)])
def test_kimura_and_jukes_cantor_query_batch_matches_oracle(cs, oracle_mod, dist_fn, mode):
    """Kimura2 / JukesCantor serving (16-bit lanes with two counter words per state, queries over
    256 residues in several passes) against the oracle's block restatement, query = s1."""
    db = _dna(240, 21, 1, 900)
    queries = _dna(7, 22, 30, 800) + [b"", b"C", _dna(1, 23, 1300, 1300)[0]]
    sm = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(sm, 16, 4, mode=mode, distance_fn=dist_fn).upload(db)
    r = eng.wait(eng.submit(queries))
    assert r["status"] == 0 and r["pairs"] == len(queries) * len(db)
    concat, off = cs.pack_sequences(list(queries) + list(db))
    nq, nd = len(queries), len(db)
    want, _ = oracle_mod.block(concat, off, 0, nq - 1, nq, nq + nd - 1, False, mode,
                               sm.Scores[:127, :127].astype(np.float32), 16.0, 4.0, 1, dist_fn)
    np.testing.assert_array_equal(r["out"], want)


def test_results_are_the_same_alone_and_in_the_mix(cs):
    db = _dna(400, 21, 20, 900)
    jobs = [_dna(k, 30 + k, 40, 1200) for k in (40, 1, 7, 3, 2, 12)]
    alone = []
    eng = _engine(cs, db)
    for q in jobs:
        alone.append(eng.wait(eng.submit(q))["out"].copy())
    eng.serve_drain()
    # all at once: several admitted together, small jobs sharing waves with the large one
    mix = _engine(cs, db, serve_wave_us=2000)
    ts = [mix.submit(q) for q in jobs]
    got = [mix.wait(t) for t in ts]
    for a, g in zip(alone, got):
        assert g["status"] == 0
        np.testing.assert_array_equal(g["out"], a)
    st = mix.serve_stats()
    assert st["completed"] == len(jobs) and st["max_active"] >= 2 and st["waves"] >= 2


def test_admission_waits_for_memory_and_slots(cs, oracle_mod):
    """A budget that holds one job's result at a time: jobs queue, each still exact."""
    db = _dna(8000, 41, 10, 120)
    jobs = [_dna(k, 50 + k, 10, 200) for k in (40, 30, 50)]
    eng = _engine(cs, db, serve_memory_mb=1, serve_slots=64)  # 1 MiB: one of these results at a time
    ts = [eng.submit(q) for q in jobs]
    for q, t in zip(jobs, ts):
        r = eng.wait(t)
        assert r["status"] == 0
        sel = np.random.default_rng(len(q)).integers(0, len(db), 300)
        want = _expected(cs, oracle_mod, q, [db[k] for k in sel], "EDNAFULL", 16, 4)
        np.testing.assert_array_equal(r["out"][:, sel], want)
    assert eng.serve_stats()["max_active"] == 1
    with pytest.raises(cs.SwError):
        eng.submit(_dna(70, 60, 10, 20))  # more queries than slots


def test_protein_database_matches_oracle(cs, oracle_mod):
    from csharp_b200 import synth
    sc = cs.ScoringMatrix.Load("BLOSUM62").Scores
    rng = np.random.default_rng(71)
    db = [s.tobytes() for s in synth.protein_family(120, 5, rng.integers(5, 300, 120), 71, sc)]
    queries = [s.tobytes() for s in synth.protein_family(4, 2, rng.integers(5, 300, 4), 72, sc)]
    eng = _engine(cs, db, "BLOSUM62", 10, 1, atype=0)
    r = eng.wait(eng.submit(queries))
    np.testing.assert_array_equal(r["out"], _expected(cs, oracle_mod, queries, db, "BLOSUM62", 10, 1, atype=0))


@pytest.mark.parametrize("matrix,atype,o,e", [("EDNAFULL", 1, 16, 4), ("BLOSUM62", 0, 10, 1)])
def test_nw_database_matches_oracle(cs, oracle_mod, matrix, atype, o, e):
    """NW (global) serving on 16-bit lanes, with a query longer than the lanes' bias covers (it
    goes to 32-bit lanes) and empty / one-residue queries."""
    from csharp_b200 import synth
    rng = np.random.default_rng(73 + atype)
    sc = cs.ScoringMatrix.Load(matrix).Scores
    if atype:
        db = _dna(150, 74, 1, 500)
        queries = _dna(6, 75, 20, 400) + [b"", b"G", _dna(1, 76, 6000, 6000)[0]]
    else:
        db = [s.tobytes() for s in synth.protein_family(120, 5, rng.integers(5, 300, 120), 77, sc)]
        queries = [s.tobytes() for s in synth.protein_family(5, 2, rng.integers(5, 300, 5), 78, sc)] + [b"W"]
    eng = cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=cs.NW, alignment_type=atype)
    eng.upload(db)
    r = eng.wait(eng.submit(queries))
    concat, off = cs.pack_sequences(list(queries) + list(db))
    nq, nd = len(queries), len(db)
    ii = np.repeat(np.arange(nq), nd)
    jj = np.tile(np.arange(nq, nq + nd), nq)
    want = oracle_mod.nw_pairs(concat, off, ii, jj, sc[:127, :127].astype(np.float32), float(o), float(e),
                               protein=not atype, threads=os.cpu_count()).reshape(nq, nd)
    np.testing.assert_array_equal(r["out"], want)


def test_submit_errors(cs):
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4)
    with pytest.raises(cs.SwError):  # no database yet
        eng.submit([b"ACGT"])
    eng.upload(_dna(10, 81, 5, 50))
    with pytest.raises(cs.SwError):  # residue outside the 127-entry table
        eng.submit([b"AC\xc8T"])
    with pytest.raises(cs.SwError):
        eng.poll(12345)
    eng.wait(eng.submit([b"ACGT"]))
    with pytest.raises(cs.SwError):  # options are read when the first job is submitted
        eng.set_option("serve_slots", 10)
