"""GPU parity through the C ABI: every distance bit-exact against the reference.

Golden vectors come from the reference's own aligner and block driver (tests/golden); larger
inputs are checked against the oracle (the CPU restatement, itself pinned to those vectors).
Tolerance: exact Int16 equality everywhere.
"""
import os

import numpy as np
import pytest

from conftest import load_npz, unpack

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cs():
    from csharp_b200 import build
    build.build()
    import csharp_b200
    return csharp_b200


_engines = {}


def engine(cs, matrix, o, e, atype=1, mode=0, lanes=0):
    key = (matrix, o, e, atype, mode, lanes)
    if key not in _engines:
        _engines[key] = cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=mode, alignment_type=atype, lanes=lanes)
    return _engines[key]


def test_align_pair_matches_reference_kats(cs, kats):
    for k in kats:
        eng = engine(cs, k["matrix"], k["o"], k["e"], k["alignment_type"])
        r = eng.align(k["s1"], k["s2"])
        got = dict(identity=r.Identity, similarity=r.Similarity, length=r.Length, start1=r.Start1,
                   start2=r.Start2, gaps=r.Gaps, distance=r.Distance)
        want = {f: k[f] for f in got}
        assert got == want, k
        if k["score"] is None:
            assert np.isinf(r.Score) and r.Score < 0
        else:
            assert r.Score == k["score"]


def _golden_engine(cs, z, mode=0, lanes=0):
    eng = cs.Engine(cs.ScoringMatrix.Load(z["matrix"].tobytes().decode()), float(z["o"]), float(z["e"]),
                    mode=mode, alignment_type=int(z["alignment_type"]), lanes=lanes)
    eng.upload(concat=z["concat"], offsets=z["offsets"])
    return eng


@pytest.mark.parametrize("name", ["mpi_p1.npz", "mpi_p3.npz", "mpi_p4.npz", "protein_mpi.npz", "identity_mpi.npz"])
@pytest.mark.parametrize("block_engine", [0, 2])
def test_block_handler_matches_reference_block_driver(cs, name, block_engine):
    """One drop-in call per block of the reference's driver, mirrored like Scatter: the plain
    per-block kernel (block_engine 0) and the batched engine (2) give the reference's values."""
    z = load_npz(name)
    eng = _golden_engine(cs, z)
    eng.set_option("block_engine", block_engine)
    N, P = len(z["offsets"]) - 1, int(z["ranks"])
    rr = cs.range_partition(N, P)
    full = np.zeros((N, N), dtype=np.int16)
    pairs = 0
    for r in range(P):
        for c in range(P):
            if not (r == c or cs.block_is_computed(r, c)):
                continue
            a, b = rr[r], rr[c]
            blk, n = eng.compute_block(a.StartIndex, a.EndIndex, b.StartIndex, b.EndIndex, r == c)
            pairs += n
            full[a.StartIndex:a.EndIndex + 1, b.StartIndex:b.EndIndex + 1] = blk
            if r != c:
                full[b.StartIndex:b.EndIndex + 1, a.StartIndex:a.EndIndex + 1] = blk.T
    assert pairs == int(z["pairs"])
    np.testing.assert_array_equal(full, z["distances"])
    eng.set_option("block_engine", 1)


@pytest.mark.parametrize("name", ["mpi_p1.npz", "mpi_p3.npz", "mpi_p4.npz", "protein_mpi.npz", "identity_mpi.npz"])
@pytest.mark.parametrize("lanes", [0, 32])
def test_engine_matches_reference_driver(cs, name, lanes):
    z = load_npz(name)
    eng = _golden_engine(cs, z, lanes=lanes)
    full, pairs, cells = eng.all_pairs(int(z["ranks"]))
    assert pairs == int(z["pairs"])
    np.testing.assert_array_equal(full, z["distances"])


@pytest.mark.parametrize("block_engine", [0, 2])
def test_block_handler_leaves_unaligned_entries_alone(cs, block_engine):
    z = load_npz("mpi_p1.npz")
    eng = _golden_engine(cs, z)
    eng.set_option("block_engine", block_engine)
    out = np.full((10, 14), 1234, dtype=np.int16)  # the block in a wider buffer (ld 14)
    blk = out[:, :10]
    eng.compute_block(3, 12, 3, 12, True, out=blk)
    assert (np.diag(blk) == 1234).all()
    assert (out[:, 10:] == 1234).all()
    np.testing.assert_array_equal(blk[~np.eye(10, dtype=bool)], z["distances"][3:13, 3:13][~np.eye(10, dtype=bool)])
    eng.set_option("block_engine", 1)


@pytest.mark.parametrize("mode", [0, 1, 2])
@pytest.mark.parametrize("matrix", ["EDNAFULL", "BLOSUM62"])
def test_engine_block_handler_equals_plain_kernel(cs, mode, matrix):
    """The block handler on the batched engine (large blocks) against the plain per-block kernel:
    diagonal and off-diagonal blocks of an uneven set, host and device output, every mode."""
    from csharp_b200 import synth
    import torch
    rng = np.random.default_rng(40 + mode)
    N = 260
    lens = synth.lognormal_lengths(N, 300, 0.6, 20, 900, rng)
    if matrix == "BLOSUM62":
        seqs = [s.tobytes() for s in synth.protein_family(N, 12, lens, 5, cs.ScoringMatrix.Load("BLOSUM62").Scores)]
        o, e, atype = 10, 1, cs.PROTEIN
    else:
        seqs = [s.tobytes() for s in synth.dna_family(N, 20, lens, seed=6)]
        o, e, atype = 16, 4, cs.NUCLEIC
    m = cs.ScoringMatrix.Load(matrix)
    plain = cs.Engine(m, o, e, mode=mode, alignment_type=atype).upload(seqs)
    plain.set_option("block_engine", 0)
    eng = cs.Engine(m, o, e, mode=mode, alignment_type=atype).upload(seqs)
    for rs, re_, cs_, ce, diag in [(0, 129, 0, 129, True), (130, 259, 0, 129, False), (20, 200, 140, 259, False),
                                   (130, 259, 130, 259, True)]:
        want, n0 = plain.compute_block(rs, re_, cs_, ce, diag)
        got, n1 = eng.compute_block(rs, re_, cs_, ce, diag)
        assert n0 == n1
        assert eng.query("launches") >= 3  # the engine ran, not the plain kernel
        np.testing.assert_array_equal(got, want)
        R, Cc = re_ - rs + 1, ce - cs_ + 1
        d = torch.zeros((R, Cc + 3), dtype=torch.int16, device="cuda")
        eng.compute_block_device(rs, re_, cs_, ce, diag, d.data_ptr(), Cc + 3)
        eng.synchronize()
        dd = d.cpu().numpy()
        assert (dd[:, Cc:] == 0).all()
        tri = diag and mode != 1
        mask = ~np.eye(R, dtype=bool) if tri else np.ones((R, Cc), dtype=bool)
        np.testing.assert_array_equal(dd[:, :Cc][mask], want[mask])
    plain.close()
    eng.close()


@pytest.mark.parametrize("name,mode", [("nw_restated.npz", 2), ("ms_restated.npz", 1),
                                       ("ms_protein_restated.npz", 1), ("nw_protein_restated.npz", 2)])
def test_nw_and_ms_modes_match_restatement(cs, name, mode):
    z = load_npz(name)
    eng = _golden_engine(cs, z, mode=mode)
    full, _, _ = eng.all_pairs(1)
    want = z["distances"].copy()
    if mode == 2:
        np.fill_diagonal(want, 0)
    np.testing.assert_array_equal(full, want)
    N = len(z["offsets"]) - 1
    blk, n = eng.compute_block(0, N - 1, 0, N - 1, True)
    if mode == 1:
        np.testing.assert_array_equal(blk, z["distances"])
    else:
        off = ~np.eye(N, dtype=bool)
        np.testing.assert_array_equal(blk[off], want[off])


def _oracle_distances(oracle, seqs, pairs, matrix, o, e, atype=1):
    from csharp_b200 import ScoringMatrix, pack_sequences
    sc = ScoringMatrix.Load(matrix).Scores[:127, :127].astype(np.float32)
    concat, off = pack_sequences(seqs)
    return oracle.pairs(concat, off, pairs[:, 0], pairs[:, 1], sc, o, e, atype)


def test_engine_long_and_uneven_sequences_against_oracle(cs, oracle_mod):
    """Multi-pass queries (up to 2600 rows), empty and 1-residue sequences, every K bin."""
    from csharp_b200 import synth
    rng = np.random.default_rng(123)
    lens = np.concatenate([rng.integers(1, 120, 40), rng.integers(400, 700, 20), rng.integers(1400, 2600, 8), [1, 2, 3]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 5, lens, seed=77)] + [b"", b"G"]
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    full, pairs, _ = eng.all_pairs(1)
    N = len(seqs)
    ii, jj = np.tril_indices(N, -1)
    sel = rng.choice(len(ii), min(len(ii), 2500), replace=False)
    pr = np.stack([ii[sel], jj[sel]], 1)
    want = _oracle_distances(oracle_mod, seqs, pr, "EDNAFULL", 16, 4)
    np.testing.assert_array_equal(full[pr[:, 0], pr[:, 1]], want)
    np.testing.assert_array_equal(full[pr[:, 1], pr[:, 0]], want)
    assert pairs == N * (N - 1) // 2
    # the drop-in block kernel agrees on the same pairs
    blk, _ = eng.compute_block(0, N - 1, 0, N - 1, True)
    off = ~np.eye(N, dtype=bool)
    np.testing.assert_array_equal(blk[off], full[off])


@pytest.mark.parametrize("opt", [("rows_per_lane", k) for k in (4, 6, 8, 10, 12, 14, 16)] +
                                [("chunk", 32), ("chunk", 1024), ("use_graph", 0)])
def test_engine_options_do_not_change_results(cs, opt):
    from csharp_b200 import synth
    rng = np.random.default_rng(5)
    lens = np.concatenate([rng.integers(20, 700, 120), [0, 1, 1500]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 6, lens, seed=9)]
    base = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    want, _, _ = base.all_pairs(1)
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    eng.set_option(*opt)
    got, _, _ = eng.all_pairs(1)
    np.testing.assert_array_equal(got, want)
    got2, _, _ = eng.all_pairs(1)  # replay
    np.testing.assert_array_equal(got2, want)


def test_tripped_16bit_lanes_rerun_in_32bit(cs):
    """Force the trip level below the scores reached: every tripped pair is redone with 32-bit
    lanes and the matrix is unchanged."""
    z = load_npz("mpi_p1.npz")
    eng = _golden_engine(cs, z)
    eng.set_option("int16_threshold", 40)
    full, _, _ = eng.all_pairs(1)
    assert eng.rerun_count() > 0
    np.testing.assert_array_equal(full, z["distances"])


def test_int16_static_guard_routes_high_scoring_pairs(cs, oracle_mod):
    """A matrix whose scores cannot stay in 16-bit lanes for long pairs goes to 32-bit lanes."""
    txt = "   A C G T\nA 300 -100 -100 -100\nC -100 300 -100 -100\nG -100 -100 300 -100\nT -100 -100 -100 300\n"
    m = cs.ScoringMatrix.Parse(txt, "HIGH")
    from csharp_b200 import synth
    lens = np.array([150, 160, 170, 40, 50, 300])
    seqs = [s.tobytes() for s in synth.dna_family(6, 1, lens, seed=3, sub_range=(0.01, 0.02), indel_range=(0.0, 0.01))]
    eng = cs.Engine(m, 16, 4).upload(seqs)
    full, _, _ = eng.all_pairs(1)
    assert eng.rerun_count() > 0
    sc = m.Scores[:127, :127].astype(np.float32)
    for i in range(6):
        for j in range(i):
            a = oracle_mod.align(seqs[i], seqs[j], sc, 16, 4)
            assert full[i, j] == oracle_mod.distance_i16(a), (i, j)


def test_rank_blocks_partition_the_job(cs):
    import torch
    z = load_npz("mpi_p4.npz")
    eng = _golden_engine(cs, z)
    N = len(z["offsets"]) - 1
    total = torch.zeros((N, N), dtype=torch.int16, device="cuda")
    npairs = 0
    for r in range(4):
        part = torch.zeros((N, N), dtype=torch.int16, device="cuda")
        npairs += eng.rank_blocks_device(r, 4, part.data_ptr(), N)
        eng.synchronize()
        assert not ((total != 0) & (part != 0)).any()
        total += part
    assert npairs == int(z["pairs"])
    np.testing.assert_array_equal(total.cpu().numpy(), z["distances"])


@pytest.mark.parametrize("name", ["mpi_p1.npz", "protein_mpi.npz", "nw_restated.npz"])
def test_balanced_row_shares_give_the_one_rank_matrix(cs, name):
    """The balanced scheme's shares (rows cut at equal DP cells, sw_compute_rows) for 1-4 ranks,
    merged as merge_row_slabs does, give the reference's one-rank matrix."""
    import torch
    from csharp_b200.driver import balanced_row_ranges, merge_row_slabs
    z = load_npz(name)
    eng = _golden_engine(cs, z, mode=int(z["mode"]) if "mode" in z else 0)
    N = len(z["offsets"]) - 1
    want = z["distances"].copy()
    np.fill_diagonal(want, 0)  # the full matrix's diagonal (NW's restatement holds self-distances)
    for world in (1, 2, 4):
        ranges = balanced_row_ranges(eng.lengths, world)
        out = torch.zeros((N, N), dtype=torch.int16, device="cuda")
        npairs = sum(eng.rows_device(lo, hi, out.data_ptr(), N) for lo, hi in ranges)
        eng.synchronize()
        assert npairs == N * (N - 1) // 2
        merge_row_slabs(out, 0, 1, [(0, N - 1)], "balanced")
        np.testing.assert_array_equal(out.cpu().numpy(), want)
    assert eng.rows_device(5, 4, out.data_ptr(), N) == 0  # no rows


def test_rows_reject_ms_and_bad_ranges(cs):
    from csharp_b200.lib import SwError
    import torch
    z = load_npz("ms_restated.npz")
    N = len(z["offsets"]) - 1
    out = torch.zeros((N, N), dtype=torch.int16, device="cuda")
    ms = _golden_engine(cs, z, mode=1)
    with pytest.raises(ValueError):
        ms.rows_device(0, N - 1, out.data_ptr(), N)
    mpi = _golden_engine(cs, load_npz("mpi_p1.npz"))
    with pytest.raises(SwError):
        mpi.rows_device(0, 10 ** 6, out.data_ptr(), N)


def test_sequence_validation(cs):
    from csharp_b200.lib import SwError
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4)
    with pytest.raises(SwError):
        eng.upload([b"ACGT", bytes([200, 65])])  # byte outside the 127-entry table
    with pytest.raises(SwError):
        eng.compute_block(0, 1, 0, 1, True)  # nothing uploaded
    eng.upload([b"ACGT", b"ACG"])
    with pytest.raises(SwError):
        eng.compute_block(0, 5, 0, 1, False)  # block outside the set
    with pytest.raises(SwError):
        eng.compute_block(0, 1, 1, 1, True)  # diagonal block must be square


def test_running_best_keeps_the_first_maximum_cell(cs):
    """The running best overwrites its own operand (BEST = max(BEST, V)); its 'keep' decision
    must still see the old value, or every pair reports the counters of the wrong cell."""
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4)
    # pairs whose best local alignment is long and partial: distance well inside (0, 32767)
    seqs = [b"ACGTACGTTTGCAACGTAGGCTA" * 3, b"TTACGTACGTTTGCAACGAAGGCTATT" * 2, b"GGGGACGTACGATTGCAACG"]
    eng.upload(seqs)
    full, _, _ = eng.all_pairs(1)
    for i in range(3):
        for j in range(i):
            r = eng.align(seqs[i], seqs[j])
            assert full[i, j] == r.Distance and 0 < r.Distance < 32767, (i, j, full[i, j], r)


def test_engine_accounts_for_every_pair(cs):
    from csharp_b200 import synth
    rng = np.random.default_rng(8)
    seqs = [s.tobytes() for s in synth.dna_family(90, 4, rng.integers(30, 900, 90), seed=21)]
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    _, pairs, _ = eng.all_pairs(1)
    assert eng.query("items") == eng.query("planned_items") > 0
    assert eng.query("lane16_pairs") + eng.rerun_count() == pairs
    assert eng.query("kernel_error") == 0  # no work item or pair outside the plan's bounds
    # the self-check word is per launch: a device-output job leaves it readable too
    import torch
    out = torch.zeros((len(seqs), len(seqs)), dtype=torch.int16, device="cuda")
    eng.set_option("two_pass", 0)
    eng.all_pairs_device(out.data_ptr(), len(seqs), 3)
    eng.synchronize()
    assert eng.query("kernel_error") == 0 and eng.query("lane16_pairs") + eng.rerun_count() == pairs


def test_protein_engine_uses_16bit_lanes_and_matches_oracle(cs, oracle_mod):
    """20-letter alphabet: two-plane profiles in the 16-bit lanes; a 2,500-residue query whose
    profile exceeds shared memory goes to 32-bit lanes.  Every pair against the oracle."""
    from csharp_b200 import synth
    sc = cs.ScoringMatrix.Load("BLOSUM62").Scores
    rng = np.random.default_rng(44)
    lens = np.concatenate([rng.integers(100, 1001, 70), [0, 1, 2500]])
    seqs = [s.tobytes() for s in synth.protein_family(len(lens), 6, lens, 44, sc)]
    eng = cs.Engine(cs.ScoringMatrix.Load("BLOSUM62"), 10, 1, alignment_type=0).upload(seqs)
    full, pairs, _ = eng.all_pairs(1)
    assert eng.query("alphabet") > 8 and eng.query("lane16_pairs") > 0
    assert eng.rerun_count() >= len(seqs) - 1  # the long query's pairs (it is s1 of every pair j < i)
    N = len(seqs)
    pr = np.array([(i, j) for i in range(N) for j in range(i)], dtype=np.int32)
    want = _oracle_distances(oracle_mod, seqs, pr, "BLOSUM62", 10.0, 1.0, atype=0)
    np.testing.assert_array_equal(full[pr[:, 0], pr[:, 1]], want)


@pytest.mark.parametrize("matrix,o,e,atype", [("EDNAFULL", 16, 4, 1), ("BLOSUM62", 10, 1, 0)])
def test_nw_engine_matches_plain_kernel(cs, matrix, o, e, atype):
    """NW on the 16-bit lanes (every rows-per-lane bin, multi-pass queries, empty and 1-residue
    sequences) equals the 32-bit plain kernel, which the NW restatement fixtures pin."""
    from csharp_b200 import synth
    rng = np.random.default_rng(61)
    lens = np.concatenate([rng.integers(1, 900, 110), [0, 1, 1, 1400]])
    if atype == 1:
        seqs = [s.tobytes() for s in synth.dna_family(len(lens), 5, lens, seed=61)]
    else:
        seqs = [s.tobytes() for s in synth.protein_family(len(lens), 5, lens, 61, cs.ScoringMatrix.Load(matrix).Scores)]
    eng = cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=cs.NW, alignment_type=atype).upload(seqs)
    full, pairs, _ = eng.all_pairs(1)
    # all but the 1,400-residue protein query's pairs (its profile exceeds shared memory)
    assert eng.query("lane16_pairs") + eng.rerun_count() == pairs
    assert eng.query("lane16_pairs") >= pairs - (len(seqs) if atype == 0 else 0)
    ref = cs.Engine(cs.ScoringMatrix.Load(matrix), o, e, mode=cs.NW, alignment_type=atype, lanes=32).upload(seqs)
    want, _, _ = ref.all_pairs(1)
    np.testing.assert_array_equal(full, want)
    for k in (4, 10, 16):  # forced rows per lane
        eng.set_option("rows_per_lane", k)
        got, _, _ = eng.all_pairs(3)
        want3, _, _ = ref.all_pairs(3)
        np.testing.assert_array_equal(got, want3)


@pytest.mark.parametrize("name", ["mpi_kimura_p3.npz", "mpi_jc_p1.npz"])
def test_kimura_and_jukes_cantor_match_reference_driver(cs, name):
    """Kimura2 / JukesCantor distances of the reference's own block driver (Alignment.cs:254-348)."""
    z = load_npz(name)
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), float(z["o"]), float(z["e"]),
                    distance_fn=int(z["dist_fn"]))
    eng.upload(concat=z["concat"], offsets=z["offsets"])
    full, pairs, _ = eng.all_pairs(int(z["ranks"]))
    assert pairs == int(z["pairs"])
    np.testing.assert_array_equal(full, z["distances"])
    N = len(z["offsets"]) - 1
    blk, _ = eng.compute_block(0, N - 1, 0, N - 1, True)
    off = ~np.eye(N, dtype=bool)
    if int(z["ranks"]) == 1:
        np.testing.assert_array_equal(blk[off], z["distances"][off])


@pytest.mark.parametrize("name", ["ms_kimura_restated.npz", "ms_jc_restated.npz"])
def test_ms_kimura_and_jukes_cantor_match_restatement(cs, name):
    z = load_npz(name)
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), float(z["o"]), float(z["e"]), mode=cs.SWG_MS,
                    distance_fn=int(z["dist_fn"]))
    eng.upload(concat=z["concat"], offsets=z["offsets"])
    full, _, _ = eng.all_pairs(1)
    np.testing.assert_array_equal(full, z["distances"])


def test_kimura_single_pair_matches_reference_kats(cs, kats):
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4, distance_fn=cs.KIMURA2)
    n = 0
    for k in kats:
        if k["matrix"] != "EDNAFULL" or k.get("kimura2") is None or (k["o"], k["e"]) != (16, 4):
            continue
        assert eng.align(k["s1"], k["s2"]).Distance == k["kimura2"], k
        n += 1
    assert n > 50


@pytest.mark.parametrize("dist_fn,mode", [(1, 0), (2, 0), (1, 1), (2, 1)])
def test_kimura_and_jukes_cantor_against_oracle(cs, oracle_mod, dist_fn, mode):
    """Uneven lengths up to 700 and multi-strip pairs: every pair against the oracle."""
    from csharp_b200 import synth
    rng = np.random.default_rng(90 + dist_fn)
    lens = np.concatenate([rng.integers(1, 700, 60), [0, 1]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 3, lens, seed=91)]
    sm = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(sm, 16, 4, mode=mode, distance_fn=dist_fn).upload(seqs)
    full, _, _ = eng.all_pairs(1)
    concat, off = cs.pack_sequences(seqs)
    N = len(seqs)
    want, _ = oracle_mod.block(concat, off, 0, N - 1, 0, N - 1, True, mode, sm.Scores[:127, :127].astype(np.float32),
                               16.0, 4.0, 1, dist_fn)
    if mode == 0:
        tri = np.tril(np.ones((N, N), dtype=bool), -1)
        np.testing.assert_array_equal(full[tri], want[tri])
        np.testing.assert_array_equal(full.T[tri], want[tri])
    else:
        np.testing.assert_array_equal(full, want)


@pytest.mark.parametrize("dist_fn,mode", [(1, 0), (2, 1)])
def test_kimura_and_jukes_cantor_16bit_lanes(cs, oracle_mod, dist_fn, mode):
    """Kimura2 / JukesCantor run on the 16-bit kernel with two counter words per state (at most 8
    rows per lane, so queries over 256 residues take several passes): every pair equals the 32-bit
    lanes and the oracle, and the pairs ran on 16-bit lanes."""
    from csharp_b200 import synth
    rng = np.random.default_rng(700 + dist_fn)
    lens = np.concatenate([rng.integers(200, 1400, 44), [0, 1, 255, 256, 257, 513]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 4, lens, seed=701)]
    sm = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(sm, 16, 4, mode=mode, distance_fn=dist_fn).upload(seqs)
    full, pairs, _ = eng.all_pairs(1)
    assert eng.query("kernel_error") == 0
    assert eng.query("lane16_pairs") + eng.rerun_count() == pairs
    assert eng.query("lane16_pairs") >= pairs - len(seqs)
    wide = cs.Engine(sm, 16, 4, mode=mode, distance_fn=dist_fn, lanes=32).upload(seqs)
    full32, pairs32, _ = wide.all_pairs(1)
    assert pairs32 == pairs
    np.testing.assert_array_equal(full, full32)
    for k in (4, 6):  # forced rows per lane
        eng.set_option("rows_per_lane", k)
        got, _, _ = eng.all_pairs(1)
        np.testing.assert_array_equal(got, full32)
    concat, off = cs.pack_sequences(seqs)
    N = len(seqs)
    r0 = N - 16  # the oracle on the last rows (the edge lengths among them)
    want, _ = oracle_mod.block(concat, off, r0, N - 1, 0, N - 1, False, mode,
                               sm.Scores[:127, :127].astype(np.float32), 16.0, 4.0, 1, dist_fn)
    for q in range(r0, N):
        cols = [d for d in range(N) if mode == 1 or d < q]
        np.testing.assert_array_equal(full[q, cols], want[q - r0, cols])


def test_jukes_cantor_log_zero_is_reported(cs, oracle_mod):
    """A matrix whose mismatches score above zero aligns AAAA with CCCC: 1 - 4/3 < 0, where
    SWG-MPI's JukesCantor throws (SW_E_THROWS) and SWG-MS gives 10."""
    txt = "   A C\nA 1 2\nC 2 1\n"
    m = cs.ScoringMatrix.Parse(txt, "POSMISMATCH")
    seqs = [b"AAAA", b"CCCC"]
    eng = cs.Engine(m, 16, 4, distance_fn=cs.JUKES_CANTOR).upload(seqs)
    with pytest.raises(cs.SwError) as ex:
        eng.all_pairs(1)
    assert ex.value.status == 8
    with pytest.raises(cs.SwError):
        eng.compute_block(0, 1, 0, 1, True)
    ms = cs.Engine(m, 16, 4, mode=cs.SWG_MS, distance_fn=cs.JUKES_CANTOR).upload(seqs)
    full, _, _ = ms.all_pairs(1)
    concat, off = cs.pack_sequences(seqs)
    want, _ = oracle_mod.block(concat, off, 0, 1, 0, 1, False, 1, m.Scores[:127, :127].astype(np.float32), 16.0, 4.0, 1, 2)
    np.testing.assert_array_equal(full, want)
    assert full[1, 0] == -10  # (short)(int)(10 * 32767): 327670 keeps its low 16 bits


def test_autotune_installs_weights_and_changes_no_result(cs):
    import torch
    z = load_npz("mpi_p3.npz")
    eng = _golden_engine(cs, z)
    N = len(z["offsets"]) - 1
    d = torch.zeros((N, N), dtype=torch.int16, device="cuda")
    w = eng.autotune(d.data_ptr(), N)
    installed = [v for v in w.values() if v]  # all 0: the built-in costs were kept
    assert not installed or min(installed) == 100
    full, _, _ = eng.all_pairs(3)
    np.testing.assert_array_equal(full, z["distances"])


def test_two_pass_equals_one_pass_and_oracle(cs, oracle_mod):
    """Score-only first pass + box kernel against the counter engine and the oracle, with
    close family members (long alignments: boxes beyond the budget go to 32-bit lanes),
    multi-pass queries, empty and 1-residue sequences."""
    from csharp_b200 import synth
    rng = np.random.default_rng(77)
    lens = np.concatenate([rng.integers(20, 1400, 140), [0, 1, 2]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 3, lens, seed=78, sub_range=(0.0, 0.05),
                                                  indel_range=(0.0, 0.05))]
    seqs += [s.tobytes() for s in synth.dna_family(60, 30, rng.integers(50, 600, 60), seed=79)]
    one = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    one.set_option("two_pass", 0)
    want, pairs, _ = one.all_pairs(1)
    two = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    got, pairs2, _ = two.all_pairs(1)
    assert pairs2 == pairs
    assert two.query("box_fallbacks") > 0  # the near-identical family members
    assert two.query("lane16_pairs") + two.rerun_count() == pairs
    np.testing.assert_array_equal(got, want)
    other = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    other.set_option("box_reg", 0)  # every box by the warp kernel
    got_o, _, _ = other.all_pairs(1)
    np.testing.assert_array_equal(got_o, want)
    other.close()
    N = len(seqs)
    sel = rng.choice(N * (N - 1) // 2, 3000, replace=False)
    pr = np.array([(i, j) for i in range(N) for j in range(i)], dtype=np.int32)[sel]
    ref = _oracle_distances(oracle_mod, seqs, pr, "EDNAFULL", 16.0, 4.0)
    np.testing.assert_array_equal(got[pr[:, 0], pr[:, 1]], ref)
    got3, _, _ = two.all_pairs(3)
    want3, _, _ = one.all_pairs(3)
    np.testing.assert_array_equal(got3, want3)


@pytest.mark.parametrize("third", [1, 0])
def test_two_pass_with_most_pairs_falling_back(cs, third):
    """Cheap gaps and close relatives: the box step gives up on most pairs; the third pass (the
    one-pass 16-bit counter kernel over them, grouped by query) or the 32-bit lanes, whose list
    must then hold them all (an overflow would raise in rerun_count), redo them."""
    from csharp_b200 import synth
    rng = np.random.default_rng(5)
    seqs = [s.tobytes() for s in synth.dna_family(90, 2, rng.integers(200, 700, 90), seed=6, sub_range=(0.0, 0.03),
                                                  indel_range=(0.0, 0.03))]
    one = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 3, 2).upload(seqs)
    one.set_option("two_pass", 0)
    want, pairs, _ = one.all_pairs(1)
    two = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 3, 2).upload(seqs)
    two.set_option("two_pass", 2)  # two passes although the default rule keeps 3/2 on one
    two.set_option("third_pass", third)
    got, _, _ = two.all_pairs(1)
    assert two.query("box_fallbacks") > pairs // 2
    if third:
        assert two.query("box_third_pass") == two.query("box_fallbacks")
        assert two.query("launches") >= 12
    else:
        assert two.query("box_third_pass") == 0
    assert two.query("lane16_pairs") + two.rerun_count() == pairs
    np.testing.assert_array_equal(got, want)
    # a block plan (rows 30..89 against columns 0..29) and a 3-rank checkerboard job
    two.set_option("block_engine", 2)
    blk, _ = two.compute_block(30, 89, 0, 29, False)
    np.testing.assert_array_equal(blk, want[30:90, 0:30])
    got3, _, _ = two.all_pairs(3)
    want3, _, _ = one.all_pairs(3)
    np.testing.assert_array_equal(got3, want3)


@pytest.mark.parametrize("o,e", [(16, 4), (10, 3), (20, 8), (4, 2)])
def test_register_box_step_on_uneven_lengths(cs, oracle_mod, o, e):
    """Lognormal lengths (median 400, sigma 0.6, clipped 50-1500) from 200 family roots, two
    passes forced at every gap setting: the register box step (one pair per thread) finishes
    nearly every pair at 16/4 and 20/8, hands wider regions to the warp box kernel and the rest to
    the 32-bit lanes (most pairs at 10/3 and 4/2).  Every entry equals the one-pass counter
    kernel's, the warp-only box step's and the default choice's; a sample equals the oracle's."""
    from csharp_b200 import synth
    rng = np.random.default_rng(91 + o)
    lens = synth.lognormal_lengths(900, 400, 0.6, 50, 1500, rng)
    seqs = [s.tobytes() for s in synth.dna_family(900, 200, lens, seed=92)]
    m = cs.ScoringMatrix.Load("EDNAFULL")
    res = {}
    for tag, opts in (("one", {"two_pass": 0}), ("warp", {"two_pass": 2, "box_reg": 0}),
                      ("reg", {"two_pass": 2}), ("auto", {})):
        eng = cs.Engine(m, o, e).upload(seqs)
        for k, v in opts.items():
            eng.set_option(k, v)
        res[tag], pairs, _ = eng.all_pairs(1)
        if tag == "reg":
            assert eng.query("lane16_pairs") + eng.rerun_count() == pairs
            assert eng.query("launches") >= 8
            if (o, e) in ((16, 4), (20, 8)):
                assert eng.query("box_spilled") + eng.query("box_fallbacks") < 0.03 * pairs
        eng.close()
    np.testing.assert_array_equal(res["reg"], res["one"])
    np.testing.assert_array_equal(res["warp"], res["one"])
    np.testing.assert_array_equal(res["auto"], res["one"])
    N = len(seqs)
    ii = rng.integers(1, N, 1500)
    jj = (rng.random(1500) * ii).astype(np.int64)
    pr = np.stack([ii, jj], 1).astype(np.int32)
    ref = _oracle_distances(oracle_mod, seqs, pr, "EDNAFULL", float(o), float(e))
    np.testing.assert_array_equal(res["reg"][pr[:, 0], pr[:, 1]], ref)


def test_reupload_of_same_shaped_set_keeps_plans_and_uses_new_residues(cs):
    """A second upload with the same lengths and letters keeps the engine's plans and graphs but
    must align the new residues: every result equals a fresh engine's on the new set."""
    from csharp_b200 import synth
    rng = np.random.default_rng(12)
    lens = synth.lognormal_lengths(300, 300, 0.6, 30, 900, rng)
    a = [s.tobytes() for s in synth.dna_family(300, 30, lens, seed=1)]
    b = [s.tobytes() for s in synth.dna_family(300, 30, lens, seed=2)]
    m = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(m, 16, 4).upload(a)
    got_a, _, _ = eng.all_pairs(3)
    blk_a, _ = eng.compute_block(0, 149, 0, 149, True)
    eng.upload(b)
    got_b, _, _ = eng.all_pairs(3)
    blk_b, _ = eng.compute_block(0, 149, 0, 149, True)
    fresh = cs.Engine(m, 16, 4).upload(b)
    want_b, _, _ = fresh.all_pairs(3)
    np.testing.assert_array_equal(got_b, want_b)
    want_blk, _ = fresh.compute_block(0, 149, 0, 149, True)  # s1 = the larger index, like the call above
    off = ~np.eye(150, dtype=bool)
    np.testing.assert_array_equal(blk_b[off], want_blk[off])
    assert not np.array_equal(got_a, got_b)
    eng.close()
    fresh.close()


def _self_score(seq, scores):
    return int(sum(int(scores[c, c]) for c in seq))


@pytest.mark.parametrize("dist_fn", [1, 2, 3])
def test_nw_kimura_jukes_cantor_minmax_against_oracle(cs, oracle_mod, dist_fn):
    """NW with Kimura2, JukesCantor (capped at 10, NW Program.cs:606-719) and MinMaxNormScore
    (:573-581) on the 32-bit lanes: every pair against the oracle's NW alignment (exact Int16)."""
    from csharp_b200 import synth
    rng = np.random.default_rng(50 + dist_fn)
    lens = np.concatenate([rng.integers(1, 300, 36), [0, 1]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 3, lens, seed=51)]
    sm = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(sm, 16, 4, mode=cs.NW, distance_fn=dist_fn).upload(seqs)
    full, _, _ = eng.all_pairs(1)
    sc = sm.Scores[:127, :127].astype(np.float32)
    N = len(seqs)
    for i in range(N):
        for j in range(i):
            a = oracle_mod.nw_align(seqs[i], seqs[j], sc, 16.0, 4.0)
            if dist_fn == 3:
                want = oracle_mod.minmax_distance_i16(int(a["score"]), _self_score(seqs[i], sm.Scores),
                                                      _self_score(seqs[j], sm.Scores), len(seqs[i]), len(seqs[j]),
                                                      16, 4, 2)
            else:
                want = oracle_mod.ms_distance_i16(a["aln1"], a["aln2"], sc, False, dist_fn)
            assert full[i, j] == want and full[j, i] == want, (i, j, dist_fn)
    eng.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_minmax_norm_score_smith_waterman(cs, oracle_mod, mode):
    """MinMaxNormScore in SWG-MS (score over the larger self score) and in SWG-MPI, whose
    ComputeDistance has no case for it (every distance 0); also through the single-pair call."""
    from csharp_b200 import synth
    rng = np.random.default_rng(60 + mode)
    lens = np.concatenate([rng.integers(1, 400, 40), [0, 1]])
    seqs = [s.tobytes() for s in synth.dna_family(len(lens), 4, lens, seed=61)]
    sm = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(sm, 16, 4, mode=mode, distance_fn=cs.MIN_MAX_NORM_SCORE).upload(seqs)
    full, _, _ = eng.all_pairs(1)
    sc = sm.Scores[:127, :127].astype(np.float32)
    N = len(seqs)
    for i in range(N):
        for j in range(N):
            if mode == 0 and j >= i:
                continue
            if mode == 0:
                want = 0
            else:
                a = oracle_mod.align(seqs[i], seqs[j], sc, 16.0, 4.0)
                s = 0 if not (len(seqs[i]) and len(seqs[j])) else int(a["score"])
                want = oracle_mod.minmax_distance_i16(s, _self_score(seqs[i], sm.Scores), _self_score(seqs[j], sm.Scores),
                                                      len(seqs[i]), len(seqs[j]), 16, 4, 1)
            assert full[i, j] == want, (i, j)
    if mode == 1:
        for i, j in [(3, 5), (0, 40), (7, 7)]:
            assert eng.align(seqs[i], seqs[j]).Distance == full[i, j]
    eng.close()


def test_ms_block_files_from_the_engine_match_the_oracle_run(cs, oracle_mod, tmp_path):
    """SWG-MS driver with the engine as block handler: every block file equals, byte for byte, the
    file a run with the oracle's block handler writes."""
    from csharp_b200 import synth
    from csharp_b200.msdriver import MSBlockRun, engine_handler
    rng = np.random.default_rng(81)
    N, W = 90, 4
    seqs = [s.tobytes() for s in synth.dna_family(N, 5, rng.integers(1, 400, N), seed=82)]
    ids = [f"s{k}" for k in range(N)]
    m = cs.ScoringMatrix.Load("EDNAFULL")
    eng = cs.Engine(m, 16, 4, mode=cs.SWG_MS).upload(seqs)
    eng.set_option("block_engine", 2)
    concat, off = cs.pack_sequences(seqs)
    sc = m.Scores[:127, :127].astype(np.float32)

    def oracle_handler(block, pm, diag, rank):
        rr, cr = block.RowRange, block.ColumnRange
        vals, n = oracle_mod.block(concat, off, rr.StartIndex, rr.EndIndex, cr.StartIndex, cr.EndIndex, diag, 1, sc, 16.0, 4.0)
        pm.block_view(block)[...] = vals
        return n
    for tag, h in (("gpu", engine_handler(eng)), ("cpu", oracle_handler)):
        d = tmp_path / tag
        d.mkdir()
        for r in range(W):
            MSBlockRun(N, h, r, W, str(d), 1, ids).Compute()
    a, b = tmp_path / "gpu", tmp_path / "cpu"
    names = sorted(os.listdir(b))
    assert sorted(os.listdir(a)) == names and names
    for f in names:
        assert (a / f).read_bytes() == (b / f).read_bytes(), f
    eng.close()


@pytest.mark.parametrize("mode,matrix,o,e,dist_fn", [(0, "EDNAFULL", 16, 4, 0), (1, "EDNAFULL", 16, 4, 0),
                                                     (2, "EDNAFULL", 16, 4, 0), (0, "BLOSUM62", 10, 1, 0),
                                                     (2, "BLOSUM62", 10, 1, 0), (0, "EDNAFULL", 5, 2, 1),
                                                     (1, "EDNAFULL", 16, 4, 3), (2, "EDNAFULL", 16, 4, 3)])
def test_alignment_strings_match_oracle_traceback(cs, oracle_mod, mode, matrix, o, e, dist_fn):
    """sw_align_strings against the oracle's traceback (SW: the NAligner restatement, NW: the NW
    restatement): the aligned strings, the counts and the context's distance (the engine's)."""
    from csharp_b200 import synth
    rng = np.random.default_rng(70 + mode)
    if matrix == "BLOSUM62":
        seqs = [s.tobytes() for s in synth.protein_family(30, 3, rng.integers(1, 250, 30), 71, cs.ScoringMatrix.Load("BLOSUM62").Scores)]
    else:
        seqs = [s.tobytes() for s in synth.dna_family(30, 3, rng.integers(1, 250, 30), seed=71)]
    seqs += [b"A" if matrix == "EDNAFULL" else b"W", b""]
    atype = cs.PROTEIN if matrix == "BLOSUM62" else cs.NUCLEIC
    sm = cs.ScoringMatrix.Load(matrix)
    eng = cs.Engine(sm, o, e, mode=mode, alignment_type=atype, distance_fn=dist_fn).upload(seqs)
    full, _, _ = eng.all_pairs(1)
    N = len(seqs)
    pairs = [(i, j) for i in range(N) for j in range(i)][::3] + [(N - 2, 0), (N - 1, 3), (5, 5)]
    got = eng.align_strings(pairs)
    sc = sm.Scores[:127, :127].astype(np.float32)
    for (i, j), (a, b, aln) in zip(pairs, got):
        if mode == 2:
            want = oracle_mod.nw_align(seqs[i], seqs[j], sc, float(o), float(e))
        else:
            want = oracle_mod.align(seqs[i], seqs[j], sc, float(o), float(e), with_strings=True)
            assert (aln.Identity, aln.Similarity, aln.Gaps, aln.Start1, aln.Start2) == \
                (want["identity"], want["similarity"], want["gaps"], want["start1"], want["start2"])
        assert (a, b) == (want["aln1"], want["aln2"]), (i, j)
        assert aln.Length == len(a)
        if i != j or mode == 1:
            assert aln.Distance == full[i, j], (i, j)
    eng.close()


def test_write_alignments_format(cs, tmp_path):
    from csharp_b200.formats import write_alignments
    seqs = [b"ACGTACGTTTGA", b"ACGTTCGTTGA", b"GGGACGT"]
    eng = cs.Engine(cs.ScoringMatrix.Load("EDNAFULL"), 16, 4).upload(seqs)
    got = eng.align_strings([(1, 0), (2, 1)])
    write_alignments(tmp_path / "a.txt", got, ["s1", "s2"], ["s0", "s1"])
    lines = (tmp_path / "a.txt").read_text().split("\n")
    assert lines[0].startswith(">s1 Kimera: ") and ", JukesCantor: " in lines[0] and ", PercentIdentity: " in lines[0]
    assert lines[1] == got[0][0].decode() and lines[3] == got[0][1].decode() and lines[4] == ""
    eng.close()
