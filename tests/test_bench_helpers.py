"""Host-side logic of bench.py, without a GPU: the 8-rank share partition and its blocks, the
pairs each configuration's parity check covers, and the end-to-end leg's split of the job among
ranks with its byte accounting (driven by a stand-in engine that records the block-handler calls).
"""
import numpy as np
import pytest
import torch

import bench


@pytest.fixture
def lens():
    rng = np.random.default_rng(3)
    return rng.integers(5, 60, 137)


def test_share_blocks_cover_each_pair_once(lens):
    """The 8 shares' blocks (the reference driver's checkerboard, Program.cs:618-642) cover every
    unordered pair exactly once, and checkerboard_share_cells adds up their DP cells."""
    n = len(lens)
    seen = np.zeros((n, n), dtype=np.int32)
    total = 0
    for s in range(bench.SHARES):
        cells = 0
        for rs, re_, cs_, ce, diag in bench.share_blocks(n, s):
            blk = np.zeros((n, n), dtype=bool)
            blk[rs:re_ + 1, cs_:ce + 1] = True
            if diag:
                blk &= np.tril(np.ones((n, n), dtype=bool), -1)
            seen += blk
            cells += int((lens[:, None] * lens[None, :])[blk].sum())
        assert cells == bench.checkerboard_share_cells(lens, s)
        total += cells
    pairs = seen + seen.T
    assert (pairs[~np.eye(n, dtype=bool)] == 1).all()
    assert (np.diag(pairs) == 0).all()
    assert total == int((np.triu(lens[:, None] * lens[None, :], 1)).sum())


def test_parity_pairs_are_oriented_and_cfg1_is_complete():
    ii, jj = bench.config_parity_pairs(50, "cfg1", np.random.default_rng(0))
    assert len(ii) == 50 * 49 // 2 and (ii > jj).all()
    assert len({(int(a), int(b)) for a, b in zip(ii, jj)}) == len(ii)
    ii, jj = bench.config_parity_pairs(1000, "cfg1_kimura2", np.random.default_rng(0))
    assert len(ii) == bench.PARITY_SAMPLE and (ii > jj).all() and (jj >= 0).all() and (ii < 1000).all()


class _Engine:
    """Stands in for csharp_b200.Engine: records uploads and block-handler calls."""

    def __init__(self):
        self.calls, self.uploads, self.plan_only = [], 0, 0

    def set_option(self, key, value):
        if key == "plan_only":
            self.plan_only = value

    def upload(self, concat=None, offsets=None):
        self.uploads += 1

    def compute_block(self, rs, re_, cs_, ce, diag, out=None):
        assert out.shape == (re_ - rs + 1, ce - cs_ + 1)
        self.calls.append((self.plan_only, rs, re_, cs_, ce, diag))


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_e2e_shares_split_the_job(world):
    got = [bench.e2e_shares(r, world) for r in range(world)]
    assert sorted(s for g in got for s in g) == list(range(bench.SHARES))
    assert max(map(len, got)) - min(map(len, got)) <= 1


def test_e2e_leg_plans_then_times_every_share(lens, monkeypatch):
    """One GPU: every block planned before timing, one untimed share, then the 8 shares through
    the block handler, each after a fresh upload; bytes per share counted from what is copied."""
    monkeypatch.setattr(torch.Tensor, "pin_memory", lambda self: self)  # no CUDA host allocator here
    n = len(lens)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    concat = np.zeros(int(off[-1]), dtype=np.uint8)
    eng = _Engine()
    r = bench.e2e_leg(None, eng, concat, off, lens, n, 0, 1)
    want = [b for s in range(bench.SHARES) for b in bench.share_blocks(n, s)]
    planned = [c[1:] for c in eng.calls if c[0] == 1]
    run = [c[1:] for c in eng.calls if c[0] == 0]
    assert planned == want
    assert run == list(bench.share_blocks(n, 0)) + want
    assert eng.uploads == bench.SHARES + 1
    assert r["h2d_bytes_per_step"] == concat.nbytes + off.nbytes
    d2h = sum((re_ - rs + 1) * (ce - cs_ + 1) * 2 for rs, re_, cs_, ce, _ in want)
    assert r["d2h_bytes_per_step"] == d2h // bench.SHARES
    assert r["unit"] == "GCUPS" and r["value"] > 0
