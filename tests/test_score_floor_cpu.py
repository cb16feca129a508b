"""The score pass floors the gap states at zero, G' = max(VO_up, G'_up - e, 0) and likewise H', and
takes V = max(F, G', H') with no floor of its own (swg_engine.cu, score_two).  Every V -- hence
every row's best and the first column reaching it, which are all the pass reports -- must equal
the reference's V = max(F, G, H, 0) (SmithWatermanGotoh.cs:154-190).  A scalar restatement of
both recurrences on random sequences, tie-heavy alphabets and cheap gaps included.
"""
import numpy as np
import pytest

NEG = -(1 << 30)


def _score_dp(a, b, S, o, e, floored):
    m, n = len(a), len(b)
    V = np.zeros((m + 1, n + 1), dtype=np.int64)
    G = np.full(n + 1, NEG, dtype=np.int64)  # per column: the gap state of the row above
    for i in range(1, m + 1):
        h = NEG
        for j in range(1, n + 1):
            f = V[i - 1, j - 1] + S[a[i - 1], b[j - 1]]
            g = max(V[i - 1, j] - o, G[j] - e)
            hh = max(V[i, j - 1] - o, h - e)
            if floored:
                g, hh = max(g, 0), max(hh, 0)
                v = max(f, g, hh)
            else:
                v = max(f, g, hh, 0)
            G[j], h = g, hh
            V[i, j] = v
    return V


@pytest.mark.parametrize("alphabet,o,e", [(4, 16, 4), (2, 3, 1), (4, 5, 2), (20, 10, 1), (2, 2, 2)])
def test_floored_gap_states_give_the_same_v(alphabet, o, e):
    rng = np.random.default_rng(100 + alphabet * 7 + o)
    S = rng.integers(-6, 7, (alphabet, alphabet))
    S = (S + S.T) // 2
    np.fill_diagonal(S, rng.integers(1, 8, alphabet))
    for _ in range(40):
        m, n = (int(x) for x in rng.integers(0, 40, 2))
        a, b = rng.integers(0, alphabet, m), rng.integers(0, alphabet, n)
        ref = _score_dp(a, b, S, o, e, floored=False)
        got = _score_dp(a, b, S, o, e, floored=True)
        np.testing.assert_array_equal(got, ref)
        if m and n:
            # the pass's outputs: per row the best V and its first column, per pair the first max
            np.testing.assert_array_equal(got[1:, 1:].max(axis=1), ref[1:, 1:].max(axis=1))
            np.testing.assert_array_equal(got[1:, 1:].argmax(axis=1), ref[1:, 1:].argmax(axis=1))
