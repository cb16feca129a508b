"""Seeded synthetic sequence sets with the shapes of the five benchmark workloads.

The reference ships no datasets; these generators stand in for its inputs.  Sequences come from
random family roots mutated by substitutions and indels (equal insertions and deletions,
geometric lengths with mean 2), then cut or extended to a target length.

* ``dna_family``     configurations 1-3 and 5 (uniform A/C/G/T roots)
* ``protein_family`` configuration 4: 20 amino acids drawn at background frequencies and
  substituted with BLOSUM62 weights, both derived from BLOSUM62 itself (row-sum normalisation
  of exp(lambda * s) with lambda = ln(2)/2 for the half-bit units), so no external table is used
"""
import numpy as np

DNA = np.frombuffer(b"ACGT", dtype=np.uint8)
AMINO = np.frombuffer(b"ARNDCQEGHILKMFPSTWYV", dtype=np.uint8)


def _mutate(root, p_sub, p_indel, rng, alphabet, sub_cdf=None):
    s = root.copy()
    n = len(s)
    # substitutions
    pos = np.nonzero(rng.random(n) < p_sub)[0]
    if len(pos):
        if sub_cdf is None:
            shift = rng.integers(1, len(alphabet), len(pos))
            s[pos] = (s[pos] + shift) % len(alphabet)
        else:
            u = rng.random(len(pos))
            s[pos] = np.array([np.searchsorted(sub_cdf[a], x) for a, x in zip(s[pos], u)], dtype=s.dtype)
    # indels: events at rate p_indel per position, half insertions, geometric length mean 2
    ev = np.nonzero(rng.random(n) < p_indel)[0]
    if len(ev) == 0:
        return s
    lens = rng.geometric(0.5, len(ev)).tolist()
    ins = (rng.random(len(ev)) < 0.5).tolist()
    # events inside a deletion are dropped; inserted codes are drawn event by event, in order
    pieces, last = [], 0
    for p, ln, isi in zip(ev.tolist(), lens, ins):
        if p < last:
            continue
        pieces.append(s[last:p])
        if isi:
            pieces.append(rng.integers(0, len(alphabet), ln).astype(s.dtype))
            last = p
        else:
            last = min(n, p + ln)
    pieces.append(s[last:n])
    return np.concatenate(pieces)


def _fit(seq, L, rng, alphabet_size):
    if len(seq) >= L:
        a = rng.integers(0, len(seq) - L + 1)
        return seq[a:a + L]
    extra = rng.integers(0, alphabet_size, L - len(seq)).astype(seq.dtype)
    return np.concatenate([seq, extra])


def family_sequences(n, nroots, lengths, rng, alphabet, sub_range, indel_range, root_len=None,
                     sub_cdf=None, background=None):
    A = len(alphabet)
    root_len = root_len or int(max(lengths))
    if background is None:
        roots = rng.integers(0, A, (nroots, root_len))
    else:
        roots = rng.choice(A, size=(nroots, root_len), p=background)
    fam = rng.integers(0, nroots, n)
    out = []
    for k in range(n):
        p_sub = rng.uniform(*sub_range)
        p_indel = rng.uniform(*indel_range)
        root = roots[fam[k]]
        w = min(root_len, int(lengths[k] * 1.1) + 4)  # mutate a window near the target length
        a = rng.integers(0, root_len - w + 1)
        s = _mutate(root[a:a + w], p_sub, p_indel, rng, alphabet, sub_cdf)
        out.append(alphabet[_fit(s, int(lengths[k]), rng, A)])
    return out


def lognormal_lengths(n, median, sigma, lo, hi, rng):
    return np.clip(np.round(np.exp(np.log(median) + sigma * rng.standard_normal(n))), lo, hi).astype(np.int64)


def dna_family(n, nroots, lengths, seed, sub_range=(0.05, 0.25), indel_range=(0.05, 0.25), root_len=None):
    rng = np.random.default_rng(seed)
    lengths = np.asarray(lengths)
    return family_sequences(n, nroots, lengths, rng, DNA, sub_range, indel_range, root_len)


def blosum62_background(scores):
    """Background frequencies and substitution CDFs from BLOSUM62 (half-bit units)."""
    lam = np.log(2.0) / 2.0
    idx = AMINO.astype(np.int64)
    S = scores[np.ix_(idx, idx)].astype(np.float64)
    W = np.exp(lam * S)
    bg = W.sum(1)
    bg /= bg.sum()
    Wo = W.copy()
    np.fill_diagonal(Wo, 0.0)
    cdf = np.cumsum(Wo / Wo.sum(1, keepdims=True), axis=1)
    cdf[:, -1] = 1.0
    return bg, cdf


def protein_family(n, nroots, lengths, seed, scores, sub_range=(0.10, 0.40), indel_range=(0.02, 0.10)):
    rng = np.random.default_rng(seed)
    bg, cdf = blosum62_background(scores)
    return family_sequences(n, nroots, np.asarray(lengths), rng, AMINO, sub_range, indel_range,
                            sub_cdf=cdf, background=bg)


# ---- the five workloads -----------------------------------------------------------------------
def config1(n=1000, seed=1):
    """Plain SWG: 1,000 DNA, 20 roots of 500 nt, lengths clipped to 200-600."""
    rng = np.random.default_rng(seed + 1000)
    lengths = np.clip(np.round(rng.normal(500, 60, n)), 200, 600).astype(np.int64)
    return dna_family(n, 20, lengths, seed, root_len=500)


def config2(n=10000, seed=2):
    """NW: 10,000 DNA, lengths uniform 300-500, 100 roots."""
    rng = np.random.default_rng(seed + 1000)
    return dna_family(n, 100, rng.integers(300, 501, n), seed)


def config3(n=20000, seed=3):
    """Batched uneven SWG: 20,000 DNA, lognormal(median 400, sigma 0.6) clipped 50-1500, 200 roots."""
    rng = np.random.default_rng(seed + 1000)
    return dna_family(n, 200, lognormal_lengths(n, 400, 0.6, 50, 1500, rng), seed)


def config4(scores, n=20000, seed=4):
    """Protein SWG: 20,000 sequences over 20 amino acids, lengths uniform 100-1000, 500 roots."""
    rng = np.random.default_rng(seed + 1000)
    return protein_family(n, 500, rng.integers(100, 1001, n), seed, scores)


def config5_db(n=100000, seed=5):
    """Serving database: 100,000 DNA, lognormal(median 500, sigma 0.6) clipped 50-2000."""
    rng = np.random.default_rng(seed + 1000)
    return dna_family(n, 1000, lognormal_lengths(n, 500, 0.6, 50, 2000, rng), seed)
