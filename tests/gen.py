"""Seeded synthetic inputs shaped like the benchmark configurations.

Test infrastructure.  Every generator takes an explicit seed (numpy PCG64),
so a case is reproducible from its parameters alone.  Shapes follow the five
all-pairs workloads: dense Bernoulli bitmaps, Zipf-sized sparse sets over
2^24, run-clustered rows over 2^26, haplotype-like 1/k carrier blocks and
density sweeps -- at sizes the CPU oracle finishes in seconds.
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def n_words(m: int) -> int:
    return (m + 63) // 64


def pack_bool_rows(bits: np.ndarray) -> np.ndarray:
    """[n, m] bool -> [n, ceil(m/64)] u64, bit b of a row = word b//64, bit b%64."""
    n, m = bits.shape
    w = n_words(m)
    padded = np.zeros((n, w * 64), dtype=np.uint8)
    padded[:, :m] = bits
    by = np.packbits(padded.reshape(n, w * 8, 8), axis=-1, bitorder="little").reshape(n, w * 8)
    return np.ascontiguousarray(by).view(np.uint64).reshape(n, w)


def bernoulli_rows(n: int, m: int, p, seed: int) -> np.ndarray:
    """Packed rows with iid Bernoulli(p) bits; p is a float or a (lo, hi) range drawn per row."""
    g = rng(seed)
    if isinstance(p, tuple):
        pr = g.uniform(p[0], p[1], size=(n, 1))
    else:
        pr = np.full((n, 1), float(p))
    bits = g.random((n, m), dtype=np.float32) < pr
    return pack_bool_rows(bits)


def rows_to_sets(words: np.ndarray, m: int):
    """Packed rows -> list of sorted u32 position arrays."""
    n, w = words.shape
    by = words.view(np.uint8).reshape(n, w * 8)
    bits = np.unpackbits(by, axis=1, bitorder="little")[:, :m]
    return [np.flatnonzero(bits[r]).astype(np.uint32) for r in range(n)]


def sets_to_rows(sets, m: int) -> np.ndarray:
    w = n_words(m)
    out = np.zeros((len(sets), w), dtype=np.uint64)
    for r, s in enumerate(sets):
        s = np.asarray(s, dtype=np.uint64)
        if s.size:
            np.bitwise_or.at(out[r], (s >> np.uint64(6)).astype(np.int64),
                             np.left_shift(np.uint64(1), s & np.uint64(63)))
    return out


def to_csr(sets):
    offs = np.zeros(len(sets) + 1, dtype=np.uint64)
    for r, s in enumerate(sets):
        offs[r + 1] = offs[r] + len(s)
    vals = np.concatenate([np.asarray(s, dtype=np.uint32) for s in sets]) if sets else np.zeros(0, np.uint32)
    return np.ascontiguousarray(vals, dtype=np.uint32), offs


def from_csr(vals, offs):
    return [vals[int(offs[r]):int(offs[r + 1])] for r in range(len(offs) - 1)]


def uniform_set(g, card: int, universe: int) -> np.ndarray:
    """`card` distinct positions uniform over [0, universe), sorted."""
    card = min(int(card), universe)
    if card * 4 > universe:
        return np.flatnonzero(g.permutation(universe) < card).astype(np.uint32)
    out = np.unique(g.integers(0, universe, size=int(card * 1.3) + 8, dtype=np.uint64))
    while out.size < card:
        out = np.unique(np.concatenate([out, g.integers(0, universe, size=card, dtype=np.uint64)]))
    return np.sort(g.choice(out, size=card, replace=False)).astype(np.uint32)


def zipf_sets(n: int, universe: int, s: float, lo: int, hi: int, seed: int):
    """Mixed-density sets: cardinality P(k) ~ k^-s on [lo, hi], elements uniform."""
    g = rng(seed)
    ks = np.arange(lo, hi + 1, dtype=np.float64)
    pk = ks ** (-s)
    pk /= pk.sum()
    cards = g.choice(ks.astype(np.int64), size=n, p=pk)
    return [uniform_set(g, int(c), universe) for c in cards]


def run_sets(n: int, universe: int, mean_runs: float, mean_len: float, seed: int):
    """Run-clustered rows: Poisson(mean_runs) runs, start uniform, length Geometric(mean_len)."""
    g = rng(seed)
    out = []
    for _ in range(n):
        k = g.poisson(mean_runs)
        starts = g.integers(0, universe, size=k)
        lens = g.geometric(1.0 / mean_len, size=k)
        bits = np.zeros(0, dtype=np.int64)
        if k:
            pieces = [np.arange(s, min(s + l, universe)) for s, l in zip(starts, lens)]
            bits = np.unique(np.concatenate(pieces)) if pieces else bits
        out.append(bits.astype(np.uint32))
    return out


def haplotype_sets(n_sites: int, n_hap: int, block: int, seed: int):
    """Rows = sites, columns = haplotypes; allele count k ~ 1/k on [1, n_hap-1];
    carriers chosen as whole contiguous haplotype blocks of `block`."""
    g = rng(seed)
    ks = np.arange(1, n_hap, dtype=np.float64)
    pk = 1.0 / ks
    pk /= pk.sum()
    n_blocks = (n_hap + block - 1) // block
    out = []
    for k in g.choice(ks.astype(np.int64), size=n_sites, p=pk):
        nb = max(1, min(n_blocks, int(np.ceil(k / block))))
        blocks = np.sort(g.choice(n_blocks, size=nb, replace=False))
        pos = (blocks[:, None] * block + np.arange(block)[None, :]).ravel()
        pos = pos[pos < n_hap]
        out.append(np.sort(pos[: int(k)]).astype(np.uint32) if pos.size > k else pos.astype(np.uint32))
    return out


def bernoulli_sets(n: int, universe: int, density: float, seed: int):
    g = rng(seed)
    cards = g.binomial(universe, density, size=n)
    return [uniform_set(g, int(c), universe) for c in cards]


def repeat_corpus(seed: int):
    """Rows whose list chunks repeat values (STORM_add keeps repeats), rows
    whose single chunk is given out of order, plain rows and bitmap-chunk
    rows beside them."""
    g = rng(seed)
    sets = []
    for k in range(50):
        kind = k % 4 if k < 46 else 4
        if kind == 0:      # sorted with many repeats, spread over three chunks
            v = np.sort(g.integers(0, 3 << 16, int(g.integers(100, 3000))))
        elif kind == 1:    # plain: sorted distinct
            v = uniform_set(g, int(g.integers(50, 3000)), 3 << 16)
        elif kind == 2:    # one chunk, distinct values out of order
            v = g.permutation(uniform_set(g, int(g.integers(20, 900)), 1 << 16))
        elif kind == 3:    # every value twice, sorted
            v = np.sort(np.repeat(uniform_set(g, int(g.integers(20, 900)), 3 << 16), 2))
        else:              # bitmap chunks (>= 4096 values) that the lists above probe
            v = uniform_set(g, int(g.integers(13000, 30000)), 3 << 16)
        sets.append(np.asarray(v, dtype=np.uint32))
    return sets


def segmentation_rows(u: int, g):
    """Rows over [0, u) that reach each EWAH-64 segmentation case (empty and
    full rows, full words at the first and last word, full runs beside
    literals and zero gaps, partial last words, several densities, runs)."""
    nw = (u + 63) // 64
    full = lambda w: list(range(64 * w, min(64 * w + 64, u)))
    rows = [[], list(range(u)), [0], [u - 1], full(0), full(nw - 1) if u % 64 == 0 else [u - 1, u - 2],
            full(0) + [70, 80] + full(3) + full(4) + [64 * 6 + 1] + full(7)]
    # alternating full words, literals and gaps, at random
    v = []
    for w in range(nw):
        t = g.integers(0, 4)
        if t == 1:
            v += full(w)
        elif t == 2:
            v += sorted(set(int(x) for x in g.integers(64 * w, min(64 * w + 64, u), size=5)))
    rows.append(v)
    # long runs of full words ending in literals and the partial last word
    rows.append(list(range(0, min(u, 64 * 40 + 17))) + list(range(max(0, u - 100), u)))
    for d in (0.0005, 0.02, 0.3, 0.5, 0.9, 0.999):
        rows.append(np.flatnonzero(g.random(u) < d).tolist())
    rows += [x.tolist() for x in run_sets(6, u, 30, 600, int(g.integers(1 << 30)))]
    return [np.array(sorted(set(x for x in r if 0 <= x < u)), np.uint32) for r in rows]
