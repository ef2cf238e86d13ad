"""Seeded synthetic genomes standing in for the reference's real-genome
workloads (none ship with the reference).

Composition: i.i.d. bases at 41% GC (A=T=0.295, C=G=0.205); soft-masked
lowercase runs of U[50, 500] bp covering ~10% of each sequence; planted
homology = target segments copied into the query with substitutions
(transition:transversion 2:1), optionally small indels (geometric length,
mean 2, cap 10, half insertions), half of them reverse-complemented.
Repeat-dense genomes add families of diverged copies and tandem repeats.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List, Tuple

import numpy as np

BASES = np.frombuffer(b"ACGT", dtype=np.uint8)
PROBS = np.array([0.295, 0.205, 0.205, 0.295])
_COMP = np.zeros(256, dtype=np.uint8)
for a, b in zip(b"ACGTacgtNn", b"TGCAtgcaNn"):
    _COMP[a] = b
# transitions A<->G, C<->T; transversions the other two
_TS = {ord("A"): ord("G"), ord("G"): ord("A"), ord("C"): ord("T"), ord("T"): ord("C")}
_TV = {ord("A"): (ord("C"), ord("T")), ord("G"): (ord("C"), ord("T")),
       ord("C"): (ord("A"), ord("G")), ord("T"): (ord("A"), ord("G"))}
_TS_T = np.arange(256, dtype=np.uint8)
_TV_T = np.zeros((2, 256), dtype=np.uint8)
for k, v in _TS.items():
    _TS_T[k] = v
for k, (x, y) in _TV.items():
    _TV_T[0, k], _TV_T[1, k] = x, y


# 200-entry table with exactly 59 A, 41 C, 41 G, 59 T (0.295 / 0.205)
_LUT200 = np.repeat(BASES, [59, 41, 41, 59])


def random_bases(rng: np.random.Generator, n: int) -> np.ndarray:
    return _LUT200[rng.integers(0, 200, size=n, dtype=np.uint8)]


def revcomp(s: np.ndarray) -> np.ndarray:
    return _COMP[s[::-1]]


def mutate(rng: np.random.Generator, seg: np.ndarray, rate: float, indel_rate: float = 0.0) -> np.ndarray:
    seg = seg.copy()
    hit = rng.random(seg.size) < rate
    idx = np.nonzero(hit)[0]
    if idx.size:
        ts = rng.random(idx.size) < 2.0 / 3.0
        pick = rng.integers(0, 2, idx.size)
        old = seg[idx]
        seg[idx] = np.where(ts, _TS_T[old], _TV_T[pick, old])
    if indel_rate > 0 and seg.size:
        n_ev = rng.binomial(seg.size, indel_rate)
        if n_ev:
            pos = np.sort(rng.integers(0, seg.size, n_ev))
            lens = np.minimum(rng.geometric(0.5, n_ev), 10)
            ins = rng.random(n_ev) < 0.5
            parts, last = [], 0
            for p, l, i in zip(pos.tolist(), lens.tolist(), ins.tolist()):
                if p < last:
                    continue
                parts.append(seg[last:p])
                if i:
                    parts.append(random_bases(rng, l))
                    last = p
                else:
                    last = p + l
            parts.append(seg[min(last, seg.size):])
            seg = np.concatenate(parts)
    return seg


def soft_mask(rng: np.random.Generator, s: np.ndarray, frac: float = 0.10, lo: int = 50, hi: int = 500):
    n = s.size
    if n == 0 or frac <= 0:
        return s
    mean = (lo + hi) / 2
    k = int(n * frac / mean) + 1
    starts = rng.integers(0, n, k)
    lens = rng.integers(lo, hi + 1, k)
    if n > (1 << 28):  # same result without an n-sized counter array
        s = s.copy()
        for a, l in zip(starts.tolist(), lens.tolist()):
            s[a: a + l] |= 0x20
        return s
    mask = np.zeros(n + 1, dtype=np.int32)
    np.add.at(mask, starts, 1)
    np.add.at(mask, np.minimum(starts + lens, n), -1)
    m = np.cumsum(mask[:n]) > 0
    s = s.copy()
    s[m] = s[m] | 0x20  # lowercase
    return s


@dataclass
class Planted:
    target_start: int
    query_start: int
    length: int
    rc: bool
    rate: float


def plant(rng, target: np.ndarray, query: np.ndarray, n_seg: int, len_lo: int, len_hi: int,
          rate_lo: float, rate_hi: float, indel_rate: float = 0.0) -> List[Planted]:
    out = []
    for _ in range(n_seg):
        L = int(rng.integers(len_lo, len_hi + 1))
        if L >= target.size or L >= query.size:
            continue
        ts = int(rng.integers(0, target.size - L))
        rate = float(rng.uniform(rate_lo, rate_hi))
        seg = mutate(rng, target[ts: ts + L], rate, indel_rate)
        rc = bool(rng.random() < 0.5)
        if rc:
            seg = revcomp(seg)
        qs = int(rng.integers(0, max(1, query.size - seg.size)))
        seg = seg[: query.size - qs]
        query[qs: qs + seg.size] = seg
        out.append(Planted(ts, qs, int(seg.size), rc, rate))
    return out


def pair(seed: int, t_len: int, q_len: int, n_seg: int, len_lo: int, len_hi: int, rate_lo: float,
         rate_hi: float, indel_rate: float = 0.0, mask_frac: float = 0.10) -> Tuple[np.ndarray, np.ndarray]:
    """Target and query ASCII blocks with planted homology."""
    rng = np.random.default_rng(seed)
    t = random_bases(rng, t_len)
    q = random_bases(rng, q_len)
    plant(rng, t, q, n_seg, len_lo, len_hi, rate_lo, rate_hi, indel_rate)
    return soft_mask(rng, t, mask_frac), soft_mask(rng, q, mask_frac)


def config1(seed: int = 1, scale: float = 1.0):
    """1 Mbp x 1 Mbp, 200 segments U[300, 2000] at 15% substitutions."""
    n = int(1_000_000 * scale)
    return pair(seed, n, n, max(1, int(200 * scale)), 300, 2000, 0.15, 0.15)


def config2(seed: int = 2, scale: float = 1.0):
    """100 Mbp target (10 bins x 10 Mbp) x 100 Mbp query; 20,000 segments
    U[200, 5000] at U[10, 30]% substitutions plus 1% small indels."""
    n = int(100_000_000 * scale)
    t, q = pair(seed, n, n, max(1, int(20_000 * scale)), 200, 5000, 0.10, 0.30, indel_rate=0.01)
    bins = 10
    step = n // bins
    return [t[i * step:(i + 1) * step] for i in range(bins)], q


def log_uniform_lengths(rng, n: int, lo: int, hi: int) -> np.ndarray:
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)


def config3(seed: int = 3, scale: float = 1.0, n_chunks: int = 512, homology_frac: float = 0.2):
    """Resident 200 Mbp target; 512 query chunks with log-uniform lengths in
    [10 kbp, 2 Mbp], each carrying planted homology at U[5, 35]% divergence
    over ~homology_frac of its length (segments U[200, 5000])."""
    rng = np.random.default_rng(seed)
    t_len = int(200_000_000 * scale)
    t = random_bases(rng, t_len)
    lens = log_uniform_lengths(rng, n_chunks, max(100, int(10_000 * scale)), max(1000, int(2_000_000 * scale)))
    chunks = []
    for L in lens.tolist():
        q = random_bases(rng, int(L))
        n_seg = max(1, int(L * homology_frac / 2600))
        plant(rng, t, q, n_seg, 200, 5000, 0.05, 0.35)
        chunks.append(soft_mask(rng, q))
    return soft_mask(rng, t), chunks


def random_genome(rng: np.random.Generator, n: int, piece: int = 1 << 26) -> np.ndarray:
    """random_bases for genome-sized n, drawn in pieces to bound host memory."""
    out = np.empty(n, dtype=np.uint8)
    for a in range(0, n, piece):
        out[a: a + piece] = random_bases(rng, min(piece, n - a))
    return out


def repeat_families(rng: np.random.Generator, n_fam: int = 500, lo: int = 300, hi: int = 6000):
    """Consensus sequences of the interspersed repeat families."""
    return [random_bases(rng, int(L)) for L in rng.integers(lo, hi + 1, n_fam)]


def repeat_genome(rng: np.random.Generator, n: int, families, rep_frac: float = 0.45,
                  tandem_frac: float = 0.03, rate_lo: float = 0.05, rate_hi: float = 0.30) -> np.ndarray:
    """Background sequence with ~rep_frac of it copies of the families (whole
    consensus, U[rate_lo, rate_hi] substitutions, half reverse-complemented)
    laid end to end between random gaps, then ~tandem_frac of it tandem arrays
    (unit U[2, 50] bp, array U[100, 5000] bp, 0-10% substitutions)."""
    s = random_genome(rng, n)
    mean_copy = float(np.mean([f.size for f in families]))
    mean_gap = mean_copy * (1.0 - rep_frac) / max(rep_frac, 1e-9)
    pos = int(rng.exponential(mean_gap))
    while pos < n:
        f = families[int(rng.integers(len(families)))]
        seg = mutate(rng, f, float(rng.uniform(rate_lo, rate_hi)))
        if rng.random() < 0.5:
            seg = revcomp(seg)
        seg = seg[: n - pos]
        s[pos: pos + seg.size] = seg
        pos += seg.size + int(rng.exponential(mean_gap))
    placed, want = 0, int(n * tandem_frac)
    while placed < want:
        unit = random_bases(rng, int(rng.integers(2, 51)))
        L = int(rng.integers(100, 5001))
        arr = mutate(rng, np.resize(unit, L), float(rng.uniform(0.0, 0.10)))
        a = int(rng.integers(0, max(1, n - L)))
        arr = arr[: n - a]
        s[a: a + arr.size] = arr
        placed += arr.size
    return s


def config4(seed: int = 4, scale: float = 1.0):
    """Repeat-dense pair: 1 Gbp target and 1 Gbp query, each ~45% copies of
    500 shared repeat families (consensus 300-6000 bp, 5-30% divergence) and
    ~3% tandem repeats (unit 2-50 bp), plus planted orthologous segments;
    the run uses a per-seed occurrence cap of 1000."""
    rng = np.random.default_rng(seed)
    n = int(1_000_000_000 * scale)
    fam = repeat_families(rng)
    t = repeat_genome(rng, n, fam)
    q = repeat_genome(rng, n, fam)
    plant(rng, t, q, max(1, int(20_000 * scale)), 200, 5000, 0.10, 0.30, indel_rate=0.01)
    return soft_mask(rng, t), soft_mask(rng, q)


def config5_target(seed: int = 5, scale: float = 1.0) -> np.ndarray:
    """Resident serving target: a 3 Gbp synthetic genome (soft-masked ~10%)."""
    rng = np.random.default_rng(seed)
    return soft_mask(rng, random_genome(rng, int(3_000_000_000 * scale)))


def request_lengths(rng: np.random.Generator, n: int, median: float = 200_000, sigma: float = 1.0,
                    cap: int = 5_000_000, lo: int = 1000) -> np.ndarray:
    """Serving request lengths: lognormal(ln median, sigma), capped."""
    return np.clip(rng.lognormal(np.log(median), sigma, n), lo, cap).astype(np.int64)


def serving_request(rng: np.random.Generator, target: np.ndarray, length: int,
                    homology_frac: float = 0.2) -> np.ndarray:
    """One query chunk with planted homology to the target over ~homology_frac
    of its length (segments U[200, 5000] at 5-35% divergence)."""
    q = random_bases(rng, int(length))
    plant(rng, target, q, max(1, int(length * homology_frac / 2600)), 200, 5000, 0.05, 0.35)
    return soft_mask(rng, q)
