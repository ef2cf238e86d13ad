"""``-D`` diagonal partition of a logical ``.segments`` output.

Mirrors hspZ ``src/partition.rs`` (its restatement of KegAlign's
``diagonal_partition.py``): an output whose HSP count reaches
``MIN_CHUNK_SIZE`` is split into files of at most a chunk size estimated
from the sizes of earlier outputs (``Partitioner``, ``:33-121``).  Records
are grouped by (reference chromosome, query chromosome) in first-appearance
order; a pair larger than the chunk (or the only pair) is sorted along its
diagonal and cut into chunks, the smaller pairs are bin-packed whole
(``split``, ``:123-196``).  Records are those of ``hsp.records``: chromosome
indices and 1-based chromosome-relative coordinates.
"""
from __future__ import annotations

from typing import List, Optional, Sequence, Tuple

import numpy as np

MIN_CHUNK_SIZE = 5000   # outputs with fewer HSPs are never partitioned
MAX_CHUNK_SIZE = 50000  # cap on an estimated chunk size


def diagonal_key(recs: np.ndarray, strand: str) -> Tuple[np.ndarray, np.ndarray]:
    """Per record (primary, secondary) sort key along the diagonal: with
    ``half = (r_end - r_start) // 2`` added to both starts as midpoints, the
    plus strand sorts by the midpoints' sum, the minus strand by their
    difference (query - reference); the reference midpoint breaks ties
    (src/hsp.rs:189-209)."""
    half = (recs["r_end"].astype(np.int64) - recs["r_start"].astype(np.int64)) // 2
    r_mid = recs["r_start"].astype(np.int64) + half
    q_mid = recs["q_start"].astype(np.int64) + half
    return (q_mid - r_mid if strand == "-" else q_mid + r_mid), r_mid


def quantiles_exclusive(sorted_sizes: Sequence[int]) -> Optional[Tuple[float, float, float]]:
    """Quartiles by the exclusive method of Python's
    ``statistics.quantiles(data, n=4)``: the k-th cut point interpolates at
    1-based position k * (n + 1) / 4, clamped to the sample."""
    n = len(sorted_sizes)
    if n < 2:
        return None

    def at(k: int) -> float:
        pos = k * (n + 1) / 4.0
        if pos < 1.0:
            return float(sorted_sizes[0])
        if pos >= n:
            return float(sorted_sizes[n - 1])
        lo = int(pos)
        frac = pos - lo
        a, b = float(sorted_sizes[lo - 1]), float(sorted_sizes[lo])
        return a + (b - a) * frac

    return at(1), at(2), at(3)


class Partitioner:
    """Chunk-size estimation over the outputs seen so far
    (src/partition.rs:33-121)."""

    def __init__(self):
        self.history: List[int] = []

    def chunk_size_for(self, count: int) -> Optional[int]:
        """The chunk size for an output of ``count`` HSPs, or None to keep it
        whole: below MIN_CHUNK_SIZE never split; with fewer than two earlier
        outputs the cap; else the median (fewer than 7 earlier outputs) or
        the upper quartile of their sizes, capped; whole when it fits."""
        if count < MIN_CHUNK_SIZE:
            return None
        if len(self.history) < 2:
            chunk = MAX_CHUNK_SIZE
        else:
            s = sorted(self.history)
            q = quantiles_exclusive(s)
            pick = q[1] if len(s) < 7 else q[2]
            chunk = min(int(pick), MAX_CHUNK_SIZE)
        return None if count <= chunk else chunk

    def observe(self, count: int):
        self.history.append(count)

    def plan(self, recs: np.ndarray, strand: str):
        """("whole", recs) or ("split", [recs of each file, in file order])."""
        count = int(recs.size)
        self.observe(count)
        chunk = self.chunk_size_for(count)
        if chunk is None:
            return "whole", recs
        return "split", split(recs, strand, chunk)


def split(recs: np.ndarray, strand: str, chunk: int) -> List[np.ndarray]:
    """Partition one output's records into files (src/partition.rs:123-196)."""
    if recs.size == 0:
        return []
    keys = list(zip(recs["r_chr"].tolist(), recs["q_chr"].tolist()))
    order: dict = {}
    for i, k in enumerate(keys):
        order.setdefault(k, []).append(i)
    pairs = list(order.items())  # first-appearance order
    query_rank: dict = {}
    for (_, q), _ in pairs:
        query_rank.setdefault(q, len(query_rank))
    multi = len(pairs) > 1
    out: List[np.ndarray] = []
    skip = []
    for key, idx in pairs:
        group = recs[np.asarray(idx)]
        if multi and group.size <= chunk:
            skip.append((key, group))
            continue
        k0, k1 = diagonal_key(group, strand)
        group = group[np.lexsort((k1, k0))]  # stable: ties keep input order
        out += [group[a: a + chunk] for a in range(0, group.size, chunk)]
    if skip:
        skip.sort(key=lambda kv: (kv[1].size, kv[0]))  # stable
        bins = [[]]
        current = 0
        for key, group in skip:
            if current + group.size <= chunk:
                current += group.size
            else:
                bins.append([])
                current = group.size
            bins[-1].append((key, group))
        for b in bins:
            if not b:
                continue
            b.sort(key=lambda kv: query_rank[kv[0][1]])  # stable
            out.append(np.concatenate([g for _, g in b]))
    return out
