"""Host-side sequence handling: FASTA records, the packed block, the device
alphabet, reverse complement, LASTZ intervals and WGA seed chunks.

Mirrors hspZ ``src/sequence.rs`` (alphabet ``:35-79``, ``pack`` ``:185-205``,
``reverse_complement`` ``:212-230``, ``chr_at`` ``:316-318``, ``intervals``
``:322-334``, FASTA reader ``:336-417``) and ``src/seed.rs`` ``chunks``
(``:488-496``).  Coordinates are block-relative; a block is every record
joined by ``&`` with the trailing separator excluded from its length.
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Iterable, List, Sequence, Tuple

import numpy as np

SEP = ord("&")

# Device alphabet (src/sequence.rs:35-44).
A_NT, C_NT, G_NT, T_NT, L_NT, N_NT, X_NT, E_NT = range(8)
NUC = 8

_ENCODE = np.full(256, X_NT, dtype=np.uint8)
for _c, _v in ((b"A", A_NT), (b"C", C_NT), (b"G", G_NT), (b"T", T_NT)):
    _ENCODE[_c[0]] = _v
for _c in b"acgt":
    _ENCODE[_c] = L_NT
_ENCODE[ord("n")] = N_NT
_ENCODE[ord("N")] = N_NT
_ENCODE[SEP] = E_NT

# 128-entry IUPAC-aware complement; bytes >= 128 complement to 'N'
# (src/sequence.rs:83-86).
_RC128 = (
    b"NNNNNNNNNNNNNNNNNNNNNNNNNNNNNNNN"
    b"NNNNNN&NNNNNNNNNNNNNNNNNNNNNNNNN"
    b"NTVGHNNCDNNMNKNNNNYSAABWNRNNNNNN"
    b"NtvghnncdnnmnknnnnysaabwnrnNNNNN"
)
_REVCOMP = np.frombuffer(_RC128 + b"N" * 128, dtype=np.uint8).copy()

# The table the device uses to encode the reverse-complement strand straight
# from forward ASCII: encode(REV_COMP[c]).
ENCODE_TABLE = _ENCODE.copy()
ENCODE_RC_TABLE = _ENCODE[_REVCOMP].copy()


def as_bytes(seq) -> np.ndarray:
    if isinstance(seq, np.ndarray):
        return seq.astype(np.uint8, copy=False)
    if isinstance(seq, str):
        seq = seq.encode()
    return np.frombuffer(bytes(seq), dtype=np.uint8)


def encode(seq) -> np.ndarray:
    """ASCII -> device alphabet (``encode``, src/sequence.rs:66-79)."""
    return _ENCODE[as_bytes(seq)]


def reverse_complement_bytes(seq) -> np.ndarray:
    """Reverse complement of an ASCII block (src/sequence.rs:212-224)."""
    return _REVCOMP[as_bytes(seq)[::-1]]


@dataclass
class Chr:
    name: str
    start: int  # offset of the first base in the block
    len: int


def pack(records: Iterable[Tuple[str, bytes]], prefix: str = "") -> Tuple[np.ndarray, List[Chr], int]:
    """Records joined by ``&``; returns (buf, chrs, block_len) where block_len
    excludes the trailing separator (src/sequence.rs:185-205)."""
    parts: List[bytes] = []
    chrs: List[Chr] = []
    at = 0
    for name, seq in records:
        b = bytes(as_bytes(seq))
        chrs.append(Chr(prefix + name, at, len(b)))
        parts.append(b)
        parts.append(b"&")
        at += len(b) + 1
    buf = np.frombuffer(b"".join(parts), dtype=np.uint8).copy()
    block_len = max(at - 1, 0)
    return buf, chrs, block_len


def reverse_complement(buf: np.ndarray, chrs: Sequence[Chr], block_len: int) -> Tuple[np.ndarray, List[Chr]]:
    """RC of a packed block plus the remapped chromosome table,
    ``start' = n - start - len`` (src/sequence.rs:212-230)."""
    n = block_len
    rc = reverse_complement_bytes(buf[:n])
    rc_chrs = [Chr(c.name, n - c.start - c.len, c.len) for c in reversed(chrs)]
    return rc, rc_chrs


def chr_at(chrs: Sequence[Chr], off: int) -> int:
    """``upper_bound(starts, off) - 1`` (src/sequence.rs:316-318)."""
    lo, hi = 0, len(chrs)
    while lo < hi:
        mid = (lo + hi) // 2
        if chrs[mid].start <= off:
            lo = mid + 1
        else:
            hi = mid
    return lo - 1


def intervals(block_len: int, seed_size: int, interval_size: int) -> List[Tuple[int, int]]:
    """LASTZ intervals ``(start, end)`` with ``end`` inclusive
    (src/sequence.rs:322-334)."""
    out = []
    if block_len <= seed_size:
        return out
    end_pos = block_len - seed_size
    cur = 0
    while cur < end_pos:
        out.append((cur, min(end_pos, cur + interval_size)))
        cur += interval_size
    return out


def chunks(start: int, end: int, wga_chunk: int) -> List[Tuple[int, int]]:
    """WGA seed chunks ``[i, min(i + wga, end + 1))`` (src/seed.rs:488-496)."""
    out = []
    i = start
    while i < end:
        out.append((i, min(i + wga_chunk, end + 1)))
        i += wga_chunk
    return out


def batches(block_len: int, seed_size: int, interval_size: int, wga_chunk: int,
            plus: bool = True, minus: bool = True) -> List[Tuple[int, bool, int, int]]:
    """The flat call list of one pass, ``(interval, rev, start, end)``: per
    interval the plus chunks then the minus chunks; the minus range is
    ``(qbl - end, qbl - start)`` with ``qbl = block_len - seed_size``
    (src/run.rs:278-299)."""
    qbl = block_len - seed_size
    out = []
    for i, (s, e) in enumerate(intervals(block_len, seed_size, interval_size)):
        if plus:
            out += [(i, False, a, b) for a, b in chunks(s, e, wga_chunk)]
        if minus:
            out += [(i, True, a, b) for a, b in chunks(qbl - e, qbl - s, wga_chunk)]
    return out


def read_fasta(path) -> List[Tuple[str, bytes]]:
    """kseq-compatible FASTA reader: the name is the first whitespace token
    after ``>``; whitespace inside sequence lines is dropped
    (src/sequence.rs:336-417).  Plain text only (no gzip / 2bit here)."""
    records: List[Tuple[str, bytearray]] = []
    with open(path, "rb") as fh:
        for line in fh.read().split(b"\n"):
            if line.startswith(b">"):
                toks = line[1:].split()
                records.append(((toks[0] if toks else b"").decode("utf-8", "replace"), bytearray()))
            elif records:
                if line.endswith(b"\r"):
                    line = line[:-1]
                records[-1][1].extend(b"".join(line.split()))
    return [(n, bytes(s)) for n, s in records]
