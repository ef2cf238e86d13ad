"""Host-side sequence handling: FASTA records, the packed block, the device
alphabet, reverse complement, LASTZ intervals and WGA seed chunks.

Mirrors hspZ ``src/sequence.rs`` (alphabet ``:35-79``, ``pack`` ``:185-205``,
``reverse_complement`` ``:212-230``, ``chr_at`` ``:316-318``, ``intervals``
``:322-334``, the FASTA / FASTA.gz / 2bit readers ``:112-176, 336-417``) and
``src/seed.rs`` ``chunks``
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


FASTA, FASTA_GZ, TWO_BIT = "fasta", "fasta.gz", "2bit"
_TWOBIT_MAGIC = 0x1A412743


def detect_format(path) -> str:
    """The reader a file needs, from its magic bytes only (src/sequence.rs:
    112-144): the 2bit signature in either byte order, the gzip magic
    ``1f 8b``, else plain FASTA."""
    with open(path, "rb") as fh:
        head = fh.read(4)
    if len(head) >= 4 and _TWOBIT_MAGIC in (int.from_bytes(head, "big"), int.from_bytes(head, "little")):
        return TWO_BIT
    if head[:2] == b"\x1f\x8b":
        return FASTA_GZ
    return FASTA


def _parse_fasta(data: bytes) -> List[Tuple[str, bytes]]:
    # A header line starts a record named by its first whitespace token; any
    # other line extends the current record with its whitespace (a trailing
    # carriage return included) removed; lines before the first header are
    # ignored (src/sequence.rs:394-417).
    records: List[Tuple[str, bytearray]] = []
    for line in data.split(b"\n"):
        if line.startswith(b">"):
            toks = line[1:].split()
            records.append(((toks[0] if toks else b"").decode("utf-8", "replace"), bytearray()))
        elif records:
            records[-1][1].extend(b"".join(line.split()))
    return [(n, bytes(s)) for n, s in records]


def read_fasta(path) -> List[Tuple[str, bytes]]:
    """FASTA records ``(name, bases)``, plain or gzip-compressed (several
    concatenated gzip members read as one stream), bases kept exactly as
    written, soft-masking included (src/sequence.rs:346-392)."""
    import gzip
    with open(path, "rb") as fh:
        data = fh.read()
    if data[:2] == b"\x1f\x8b":
        data = gzip.decompress(data)
    return _parse_fasta(data)


# 2bit bases, two bits each, first base in the high bits: T, C, A, G.
_TWOBIT_BASES = np.frombuffer(b"TCAG", dtype=np.uint8)


def read_2bit(path) -> List[Tuple[str, bytes]]:
    """Records of a UCSC .2bit file in its index order (src/sequence.rs:
    153-176, which reads it through the `twobit` crate 0.2.2 with soft masks
    on).  The format, restated: a 16-byte header (signature 0x1A412743 in
    the file's byte order, version 0 or 1, sequence count, reserved), an
    index of (u8 name length, name, offset -- u32, or u64 in version 1), and
    per sequence: base count, N-block count, N-block starts, N-block sizes,
    mask-block count, mask-block starts, mask-block sizes, a reserved u32,
    then the packed bases.  N blocks read as 'N', mask blocks lowercase."""
    with open(path, "rb") as fh:
        data = fh.read()
    if len(data) < 16:
        raise ValueError(f"{path}: too short for a 2bit header")
    if int.from_bytes(data[:4], "little") == _TWOBIT_MAGIC:
        end = "<"
    elif int.from_bytes(data[:4], "big") == _TWOBIT_MAGIC:
        end = ">"
    else:
        raise ValueError(f"{path}: not a 2bit file")
    u32 = np.dtype(end + "u4")
    version, count = np.frombuffer(data, u32, 2, 4)
    if version not in (0, 1):
        raise ValueError(f"{path}: unsupported 2bit version {version}")
    off_t = np.dtype(end + ("u8" if version == 1 else "u4"))
    at = 16
    index = []
    for _ in range(int(count)):
        n = data[at]
        name = data[at + 1: at + 1 + n].decode("utf-8", "replace")
        at += 1 + n
        index.append((name, int(np.frombuffer(data, off_t, 1, at)[0])))
        at += off_t.itemsize
    out = []
    for name, off in index:
        dna, nb = (int(x) for x in np.frombuffer(data, u32, 2, off))
        off += 8
        n_starts = np.frombuffer(data, u32, nb, off).astype(np.int64)
        n_sizes = np.frombuffer(data, u32, nb, off + 4 * nb).astype(np.int64)
        off += 8 * nb
        mb = int(np.frombuffer(data, u32, 1, off)[0])
        off += 4
        m_starts = np.frombuffer(data, u32, mb, off).astype(np.int64)
        m_sizes = np.frombuffer(data, u32, mb, off + 4 * mb).astype(np.int64)
        off += 8 * mb + 4  # the reserved word
        packed = np.frombuffer(data, np.uint8, (dna + 3) // 4, off)
        codes = np.stack([(packed >> s) & 3 for s in (6, 4, 2, 0)], axis=1).reshape(-1)[:dna]
        seq = _TWOBIT_BASES[codes]
        for a, l in zip(n_starts.tolist(), n_sizes.tolist()):
            seq[a: a + l] = ord("N")
        for a, l in zip(m_starts.tolist(), m_sizes.tolist()):
            seq[a: a + l] |= 0x20
        out.append((name, seq.tobytes()))
    return out


def read_records(path) -> Tuple[str, List[Tuple[str, bytes]]]:
    """(format, records) of FASTA, gzipped FASTA or 2bit, chosen by magic
    bytes (src/sequence.rs:112-176)."""
    fmt = detect_format(path)
    return fmt, (read_2bit(path) if fmt == TWO_BIT else read_fasta(path))


@dataclass
class Genome:
    """One loaded sequence file packed into a single block
    (``Genome``, src/sequence.rs:93-311)."""
    buf: np.ndarray
    chrs: List[Chr]
    block_len: int
    format: str
    bytes_read: int

    def digest(self) -> int:
        """64-bit FNV-1a over every chromosome's name, start (8 bytes LE)
        and length (4 bytes LE), the block bytes and the block length
        (8 bytes LE) -- identical inputs load to identical digests
        (src/sequence.rs:289-305)."""
        h = 0xCBF29CE484222325
        parts = []
        for c in self.chrs:
            parts += [c.name.encode(), int(c.start).to_bytes(8, "little"), int(c.len).to_bytes(4, "little")]
        parts += [bytes(self.buf), int(self.block_len).to_bytes(8, "little")]
        for b in b"".join(parts):
            h = ((h ^ b) * 0x100000001B3) & 0xFFFFFFFFFFFFFFFF
        return h

    def reverse_complement(self):
        return reverse_complement(self.buf, self.chrs, self.block_len)


def load_genome(path, prefix: str = "", seq_block_size: int = 10_000_000_000) -> Genome:
    """Loads FASTA / FASTA.gz / 2bit and packs it into one block; a block
    longer than ``seq_block_size`` is refused (``Genome::load``,
    src/sequence.rs:254-287)."""
    import os
    fmt, records = read_records(path)
    buf, chrs, block_len = pack(records, prefix)
    if block_len > seq_block_size:
        raise ValueError(f"{path} exceeds one sequence block ({block_len} > {seq_block_size} bytes)")
    return Genome(buf, chrs, block_len, fmt, os.path.getsize(path))
