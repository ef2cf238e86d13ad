"""The HSP record, its orderings, and the ``.segments`` writer.

Mirrors hspZ ``src/hsp.rs``: ``SegmentPair`` (``:31-41``), ``by_diagonal``
(``:62-68``), ``by_lastz`` (``:71-77``), ``contained`` (``:83-87``),
``dedup_and_order`` (``:94-126``) and the ``.segments`` rendering
(``:213-292``).  The device kernels produce the same 16-byte records; this
module is the host-side view used for rendering, digests and parity checks.
"""
from __future__ import annotations

import hashlib
from typing import Dict, List, Sequence, Tuple

import numpy as np

from .sequence import Chr, chr_at

SEGMENT_PAIR = np.dtype([("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])
# One output record of a pass: interval index, strand (0 '+', 1 '-') and the HSP.
PASS_RECORD = np.dtype([("interval", "<u4"), ("strand", "<u4"), ("ref_start", "<u4"),
                        ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])


def diagonal(h) -> int:
    return (int(h["ref_start"]) - int(h["query_start"])) & 0xFFFFFFFF


def _diag_key(h):
    return (diagonal(h), int(h["ref_start"]), int(h["len"]), -int(h["score"]))


def _lastz_key(h):
    return (int(h["query_start"]), int(h["ref_start"]), int(h["len"]), -int(h["score"]))


def contained(x, y) -> bool:
    xe = (int(x["ref_start"]) + int(x["len"])) & 0xFFFFFFFF
    ye = (int(y["ref_start"]) + int(y["len"])) & 0xFFFFFFFF
    xs, ys = int(x["ref_start"]), int(y["ref_start"])
    return diagonal(x) == diagonal(y) and ((xs >= ys and xe <= ye) or (ys >= xs and ye <= xe))


def dedup_and_order(hsps: np.ndarray) -> np.ndarray:
    """Sort by diagonal, drop records contained in the previous INPUT record,
    then sort by LASTZ order (src/hsp.rs:94-126).  Host reference used for
    small checks; the engine does this per dedup scope itself."""
    a = sorted(hsps.tolist(), key=lambda t: ((t[0] - t[1]) & 0xFFFFFFFF, t[0], t[2], -t[3]))
    arr = np.array(a, dtype=SEGMENT_PAIR)
    kept = [arr[i] for i in range(len(arr)) if i == 0 or not contained(arr[i - 1], arr[i])]
    kept.sort(key=_lastz_key)
    return np.array([tuple(k) for k in kept], dtype=SEGMENT_PAIR)


def render_segments(hsps: np.ndarray, r_chrs: Sequence[Chr], q_chrs: Sequence[Chr], strand: str) -> str:
    """``.segments`` text: 1-based, chromosome-relative, inclusive ends; the
    minus strand prints in reverse order (src/hsp.rs:266-292)."""
    rows = hsps[::-1] if strand == "-" else hsps
    out = []
    for e in rows:
        rs, qs, ln, sc = int(e["ref_start"]), int(e["query_start"]), int(e["len"]), int(e["score"])
        r = r_chrs[chr_at(r_chrs, rs)]
        q = q_chrs[chr_at(q_chrs, qs)]
        out.append(f"{r.name}\t{rs + 1 - r.start}\t{rs + ln + 1 - r.start}\t{q.name}\t"
                   f"{qs + 1 - q.start}\t{qs + ln + 1 - q.start}\t{strand}\t{sc}\n")
    return "".join(out)


def render_pass(records: np.ndarray, r_chrs, q_chrs, rc_chrs, query_bin: int = 0,
                ref_bin: int = 0) -> Dict[str, str]:
    """Every ``tmp<n>.block<q>.r<r>.{plus,minus}.segments`` file of one
    reference-bin x query-bin unit (src/run.rs:568-626), as {name: text}."""
    files = {}
    if records.size == 0:
        return files
    n_int = int(records["interval"].max()) + 1
    for n in range(n_int):
        for strand_id, (chrs, sym, word) in enumerate(((q_chrs, "+", "plus"), (rc_chrs, "-", "minus"))):
            sel = records[(records["interval"] == n) & (records["strand"] == strand_id)]
            if sel.size == 0:
                continue
            h = np.zeros(sel.size, dtype=SEGMENT_PAIR)
            for f in SEGMENT_PAIR.names:
                h[f] = sel[f]
            files[f"tmp{n + 1}.block{query_bin}.r{ref_bin}.{word}.segments"] = render_segments(h, r_chrs, chrs, sym)
    return files


def sorted_digest(files: Dict[str, str]) -> Tuple[int, str]:
    """``cat *.segments | LC_ALL=C sort | sha256sum | cut -c1-16`` and the
    line count (assets/container/smoke.sh:66-68)."""
    lines: List[bytes] = []
    for text in files.values():
        lines += [l + b"\n" for l in text.encode().split(b"\n") if l]
    lines.sort()
    return len(lines), hashlib.sha256(b"".join(lines)).hexdigest()[:16]


def parity_set(records: np.ndarray) -> List[Tuple[int, int, int, int, int]]:
    """Sorted (strand, ref_start, query_start, len, score) multiset of a pass:
    the bit-exact parity object."""
    return sorted(zip(records["strand"].tolist(), records["ref_start"].tolist(),
                      records["query_start"].tolist(), records["len"].tolist(),
                      records["score"].tolist()))
