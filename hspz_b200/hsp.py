"""The HSP record, its orderings, and the ``.segments`` writer.

Mirrors hspZ ``src/hsp.rs``: ``SegmentPair`` (``:31-41``), ``by_diagonal``
(``:62-68``), ``by_lastz`` (``:71-77``), ``contained`` (``:83-87``),
``dedup_and_order`` (``:94-126``), the ``.segments`` records and rendering
(``:179-292``) and the per-unit file naming of ``src/run.rs:568-626``.  The device kernels produce the same 16-byte records; this
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


# One .segments line as numbers (hsp::Record, src/hsp.rs:179-187): chromosome
# indices and 1-based chromosome-relative coordinates; laid out like the C
# ABI's hz_segment_record so arrays pass to the native renderer as they are.
RECORD = np.dtype([("r_chr", "<u4"), ("q_chr", "<u4"), ("r_start", "<u8"), ("r_end", "<u8"),
                   ("q_start", "<u8"), ("q_end", "<u8"), ("score", "<i4"), ("pad", "<u4")])


def records(hsps: np.ndarray, r_chrs: Sequence[Chr], q_chrs: Sequence[Chr], strand: str) -> np.ndarray:
    """The records ``render_segments`` prints, in printed order: reversed on
    the minus strand, chromosome by ``chr_at`` (src/hsp.rs:213-232)."""
    h = hsps[::-1] if strand == "-" else hsps
    out = np.zeros(h.size, dtype=RECORD)
    if h.size == 0:
        return out
    rs = h["ref_start"].astype(np.int64)
    qs = h["query_start"].astype(np.int64)
    ln = h["len"].astype(np.int64)
    r_start = np.array([c.start for c in r_chrs], dtype=np.int64)
    q_start = np.array([c.start for c in q_chrs], dtype=np.int64)
    ri = np.searchsorted(r_start, rs, side="right") - 1  # upper_bound - 1
    qi = np.searchsorted(q_start, qs, side="right") - 1
    out["r_chr"], out["q_chr"] = ri, qi
    out["r_start"] = rs + 1 - r_start[ri]
    out["r_end"] = rs + ln + 1 - r_start[ri]
    out["q_start"] = qs + 1 - q_start[qi]
    out["q_end"] = qs + ln + 1 - q_start[qi]
    out["score"] = h["score"]
    return out


def render_records_py(recs: np.ndarray, r_chrs: Sequence[Chr], q_chrs: Sequence[Chr], strand: str) -> str:
    """``render_records`` (src/hsp.rs:234-252) in Python."""
    return "".join(f"{r_chrs[r['r_chr']].name}\t{r['r_start']}\t{r['r_end']}\t{q_chrs[r['q_chr']].name}\t"
                   f"{r['q_start']}\t{r['q_end']}\t{strand}\t{r['score']}\n" for r in recs)


def render_records(recs: np.ndarray, r_chrs: Sequence[Chr], q_chrs: Sequence[Chr], strand: str) -> str:
    """``render_records`` (src/hsp.rs:234-252) through the library's native
    renderer (hz_render_records)."""
    import ctypes as C
    from . import _native as N
    a = np.ascontiguousarray(recs, dtype=RECORD)
    rn = (C.c_char_p * max(len(r_chrs), 1))(*[c.name.encode() for c in r_chrs])
    qn = (C.c_char_p * max(len(q_chrs), 1))(*[c.name.encode() for c in q_chrs])
    out, n = C.c_void_p(), C.c_uint64()
    N.check(N.lib().hz_render_records(a.ctypes.data_as(C.c_void_p), a.size, rn, len(r_chrs), qn, len(q_chrs),
                                      strand.encode(), C.byref(out), C.byref(n)))
    try:
        return C.string_at(out, n.value).decode() if n.value else ""
    finally:
        N.lib().hz_free(out)


def emit_unit(records_of_pass: np.ndarray, r_chrs, q_chrs, rc_chrs, query_bin: int = 0, ref_bin: int = 0,
              partitioner=None, native: bool = True) -> Dict[str, str]:
    """Every output file of one reference-bin x query-bin unit, {name: text}
    (``Emitter::emit_unit``, src/run.rs:568-626): ``tmp<n>.block<q>.r<r>.
    {plus,minus}.segments`` per LASTZ interval and strand, or, with a
    ``partition.Partitioner`` (``-D``), ``....split<k>.segments`` pieces."""
    files: Dict[str, str] = {}
    if records_of_pass.size == 0:
        return files
    render = render_records if native else render_records_py
    n_int = int(records_of_pass["interval"].max()) + 1
    for n in range(n_int):
        base = f"tmp{n + 1}.block{query_bin}.r{ref_bin}"
        for strand_id, (chrs, sym, word) in enumerate(((q_chrs, "+", "plus"), (rc_chrs, "-", "minus"))):
            sel = records_of_pass[(records_of_pass["interval"] == n) & (records_of_pass["strand"] == strand_id)]
            if sel.size == 0:
                continue
            h = np.zeros(sel.size, dtype=SEGMENT_PAIR)
            for f in SEGMENT_PAIR.names:
                h[f] = sel[f]
            recs = records(h, r_chrs, chrs, sym)
            plan = partitioner.plan(recs, sym) if partitioner is not None else ("whole", recs)
            stem = f"{base}.{word}"
            if plan[0] == "whole":
                files[f"{stem}.segments"] = render(recs, r_chrs, chrs, sym)
            else:
                for k, piece in enumerate(plan[1], 1):
                    files[f"{stem}.split{k}.segments"] = render(piece, r_chrs, chrs, sym)
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
