"""Scores for the extension kernels: the 8x8 substitution matrix indexed by
the device alphabet, and a reader for LASTZ score-set files.

The matrix follows hspZ ``src/scoring.rs`` (``build_sub_mat``, ``:41-120``):
the ACGT block is blastz/HOXD70 unless a score file replaces it; the rows and
columns of soft-masked (L), N, other (X) and separator (E) codes are always
derived from fixed values and the ``--ambiguous`` mode, never from the file;
and the separator scores ``-10 * xdrop`` so that no extension crosses a
record boundary.

The reader accepts the LASTZ score-set format as KegAlign consumes it
(``src/scoring.rs:122-278``): ``#`` comments, ``key = value`` settings before
the matrix (``bad_score`` and ``fill_score`` are used, every other LASTZ
setting is accepted and has no effect here), one line of column symbols,
then rows that either start with their own symbol or, blastz style, follow
the column order.  Pairs the file leaves out take ``fill_score``; a
nucleotide named by ``bad_score`` takes that score in its row or column.
"""
from __future__ import annotations

import re
from typing import Dict, Iterator, List, Optional, Tuple

from .sequence import E_NT, L_NT, N_NT, NUC, X_NT

BAD = -1000   # soft-masked / unusable pairs
FILL = -100   # pairs with an unknown (X) base

# blastz / HOXD70 (src/scoring.rs:26-31)
DEFAULT_ACGT = [
    [91, -114, -31, -123],
    [-114, 100, -125, -31],
    [-31, -125, 100, -114],
    [-123, -31, -114, 91],
]


class ScoringError(ValueError):
    pass


# ---------------------------------------------------------------------------
# The 8x8 matrix

_SIGNED = re.compile(r"[+-]?[0-9]+\Z")


def _as_i32(v: int) -> int:
    """Two's-complement wrap to 32 bits, as the reference's i32 arithmetic."""
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v & 0x80000000 else v


def _strict_int(text: str) -> Optional[int]:
    """An i32 written as an optional sign and decimal digits, else None."""
    if not _SIGNED.match(text):
        return None
    v = int(text)
    return v if -(1 << 31) <= v < (1 << 31) else None


def _ambiguity(spec: str) -> Tuple[str, int, int]:
    """(mode, reward, penalty) of an ``--ambiguous`` value.

    The mode is the text before the first comma.  With exactly three
    comma-separated parts the other two give the reward for an N/IUPAC code
    against itself and the (positive) penalty against anything else; the
    bare modes ``n`` and ``iupac`` score both as 0, and anything else leaves
    them at -100."""
    parts = spec.split(",")
    mode = parts[0]
    if len(parts) == 3:
        reward = _strict_int(parts[1])
        if reward is None:
            raise ScoringError(f"--ambiguous {spec!r}: the reward {parts[1]!r} is not an integer")
        penalty = _strict_int(parts[2])
        if penalty is None:
            raise ScoringError(f"--ambiguous {spec!r}: the penalty {parts[2]!r} is not an integer")
        return mode, reward, _as_i32(-penalty)
    if spec in ("n", "iupac"):
        return mode, 0, 0
    return mode, -100, -100


def build_sub_mat(ambiguous: str = "", xdrop: int = 910, scoring: Optional[str] = None) -> List[int]:
    """The row-major 8x8 matrix ``m[ref_code * 8 + query_code]``."""
    acgt = load_scoring_matrix(scoring) if scoring else [list(r) for r in DEFAULT_ACGT]
    mode, reward, penalty = _ambiguity(ambiguous)
    separator = _as_i32(-10 * xdrop)
    n_scored = mode in ("n", "iupac")

    def pair(r: int, c: int) -> int:
        # every non-ACGT row and column is symmetric; the higher code decides
        hi, lo = max(r, c), min(r, c)
        if hi == E_NT:
            return separator
        if hi == X_NT:
            if mode == "iupac":
                return reward if lo == X_NT else penalty
            # X against a nucleotide or itself is a fill; against L or N, bad
            return FILL if (lo < L_NT or lo == X_NT) else BAD
        if hi == N_NT:
            if n_scored:
                return reward if lo == N_NT else penalty
            return BAD
        if hi == L_NT:
            return BAD
        return acgt[r][c]

    return [pair(r, c) for r in range(NUC) for c in range(NUC)]


# ---------------------------------------------------------------------------
# LASTZ score-set files

_HEX2 = re.compile(r"\+?[0-9A-Fa-f]{1,2}\Z")


def _symbol(tok: str, where: str) -> int:
    """A matrix symbol: one ASCII character, or its code as two hex digits."""
    if "~" in tok:
        raise ScoringError(f"{where}: `{tok}` is a quantum-alphabet symbol; only nucleotide symbols are read")
    if len(tok) == 1:
        code = ord(tok)
    elif len(tok) == 2 and _HEX2.match(tok):
        code = int(tok, 16)
    else:
        raise ScoringError(f"{where}: `{tok}` is neither one character nor two hex digits")
    if not 0 < code < 128:
        raise ScoringError(f"{where}: symbol `{tok}` is not a printable ASCII code")
    return code


def _score(tok: str, where: str) -> int:
    v = _strict_int(tok)
    if v is None:
        raise ScoringError(f"{where}: `{tok}` is not an integer score")
    return v


def _content(text: str) -> Iterator[Tuple[int, str]]:
    """(line number, text) of every line that still has text once its
    ``#`` comment and surrounding blanks are gone."""
    for no, raw in enumerate(text.splitlines(), start=1):
        body = raw.partition("#")[0].strip()
        if body:
            yield no, body


class _Settings:
    def __init__(self):
        self.bad = BAD
        self.fill = FILL
        self.bad_row: Optional[int] = None
        self.bad_col: Optional[int] = None

    def apply(self, key: str, value: str, where: str) -> None:
        if key == "fill_score":
            self.fill = _score(value, where)
        elif key == "bad_score":
            # `score`, `symbol:score` (row and column) or `row:column:score`
            spec = value.split(":")
            if len(spec) > 3:
                raise ScoringError(f"{where}: bad_score takes score, symbol:score or row:column:score")
            self.bad = _score(spec[-1], where)
            if len(spec) >= 2:
                self.bad_row = _symbol(spec[0], where) if spec[0] else None
                self.bad_col = self.bad_row
            if len(spec) == 3:
                self.bad_col = _symbol(spec[1], where) if spec[1] else None
        # gap penalties, thresholds and the like do not reach the ACGT block


def load_scoring_matrix(path: str) -> List[List[int]]:
    """The 4x4 ACGT block of a LASTZ score-set file."""
    with open(path, "r") as fh:
        lines = list(_content(fh.read()))

    def where(no: int) -> str:
        return f"{path}, line {no}"

    settings = _Settings()
    k = 0
    while k < len(lines) and "=" in lines[k][1]:
        no, body = lines[k]
        key, _, value = body.partition("=")
        settings.apply(key.strip(), value.strip(), where(no))
        k += 1
    if k == len(lines):
        raise ScoringError(f"{path}: no matrix header line (column symbols) after the settings")
    header_no, header = lines[k]
    columns = [_symbol(tok, where(header_no)) for tok in header.split()]

    scores: Dict[Tuple[int, int], int] = {}
    width = None  # fields per row, fixed by the first row
    unlabelled = 0
    for no, body in lines[k + 1:]:
        toks = body.split()
        if width is None:
            if len(toks) not in (len(columns), len(columns) + 1):
                raise ScoringError(f"{where(no)}: a matrix row holds {len(columns)} scores, optionally after "
                                   f"its symbol; this one has {len(toks)} fields")
            width = len(toks)
        elif len(toks) != width:
            raise ScoringError(f"{where(no)}: {len(toks)} fields where the rows above have {width}")
        if width == len(columns):
            if unlabelled == len(columns):
                raise ScoringError(f"{where(no)}: more unlabelled rows than column symbols")
            row = columns[unlabelled]
            unlabelled += 1
        else:
            row = _symbol(toks[0], where(no))
            toks = toks[1:]
        for col, tok in zip(columns, toks):
            scores[(row, col)] = _score(tok, where(no))
    if width is None:
        raise ScoringError(f"{path}: the matrix has column symbols but no rows")

    block = []
    for r in b"ACGT":
        out_row = []
        for c in b"ACGT":
            if r == settings.bad_row or c == settings.bad_col:
                out_row.append(settings.bad)
            else:
                out_row.append(scores.get((r, c), settings.fill))
        block.append(out_row)
    return block
