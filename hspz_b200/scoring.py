"""The 8x8 substitution matrix the extension kernels index with the device
alphabet, and the LASTZ score-set reader.

Mirrors hspZ ``src/scoring.rs``: ``build_sub_mat`` (``:41-120``) and
``load_scoring_matrix`` (``:130-248``).  Only the ACGT block comes from a
scoring file; the soft-mask / N / X / separator rows are always rebuilt from
the fixed bad (-1000) and fill (-100) scores, and the separator scores
``-10 * xdrop`` so that no extension crosses a record boundary.
"""
from __future__ import annotations

import re
from typing import List, Optional

from .sequence import E_NT, L_NT, N_NT, NUC, X_NT

BAD = -1000
FILL = -100

# blastz / HOXD70 (src/scoring.rs:26-31)
DEFAULT_ACGT = [
    [91, -114, -31, -123],
    [-114, 100, -125, -31],
    [-31, -125, 100, -114],
    [-123, -31, -114, 91],
]


class ScoringError(ValueError):
    pass


# Rust's `str::parse::<i32>`: one optional sign, ASCII digits only.
_INT_RE = re.compile(r"[+-]?[0-9]+")


def build_sub_mat(ambiguous: str = "", xdrop: int = 910, scoring: Optional[str] = None) -> List[int]:
    acgt = load_scoring_matrix(scoring) if scoring else [row[:] for row in DEFAULT_ACGT]
    fields = ambiguous.split(",")
    field = fields[0]
    if len(fields) == 3:
        try:
            reward = int(fields[1])
        except ValueError as e:
            raise ScoringError(f"--ambiguous reward: {e}")
        try:
            penalty = -int(fields[2])
        except ValueError as e:
            raise ScoringError(f"--ambiguous penalty: {e}")
    elif ambiguous in ("n", "iupac"):
        reward, penalty = 0, 0
    else:
        reward, penalty = -100, -100

    m = [0] * (NUC * NUC)
    l, n, x, e = L_NT, N_NT, X_NT, E_NT
    for i in range(l):
        for j in range(l):
            m[i * NUC + j] = acgt[i][j]
    for i in range(l):
        m[i * NUC + l] = BAD
        m[l * NUC + i] = BAD
    m[l * NUC + l] = BAD

    n_score = (penalty, reward) if field in ("n", "iupac") else (BAD, BAD)
    for i in range(n):
        m[i * NUC + n] = n_score[0]
        m[n * NUC + i] = n_score[0]
    m[n * NUC + n] = n_score[1]

    if field == "iupac":
        for i in range(x):
            m[i * NUC + x] = penalty
            m[x * NUC + i] = penalty
        m[x * NUC + x] = reward
    else:
        for i in range(l):
            m[i * NUC + x] = FILL
            m[x * NUC + i] = FILL
        for i in range(l, x):
            m[i * NUC + x] = BAD
            m[x * NUC + i] = BAD
        m[x * NUC + x] = FILL

    sep = _wrap_i32(-10 * xdrop)
    for i in range(e):
        m[i * NUC + e] = sep
        m[e * NUC + i] = sep
    m[e * NUC + e] = sep
    return m


def _wrap_i32(v: int) -> int:
    v &= 0xFFFFFFFF
    return v - (1 << 32) if v >= 1 << 31 else v


def _parse_char_code(field: str, at: str) -> Optional[int]:
    if not field:
        return None
    if "~" in field:
        raise ScoringError(
            f"quantum alphabet column `{field}` is not supported ({at}); only the ACGT block is used")
    if len(field) == 1:
        code = ord(field)
    elif len(field) == 2:
        try:
            code = int(field, 16)
        except ValueError:
            raise ScoringError(f"invalid character code `{field}` ({at})")
    else:
        raise ScoringError(f"invalid character code `{field}` ({at})")
    if code == 0 or code >= 128:
        raise ScoringError(f"character code `{field}` out of range ({at})")
    return code


def _parse_score(field: str, at: str) -> int:
    try:
        if not _INT_RE.fullmatch(field):
            raise ValueError
        v = int(field)
        if not -(1 << 31) <= v < (1 << 31):
            raise ValueError
        return v
    except ValueError:
        raise ScoringError(f"invalid score `{field}` ({at}); scores must be integers")


def load_scoring_matrix(path: str) -> List[List[int]]:
    """ACGT block of a LASTZ score-set file (src/scoring.rs:130-248)."""
    with open(path, "r") as fh:
        text = fh.read()
    lines = []
    for i, raw in enumerate(text.splitlines()):
        l = raw.split("#", 1)[0].strip()
        if l:
            lines.append((i + 1, l))
    at = lambda n: f"{path}: line {n}"

    bad_score, fill_score = BAD, FILL
    bad_row = bad_col = None
    header = None
    idx = 0
    while idx < len(lines):
        n, line = lines[idx]
        idx += 1
        if "=" not in line:
            header = (n, line)
            break
        key, value = line.split("=", 1)
        key, value = key.strip(), value.strip()
        if key == "bad_score":
            parts = value.split(":")
            bad_score = _parse_score(parts[-1], at(n))
            if len(parts) == 1:
                pass
            elif len(parts) == 2:
                bad_row = _parse_char_code(parts[0], at(n))
                bad_col = bad_row
            elif len(parts) == 3:
                bad_row = _parse_char_code(parts[0], at(n))
                bad_col = _parse_char_code(parts[1], at(n))
            else:
                raise ScoringError(f"malformed bad_score ({at(n)})")
        elif key == "fill_score":
            fill_score = _parse_score(value, at(n))
    if header is None:
        raise ScoringError(f"{path}: no scoring matrix")
    hn, hline = header
    col_chars = []
    for f in hline.split():
        c = _parse_char_code(f, at(hn))
        if c is None:
            raise ScoringError(f"empty column label ({at(hn)})")
        col_chars.append(c)
    num_cols = len(col_chars)
    if num_cols == 0:
        raise ScoringError(f"{path}: no score columns")

    sub = {}
    num_fields = None
    implicit_row = 0
    for n, line in lines[idx:]:
        fields = line.split()
        if num_fields is None:
            if len(fields) not in (num_cols, num_cols + 1):
                raise ScoringError(
                    f"wrong number of score columns: got {len(fields)}, expected {num_cols} or "
                    f"{num_cols + 1} ({at(n)})")
            num_fields = len(fields)
        elif num_fields != len(fields):
            raise ScoringError(f"inconsistent number of score columns ({at(n)})")
        if len(fields) == num_cols:
            if implicit_row >= num_cols:
                raise ScoringError(f"too many score rows ({at(n)})")
            implicit_row += 1
            row_char, values = col_chars[implicit_row - 1], fields
        else:
            row_char = _parse_char_code(fields[0], at(n))
            if row_char is None:
                raise ScoringError(f"invalid row character code ({at(n)})")
            values = fields[1:]
        for ix, v in enumerate(values):
            sub[(row_char, col_chars[ix])] = _parse_score(v, at(n))
    if num_fields is None:
        raise ScoringError(f"{path}: contains no score rows")

    out = [[0] * 4 for _ in range(4)]
    for xi, r in enumerate(b"ACGT"):
        for yi, c in enumerate(b"ACGT"):
            if bad_row == r or bad_col == c:
                out[xi][yi] = bad_score
            else:
                out[xi][yi] = sub.get((r, c), fill_score)
    return out
