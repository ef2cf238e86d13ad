"""HSP orderings and dedup (src/hsp.rs:334-390 restated) through every
implementation here: the oracle, the library's host dedup (hz_dedup_and_order,
which the plain form uses) and the Python restatement."""
import numpy as np
import pytest

import oracle
from hspz_b200 import engine as E
from hspz_b200 import hsp as H
from hspz_b200.build import build


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


def sp(*rows):
    return np.array(list(rows), dtype=H.SEGMENT_PAIR)


def dedups(a):
    return {"oracle": oracle.dedup_and_order(a.copy()), "library": E.dedup_and_order(a.copy()),
            "python": H.dedup_and_order(a.copy())}


def as_set(a):
    return {tuple(int(x) for x in r) for r in a.tolist()}


def test_diagonal_wraps_like_uint32():
    assert H.diagonal(sp((10, 4, 0, 0))[0]) == 6
    assert H.diagonal(sp((4, 10, 0, 0))[0]) == 0xFFFFFFFF - 5


def test_dedup_drops_contained_segments_on_the_same_diagonal():
    v = sp((0, 0, 10, 50), (0, 0, 5, 40), (6, 6, 2, 30), (0, 1, 4, 20))
    for name, got in dedups(v).items():
        assert as_set(got) == {(0, 1, 4, 20), (0, 0, 5, 40)}, name


def test_dedup_compares_against_previous_input_not_last_kept():
    v = sp((0, 0, 5, 10), (0, 0, 10, 20), (6, 6, 2, 30))
    for name, got in dedups(v).items():
        assert got.tolist() == [(0, 0, 5, 10)], name


def test_diagonal_sort_key_then_lastz_order():
    # no containment among these: dedup only reorders them into LASTZ order
    # (query start, reference start, length, score descending)
    v = sp((9, 5, 1, 1), (1, 2, 1, 1), (0, 5, 1, 1), (5, 0, 3, 100), (5, 0, 3, 900))
    want = [(1, 2, 1, 1), (0, 5, 1, 1), (9, 5, 1, 1)]
    for name, got in dedups(v).items():
        rows = [tuple(r) for r in got.tolist()]
        assert [r for r in rows if r[1] != 0] == want, name
        # the two identical segments on one diagonal: the higher score sorts
        # first, the lower one is contained in it and dropped
        assert [r for r in rows if r[1] == 0] == [(5, 0, 3, 900)], name
