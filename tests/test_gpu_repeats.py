"""Repeat-dense workload (the shape of the 1 Gbp repeat-family benchmark,
scaled down): long bucket tails, tandem arrays, and the per-seed occurrence
cap applied identically in the plain form, the batched form and the oracle.
At this size no bucket reaches the benchmark's cap of 1000, so a cap of 50
is tested too, which does drop repeat tails."""
import numpy as np
import pytest

from hspz_b200 import Engine, EngineConfig
from hspz_b200 import synth
from hspz_b200.build import build
from tests.test_gpu_parity import oracle_run

pytestmark = pytest.mark.gpu

FIELDS = ("interval", "strand", "ref_start", "query_start", "len", "score")


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


@pytest.fixture(scope="module")
def pair():
    return synth.config4(seed=44, scale=0.004)  # 4 Mbp x 4 Mbp


@pytest.mark.parametrize("cap", [1000, 50])
def test_repeat_dense_plain_equals_oracle(pair, cap):
    t, q = pair
    sm = EngineConfig().sub_mat
    want, st_o = oracle_run(t, q, sm, occ_cap=cap)
    with Engine(EngineConfig(occ_cap=cap)) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
    assert want.size > 100
    assert got.tobytes() == want.tobytes()
    for k in ("hits", "raw_hsps", "hsps", "cells"):
        assert st[k] == st_o[k], k


def test_occurrence_cap_drops_repeat_tails(pair):
    t, q = pair
    with Engine(EngineConfig(occ_cap=50)) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        _, capped = e.run_pass()
    with Engine(EngineConfig(occ_cap=0)) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        _, full = e.run_pass()
    assert capped["hits"] < full["hits"]


def test_repeat_dense_batched_equals_plain(pair):
    t, q = pair
    # the query cut into uneven chunks, all staged and run in shared waves
    cuts = [0, 300_000, 310_000, 1_500_000, 1_500_500, 2_900_000, q.size]
    chunks = [q[a:b] for a, b in zip(cuts[:-1], cuts[1:])]
    with Engine(EngineConfig(occ_cap=1000)) as e:
        e.load_target(t)
        e.stage_queries(chunks)
        got, st = e.run_batched()
        hits = 0
        for i, c in enumerate(chunks):
            e.select_query(i)
            want, s = e.run_pass()
            hits += s["hits"]
            sel = got[got["query"] == i]
            for f in FIELDS:
                assert np.array_equal(sel[f], want[f]), (i, f)
    assert st["hits"] == hits


@pytest.mark.parametrize("gate_version", [2, 1])
@pytest.mark.parametrize("gate_cap", [8, 64])
def test_long_extensions(pair, gate_cap, gate_version):
    """A small gate cap sends most hits on as long candidates: with the
    lockstep gate to the lane-per-candidate long kernel (maxima and their
    first positions from its 48-cell rounds), with the lane-refill gate to
    the warp kernel (four cells per lane).  Records and counts still equal
    the oracle's."""
    t, q = pair
    sm = EngineConfig().sub_mat
    want, st_o = oracle_run(t, q, sm, occ_cap=1000)
    with Engine(EngineConfig(occ_cap=1000)) as e:
        e.set_tuning(gate_cap=gate_cap, gate_version=gate_version)
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
    assert got.tobytes() == want.tobytes()
    for k in ("hits", "raw_hsps", "hsps", "cells"):
        assert st[k] == st_o[k], k
