"""The serving loop: query blocks submitted while others run are batched by
the workers, yet each request's records must equal what hz_run_pass gives for
that query alone.  Also covers admission against the memory budget,
cancellation, a failing request surfacing as its own error, and polling."""
import time

import numpy as np
import pytest

from hspz_b200 import Engine, EngineConfig
from hspz_b200 import _native as N
from hspz_b200 import synth
from hspz_b200.build import build

pytestmark = pytest.mark.gpu

FIELDS = ("interval", "strand", "ref_start", "query_start", "len", "score")


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


@pytest.fixture(scope="module")
def workload():
    return synth.config3(seed=47, scale=0.05, n_chunks=24)


def rows(recs):
    return [tuple(int(r[f]) for f in FIELDS) for r in recs]


@pytest.fixture(scope="module")
def alone(workload):
    """Each query's records from run_pass, one query at a time."""
    target, chunks = workload
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        out = []
        for q in chunks:
            e.swap_query_ascii(q)
            out.append(rows(e.run_pass()[0]))
    assert sum(len(r) for r in out) > 30
    return out


def test_served_requests_equal_run_pass_alone(workload, alone):
    target, chunks = workload
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.serve_start(budget_bytes=8 << 30, workers=2)
        tickets = []
        for i, q in enumerate(chunks):
            tickets.append(e.serve_submit(q))
            if i % 6 == 5:
                time.sleep(0.002)  # later arrivals join batches that form while others run
        batches = []
        for t, want in zip(tickets, alone):
            got, tm = e.serve_poll(t)
            assert rows(got) == want
            assert tm["total_ms"] >= tm["service_ms"] >= 0 and tm["queued_ms"] >= 0
            batches.append(tm["batch_queries"])
        e.serve_stop()
    assert max(batches) > 1  # requests were batched


def test_budget_admits_one_request_at_a_time_and_refuses_oversized(workload, alone):
    target, chunks = workload
    n = 20_000
    qs = [c[:n] for c in chunks if len(c) >= n][:6]
    assert len(qs) >= 3
    with Engine(EngineConfig()) as ref:
        ref.load_target(target)
        want = []
        for q in qs:
            ref.swap_query_ascii(q)
            want.append(rows(ref.run_pass()[0]))
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.serve_start(budget_bytes=1 << 40, workers=2)
        est = e.serve_estimate(n)  # what one request of n bases is expected to need
        assert e.serve_estimate(2 * n) > est + 1000
        e.serve_stop()
        e.serve_start(budget_bytes=est + 1000, workers=2)
        with pytest.raises(N.HzError) as ex:
            e.serve_submit(b"A" * (2 * n))
        assert ex.value.code == N.HZ_E_BUDGET
        tickets = [e.serve_submit(q) for q in qs]
        for t, w in zip(tickets, want):
            got, tm = e.serve_poll(t)
            assert rows(got) == w
            assert tm["batch_queries"] == 1  # two never fit the budget together
        e.serve_stop()


def test_cancel_poll_timeout_and_tickets(workload, alone):
    target, chunks = workload
    big = max(range(len(chunks)), key=lambda i: len(chunks[i]))
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.serve_start(budget_bytes=8 << 30, workers=1, max_batch_queries=1)
        tickets = [e.serve_submit(chunks[big]) for _ in range(6)]
        # the last ones are still queued behind the single worker
        with pytest.raises(N.HzError) as ex:
            e.serve_poll(tickets[-1], timeout_ms=0)
        assert ex.value.code == N.HZ_E_TIMEOUT
        cancelled = []
        for t in tickets[3:]:
            try:
                e.serve_cancel(t)
                cancelled.append(t)
            except N.HzError as err:
                assert err.code == N.HZ_E_STATE  # a worker took it first
        assert cancelled
        for t in tickets:
            if t in cancelled:
                with pytest.raises(N.HzError) as ex:
                    e.serve_poll(t)
                assert ex.value.code == N.HZ_E_STATE
            else:
                got, _ = e.serve_poll(t)
                assert rows(got) == alone[big]
        with pytest.raises(N.HzError) as ex:  # consumed
            e.serve_poll(tickets[0])
        assert ex.value.code == N.HZ_E_INVALID
        with pytest.raises(N.HzError) as ex:
            e.serve_poll(10 ** 9)
        assert ex.value.code == N.HZ_E_INVALID
        t = e.serve_submit(b"")  # empty query block
        got, _ = e.serve_poll(t)
        assert got.size == 0
        with pytest.raises(N.HzError) as ex:  # the target is shared with the workers
            e.load_target(target)
        assert ex.value.code == N.HZ_E_STATE
        e.serve_stop()
        e.load_target(target)  # allowed again once stopped


def test_failing_request_reports_its_own_error():
    rng = np.random.default_rng(5)
    rep = synth.random_bases(rng, 2000)
    target = np.concatenate([synth.random_bases(rng, 50_000), rep, synth.random_bases(rng, 3000), rep,
                             synth.random_bases(rng, 3000), rep])
    clean = synth.random_bases(rng, 20_000)
    # max_hits=1: the repeat's first seed holds 3 hits, so its MAX_HITS walk has no valid cut
    with Engine(EngineConfig(max_hits=1)) as e:
        e.load_target(target)
        e.swap_query_ascii(rep)
        with pytest.raises(N.HzError) as want:
            e.run_pass()
        e.serve_start(budget_bytes=1 << 30, workers=1, max_batch_queries=1)
        bad = e.serve_submit(rep)
        good = e.serve_submit(clean)
        with pytest.raises(N.HzError) as ex:
            e.serve_poll(bad)
        assert ex.value.code == want.value.code == N.HZ_E_INVALID
        got, _ = e.serve_poll(good)  # the worker carries on after a failed request
        e.serve_stop()
        e.swap_query_ascii(clean)
        assert rows(got) == rows(e.run_pass()[0])


def test_a_failing_request_fails_alone_in_its_batch():
    """A batch holding one request that fails on its own: the batch is rerun
    request by request, so only that request reports the error and the
    others return exactly what run_pass gives them alone.  One worker is kept
    busy with a long request while the next three queue behind it; the
    scenario repeats until the three shared one batch (they almost always do
    at once), and every repetition must give the right results."""
    rng = np.random.default_rng(6)
    rep = synth.random_bases(rng, 2000)
    target = np.concatenate([synth.random_bases(rng, 50_000), rep, synth.random_bases(rng, 3000), rep,
                             synth.random_bases(rng, 3000), rep])
    busy = synth.random_bases(rng, 20_000_000)
    good = [synth.random_bases(rng, 30_000), synth.random_bases(rng, 25_000)]
    with Engine(EngineConfig(max_hits=1)) as e:  # the repeat's first seed holds 3 hits: no valid MAX_HITS cut
        e.load_target(target)
        want = []
        for q in [busy] + good:
            e.swap_query_ascii(q)
            want.append(rows(e.run_pass()[0]))
        shared = False
        for _ in range(5):
            e.serve_start(budget_bytes=1 << 30, workers=1, max_batch_queries=8)
            t_busy = e.serve_submit(busy)  # keeps the one worker while the next three queue
            t = [e.serve_submit(good[0]), e.serve_submit(rep), e.serve_submit(good[1])]
            got, _ = e.serve_poll(t_busy)
            assert rows(got) == want[0]
            with pytest.raises(N.HzError) as ex:
                e.serve_poll(t[1])
            assert ex.value.code == N.HZ_E_INVALID
            sizes = []
            for ticket, w in ((t[0], want[1]), (t[2], want[2])):
                got, tm = e.serve_poll(ticket)
                assert rows(got) == w
                sizes.append(tm["batch_queries"])
            e.serve_stop()
            if sizes == [3, 3]:  # they shared a batch with the failing request
                shared = True
                break
        assert shared


def test_many_workers_random_poll_order_and_totals():
    """Four workers, batches of up to eight, requests polled in random order:
    every result equals run_pass alone, and the loop's hit total is the sum
    of the requests' own totals."""
    rng = np.random.default_rng(11)
    target, chunks = synth.config3(seed=53, scale=0.01, n_chunks=40)
    with Engine(EngineConfig()) as ref:
        ref.load_target(target)
        want, hits = [], 0
        for q in chunks:
            ref.swap_query_ascii(q)
            r, st = ref.run_pass()
            want.append(rows(r))
            hits += st["hits"]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.serve_start(budget_bytes=4 << 30, workers=4, max_batch_queries=8)
        tickets = [e.serve_submit(q) for q in chunks]
        order = rng.permutation(len(chunks))
        for i in order:
            got, _ = e.serve_poll(tickets[i])
            assert rows(got) == want[i], i
        totals, queued, running = e.serve_stats()
        assert (queued, running) == (0, 0)
        assert totals["hits"] == hits
        e.serve_stop()
