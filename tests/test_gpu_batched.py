"""The batched form against the plain per-chunk form and the oracle: many
query chunks of uneven length through shared waves must give, per query,
exactly the records the plain form gives for that query alone."""
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
def workload():
    # config 3 shape, scaled: 4 Mbp resident target, 48 chunks with
    # log-uniform lengths, planted homology at 5-35% divergence
    return synth.config3(seed=31, scale=0.02, n_chunks=48)


def per_query(recs, nq):
    out = []
    for q in range(nq):
        sel = recs[recs["query"] == q]
        out.append([tuple(int(r[f]) for f in FIELDS) for r in sel])
    return out


def plain_records(e, q):
    e.swap_query_ascii(q)
    recs, st = e.run_pass()
    return [tuple(int(r[f]) for f in FIELDS) for r in recs], st


def test_batched_equals_plain_per_query(workload):
    target, chunks = workload
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries(chunks)
        got, st = e.run_batched()
        want = []
        hits = 0
        for q in chunks:
            r, s = plain_records(e, q)
            want.append(r)
            hits += s["hits"]
    assert sum(len(w) for w in want) > 50
    assert per_query(got, len(chunks)) == want
    assert st["hits"] == hits


@pytest.mark.parametrize("tuning", [dict(wave_positions=50_000), dict(gate_cap=8), dict(gate_cap=4096),
                                    dict(gate_tile=128, gate_blocks_per_sm=1), dict(gate_tile=256),
                                    dict(gate_tile=64), dict(device_dedup=0),
                                    dict(device_dedup=0, wave_positions=5_000), dict(graph=1),
                                    dict(graph=1, wave_positions=20_000, gate_tile=64),
                                    dict(gate_version=1), dict(gate_version=1, gate_tile=64, gate_cap=8),
                                    dict(gate_sparse=0), dict(gate_sparse=1), dict(gate_sparse=0, gate_cap=8),
                                    dict(wave_hits_cap=1 << 20)])
def test_launch_shapes_do_not_change_results(workload, tuning):
    target, chunks = workload
    chunks = chunks[:16]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries(chunks)
        base, st0 = e.run_batched()
        e.set_tuning(**tuning)
        got, st1 = e.run_batched()
    assert got.tobytes() == base.tobytes()
    assert (st1["hits"], st1["cells"], st1["raw_hsps"]) == (st0["hits"], st0["cells"], st0["raw_hsps"])


def test_batched_matches_oracle(workload):
    target, chunks = workload
    sm = EngineConfig().sub_mat
    pick = [0, 5, 11, 17]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries([chunks[i] for i in pick])
        got, st = e.run_batched()
    got_q = per_query(got, len(pick))
    for k, i in enumerate(pick):
        want, _ = oracle_run(target, chunks[i], sm)
        assert got_q[k] == [tuple(int(r[f]) for f in FIELDS) for r in want]


def test_empty_and_tiny_queries_in_a_batch(workload):
    target, chunks = workload
    qs = [b"", b"ACGT", chunks[0], b"ACGTACGTACGTACGTACGTAC", chunks[1]]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries(qs)
        got, _ = e.run_batched()
        want = [plain_records(e, q)[0] for q in qs]
    assert per_query(got, len(qs)) == want


def test_graph_replay_profiles_and_autotune_keep_results(workload):
    """The wave chain replayed as a CUDA graph (updated in place from wave to
    wave) gives the same records; its kernels are still timed one by one; the
    autotuner picks a valid shape and the results stay identical."""
    target, chunks = workload
    chunks = chunks[:20]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries(chunks)
        base, st0 = e.run_batched()
        e.set_tuning(graph=1, wave_positions=30_000)  # many waves through one instantiated graph
        e.set_profiling(True)
        e.profile_reset()
        got, st1 = e.run_batched()
        prof = e.profile()
        e.set_profiling(False)
        assert got.tobytes() == base.tobytes()
        assert prof["gate"][1] >= 2 and prof["gate"][0] > 0
        assert prof["lookup_count"][1] == prof["gate"][1]
        tune = e.autotune(sample_positions=200_000)
        assert tune["gate_tile"] in (64, 128, 256)
        assert tune["gate_cap"] in (64, 128, 256, 512, 1024)
        assert tune["candidates"] == 30 and tune["sample_calls"] >= 1
        assert 0 < tune["best_ms"] <= tune["start_ms"]
        again, st2 = e.run_batched()
    assert again.tobytes() == base.tobytes()
    assert (st2["hits"], st2["cells"]) == (st0["hits"], st0["cells"])


def test_capacity_overflow_reruns_give_the_same_records(workload):
    """Starting capacities far too small: every wave overflows its tile
    table, candidate list and raw-HSP list, grows them and runs again; the
    records and counts are unchanged, in both forms."""
    target, chunks = workload
    chunks = chunks[:12]
    with Engine(EngineConfig()) as e:
        e.load_target(target)
        e.stage_queries(chunks)
        base, st0 = e.run_batched()
        e.select_query(3)
        plain0, _ = e.run_pass()
    with Engine(EngineConfig()) as e:
        e.set_tuning(tile_cap=16, cand_cap=16, raw_cap=16)
        e.load_target(target)
        e.stage_queries(chunks)
        got, st1 = e.run_batched()
        e.set_tuning(tile_cap=16, cand_cap=16, raw_cap=16)
        e.select_query(3)
        plain1, _ = e.run_pass()
    assert got.tobytes() == base.tobytes()
    assert plain1.tobytes() == plain0.tobytes()
    assert (st1["hits"], st1["cells"], st1["raw_hsps"]) == (st0["hits"], st0["cells"], st0["raw_hsps"])


@pytest.mark.parametrize("kw", [dict(strand="minus"), dict(strand="plus"), dict(transitions=False),
                                dict(noentropy=True), dict(wga_chunk=30_000, interval=100_000),
                                dict(seed="111010010100110111"), dict(max_hits=5000)])
def test_batched_equals_plain_under_flags(workload, kw):
    target, chunks = workload
    chunks = chunks[:10]
    with Engine(EngineConfig(**kw)) as e:
        e.load_target(target)
        e.stage_queries(chunks)
        got, st = e.run_batched()
        want = []
        for i in range(len(chunks)):
            e.select_query(i)
            r, _ = e.run_pass()
            want.append([tuple(int(x[f]) for f in FIELDS) for x in r])
    assert per_query(got, len(chunks)) == want
