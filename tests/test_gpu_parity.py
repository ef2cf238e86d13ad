"""GPU parity: the CUDA path through the C ABI against the oracle and the
golden fixtures.  Integer/index work must be bit-exact; the entropy is the
same IEEE double sequence on both sides, so HSP scores are compared exactly
too (tolerance 0)."""
import json
import os

import numpy as np
import pytest

import oracle
from hspz_b200 import Engine, EngineConfig
from hspz_b200 import _native as N
from hspz_b200 import hsp as H
from hspz_b200 import sequence as S
from hspz_b200 import synth
from hspz_b200.build import build
from tests.golden.fixture_pass import MAX_HITS, load

pytestmark = pytest.mark.gpu
EXPECTED = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "expected.json")))


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


def oracle_run(ref_ascii, qry_ascii, sub_mat, **kw):
    ref = oracle.encode(bytes(ref_ascii))
    qf = oracle.encode(bytes(qry_ascii))
    qr = oracle.encode(bytes(S.reverse_complement_bytes(qry_ascii)))
    sh = oracle.shape(kw.pop("seed", "12of19"))
    idx, pos = oracle.seed_table(ref, sh, kw.pop("step", 1))
    kw.setdefault("threads", os.cpu_count() or 1)
    p = oracle.params(sub_mat, **kw)
    return oracle.seed_and_filter_all(p, sh, ref, idx, pos, qf, qr)


def engine_for(sub_mat, **kw):
    return Engine(EngineConfig(sub_mat=list(sub_mat), **kw))


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_fixture_digest_device_tables(name):
    d = load(name)
    with engine_for(d["sub_mat"], max_hits=MAX_HITS) as e:
        e.load_target(d["ref_ascii"])
        e.swap_query_ascii(d["qry_ascii"])
        recs, st = e.run_pass()
    files = H.render_pass(recs, d["rchrs"], d["qchrs"], d["rcchrs"])
    n, digest = H.sorted_digest(files)
    want = EXPECTED[name]
    assert (n, len(files), digest) == (want["hsps"], want["files"], want["digest"])
    assert (st["hits"], st["raw_hsps"], st["cells"]) == (want["hits"], want["raw_hsps"], want["cells"])


@pytest.mark.parametrize("name", ["repeat", "multi", "revcomp", "ambiguous"])
def test_fixture_host_tables_and_encoded_query(name):
    """Engine::new-style host tables (the oracle's SeedTable) + encoded query."""
    d = load(name)
    ref = oracle.encode(d["ref_ascii"].tobytes())
    idx, pos = oracle.seed_table(ref, oracle.shape("12of19"))
    with engine_for(d["sub_mat"]) as e:
        e.load_tables(idx, pos, ref)
        e.swap_query(S.encode(d["qry_ascii"]), S.encode(d["qrc_ascii"]))
        recs, _ = e.run_pass()
    n, digest = H.sorted_digest(H.render_pass(recs, d["rchrs"], d["qchrs"], d["rcchrs"]))
    assert (n, digest) == (EXPECTED[name]["hsps"], EXPECTED[name]["digest"])


def test_device_seed_table_is_byte_identical():
    """SeedTable::build on device == the oracle's, bucket order included
    (src/seed.rs:546-597), at step 1 and 3, with N / soft-mask / separators."""
    rng = np.random.default_rng(20260811)
    alpha = np.frombuffer(b"ACGTNacgt&", dtype=np.uint8)
    seq = rng.choice(alpha, size=400_000, p=[.245, .245, .245, .195, .02, .012, .012, .011, .01, .005])
    sm = EngineConfig().sub_mat
    for step in (1, 3):
        idx_o, pos_o = oracle.seed_table(oracle.encode(seq.tobytes()), oracle.shape("12of19"), step)
        with engine_for(sm, step=step) as e:
            e.load_target(seq)
            idx_d, pos_d = e.read_tables()
        assert np.array_equal(idx_d, idx_o)
        assert np.array_equal(pos_d, pos_o)
    # other seed patterns: short, spaced, with explicit transition marks
    for spec in ("1111", "11011", "1T1T11", "111010010100110111"):
        idx_o, pos_o = oracle.seed_table(oracle.encode(seq[:50_000].tobytes()), oracle.shape(spec), 1)
        with engine_for(sm, seed=spec) as e:
            e.load_target(seq[:50_000])
            idx_d, pos_d = e.read_tables()
        assert np.array_equal(idx_d, idx_o), spec
        assert np.array_equal(pos_d, pos_o), spec


@pytest.mark.parametrize("gate_version", [2, 1])
def test_config1_full_parity(gate_version):
    """1 Mbp x 1 Mbp synthetic pair (41% GC, 10% soft-masked, 200 planted
    segments at 15%), both strands: identical record list, order included,
    through the lockstep gate and through the lane-refill gate."""
    t, q = synth.config1(seed=1)
    sm = EngineConfig().sub_mat
    want, st_o = oracle_run(t, q, sm)
    with engine_for(sm) as e:
        e.set_tuning(gate_version=gate_version)
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
    assert want.size > 100
    assert got.tobytes() == want.tobytes()
    for k in ("hits", "raw_hsps", "hsps", "cells"):
        assert st[k] == st_o[k], k


def test_plain_pass_on_one_to_four_streams():
    """The plain pass runs its calls over several workspaces (host threads and
    streams; four by default); on one it must give the same records,
    statistics, kernel launches and profiled kernels, also after the target
    and the query change between passes."""
    sm = EngineConfig().sub_mat
    t1, q1 = synth.config1(seed=21, scale=0.2)
    t2, q2 = synth.config1(seed=22, scale=0.15)
    with engine_for(sm, wga_chunk=20_000) as e:
        runs = {}
        for streams in (1, 2, 3, 4):
            e.set_tuning(plain_streams=streams)
            out = []
            for t, q in ((t1, q1), (t2, q2)):
                e.load_target(t)
                e.swap_query_ascii(q)
                e.set_profiling(True)
                e.profile_reset()
                l0 = e.launches
                got, st = e.run_pass()
                prof = {k: v[1] for k, v in e.profile().items()}
                e.set_profiling(False)
                out.append((got.tobytes(), st, e.launches - l0, prof))
            runs[streams] = out
    assert st["calls"] >= 10
    for streams in (2, 3, 4):
        for one, many in zip(runs[1], runs[streams]):
            assert one[0] == many[0] and one[1] == many[1], streams
            assert one[2] == many[2] and one[3] == many[3], streams
    want, _ = oracle_run(t2, q2, sm, wga_chunk=20_000)
    assert runs[4][1][0] == want.tobytes()


@pytest.mark.parametrize("max_hits", [1000, 37, 250_000])
def test_max_hits_chunking_parity(max_hits):
    """Small MAX_HITS forces the lower_bound walk (chunk_limits,
    src/gpu/mod.rs:2394-2420); each chunk is its own dedup scope."""
    t, q = synth.config1(seed=4, scale=0.2)
    sm = EngineConfig().sub_mat
    want, st_o = oracle_run(t, q, sm, max_hits=max_hits)
    with engine_for(sm, max_hits=max_hits) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
    assert got.tobytes() == want.tobytes()
    assert (st["hits"], st["raw_hsps"], st["cells"]) == (st_o["hits"], st_o["raw_hsps"], st_o["cells"])


def test_occurrence_cap_parity():
    d = load("repeat")
    for cap in (1, 5, 29, 1000):
        want, st_o = oracle_run(d["ref_ascii"], d["qry_ascii"], d["sub_mat"], occ_cap=cap)
        with engine_for(d["sub_mat"], occ_cap=cap) as e:
            e.load_target(d["ref_ascii"])
            e.swap_query_ascii(d["qry_ascii"])
            got, st = e.run_pass()
        assert got.tobytes() == want.tobytes(), cap
        assert st["hits"] == st_o["hits"]


@pytest.mark.parametrize("kw", [dict(noentropy=True), dict(transitions=False), dict(strand="minus"),
                                dict(hspthresh=2000, xdrop=500), dict(seed="111010010100110111"),
                                dict(wga_chunk=7_000, interval=60_000)])
def test_flag_variants_parity(kw):
    t, q = synth.config1(seed=9, scale=0.15)
    sm = EngineConfig().sub_mat
    okw = dict(kw)
    if "noentropy" in okw:
        okw["noentropy"] = True
    if "strand" in okw:
        okw["strand"] = {"plus": 1, "minus": 2, "both": 3}[okw["strand"]]
    want, st_o = oracle_run(t, q, sm, **okw)
    with engine_for(sm, **kw) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
    assert got.tobytes() == want.tobytes()
    # xdrop 500 < 7 * 100: an extension dropping inside a group may not end with
    # the group's final maximum, so the gate takes its general path there
    assert (st["hits"], st["raw_hsps"], st["cells"]) == (st_o["hits"], st_o["raw_hsps"], st_o["cells"])


@pytest.mark.parametrize("cap", [128, 1024])
def test_scaled_matrix_parity(cap):
    """Scores, xdrop and threshold x 1000: gate totals can pass 2^24, where
    (i32)(f32)total may differ from total, so the gate rounds through f32."""
    t, q = synth.config1(seed=17, scale=0.1)
    sm = [v * 1000 for v in EngineConfig().sub_mat]
    want, st_o = oracle_run(t, q, sm, xdrop=910_000, hspthresh=3_000_000)
    with engine_for(sm, xdrop=910_000, hspthresh=3_000_000) as e:
        e.set_tuning(gate_cap=cap)
        e.load_target(t)
        e.swap_query_ascii(q)
        got, st = e.run_pass()
        e.stage_queries([q])
        bgot, bst = e.run_batched()
    assert len(want) > 0
    assert got.tobytes() == want.tobytes()
    assert (st["hits"], st["raw_hsps"], st["cells"]) == (st_o["hits"], st_o["raw_hsps"], st_o["cells"])
    fields = ("interval", "strand", "ref_start", "query_start", "len", "score")
    assert all((bgot[f] == got[f]).all() for f in fields) and bst["cells"] == st["cells"]


def test_single_call_uploaded_vs_generated_seeds():
    """upload_seeds (host chunk_seeds) and generate_seeds give the same call."""
    t, q = synth.config1(seed=12, scale=0.1)
    sm = EngineConfig().sub_mat
    ref = oracle.encode(t.tobytes())
    qf = oracle.encode(q.tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(ref, sh)
    start, end = 1000, 60_000
    want, st_o = oracle.seed_and_filter(oracle.params(sm), sh, ref, idx, pos, qf, start, end)
    # host seeds in chunk_seeds order (src/seed.rs:385-398)
    seeds = []
    for j in range(start, end):
        w = qf[j: j + 19]
        if np.all(w < 4):
            k = 0
            for p_ in list(sh.pos)[:12]:
                k = (k << 2) + int(qf[j + p_])
            seeds.append((k << 32) | j)
            seeds += [((k ^ (2 << (2 * t_))) << 32) | j for t_ in range(12)]
    with engine_for(sm) as e:
        e.load_target(t)
        e.swap_query_ascii(q)
        n = e.generate_seeds(0, False, (start, end))
        assert n == len(seeds) == st_o["seeds"]
        got_g, st_g = e.seed_and_filter(0, False)
        e.upload_seeds(1, np.array(seeds, dtype=np.uint64))
        got_u, st_u = e.seed_and_filter(1, False)
    assert got_g.tobytes() == want.tobytes()
    assert got_u.tobytes() == want.tobytes()
    assert st_g["hits"] == st_u["hits"] == st_o["hits"]


def test_errors_are_loud():
    sm = EngineConfig().sub_mat
    with engine_for(sm) as e:
        with pytest.raises(N.HzError) as ei:
            e.run_pass()
        assert ei.value.code == N.HZ_E_STATE  # no query swapped in (src/gpu/mod.rs:1515-1519)
        e.load_target(b"ACGT" * 100)
        e.swap_query_ascii(b"ACGT" * 50)
        with pytest.raises(N.HzError):
            e.generate_seeds(0, False, (0, 190))  # window past the query end
        with pytest.raises(N.HzError):
            e.upload_seeds(0, np.array([(1 << 56) | 5], dtype=np.uint64))
            e.seed_and_filter(0, False)
        with pytest.raises(N.HzError):
            e.load_tables(np.zeros(10, np.uint32), np.zeros(0, np.uint32), np.zeros(5, np.uint8))


def test_tiny_and_empty_inputs():
    sm = EngineConfig().sub_mat
    with engine_for(sm) as e:
        e.load_target(b"")
        e.swap_query_ascii(b"ACGTACGTACGTACGTACG")
        recs, st = e.run_pass()
        assert recs.size == 0 and st["hits"] == 0
        e.load_target(b"ACGTTGCA" * 10)
        e.swap_query_ascii(b"")
        recs, st = e.run_pass()
        assert recs.size == 0


def test_plain_form_device_dedup_for_large_calls():
    """A plain-form call with many raw HSPs dedups on the device; with the
    threshold at 1 every call does, and the records stay the oracle's."""
    t, q = synth.config1(seed=4, scale=0.2)
    sm = EngineConfig().sub_mat
    want, _ = oracle_run(t, q, sm)
    with engine_for(sm) as e:
        e.set_tuning(device_dedup_min=1)
        e.load_target(t)
        e.swap_query_ascii(q)
        got, _ = e.run_pass()
    assert want.size > 10
    assert got.tobytes() == want.tobytes()


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_files_in_files_out_reproduce_the_frozen_digests(tmp_path, form):
    """Sequence files -> device seed table -> pass -> .segments files: the
    frozen smoke digests, with the inputs as FASTA and as gzipped FASTA."""
    import gzip
    import shutil
    from hspz_b200.pipeline import seed_and_filter_files
    from tests.golden.fixture_pass import FIXTURES
    for name in sorted(EXPECTED):
        d = load(name)
        ref = os.path.join(FIXTURES, f"{name}.ref.fa")
        qry = tmp_path / f"{name}.qry.fa.gz"
        with open(os.path.join(FIXTURES, f"{name}.qry.fa"), "rb") as src, gzip.open(qry, "wb") as dst:
            shutil.copyfileobj(src, dst)
        out = tmp_path / f"out_{name}_{form}"
        files = seed_and_filter_files(ref, qry, out_dir=str(out), form=form,
                                      config=EngineConfig(sub_mat=d["sub_mat"], max_hits=MAX_HITS))
        n, digest = H.sorted_digest(files)
        assert (n, len(files), digest) == (EXPECTED[name]["hsps"], EXPECTED[name]["files"],
                                           EXPECTED[name]["digest"]), name
        assert sorted(os.listdir(out)) == sorted(files)


@pytest.mark.parametrize("ambiguous", ["n", "iupac", "iupac,5,7"])
def test_ambiguous_scoring_parity(ambiguous):
    """--ambiguous scoring (N and IUPAC codes rewarded or penalised) on the
    fixture with ambiguous bases: the oracle's records."""
    from hspz_b200.scoring import build_sub_mat
    d = load("ambiguous")
    sm = build_sub_mat(ambiguous, 910)
    want, st_o = oracle_run(d["ref_ascii"], d["qry_ascii"], sm, max_hits=MAX_HITS)
    with engine_for(sm, max_hits=MAX_HITS) as e:
        e.load_target(d["ref_ascii"])
        e.swap_query_ascii(d["qry_ascii"])
        got, st = e.run_pass()
    assert got.tobytes() == want.tobytes()
    assert (st["hits"], st["cells"]) == (st_o["hits"], st_o["cells"])
