"""The output side of a pass: .segments records, the native renderer, the
per-unit file naming and the -D diagonal partition (src/hsp.rs:179-292,
src/run.rs:568-626, src/partition.rs).  Host code only."""
import numpy as np
import pytest

import oracle
from hspz_b200 import _native as N
from hspz_b200 import hsp as H
from hspz_b200 import partition as P
from hspz_b200 import sequence as S
from hspz_b200.build import build
from tests.golden.fixture_pass import MAX_HITS, load

EXPECTED = {"repeat": (57, 1, "d01edd2118cf5fa5"), "multi": (3, 2, "0da3bbda656e4f7b")}


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


def random_hsps(seed, n, chrs):
    rng = np.random.default_rng(seed)
    h = np.zeros(n, dtype=H.SEGMENT_PAIR)
    end = chrs[-1].start + chrs[-1].len
    h["ref_start"] = rng.integers(0, end - 1000, n)
    h["query_start"] = rng.integers(0, end - 1000, n)
    h["len"] = rng.integers(0, 900, n)
    h["score"] = rng.integers(-5000, 90000, n)
    return h


def test_native_renderer_equals_the_restatements():
    chrs = [S.Chr(f"chr{i}", i * 100_001, 100_000) for i in range(7)]
    h = random_hsps(3, 5000, chrs)
    for strand in "+-":
        recs = H.records(h, chrs, chrs, strand)
        native = H.render_records(recs, chrs, chrs, strand)
        assert native == H.render_records_py(recs, chrs, chrs, strand)
        assert native == H.render_segments(h, chrs, chrs, strand)
    assert H.render_records(H.records(h[:0], chrs, chrs, "+"), chrs, chrs, "+") == ""


def test_native_renderer_refuses_unknown_chromosomes():
    chrs = [S.Chr("a", 0, 10)]
    recs = np.zeros(1, dtype=H.RECORD)
    recs["q_chr"] = 3
    with pytest.raises(N.HzError) as ex:
        H.render_records(recs, chrs, chrs, "+")
    assert ex.value.code == N.HZ_E_INVALID


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_emitted_files_reproduce_the_frozen_digests(name):
    d = load(name)
    ref = oracle.encode(d["ref_ascii"].tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(ref, sh)
    p = oracle.params(d["sub_mat"], max_hits=MAX_HITS, threads=2)
    out, _ = oracle.seed_and_filter_all(p, sh, ref, idx, pos, oracle.encode(d["qry_ascii"].tobytes()),
                                        oracle.encode(d["qrc_ascii"].tobytes()))
    native = H.emit_unit(out, d["rchrs"], d["qchrs"], d["rcchrs"])
    assert native == H.render_pass(out, d["rchrs"], d["qchrs"], d["rcchrs"])
    n, digest = H.sorted_digest(native)
    assert (n, len(native), digest) == EXPECTED[name]


# ---- -D diagonal partition (the reference's unit tests, src/partition.rs:199-302) ----

def rec(rc, qc, rs, qs, ln, score=100):
    r = np.zeros(1, dtype=H.RECORD)
    r["r_chr"], r["q_chr"], r["r_start"], r["r_end"] = rc, qc, rs, rs + ln
    r["q_start"], r["q_end"], r["score"] = qs, qs + ln, score
    return r


def cat(rs):
    return np.concatenate(rs)


def test_plus_sorts_by_sum_minus_by_difference():
    a, b, c = rec(0, 0, 100, 10, 0), rec(0, 0, 10, 100, 0), rec(0, 0, 1, 1, 0)
    k = lambda r, s: int(P.diagonal_key(r, s)[0][0])
    assert k(c, "+") == 2
    assert k(a, "+") == k(b, "+")
    assert k(a, "-") < k(c, "-") < k(b, "-")


def test_midpoint_uses_the_reference_half_length():
    k0, k1 = P.diagonal_key(rec(0, 0, 10, 100, 7), "+")
    assert (int(k0[0]), int(k1[0])) == (13 + 103, 13)


def test_chunk_size_estimation():
    p = P.Partitioner()
    assert p.chunk_size_for(P.MIN_CHUNK_SIZE - 1) is None
    assert p.chunk_size_for(P.MAX_CHUNK_SIZE) is None
    assert p.chunk_size_for(P.MAX_CHUNK_SIZE + 1) == P.MAX_CHUNK_SIZE
    for c in (6000, 8000, 10000):
        p.observe(c)
    assert p.chunk_size_for(9000) == 8000          # fewer than 7 outputs: the median
    for c in (12000, 14000, 16000, 18000):
        p.observe(c)
    assert p.chunk_size_for(20000) == 16000        # 7 or more: the upper quartile
    assert p.chunk_size_for(15000) is None         # fits in one chunk


def test_quantiles_match_the_exclusive_method():
    q = P.quantiles_exclusive([1, 2, 3, 4])
    assert np.allclose(q, (1.25, 2.5, 3.75))
    assert P.quantiles_exclusive([5]) is None


def test_a_single_pair_is_split_even_when_it_would_fit():
    files = P.split(cat([rec(0, 0, i * 10, i * 10, 5) for i in range(10)]), "+", 4)
    assert [f.size for f in files] == [4, 4, 2]


def test_small_pairs_are_aggregated():
    recs = cat([rec(0, 0, i * 10, i * 10, 1) for i in range(6)] + [rec(1, 1, i * 10, i * 10, 1) for i in range(2)]
               + [rec(2, 2, i * 10, i * 10, 1) for i in range(2)])
    files = P.split(recs, "+", 4)
    assert sorted(f.size for f in files) == [2, 4, 4]
    assert sum(f.size for f in files) == 10


def test_partition_union_preserves_the_multiset():
    recs = cat([rec(c, c, i * 3, i * 5, 2) for c in range(3) for i in range(7)])
    files = P.split(recs, "-", 3)
    key = lambda a: sorted(zip(a["r_chr"].tolist(), a["q_chr"].tolist(), a["r_start"].tolist(),
                               a["q_start"].tolist(), a["score"].tolist()))
    assert key(np.concatenate(files)) == key(recs)


def test_emit_unit_names_split_files():
    chrs = [S.Chr("r", 0, 5_000_000)]
    rng = np.random.default_rng(9)
    n = 12_000
    pr = np.zeros(n, dtype=H.PASS_RECORD)
    pr["ref_start"] = np.sort(rng.integers(0, 4_000_000, n))
    pr["query_start"] = rng.integers(0, 4_000_000, n)
    pr["len"] = 50
    pr["score"] = 4000
    part = P.Partitioner()
    part.observe(2000)
    part.observe(3000)
    # the plan counts this output too: sizes 2000, 3000, 12000 -> median chunk 3000
    files = H.emit_unit(pr, chrs, chrs, chrs, query_bin=2, ref_bin=1, partitioner=part)
    assert list(files) == [f"tmp1.block2.r1.plus.split{k}.segments" for k in range(1, 5)]
    assert [t.count("\n") for t in files.values()] == [3000] * 4
    assert sum(t.count("\n") for t in files.values()) == n
    whole = H.emit_unit(pr, chrs, chrs, chrs, query_bin=2, ref_bin=1)
    assert list(whole) == ["tmp1.block2.r1.plus.segments"]
    assert sorted(whole["tmp1.block2.r1.plus.segments"].splitlines()) == \
        sorted(l for t in files.values() for l in t.splitlines())
