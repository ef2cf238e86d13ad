"""Pins the CPU oracle to the reference's own golden answers before anything
is compared against it.

* The frozen smoke digests (assets/container/smoke.sh:11-12,78-79):
  repeat -> 57 HSPs in 1 file, d01edd2118cf5fa5; multi -> 3 HSPs in 2 files,
  0da3bbda656e4f7b, at --max-hits 16711680.
* The unit-test expectations of src/seed.rs, src/hsp.rs, src/scoring.rs and
  src/gpu/mod.rs (cited per test).
"""
import json
import os

import numpy as np
import pytest

import oracle
from hspz_b200 import hsp as H
from hspz_b200 import scoring
from hspz_b200 import sequence as S
from tests.golden.fixture_pass import oracle_pass

EXPECTED = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "expected.json")))


@pytest.mark.parametrize("name", ["repeat", "multi"])
def test_frozen_smoke_digests(name):
    n, files, digest, _ = oracle_pass(name)
    want = {"repeat": (57, 1, "d01edd2118cf5fa5"), "multi": (3, 2, "0da3bbda656e4f7b")}[name]
    assert (n, files, digest) == want


@pytest.mark.parametrize("name", sorted(EXPECTED))
def test_all_fixtures_match_recorded_answers(name):
    n, files, digest, st = oracle_pass(name)
    e = EXPECTED[name]
    assert (n, files, digest) == (e["hsps"], e["files"], e["digest"])
    assert (st["seeds"], st["hits"], st["raw_hsps"], st["cells"]) == (e["seeds"], e["hits"], e["raw_hsps"], e["cells"])


def test_shape_12of19_matches_kegalign():  # src/seed.rs:502-509
    s = oracle.shape("12of19")
    assert (s.size, s.kmer_size) == (19, 12)
    assert list(s.pos)[:12] == [0, 1, 2, 4, 7, 8, 11, 13, 15, 16, 17, 18]
    assert all(s.transition[i] for i in range(12))
    with pytest.raises(ValueError):
        oracle.shape("101")


def test_seed_table_skips_position_zero():  # src/seed.rs:614-623
    sh = oracle.shape("1111")
    idx, pos = oracle.seed_table(oracle.encode(b"AAAAACGTA"), sh)
    assert pos.size == 5
    assert list(pos[: idx[0]]) == [1]
    assert idx[-1] == 5


def test_seed_table_buckets_ascending_with_separators_and_masks():  # src/seed.rs:546-597
    rng = np.random.default_rng(7)
    seq = rng.choice(np.frombuffer(b"ACGTNacgt&", dtype=np.uint8), size=40000,
                     p=[.24, .24, .24, .2, .02, .015, .015, .015, .01, .005])
    codes = oracle.encode(seq.tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(codes, sh)
    starts = np.concatenate([[0], idx[:-1]])
    nz = np.nonzero(idx - starts)[0]
    for k in nz[:2000]:
        b = pos[starts[k]: idx[k]]
        assert np.all(np.diff(b.astype(np.int64)) > 0)
    # every indexed position's window is all-uppercase ACGT
    for p in pos[:2000]:
        assert np.all(codes[p: p + 19] < 4)


def test_chunking_matches_seeder_loop():  # src/seed.rs:648-656
    assert S.chunks(0, 376657, 250_000) == [(0, 250_000), (250_000, 376_658)]
    assert S.chunks(0, 10, 250_000) == [(0, 11)]


def test_encode_and_revcomp_match_oracle():  # src/sequence.rs:66-86
    allb = bytes(range(256))
    assert np.array_equal(S.encode(allb), oracle.encode(allb))
    assert np.array_equal(S.reverse_complement_bytes(allb), oracle.revcomp(allb))
    assert list(S.encode(b"Acgt&")) == [0, 4, 4, 4, 7]
    # the device rc table == encode(revcomp(c)) per byte
    assert np.array_equal(S.ENCODE_RC_TABLE, oracle.encode(oracle.revcomp(allb)[::-1].tobytes()))


def test_default_sub_mat_matches_kegalign():  # src/scoring.rs:295-306
    m = scoring.build_sub_mat("", 910)
    assert m[0] == 91 and m[3] == -123 and m[2 * 8 + 2] == 100
    assert m[4 * 8 + 4] == -1000 and m[5 * 8 + 5] == -1000 and m[6 * 8 + 6] == -100
    assert m[7 * 8 + 7] == -9100 and m[7] == -9100
    n = scoring.build_sub_mat("n", 910)
    assert n[5 * 8 + 5] == 0 and n[5] == 0 and n[6 * 8 + 6] == -100
    t = scoring.build_sub_mat("iupac,5,7", 910)
    assert t[5 * 8 + 5] == 5 and t[5] == -7 and t[6 * 8 + 6] == 5


def test_dedup_compares_against_previous_input():  # src/hsp.rs:334-361
    sp = lambda r, q, l, s: (r, q, l, s)
    v = np.array([sp(0, 0, 5, 10), sp(0, 0, 10, 20), sp(6, 6, 2, 30)], dtype=oracle.HSP_DTYPE)
    assert oracle.dedup_and_order(v).tolist() == [(0, 0, 5, 10)]
    v = np.array([sp(0, 0, 10, 50), sp(0, 0, 5, 40), sp(6, 6, 2, 30), sp(0, 1, 4, 20)], dtype=oracle.HSP_DTYPE)
    got = oracle.dedup_and_order(v).tolist()
    assert len(got) == 2 and (0, 1, 4, 20) in got and (0, 0, 5, 40) in got
    # the host mirror agrees with the oracle on random inputs
    rng = np.random.default_rng(3)
    for _ in range(50):
        a = np.zeros(40, dtype=oracle.HSP_DTYPE)
        a["ref_start"] = rng.integers(0, 30, 40)
        a["query_start"] = rng.integers(0, 30, 40)
        a["len"] = rng.integers(0, 12, 40)
        a["score"] = rng.integers(0, 5, 40)
        assert oracle.dedup_and_order(a).tolist() == H.dedup_and_order(a).tolist()


def test_ln_series_is_close_to_libm():  # src/gpu/kernels.rs:1879-1908
    # The series stops at z^7 (z <= 0.0295), so its truncation error near a
    # reduced mantissa of sqrt(2) is ~4e-14 relative; parity needs the same
    # series on both sides, not libm accuracy.
    for x in [1.0, 0.5, 0.25, 1e-3, 0.3333333333, 0.999999, 0.7071, 0.70710678118654757]:
        assert abs(oracle.ln(x) - np.log(x)) < 1e-13 * max(1.0, abs(np.log(x)))


def test_chunk_limits_walk():  # src/gpu/mod.rs:2644-2668
    assert oracle.chunk_limits([2, 5, 9], 1000) == [(0, 2, 0, 9)]
    ch = oracle.chunk_limits([3, 7, 11, 15], 5)
    assert len(ch) == 4
    assert ch[0] == (0, 0, 0, 3)  # the first chunk stops before overshooting 5
    assert all(b[0] == a[1] + 1 for a, b in zip(ch, ch[1:]))  # chunks tile the seed range
    assert ch[-1][1] == 3
    with pytest.raises(ValueError):  # a first seed above the limit has no cut
        oracle.chunk_limits([10, 12], 5)


def test_gate_threshold_uses_the_f32_rounded_total():  # src/gpu/kernels.rs:2029-2042
    import struct
    f32 = lambda v: struct.unpack("f", struct.pack("f", float(v)))[0]
    right, left, threshold = 1400, 1600, 3000
    assert right < threshold and int(f32(right + left)) >= threshold
    raw, threshold = 16_777_219, 16_777_220  # above 2^24 the f32 conversion can round up
    assert raw < threshold and int(f32(raw)) >= threshold


def test_shapes_and_kmers_restated():  # src/seed.rs:512-538
    from hspz_b200 import _native as N
    from hspz_b200 import shape_info
    assert shape_info("1111") == (4, 4)
    assert shape_info("11011") == (5, 4)
    for bad in ("101", "1" * 16):  # care positions must number 4..15
        with pytest.raises(N.HzError):
            shape_info(bad)
    # "1111" packs A C G T as 00 01 10 11; a separator anywhere in the window
    # (a don't-care position included) kills it; step 1 skips position 0
    for spec, seq, k, want in (("1111", b"AACGTA&ACGTT", 0b00011011, [1, 7]),
                               ("11011", b"TACAGT&AC&GT", 0b00011011, [1])):
        idx, pos = oracle.seed_table(oracle.encode(seq), oracle.shape(spec))
        lo = int(idx[k - 1]) if k else 0
        assert pos[lo: int(idx[k])].tolist() == want, spec
