"""Host-side mirror of the reference's config surface: scoring files
(src/scoring.rs tests :280-404), sequence helpers and synthetic inputs."""
import numpy as np
import pytest

from hspz_b200 import scoring, synth
from hspz_b200 import sequence as S
from hspz_b200.scoring import DEFAULT_ACGT, ScoringError, load_scoring_matrix


def write(tmp_path, name, body):
    p = tmp_path / name
    p.write_text(body)
    return str(p)


def test_reads_the_documented_lastz_example(tmp_path):
    p = write(tmp_path, "ex", "# blastz default\nbad_score = X:-1000\nfill_score = -100\n"
              "gap_open_penalty = 30\ngap_extend_penalty = 400\n\n"
              "     A     C     G     T\nA   91  -114   -31  -123\nC -114   100  -125   -31\n"
              "G  -31  -125   100  -114\nT -123   -31  -114    91\n")
    assert load_scoring_matrix(p) == DEFAULT_ACGT
    assert scoring.build_sub_mat("", 910, p) == scoring.build_sub_mat("", 910)


def test_blastz_rows_without_labels(tmp_path):
    p = write(tmp_path, "bz", "  A C G T\n 91 -114 -31 -123\n-114 100 -125 -31\n-31 -125 100 -114\n-123 -31 -114 91\n")
    assert load_scoring_matrix(p) == DEFAULT_ACGT


def test_undefined_pairs_take_fill(tmp_path):
    m = load_scoring_matrix(write(tmp_path, "p", "fill_score = -7\n   A\nA  5\n"))
    assert m[0][0] == 5 and m[1][1] == -7 and m[3][0] == -7


@pytest.mark.parametrize("body,want", [
    ("  A  C\nA 1 2\nC 3\n", "where the rows above have 3"),
    ("  A  C\nA 1 2 3 4\n", "holds 2 scores, optionally after its symbol"),
    ("  A\nA 1.5\n", "is not an integer score"),
    ("  A~T\nA 1\n", "quantum-alphabet symbol"),
    ("fill_score = -1\n", "no matrix header line"),
    ("  A  C\n", "column symbols but no rows"),
])
def test_rejects_malformed(tmp_path, body, want):
    with pytest.raises(ScoringError, match=want):
        load_scoring_matrix(write(tmp_path, "bad", body))


def test_bad_score_aimed_at_a_nucleotide(tmp_path):
    m = load_scoring_matrix(write(tmp_path, "b", "bad_score = A:-500\n  A  C\nA 1 2\nC 3 4\n"))
    assert m[0][0] == -500 and m[0][1] == -500 and m[1][0] == -500 and m[1][1] == 4


def test_intervals_and_batches():
    assert S.intervals(19, 19, 10) == []
    assert S.intervals(100, 19, 50) == [(0, 50), (50, 81)]
    b = S.batches(100, 19, 50, 30)
    # per interval: plus chunks, then minus chunks over (qbl - end, qbl - start)
    assert b[:3] == [(0, False, 0, 30), (0, False, 30, 51), (0, True, 31, 61)]


def test_pack_and_revcomp_remap():
    buf, chrs, bl = S.pack([("a", b"ACGT"), ("b", b"GG")])
    assert bytes(buf) == b"ACGT&GG&" and bl == 7
    rc, rchrs = S.reverse_complement(buf, chrs, bl)
    assert bytes(rc) == b"CC&ACGT"
    assert [(c.name, c.start, c.len) for c in rchrs] == [("b", 0, 2), ("a", 3, 4)]
    assert S.chr_at(chrs, 0) == 0 and S.chr_at(chrs, 5) == 1


def test_synthetic_inputs_are_seeded():
    a1, b1 = synth.config1(seed=5, scale=0.01)
    a2, b2 = synth.config1(seed=5, scale=0.01)
    assert np.array_equal(a1, a2) and np.array_equal(b1, b2)
    low = np.mean((a1 >= ord("a")))
    assert 0.03 < low < 0.2
    gc = np.mean(np.isin(a1 & 0xDF, np.frombuffer(b"GC", dtype=np.uint8)))
    assert 0.37 < gc < 0.45


def test_ambiguous_scoring_variants():  # src/scoring.rs:295-323
    from hspz_b200.scoring import build_sub_mat
    nuc = 8
    m = build_sub_mat("", 910)
    assert (m[2 * nuc + 2], m[4 * nuc + 4], m[5 * nuc + 5]) == (100, -1000, -1000)
    assert (m[6 * nuc + 6], m[7 * nuc + 7], m[7]) == (-100, -9100, -9100)
    m = build_sub_mat("n", 910)
    assert (m[5 * nuc + 5], m[5], m[6 * nuc + 6]) == (0, 0, -100)
    m = build_sub_mat("iupac,5,7", 910)
    assert (m[5 * nuc + 5], m[5], m[6 * nuc + 6]) == (5, -7, 5)
