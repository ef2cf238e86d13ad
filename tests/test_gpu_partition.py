"""-D end to end on the GPU: FASTA files in, .segments files out through the
device pass and the diagonal partition (src/partition.rs:62-196), checked
file by file against the oracle's records of the same inputs cut by the same
restated rules, and against the unpartitioned output line for line."""
import numpy as np
import pytest

import oracle
from hspz_b200 import EngineConfig, synth
from hspz_b200 import hsp as H
from hspz_b200.partition import MIN_CHUNK_SIZE, Partitioner
from hspz_b200.pipeline import seed_and_filter_files
from hspz_b200.sequence import load_genome
from hspz_b200.build import build

pytestmark = pytest.mark.gpu

MAX_HITS = 16711680
INTERVAL = 1_000_000  # several LASTZ intervals, so the partitioner has earlier outputs to size chunks from


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


def write_fasta(path, records):
    with open(path, "w") as fh:
        for name, seq in records:
            fh.write(f">{name}\n")
            s = seq.tobytes().decode()
            for a in range(0, len(s), 80):
                fh.write(s[a:a + 80] + "\n")


@pytest.fixture(scope="module")
def inputs(tmp_path_factory):
    """A four-record target and a three-record query whose second LASTZ
    interval is packed with short copies of the target (thousands of HSPs in
    one output, across several chromosome pairs); the first interval holds
    far fewer."""
    rng = np.random.default_rng(91)
    target = [synth.random_bases(rng, 600_000) for _ in range(4)]
    flat = np.concatenate(target)

    def copies(n, lo, hi):
        out = []
        for _ in range(n):
            L = int(rng.integers(lo, hi))
            a = int(rng.integers(0, flat.size - L))
            seg = synth.mutate(rng, flat[a:a + L], 0.03)
            out += [seg, synth.random_bases(rng, int(rng.integers(5, 15)))]
        return np.concatenate(out)

    sparse = np.concatenate([synth.random_bases(rng, 900_000), copies(600, 100, 140)])[:INTERVAL - 50_000]
    dense = copies(8000, 95, 105)
    tail = synth.random_bases(rng, 200_000)
    q = np.concatenate([sparse, dense, tail])
    cuts = [0, 700_000, 1_500_000, q.size]
    query = [q[cuts[i]:cuts[i + 1]] for i in range(3)]
    d = tmp_path_factory.mktemp("part")
    ref_path, qry_path = str(d / "ref.fa"), str(d / "qry.fa")
    write_fasta(ref_path, [(f"chr{i + 1}", s) for i, s in enumerate(target)])
    write_fasta(qry_path, [(f"q{i + 1}", s) for i, s in enumerate(query)])
    return ref_path, qry_path


def oracle_files(ref_path, qry_path, partition):
    ref, qry = load_genome(ref_path), load_genome(qry_path)
    qrc, rc_chrs = qry.reverse_complement()
    r = oracle.encode(ref.buf[: ref.block_len].tobytes())
    qf = oracle.encode(qry.buf[: qry.block_len].tobytes())
    qr = oracle.encode(qrc.tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(r, sh)
    p = oracle.params(EngineConfig().sub_mat, max_hits=MAX_HITS, interval=INTERVAL, threads=8)
    out, _ = oracle.seed_and_filter_all(p, sh, r, idx, pos, qf, qr)
    return H.emit_unit(out, ref.chrs, qry.chrs, rc_chrs, partitioner=Partitioner() if partition else None)


@pytest.mark.parametrize("form", ["batched", "plain"])
def test_partitioned_output_equals_the_oracle_files(inputs, form):
    ref_path, qry_path = inputs
    cfg = EngineConfig(max_hits=MAX_HITS, interval=INTERVAL)
    got = seed_and_filter_files(ref_path, qry_path, config=cfg, form=form, partition=True)
    want = oracle_files(ref_path, qry_path, partition=True)
    split = [k for k in got if ".split" in k]
    assert len(split) >= 2  # the dense output was cut
    assert sorted(got) == sorted(want)
    for name in want:
        assert got[name] == want[name], name


def test_split_files_hold_exactly_the_unsplit_lines(inputs):
    ref_path, qry_path = inputs
    cfg = EngineConfig(max_hits=MAX_HITS, interval=INTERVAL)
    whole = seed_and_filter_files(ref_path, qry_path, config=cfg, partition=False)
    parts = seed_and_filter_files(ref_path, qry_path, config=cfg, partition=True)
    lines = lambda files: sorted(l for t in files.values() for l in t.splitlines())
    assert lines(whole) == lines(parts)
    # the output that was cut reached the partition threshold
    for stem in {k.split(".split")[0] for k in parts if ".split" in k}:
        assert whole[stem + ".segments"].count("\n") >= MIN_CHUNK_SIZE
