"""Loads one golden fixture and runs it through the oracle: the shared
set-up of tests/test_oracle_golden.py and the GPU parity tests."""
import os

import oracle
from hspz_b200 import hsp as H
from hspz_b200 import scoring
from hspz_b200 import sequence as S

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = os.path.join(HERE, "fixtures")
MAX_HITS = 16711680  # the smoke value, pinned (assets/container/smoke.sh:20)


def load(name):
    """Packed + encoded inputs of a fixture, the way a run prepares them
    (src/run.rs:70-130)."""
    r = S.read_fasta(os.path.join(FIXTURES, f"{name}.ref.fa"))
    q = S.read_fasta(os.path.join(FIXTURES, f"{name}.qry.fa"))
    rbuf, rchrs, rbl = S.pack(r)
    qbuf, qchrs, qbl = S.pack(q)
    qrc, rcchrs = S.reverse_complement(qbuf, qchrs, qbl)
    sm_path = os.path.join(FIXTURES, "scoring.matrix") if name == "scoring" else None
    return dict(ref_ascii=rbuf[:rbl], qry_ascii=qbuf[:qbl], qrc_ascii=qrc, rchrs=rchrs, qchrs=qchrs,
                rcchrs=rcchrs, sub_mat=scoring.build_sub_mat("", 910, sm_path))


def oracle_pass(name, **kw):
    d = load(name)
    ref = oracle.encode(d["ref_ascii"].tobytes())
    qf = oracle.encode(d["qry_ascii"].tobytes())
    qr = oracle.encode(d["qrc_ascii"].tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(ref, sh)
    p = oracle.params(d["sub_mat"], max_hits=kw.get("max_hits", MAX_HITS), threads=2)
    out, st = oracle.seed_and_filter_all(p, sh, ref, idx, pos, qf, qr)
    files = H.render_pass(out, d["rchrs"], d["qchrs"], d["rcchrs"])
    n, digest = H.sorted_digest(files)
    return n, len(files), digest, st
