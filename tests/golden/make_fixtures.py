"""Regenerates tests/golden/fixtures/ from the reference's own fixture
generator (hspZ assets/tests/gen_fixtures.py, deterministic seed 20260811).

Run with the root of an hspZ checkout, as an argument or in HSPZ_REFERENCE:
    python tests/golden/make_fixtures.py /path/to/hspZ
The FASTA files it writes are committed, so nothing at test time needs the
reference.  expected.json records, per fixture, the HSP count, file count and
sorted digest; `repeat` and `multi` are the reference's frozen smoke answers
(assets/container/smoke.sh:11-12), the rest are the oracle's answers on the
same bytes.
"""
import importlib.util
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    spec = importlib.util.spec_from_file_location(
        "gen_fixtures", os.path.join(ref_root, "assets", "tests", "gen_fixtures.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.main(os.path.join(HERE, "fixtures"))
    write_expected()


# The reference's frozen smoke answers (assets/container/smoke.sh:11-12,78-79).
FROZEN = {"repeat": (57, 1, "d01edd2118cf5fa5"), "multi": (3, 2, "0da3bbda656e4f7b")}


def write_expected():
    import json
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from tests.golden.fixture_pass import oracle_pass

    out = {}
    for name in sorted(f[:-7] for f in os.listdir(os.path.join(HERE, "fixtures")) if f.endswith(".ref.fa")):
        n, nfiles, digest, stats = oracle_pass(name)
        if name in FROZEN and FROZEN[name] != (n, nfiles, digest):
            raise SystemExit(f"oracle disagrees with the frozen answer for {name}")
        out[name] = {"hsps": n, "files": nfiles, "digest": digest, "seeds": stats["seeds"],
                     "hits": stats["hits"], "raw_hsps": stats["raw_hsps"], "cells": stats["cells"],
                     "frozen_by_reference": name in FROZEN}
    with open(os.path.join(HERE, "expected.json"), "w") as fh:
        json.dump(out, fh, indent=1, sort_keys=True)


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("HSPZ_REFERENCE")
    if not root:
        raise SystemExit("usage: make_fixtures.py <hspZ checkout> (or set HSPZ_REFERENCE)")
    main(root)
