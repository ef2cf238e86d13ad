"""One reference-bin x query-bin unit end to end, from sequence files to
``.segments`` files: the host flow around the path that hspZ's ``run_bins``
(src/run.rs:816-887) and ``Emitter::emit_unit`` (src/run.rs:568-626) drive,
over this library's engine.

    files = seed_and_filter_files("ref.2bit", "qry.fa.gz", out_dir="out")

Both inputs are read by magic bytes (FASTA, FASTA.gz or 2bit) and packed as
one block each; the reference's seed table is built on the device; the query
runs as one pass in the batched form (or the plain per-chunk form) and the
records are rendered by the native writer, optionally cut by the -D
partition.  A file-level planner (several bins, several GPUs) stays out of
this module: callers loop over their own bins.
"""
from __future__ import annotations

import os
from typing import Dict, Optional

from . import hsp as H
from .engine import Engine, EngineConfig
from .partition import Partitioner
from .sequence import load_genome


def seed_and_filter_files(target_path, query_path, out_dir: Optional[str] = None,
                          config: Optional[EngineConfig] = None, form: str = "batched",
                          partition: bool = False, ref_prefix: str = "", query_prefix: str = "",
                          ref_bin: int = 0, query_bin: int = 0, device: int = 0) -> Dict[str, str]:
    """{file name: text} of the unit; written into ``out_dir`` when given."""
    if form not in ("batched", "plain"):
        raise ValueError("form must be 'batched' or 'plain'")
    ref = load_genome(target_path, ref_prefix)
    qry = load_genome(query_path, query_prefix)
    _, rc_chrs = qry.reverse_complement()
    with Engine(config or EngineConfig(), device=device) as e:
        e.load_target(ref.buf[: ref.block_len])
        if form == "batched":
            e.stage_queries([qry.buf[: qry.block_len]])
            recs, _ = e.run_batched()
        else:
            e.swap_query_ascii(qry.buf[: qry.block_len])
            recs, _ = e.run_pass()
    files = H.emit_unit(recs, ref.chrs, qry.chrs, rc_chrs, query_bin=query_bin, ref_bin=ref_bin,
                        partitioner=Partitioner() if partition else None)
    if out_dir is not None:
        os.makedirs(out_dir, exist_ok=True)
        for name, text in files.items():
            with open(os.path.join(out_dir, name), "w") as fh:
                fh.write(text)
    return files
