"""bench.py's multi-rank logic on CPU: world_size-2 gloo ranks reduce the
timed window (max over ranks) and the work done (sum over ranks) the way the
NCCL ranks do on GPUs, and non-zero ranks print nothing."""
import contextlib
import io
import os
import socket
import types

import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = bench.over_ranks([10.0 + 5 * rank], "max", torch.device("cpu"))
        tot = bench.over_ranks([100 * (rank + 1), rank], "sum", torch.device("cpu"))
        out.put((rank, ms, tot))
    finally:
        dist.destroy_process_group()


def test_reductions_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get() for _ in range(2))
    for rank, ms, tot in got:
        assert ms == [15.0]          # the slowest rank's window
        assert tot == [300.0, 1.0]   # work of both ranks


def test_reference_arm_prints_only_on_rank_zero():
    args = types.SimpleNamespace(config=2, scale=0.001, warmup=0, steps=1, ref_frac=0.01, gpus=2)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, rank=1)
    assert buf.getvalue() == ""


def test_reference_arm_prints_the_contract_line():
    """bench.py --impl reference on a small CPU case: one JSON line with the
    contract's keys, its cpu_baseline and e2e describing the same run."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--config", "1",
                          "--scale", "0.05", "--steps", "1", "--warmup", "0"],
                         capture_output=True, text=True, timeout=300, check=True).stdout
    lines = [l for l in out.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
              "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["cpu_baseline"]["value"] == d["value"] and d["cpu_baseline"]["kind"] == "port"
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}


def test_sample_call_counts_match_the_oracle_batch_list():
    """The CPU sample's 'first n intervals' equals that many calls of the
    reference's batch order (per interval: plus chunks, then minus chunks)."""
    import ctypes as C

    import numpy as np
    import oracle
    L = oracle.lib()
    for qlen in (5_000, 250_019, 9_999_999, 10_000_019, 23_456_789, 100_000_000):
        nb = L.hzo_batches(qlen, 19, 10_000_000, 250_000, 3, None)
        b = np.zeros((max(nb, 1), 4), dtype=np.uint32)
        L.hzo_batches(qlen, 19, 10_000_000, 250_000, 3, b.ctypes.data_as(C.c_void_p))
        for n_iv in (1, 2, 3):
            want = int(np.sum(b[:nb, 0] < n_iv))
            assert bench.CpuOracle._calls_in_intervals(qlen, n_iv) == want, (qlen, n_iv)


def test_parity_digest_is_the_sorted_set():
    import numpy as np
    from hspz_b200.hsp import PASS_RECORD
    a = np.zeros(4, dtype=PASS_RECORD)
    a["strand"] = [1, 0, 0, 1]
    a["ref_start"] = [5, 9, 2, 5]
    a["score"] = [3000, 3100, 3200, 3300]
    b = a[::-1].copy()
    assert bench.parity_digest([a]) == bench.parity_digest([b])
    c = a.copy()
    c["len"][2] = 1
    assert bench.parity_digest([a]) != bench.parity_digest([c])
    assert bench.parity_digest([a[:2], a[2:]]) != bench.parity_digest([a])  # per-query boundaries count


def test_reference_arm_on_the_chunked_workload():
    """The default (chunked) workload's reference arm: a seeded sample of
    whole chunks per step, and a config that names the batched form like the
    GPU arm's line."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--impl", "reference", "--config", "3",
                          "--scale", "0.002", "--steps", "1", "--warmup", "0", "--ref-frac", "0.05"],
                         capture_output=True, text=True, timeout=300, check=True).stdout
    d = json.loads([l for l in out.splitlines() if l.startswith("{")][0])
    assert d["config"]["form"] == "batched" and d["config"]["queries"] == 512
    assert "query chunks" in d["cpu_baseline"]["sample"] and d["value"] > 0
