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
    args = types.SimpleNamespace(config=2, scale=0.001, warmup=0, steps=1, cpu_batches=1, gpus=2)
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        bench.run_reference(args, rank=1)
    assert buf.getvalue() == ""
