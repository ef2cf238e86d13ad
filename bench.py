#!/usr/bin/env python
"""Seed-and-filter benchmark on one node.

Workload (the reference's "plain per-chunk at scale" configuration): a
100 Mbp synthetic target split into 10 bins of 10 Mbp against a 100 Mbp
synthetic query (41% GC, 10% soft-masked, 20,000 planted segments of
200-5000 bp at 10-30% substitutions plus 1% small indels), 12of19 seed with
one transition, HOXD70, X-drop 910, HSP threshold 3000, both strands.
A step is one full pass: every bin x every interval x strand x WGA chunk.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--form plain|batched] [--scale S]

One JSON line on rank 0.  `value` is seed hits/s over all ranks with the
targets and query resident in HBM; `e2e` is the same metric through the C
ABI from pinned host buffers (uploads, on-device index builds and result
read-back inside the timed region).  Multi-GPU runs are independent replicas
(weak scaling; the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "seed hits/s"
UNIT = "hits/s"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload(scale: float):
    from hspz_b200 import synth
    bins, query = synth.config2(seed=2, scale=scale)
    return bins, query


def config_block(args, n_gpus):
    return {"workload": "config2: 100 Mbp target as 10 bins x 10 Mbp vs 100 Mbp query, both strands"
            if args.scale == 1.0 else f"config2 scaled x{args.scale}",
            "target_bp": int(100_000_000 * args.scale), "query_bp": int(100_000_000 * args.scale),
            "bins": 10, "seed": "12of19", "transitions": True, "xdrop": 910, "hspthresh": 3000,
            "max_hits": 16711680, "wga_chunk": 250000, "interval": 10000000, "form": args.form,
            "parallelism": f"replicas x{n_gpus}", "l2": "inputs larger than L2 (126 MB)"}


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f".clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9 and f[1].isdigit():
                    rows.append(f)
            os.remove(self.path)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [int(r[1]) for r in rows]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for n, v in zip(names, r[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": int(rows[0][2]), "reasons": sorted(reasons),
                "samples": len(rows)}


# ---------------------------------------------------------------------------
def cpu_sample(bins, query, threads: int, budget_batches: int):
    """The oracle (C restatement of the reference's path) on bin 0 x the first
    `budget_batches` calls of the pass; returns (hits/s, stats, seconds)."""
    import oracle
    from hspz_b200 import build_sub_mat
    from hspz_b200 import sequence as S
    ref = oracle.encode(bins[0].tobytes())
    qf = oracle.encode(query.tobytes())
    qr = oracle.encode(S.reverse_complement_bytes(query).tobytes())
    sh = oracle.shape("12of19")
    idx, pos = oracle.seed_table(ref, sh)
    p = oracle.params(build_sub_mat("", 910), threads=threads)
    t0 = time.perf_counter()
    _, st = oracle.seed_and_filter_all(p, sh, ref, idx, pos, qf, qr, max_batches=budget_batches)
    dt = time.perf_counter() - t0
    return st["hits"] / dt, st, dt


def run_reference(args, rank):
    """The reference arm: its CPU path (the oracle restatement; the Rust
    reference cannot be built here and has no CPU extension path) on the host
    cores, a bounded sample per step."""
    if rank != 0:
        return
    bins, query = workload(args.scale)
    threads = os.cpu_count() or 1
    vals = []
    st = None
    for i in range(args.warmup + args.steps):
        v, st, dt = cpu_sample(bins, query, threads, args.cpu_batches)
        if i >= args.warmup:
            vals.append((v, dt))
    v = statistics.median([x[0] for x in vals])
    ms = statistics.median([x[1] for x in vals]) * 1000
    sample = f"bin 0 x first {args.cpu_batches} of 80 calls of the pass ({st['hits']} hits)"
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": config_block(args, args.gpus),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import torch
    from hspz_b200 import Engine, EngineConfig
    from hspz_b200.build import build

    if rank == 0 or world == 1:
        build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    bins, query = workload(args.scale)
    cfg = EngineConfig()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], device=dev, dtype=torch.float64)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # ---- device-resident: one engine per bin, tables and query resident ----
    engines = []
    for b in bins:
        e = Engine(cfg, device=local_rank)
        e.set_stream(stream.cuda_stream)
        e.load_target(b)
        e.swap_query_ascii(query)
        engines.append(e)

    def step():
        tot = {"hits": 0, "cells": 0, "raw_hsps": 0, "hsps": 0, "seeds": 0}
        nrec = 0
        for e in engines:
            recs, st = e.run_pass()
            nrec += recs.size
            for k in tot:
                tot[k] += st[k]
        return tot, nrec

    for _ in range(args.warmup):
        step()
    for e in engines:
        e.set_profiling(True)
        e.profile_reset()
    l0 = sum(e.launches for e in engines)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local_rank) as clk:
        ev0.record(stream)
        totals = []
        for _ in range(args.steps):
            totals.append(step())
        ev1.record(stream)
        barrier()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms)
    launches = sum(e.launches for e in engines) - l0
    prof = {}
    for e in engines:
        for k, (t, n) in e.profile().items():
            a = prof.setdefault(k, [0.0, 0])
            a[0] += t
            a[1] += n
        e.set_profiling(False)
    tot, nrec = totals[-1]
    hits_step = tot["hits"]
    cells_step = tot["cells"]
    value = hits_step * args.steps * world / (ms / 1000)
    bp_s = cells_step * args.steps * world / (ms / 1000)

    # roofline of the dominant kernel (the X-drop extension): algorithmic
    # bytes = 2 B per scored cell (1 B reference + 1 B query code)
    peak, peak_kind = peaks()
    ext_ms, ext_n = prof.get("extend", (0.0, 0))
    ext_bytes = 2.0 * cells_step * args.steps
    ext_avg_ms = ext_ms / max(ext_n, 1)
    achieved = (ext_bytes / max(ext_n, 1)) / (ext_avg_ms / 1000) / 1e9 if ext_ms > 0 else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "extend_traffic.json")
    if os.path.exists(tfile) and ext_n:
        tr = json.load(open(tfile))
        traffic = tr["dram_bytes_per_cell"] * cells_step * args.steps / ext_n
    lookup_names = ("seed_count", "pair", "scan", "seed_compact", "expand")
    lk_ms = sum(prof.get(k, (0.0, 0))[0] for k in lookup_names)
    seeds_step = tot["seeds"]
    # B_lookup = 1 B/query base per strand + 8 B per seed (two index words) + 4 B per hit (pos_table)
    # + 8 B per hit (anchors written by expand)
    qlen = query.size
    lk_bytes = (2 * qlen * len(bins) + 8 * seeds_step + 12 * hits_step) * args.steps
    lookup_gbs = lk_bytes / (lk_ms / 1000) / 1e9 if lk_ms > 0 else None

    # ---- end to end through the C ABI from pinned host buffers ------------
    e2e = None
    if not args.no_e2e:
        pin_q = torch.from_numpy(query).pin_memory()
        pin_bins = [torch.from_numpy(b).pin_memory() for b in bins]
        e2 = Engine(cfg, device=local_rank)
        e2.set_stream(stream.cuda_stream)
        from hspz_b200 import _native as N
        import ctypes as C
        L = N.lib()

        def e2e_step():
            N.check(L.hz_swap_query_ascii(e2._h, C.c_void_p(pin_q.data_ptr()), pin_q.numel()))
            hits = 0
            d2h = 0
            for pb in pin_bins:
                N.check(L.hz_engine_load_target(e2._h, C.c_void_p(pb.data_ptr()), pb.numel()))
                recs, st = e2.run_pass()
                hits += st["hits"]
                d2h += recs.nbytes
            return hits, d2h

        for _ in range(max(1, args.warmup)):
            e2e_step()
        barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        res = [e2e_step() for _ in range(args.steps)]
        t1.record(stream)
        barrier()
        ems = max_over_ranks(t0.elapsed_time(t1))
        hits_e = res[-1][0]
        e2e = {"value": hits_e * args.steps * world / (ems / 1000), "unit": UNIT,
               "h2d_bytes_per_step": int(pin_q.numel() + sum(p.numel() for p in pin_bins)),
               "d2h_bytes_per_step": int(res[-1][1]), "ms_per_step": ems / args.steps}
        e2.close()

    cpu = None
    if rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        v, st, dt = cpu_sample(bins, query, threads, args.cpu_batches)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"bin 0 x first {args.cpu_batches} of 80 calls of the pass ({st['hits']} hits, {dt:.1f} s)"}

    for e in engines:
        e.close()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": config_block(args, world),
            "extended_bp_per_s": bp_s, "hits_per_step": hits_step, "cells_per_step": cells_step,
            "hsps_per_step": tot["hsps"], "raw_hsps_per_step": tot["raw_hsps"],
            "roofline": {"bound": "hbm", "kernel": "extend", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": traffic,
                         "peak_kind": peak_kind,
                         "note": "X-drop extension is issue-bound; algorithmic bytes = 2 B per scored cell"},
            "lookup_roofline": {"kernels": list(lookup_names), "achieved": lookup_gbs, "peak": peak, "unit": "GB/s",
                                "frac": lookup_gbs / peak if lookup_gbs else None},
            "kernel_ms": {k: round(v[0], 3) for k, v in prof.items()},
            "kernel_launches": {k: v[1] for k, v in prof.items()},
            "gpu_launches": launches, "clocks": clk.summary(), "e2e": e2e, "cpu_baseline": cpu}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--form", default="plain", choices=["plain"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-batches", type=int, default=80)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
