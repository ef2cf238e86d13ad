#!/usr/bin/env python
"""Seed-and-filter benchmark on one node.

Default workload (the reference's batched configuration, on which the
batched-versus-plain target is quoted): a resident 200 Mbp synthetic target
(41% GC, 10% soft-masked) against 512 query chunks with log-uniform lengths in
10 kbp-2 Mbp carrying planted homology at 5-35% divergence; 12of19 seed with
one transition, HOXD70, X-drop 910, HSP threshold 3000, both strands.

--config 2: 100 Mbp target as 10 bins of 10 Mbp against a 100 Mbp query
(20,000 planted segments of 200-5000 bp at 10-30% plus 1% small indels).
--config 1: the reference's CPU-sized case, 1 Mbp x 1 Mbp.  --config 4:
repeat-dense 1 Gbp target (10 bins) vs 1 Gbp query with a per-seed occurrence
cap of 1000.  --config 5: the serving loop alone over a resident 3 Gbp target
under a Poisson request stream (p50/p99 latency and throughput).

A step is one full pass of every bin x every query x interval x strand x WGA
chunk.  Two forms are timed: the plain per-chunk form (one launch chain and
one read-back per seed_and_filter call, as the reference runs) and the
batched form (all calls in shared waves: one lookup, one persistent gate
launch over a device work queue, one read-back per wave).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--config 1|2|3|4|5] [--form both|batched|plain] [--scale S]

One JSON line on rank 0.  `value` is seed hits/s over all ranks for the
batched form with targets and queries resident in HBM; `e2e` is the same
metric through the C ABI from pinned host buffers (uploads, on-device seed
table builds, query encoding and result read-back inside the timed region).
`parity` holds the in-run checks: the oracle's records for a sample of the
workload against both forms' records of exactly that sample, and the two
forms against each other over the whole workload (any difference exits
non-zero).  On the default workload a `serving` block adds the serving loop
(config 5 on a smaller resident target, stated in the block) with p50/p99
latency and per-request parity.  Multi-GPU runs are independent replicas
(weak scaling; no exchange step).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "seed hits/s"
UNIT = "hits/s"
FALLBACK_HBM_GBS = 6650.0


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def workload(config: int, scale: float):
    """(target bins, query blocks) as ASCII arrays."""
    from hspz_b200 import synth
    if config == 1:
        t, q = synth.config1(seed=1, scale=scale)
        return [t], [q]
    if config == 3:
        target, chunks = synth.config3(seed=3, scale=scale)
        return [target], chunks
    if config == 4:
        t, q = synth.config4(seed=4, scale=scale)
        step = -(-t.size // 10)
        return [t[i:i + step] for i in range(0, t.size, step)], [q]
    bins, query = synth.config2(seed=2, scale=scale)
    return bins, [query]


def occ_cap(config: int) -> int:
    return 1000 if config == 4 else 0


WORKLOADS = {
    1: "config1: 1 Mbp target vs 1 Mbp query, 200 planted segments at 15%",
    2: "config2: 100 Mbp target as 10 bins x 10 Mbp vs 100 Mbp query",
    3: "config3: 200 Mbp resident target vs 512 query chunks (log-uniform 10 kbp-2 Mbp)",
    4: "config4: repeat-dense 1 Gbp target as 10 bins vs 1 Gbp query (45% from 500 repeat families, "
       "3% tandem), occurrence cap 1000",
    5: "config5: serving, resident 3 Gbp target, Poisson arrivals, lognormal(200 kbp, sigma 1) requests "
       "capped at 5 Mbp, 40 GB admission budget",
}


def config_block(args, n_gpus, bins, queries):
    name = WORKLOADS[args.config]
    if args.scale != 1.0:
        name += f", scaled x{args.scale}"
    return {"workload": name + ", both strands", "target_bp": int(sum(b.size for b in bins)),
            "query_bp": int(sum(q.size for q in queries)), "bins": len(bins), "queries": len(queries),
            "seed": "12of19", "transitions": True, "xdrop": 910, "hspthresh": 3000, "max_hits": 16711680,
            "occ_cap": occ_cap(args.config), "wga_chunk": 250000, "interval": 10000000,
            "parallelism": f"replicas x{n_gpus}", "l2": "inputs larger than L2 (126 MB)"}


def over_ranks(vals, op: str, device) -> list:
    """Element-wise max or sum of `vals` over all ranks (every rank calls it
    at the same point, with the same length)."""
    import torch
    t = torch.tensor([float(v) for v in vals], dtype=torch.float64, device=device)
    red = {"max": torch.distributed.ReduceOp.MAX, "sum": torch.distributed.ReduceOp.SUM}[op]
    torch.distributed.all_reduce(t, op=red)
    return [float(x) for x in t.tolist()]


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        import tempfile
        self.path = os.path.join(tempfile.gettempdir(), f"hz_clocks_{os.getpid()}_{device}.csv")

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
# The CPU side: the oracle (C restatement of the reference's path) on bin 0
# and a bounded sample of the queries, on all host cores.

def sample_picks(config: int, queries, frac: float, seed: int):
    """[(query index, calls)] of a sample: for the chunked workload a seeded
    set of whole chunks covering about `frac` of the query bases (all calls of
    each); otherwise query 0's first LASTZ interval (its plus and minus
    calls), or the whole pass for config 1."""
    import numpy as np
    if config == 1:
        return [(0, 0)]
    if len(queries) == 1:
        return [(0, 1)]  # one interval
    lens = np.array([q.size for q in queries], dtype=np.int64)
    order = np.random.default_rng(seed).permutation(len(queries))
    picks, got = [], 0
    for qi in order.tolist():
        picks.append((int(qi), 0))
        got += int(lens[qi])
        if got >= frac * lens.sum():
            break
    return sorted(picks)


class CpuOracle:
    """Bin 0's seed table on the host and the oracle passes of sampled queries."""

    def __init__(self, bins, queries, cap: int, threads: int):
        import oracle
        from hspz_b200 import build_sub_mat
        self.oracle = oracle
        self.queries = queries
        self.ref = oracle.encode(bins[0].tobytes())
        self.sh = oracle.shape("12of19")
        self.idx, self.pos = oracle.seed_table(self.ref, self.sh)
        self.threads = threads
        self.sub = build_sub_mat("", 910)
        self.cap = cap
        self.enc = {}

    def _encoded(self, qi):
        from hspz_b200 import sequence as S
        if qi not in self.enc:
            q = self.queries[qi]
            self.enc[qi] = (self.oracle.encode(q.tobytes()),
                            self.oracle.encode(S.reverse_complement_bytes(q).tobytes()))
        return self.enc[qi]

    def run(self, picks):
        """{query: records}, summed stats, seconds.  Passes of different
        queries run side by side, each over all host threads (its calls are
        its unit of parallelism), so short chunks do not leave cores idle."""
        from concurrent.futures import ThreadPoolExecutor
        for qi, _ in picks:
            self._encoded(qi)
        p = self.oracle.params(self.sub, threads=self.threads, occ_cap=self.cap)
        # intervals -> calls: an interval of one query is its plus chunks then its minus chunks
        def one(pick):
            qi, n_iv = pick
            qf, qr = self.enc[qi]
            max_batches = 0 if n_iv == 0 else self._calls_in_intervals(qf.size, n_iv)
            return qi, self.oracle.seed_and_filter_all(p, self.sh, self.ref, self.idx, self.pos, qf, qr,
                                                       max_batches=max_batches)
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=max(1, min(len(picks), 4))) as ex:
            out = list(ex.map(one, picks))
        dt = time.perf_counter() - t0
        recs, st = {}, {}
        for qi, (r, s1) in out:
            recs[qi] = r
            for k, v in s1.items():
                st[k] = st.get(k, 0) + v
        return recs, st, dt

    @staticmethod
    def _calls_in_intervals(qlen: int, n_iv: int, interval: int = 10_000_000, chunk: int = 250_000):
        """Calls of the first n_iv LASTZ intervals of a query (both strands)."""
        end = max(qlen - 19, 0)
        calls = 0
        for i in range(n_iv):
            a, b = i * interval, min(end, (i + 1) * interval)
            if a >= end:
                break
            calls += 2 * (-(-(b - a) // chunk))
        return calls


def sample_text(config: int, queries, picks, st, dt):
    if config == 1:
        return f"the whole pass ({st['calls']} seed_and_filter calls, {st['hits']} hits, {dt:.1f} s)"
    if len(queries) == 1:
        return (f"bin 0 x the first LASTZ interval of the query ({st['calls']} seed_and_filter calls, "
                f"{st['hits']} hits, {dt:.1f} s)")
    bp = sum(queries[qi].size for qi, _ in picks)
    return (f"bin 0 x {len(picks)} seeded-random query chunks, {bp} bp ({st['calls']} seed_and_filter calls, "
            f"{st['hits']} hits, {dt:.1f} s)")


FIELDS = ("interval", "strand", "ref_start", "query_start", "len", "score")


def parity_digest(arrays) -> str:
    """sha256 over the records of each array in turn, each sorted by
    (strand, ref_start, query_start, len, score): the HSP-set digest."""
    import hashlib
    import numpy as np
    h = hashlib.sha256()
    for a in arrays:
        if a.size == 0:
            h.update(b"|")
            continue
        keys = np.stack([a["strand"].astype(np.int64), a["ref_start"].astype(np.int64),
                         a["query_start"].astype(np.int64), a["len"].astype(np.int64),
                         a["score"].astype(np.int64)], axis=1)
        keys = keys[np.lexsort(keys.T[::-1])]
        h.update(keys.astype("<i8").tobytes())
        h.update(b"|")
    return h.hexdigest()


def same_records(a, b) -> bool:
    import numpy as np
    return a.size == b.size and all(np.array_equal(a[f], b[f]) for f in FIELDS)


def run_reference(args, rank):
    """The reference arm: its CPU path -- the oracle restatement, since the
    Rust reference cannot be built here and has no CPU extension path -- on
    the host cores, a bounded sample of the same workload per step."""
    if rank != 0:
        return
    bins, queries = workload(args.config, args.scale)
    threads = os.cpu_count() or 1
    cpu = CpuOracle(bins, queries, occ_cap(args.config), threads)
    picks = sample_picks(args.config, queries, args.ref_frac, seed=7)
    vals = []
    st = dt = None
    for i in range(args.warmup + args.steps):
        _, st, dt = cpu.run(picks)
        if i >= args.warmup:
            vals.append((st["hits"] / dt, dt))
    v = statistics.median([x[0] for x in vals])
    ms = statistics.median([x[1] for x in vals]) * 1000
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(config_block(args, args.gpus, bins, queries), form="batched"),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": sample_text(args.config, queries, picks, st, dt)},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    from hspz_b200 import Engine, EngineConfig
    from hspz_b200 import _native as N
    from hspz_b200.build import build

    if rank == 0:
        build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    bins, queries = workload(args.config, args.scale)
    cfg = EngineConfig(occ_cap=occ_cap(args.config))

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x: float) -> float:
        return x if world == 1 else over_ranks([x], "max", dev)[0]

    # ---- device-resident: one engine per bin, target and queries resident ----
    engines = []
    for b in bins:
        e = Engine(cfg, device=local_rank)
        e.set_stream(stream.cuda_stream)
        if args.tuning:
            e.set_tuning(**json.loads(args.tuning))
        e.load_target(b)
        e.stage_queries(queries)
        engines.append(e)

    tuning = None
    if not args.no_autotune:
        # launch shapes timed on a sample of this workload (outside the timed
        # region), then used by every engine of both forms
        tuning = engines[0].autotune(sample_positions=args.tune_positions)
        knobs = {k: tuning[k] for k in ("gate_tile", "gate_cap", "graph")}
        for e in engines:
            e.set_tuning(**knobs)

    def step(form):
        tot = {"hits": 0, "cells": 0, "raw_hsps": 0, "hsps": 0, "seeds": 0, "calls": 0}
        recs = []
        for e in engines:
            if form == "batched":
                r, st = e.run_batched()
                recs.append(r)
                for k in tot:
                    tot[k] += st[k]
            else:
                for qi in range(len(queries)):
                    e.select_query(qi)
                    r, st = e.run_pass()
                    recs.append(r)
                    for k in tot:
                        tot[k] += st[k]
        return tot, recs

    def timed(form, steps, warmup):
        for _ in range(warmup):
            step(form)
        for e in engines:
            e.set_profiling(True)
            e.profile_reset()
        l0 = sum(e.launches for e in engines)
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local_rank) as clk:
            ev0.record(stream)
            res = [step(form) for _ in range(steps)]
            ev1.record(stream)
            barrier()
        ms = max_over_ranks(ev0.elapsed_time(ev1))
        prof = {}
        for e in engines:
            for k, (t, n) in e.profile().items():
                a = prof.setdefault(k, [0.0, 0])
                a[0] += t
                a[1] += n
            e.set_profiling(False)
        launches = sum(e.launches for e in engines) - l0
        tot, recs = res[-1]
        return {"ms": ms, "tot": tot, "recs": recs, "prof": prof, "launches": launches, "clocks": clk.summary(),
                "steps": steps, "warmup": warmup}

    forms = ["batched", "plain"] if args.form == "both" else [args.form]
    runs = {}
    for f in forms:
        if f == "batched" or len(forms) == 1:
            runs[f] = timed(f, args.steps, args.warmup)
        else:  # the comparison form: fewer steps (stated in its block)
            runs[f] = timed(f, min(args.steps, args.plain_steps), min(args.warmup, 1))

    # ---- records of each query, per form ----------------------------------
    nq = len(queries)

    def per_query(form):
        """records[bin][query] of a form's last step (PASS_RECORD fields)."""
        r = runs[form]["recs"]
        out = []
        for bi in range(len(bins)):
            if form == "batched":
                br = r[bi]
                out.append([br[br["query"] == qi] for qi in range(nq)])
            else:
                out.append(r[bi * nq:(bi + 1) * nq])
        return out

    recs_by = {f: per_query(f) for f in runs}
    parity = {}
    bad = []
    if len(runs) == 2:
        a, b = recs_by["batched"], recs_by["plain"]
        for bi in range(len(bins)):
            for qi in range(nq):
                if not same_records(a[bi][qi], b[bi][qi]):
                    bad.append(f"batched != plain for bin {bi} query {qi}")
        da = parity_digest([x for row in a for x in row])
        db = parity_digest([x for row in b for x in row])
        parity["batched_vs_plain"] = {"bins": len(bins), "queries": nq,
                                      "hsps": int(sum(x.size for row in a for x in row)),
                                      "sha256_batched": da, "sha256_plain": db, "equal": not bad and da == db}

    peak, peak_kind = peaks()

    knobs = json.loads(args.tuning) if args.tuning else {}
    cell_bytes = 2.0 if knobs.get("gate_version") == 1 else 0.75

    def summarize(r):
        ms, tot, prof, steps = r["ms"], r["tot"], r["prof"], r["steps"]
        per_s = steps * world / (ms / 1000)
        gate_ms, gate_n = prof.get("gate", (0.0, 0))
        # dominant kernel: the fused expansion + X-drop gate.  Algorithmic
        # bytes: per scored cell the reference and query codes -- 0.75 B at
        # 2 bits + 1 special bit per base (the lockstep gate), 2 B at 8-bit
        # codes (the lane-refill gate) -- and 4 B per hit (its pos_table entry)
        gate_bytes = (cell_bytes * tot["cells"] + 4.0 * tot["hits"]) * steps
        gate_gbs = gate_bytes / (gate_ms / 1000) / 1e9 if gate_ms else None
        lk_ms = prof.get("lookup_count", (0.0, 0))[0]
        # seed lookup per valid query position: its base at 2 bits + 1 special
        # bit, one 4-byte neighbourhood hit count (the per-k-mer table built
        # with the target holds the capped hits of all 13 seeds), and the
        # count and the k-mer written (4 B each; the gate's tile setup reads
        # the k-mer back)
        positions = tot["seeds"] / 13.0
        lk_bytes = positions * 12.375 * steps
        lk_gbs = lk_bytes / (lk_ms / 1000) / 1e9 if lk_ms else None
        return {"hits_per_s": tot["hits"] * per_s, "extended_bp_per_s": tot["cells"] * per_s,
                "ms_per_step": ms / steps, "steps": steps, "warmup": r["warmup"],
                "hits_per_step": tot["hits"], "cells_per_step": tot["cells"],
                "hsps_per_step": tot["hsps"], "raw_hsps_per_step": tot["raw_hsps"], "calls_per_step": tot["calls"],
                "gpu_launches": r["launches"],
                "kernel_ms_per_step": {k: round(v[0] / steps, 3) for k, v in prof.items()},
                "kernel_launches_per_step": {k: v[1] // steps for k, v in prof.items()},
                "gate": {"achieved": gate_gbs, "avg_launch_ms": gate_ms / max(gate_n, 1),
                         "bytes_per_launch": gate_bytes / max(gate_n, 1),
                         "cells_per_s": tot["cells"] * steps / (gate_ms / 1000) if gate_ms else None},
                "lookup": {"achieved": lk_gbs, "frac": lk_gbs / peak if lk_gbs else None,
                           "seed_lookups_per_s": tot["seeds"] * steps / (lk_ms / 1000) if lk_ms else None},
                "clocks": r["clocks"]}

    summ = {f: summarize(r) for f, r in runs.items()}
    head = summ["batched"] if "batched" in summ else summ["plain"]
    head_form = "batched" if "batched" in summ else "plain"

    traffic = None
    tfile = os.path.join(ROOT, "profiles", "gate_traffic.json")
    if os.path.exists(tfile):
        tr = json.load(open(tfile))
        traffic = tr.get("dram_bytes_per_hit", 0) * head["hits_per_step"] * head["steps"] / max(
            runs[head_form]["prof"].get("gate", (0, 1))[1], 1)

    # ---- end to end through the C ABI from pinned host buffers ------------
    e2e = None
    if not args.no_e2e:
        pin_q = [torch.from_numpy(q).pin_memory() for q in queries]
        pin_b = [torch.from_numpy(b).pin_memory() for b in bins]
        e2 = Engine(cfg, device=local_rank)
        e2.set_stream(stream.cuda_stream)
        if args.tuning:
            e2.set_tuning(**json.loads(args.tuning))
        if tuning:
            e2.set_tuning(**{k: tuning[k] for k in ("gate_tile", "gate_cap", "graph")})
        L = N.lib()
        qarr = (N.QueryC * len(pin_q))()
        for i, t in enumerate(pin_q):
            qarr[i].ascii = t.data_ptr() if t.numel() else None
            qarr[i].len = t.numel()

        parts = {"load_target": 0.0, "stage_queries": 0.0, "run_batched": 0.0}

        def e2e_step():
            # each call returns once its work is done, so the host clock
            # splits the step into its parts
            hits = d2h = 0
            for pb in pin_b:  # per reference bin: Engine::new + swap_query (src/run.rs:816-887)
                t0 = time.perf_counter()
                N.check(L.hz_engine_load_target(e2._h, C.c_void_p(pb.data_ptr()), pb.numel()))
                t1 = time.perf_counter()
                N.check(L.hz_stage_queries(e2._h, qarr, len(pin_q)))
                t2 = time.perf_counter()
                recs, st = e2.run_batched()
                t3 = time.perf_counter()
                parts["load_target"] += t1 - t0
                parts["stage_queries"] += t2 - t1
                parts["run_batched"] += t3 - t2
                hits += st["hits"]
                d2h += recs.nbytes
            return hits, d2h

        e_steps = min(args.steps, args.e2e_steps)
        for _ in range(1):
            e2e_step()
        barrier()
        for k in parts:
            parts[k] = 0.0
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        res = [e2e_step() for _ in range(e_steps)]
        t1.record(stream)
        barrier()
        ems = max_over_ranks(t0.elapsed_time(t1))
        e2e = {"value": res[-1][0] * e_steps * world / (ems / 1000), "unit": UNIT,
               "h2d_bytes_per_step": int(sum(p.numel() for p in pin_b) + len(pin_b) * sum(p.numel() for p in pin_q)),
               "d2h_bytes_per_step": int(res[-1][1]), "ms_per_step": ems / e_steps, "steps": e_steps,
               "warmup": 1, "form": "batched",
               "host_ms_per_step": {k: round(v * 1000 / e_steps, 2) for k, v in parts.items()}}
        e2.close()

    for e in engines:
        e.close()

    # ---- the oracle on a sample of the workload, checked against both forms
    cpu = None
    if rank == 0 and not args.no_cpu and args.cpu_query_bp and len(queries) == 1:
        # a prefix of the one query as its own query block against bin 0: the
        # oracle and both forms on exactly that block (for workloads whose
        # first interval alone is too dense for a bounded CPU sample)
        threads = os.cpu_count() or 1
        sub = queries[0][: args.cpu_query_bp]
        oc = CpuOracle(bins, [sub], occ_cap(args.config), threads)
        picks = [(0, 0)]
        o_recs, st, dt = oc.run(picks)
        cpu = {"value": st["hits"] / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"bin 0 x the query's first {sub.size} bp as one query block ({st['calls']} "
                         f"seed_and_filter calls, {st['hits']} hits, {dt:.1f} s)"}
        with Engine(cfg, device=local_rank) as e0:
            if tuning:
                e0.set_tuning(**{k: tuning[k] for k in ("gate_tile", "gate_cap", "graph")})
            e0.load_target(bins[0])
            e0.stage_queries([sub])
            gb, _ = e0.run_batched()
            e0.select_query(0)
            gp, _ = e0.run_pass()
        checked = {"batched": same_records(gb, o_recs[0]), "plain": same_records(gp, o_recs[0])}
        for f, ok in checked.items():
            if not ok:
                bad.append(f"{f} form != oracle on the query prefix")
        parity["oracle"] = {"bin": 0, "query_prefix_bp": int(sub.size), "calls": int(st["calls"]),
                            "hits": int(st["hits"]), "raw_hsps": int(st["raw_hsps"]), "hsps": int(st["hsps"]),
                            "cells": int(st["cells"]), "sha256": parity_digest([o_recs[0]]), "equal": checked}
    elif rank == 0 and not args.no_cpu:
        threads = os.cpu_count() or 1
        oc = CpuOracle(bins, queries, occ_cap(args.config), threads)
        picks = sample_picks(args.config, queries, args.cpu_frac, seed=11)
        o_recs, st, dt = oc.run(picks)
        cpu = {"value": st["hits"] / dt, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": sample_text(args.config, queries, picks, st, dt)}
        checked = {}
        for f in runs:
            ok = True
            for qi, n_iv in picks:
                g = recs_by[f][0][qi]
                if n_iv:
                    g = g[g["interval"] < n_iv]
                if not same_records(g, o_recs[qi]):
                    ok = False
                    bad.append(f"{f} form != oracle for bin 0 query {qi}")
            checked[f] = ok
        parity["oracle"] = {"bin": 0, "queries": [qi for qi, _ in picks], "calls": int(st["calls"]),
                            "hits": int(st["hits"]), "raw_hsps": int(st["raw_hsps"]), "hsps": int(st["hsps"]),
                            "cells": int(st["cells"]),
                            "sha256": parity_digest([o_recs[qi] for qi, _ in picks]),
                            "equal": {f: v for f, v in checked.items()}}

    # ---- the serving loop on the default workload ---------------------------
    serving = None
    if args.config == 3 and not args.no_serving:
        try:
            serving = serving_block(args, local_rank, tuning)
            if not serving.get("parity", {}).get("equal", True):
                bad.append("a served request differs from run_pass alone")
        except Exception as ex:  # reported in the line; the headline stands
            serving = {"error": f"{type(ex).__name__}: {ex}"}

    if rank != 0:
        if bad:
            raise SystemExit("parity failed: " + "; ".join(bad[:5]))
        return
    g = head["gate"]
    line = {"metric": METRIC, "value": head["hits_per_s"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": dict(config_block(args, world, bins, queries), form=head_form),
            "extended_bp_per_s": head["extended_bp_per_s"],
            "roofline": {"bound": "hbm", "kernel": "gate (fused hit expansion + X-drop score gate)",
                         "achieved": g["achieved"], "peak": peak, "unit": "GB/s",
                         "frac": g["achieved"] / peak if g["achieved"] else None, "traffic": traffic,
                         "peak_kind": peak_kind, "spec_peak": 8000.0,
                         "frac_of_spec": g["achieved"] / 8000.0 if g["achieved"] else None,
                         "note": f"issue-bound integer kernel; algorithmic bytes = {cell_bytes:g} B per scored "
                                 f"cell + 4 B per hit"},
            "lookup_roofline": dict(head["lookup"], kernel="lookup_count", peak=peak, unit="GB/s",
                                    note="12.375 B per valid query position: packed base (0.375 B), "
                                         "neighbourhood count, count and k-mer written"),
            "forms": summ,
            "batched_over_plain": (summ["batched"]["hits_per_s"] / summ["plain"]["hits_per_s"]
                                   if len(summ) == 2 else None),
            "parity": dict(parity, ok=not bad),
            "gpu_launches": head["gpu_launches"], "clocks": head["clocks"], "e2e": e2e, "cpu_baseline": cpu,
            "serving": serving, "autotune": tuning}
    print(json.dumps(line), flush=True)
    if bad:
        print("parity failed: " + "; ".join(bad[:5]), file=sys.stderr, flush=True)
        raise SystemExit(3)


# ---------------------------------------------------------------------------
def percentile(xs, q):
    import numpy as np
    return float(np.percentile(np.asarray(xs, dtype=np.float64), q)) if len(xs) else None


def serve_window(e, target, rng, rate: float, n_req: int, keep: int = 0):
    """One window of an open-loop Poisson request stream on a running
    serving loop: a submit thread issues each request at its arrival time
    while this thread collects the results.  Latency is submit -> finished,
    as the library records it; the window's makespan runs from the first
    arrival to the last completion, so queueing is inside both.  The first
    `keep` requests are returned with their records for a parity check."""
    import queue
    import threading

    import numpy as np
    from hspz_b200 import synth
    lens = synth.request_lengths(rng, n_req)
    reqs = [synth.serving_request(rng, target, int(L)) for L in lens]
    arrive = np.cumsum(rng.exponential(1.0 / rate, n_req))
    arrive -= arrive[0]
    st0, _, _ = e.serve_stats()
    tq = queue.Queue()
    t0 = time.perf_counter()

    def submitter():
        for a, r in zip(arrive.tolist(), reqs):
            d = t0 + a - time.perf_counter()
            if d > 0:
                time.sleep(d)
            ts = time.perf_counter() - t0
            tq.put((e.serve_submit(r), ts))

    th = threading.Thread(target=submitter)
    th.start()
    out, kept = [], []
    for i in range(n_req):
        ticket, ts = tq.get()
        recs, tm = e.serve_poll(ticket)
        out.append(dict(tm, submit_s=ts, records=int(recs.size), bytes_out=int(recs.nbytes)))
        if i < keep:
            kept.append((reqs[i], recs))
    th.join()
    st1, _, _ = e.serve_stats()
    makespan = max(o["submit_s"] + o["total_ms"] / 1000 for o in out)
    d = {k: st1[k] - st0[k] for k in st1}
    return {"makespan_s": makespan, "stats": d, "reqs": out, "bases": int(sum(lens)), "rate": rate, "kept": kept}


def window_summary(w):
    import numpy as np
    lat = [o["total_ms"] for o in w["reqs"]]
    return {"rate_req_per_s": w["rate"], "requests": len(w["reqs"]),
            "p50_ms": percentile(lat, 50), "p99_ms": percentile(lat, 99),
            "hits_per_s": w["stats"]["hits"] / w["makespan_s"],
            "served_req_per_s": len(w["reqs"]) / w["makespan_s"],
            "mean_batch": float(np.mean([o["batch_queries"] for o in w["reqs"]]))}


def check_served(e, kept):
    """Each kept request's served records against hz_run_pass on that query
    alone (after the loop has stopped)."""
    n = 0
    ok = True
    for q, got in kept:
        e.swap_query_ascii(q)
        want, _ = e.run_pass()
        ok = ok and same_records(got, want)
        n += int(want.size)
    return {"requests": len(kept), "hsps": n, "equal": ok}


def serving_block(args, local_rank, tuning):
    """The serving loop beside the default workload: a resident synthetic
    target of --serve-scale x 3 Gbp, one window of Poisson arrivals at
    --rate, and the per-request parity check."""
    import numpy as np
    from hspz_b200 import Engine, EngineConfig, synth
    t_gen = time.perf_counter()
    target = synth.config5_target(seed=5, scale=args.serve_scale)
    t_gen = time.perf_counter() - t_gen
    rng = np.random.default_rng(55)
    with Engine(EngineConfig(), device=local_rank) as e:
        t_load = time.perf_counter()
        e.load_target(target)
        t_load = time.perf_counter() - t_load
        if tuning:
            e.set_tuning(**{k: tuning[k] for k in ("gate_tile", "gate_cap")})
        budget = int(args.budget_gb * (1 << 30))
        e.serve_start(budget_bytes=budget, workers=args.workers, max_batch_queries=args.max_batch)
        serve_window(e, target, rng, args.rate, 4)  # warm-up
        with Clocks(local_rank) as clk:
            w = serve_window(e, target, rng, args.rate, args.requests, keep=args.serve_check)
        e.serve_stop()
        par = check_served(e, w["kept"])
    lat = [o["total_ms"] for o in w["reqs"]]
    return {"workload": f"config5 scaled: resident {target.size} bp synthetic target (x{args.serve_scale} of 3 Gbp), "
                        f"Poisson arrivals at {args.rate} req/s, lognormal(200 kbp, sigma 1) requests capped at "
                        f"5 Mbp, {args.budget_gb:g} GB admission budget, {args.workers} workers",
            "requests": len(w["reqs"]), "latency_ms": {"p50": percentile(lat, 50), "p99": percentile(lat, 99),
                                                      "mean": float(np.mean(lat))},
            "hits_per_s": w["stats"]["hits"] / w["makespan_s"],
            "extended_bp_per_s": w["stats"]["cells"] / w["makespan_s"],
            "served_req_per_s": len(w["reqs"]) / w["makespan_s"],
            "mean_batch_queries": float(np.mean([o["batch_queries"] for o in w["reqs"]])),
            "timing": "host clock, submit -> finished", "parity": par, "clocks": clk.summary(),
            "setup_s": {"target_generation": round(t_gen, 1), "load_target": round(t_load, 2)}}


def run_serving(args, rank, world, local_rank):
    """Config 5: the serving loop under an open-loop Poisson request stream.

    A step is one window of --requests query chunks (serve_window).  Serving
    is host-observed end to end by construction: each request's bases go host
    -> device and its records device -> host inside the window."""
    import numpy as np
    import torch
    from hspz_b200 import Engine, EngineConfig, synth
    from hspz_b200.build import build

    if rank == 0:
        build()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    t_gen = time.perf_counter()
    target = synth.config5_target(seed=5, scale=args.scale)
    rng = np.random.default_rng(50 + rank)
    t_gen = time.perf_counter() - t_gen
    e = Engine(EngineConfig(), device=local_rank)
    t_load = time.perf_counter()
    e.load_target(target)
    t_load = time.perf_counter() - t_load
    budget = int(args.budget_gb * (1 << 30))
    tuning = None
    if not args.no_autotune:
        # launch shapes tuned on a few requests of this stream before it starts;
        # the workers inherit them
        e.stage_queries([synth.serving_request(rng, target, int(L)) for L in synth.request_lengths(rng, 4)])
        tuning = e.autotune(sample_positions=1 << 22)
    e.serve_start(budget_bytes=budget, workers=args.workers, max_batch_queries=args.max_batch)

    for _ in range(args.warmup):
        serve_window(e, target, rng, args.rate, 4)
    l0 = e.launches
    with Clocks(local_rank) as clk:
        runs = [serve_window(e, target, rng, args.rate, args.requests, keep=args.serve_check if i == 0 else 0)
                for i in range(args.steps)]
    launches = e.launches - l0
    sweep = []
    for r in [float(x) for x in args.sweep.split(",") if x.strip()]:
        sweep.append(window_summary(serve_window(e, target, rng, r, args.sweep_requests)))
    e.serve_stop()
    par = check_served(e, runs[0]["kept"])
    e.close()

    span = sum(r["makespan_s"] for r in runs)
    hits = sum(r["stats"]["hits"] for r in runs)
    cells = sum(r["stats"]["cells"] for r in runs)
    n_req = sum(len(r["reqs"]) for r in runs)
    if world > 1:
        span_all = over_ranks([span], "max", dev)[0]
        hits_all, cells_all = over_ranks([hits, cells], "sum", dev)
    else:
        span_all, hits_all, cells_all = span, hits, cells
    if rank != 0:
        return
    lat = [o["total_ms"] for r in runs for o in r["reqs"]]
    qd = [o["queued_ms"] for r in runs for o in r["reqs"]]
    sv = [o["service_ms"] for r in runs for o in r["reqs"]]
    mean_hits = hits / max(n_req, 1)
    h2d = sum(r["bases"] for r in runs) // max(args.steps, 1)
    d2h = sum(o["bytes_out"] for r in runs for o in r["reqs"]) // max(args.steps, 1)
    value = hits_all / span_all
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": span_all / args.steps * 1000, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": WORKLOADS[5] + (f", target scaled x{args.scale}" if args.scale != 1.0 else ""),
                       "target_bp": int(target.size), "rate_req_per_s": args.rate,
                       "requests_per_step": args.requests, "workers": args.workers,
                       "max_batch_queries": args.max_batch, "budget_bytes": budget,
                       "seed": "12of19", "transitions": True, "xdrop": 910, "hspthresh": 3000,
                       "max_hits": 16711680, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (126 MB)", "timing": "host clock, submit -> finished"},
            "latency_ms": {"p50": percentile(lat, 50), "p99": percentile(lat, 99), "mean": float(np.mean(lat)),
                           "queued_p50": percentile(qd, 50), "queued_p99": percentile(qd, 99),
                           "service_p50": percentile(sv, 50), "service_p99": percentile(sv, 99)},
            "served_req_per_s": n_req / span, "offered_req_per_s": args.rate,
            "mean_hits_per_request": mean_hits, "offered_hits_per_s": mean_hits * args.rate,
            "extended_bp_per_s": cells_all / span_all,
            "mean_batch_queries": float(np.mean([o["batch_queries"] for r in runs for o in r["reqs"]])),
            "rate_sweep": sweep, "gpu_launches": launches, "clocks": clk.summary(), "autotune": tuning,
            "parity": par,
            "setup_s": {"target_generation": t_gen, "load_target": t_load},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "note": "serving is measured end to end; value and e2e are the same measurement"},
            "cpu_baseline": None,
            "cpu_note": "the CPU path is timed on configs 1-4; a 3 Gbp host seed table is out of a bench budget"}
    print(json.dumps(line), flush=True)
    if not par["equal"]:
        print("parity failed: a served request differs from run_pass alone", file=sys.stderr, flush=True)
        raise SystemExit(3)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=3, choices=[1, 2, 3, 4, 5])
    ap.add_argument("--form", default="both", choices=["both", "batched", "plain"])
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--cpu-frac", type=float, default=0.01,
                    help="share of the query bases the oracle checks (chunked workload)")
    ap.add_argument("--ref-frac", type=float, default=0.002,
                    help="reference arm: share of the query bases timed per step (chunked workload)")
    ap.add_argument("--cpu-query-bp", type=int, default=0,
                    help="one-query workloads: check the oracle on this prefix of the query as its own block")
    ap.add_argument("--plain-steps", type=int, default=3, help="timed steps of the plain form (at most --steps)")
    ap.add_argument("--e2e-steps", type=int, default=5, help="timed steps of the e2e leg (at most --steps)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving block of the default workload")
    ap.add_argument("--serve-scale", type=float, default=1.0 / 3.0,
                    help="serving block: resident target as a share of 3 Gbp")
    ap.add_argument("--serve-check", type=int, default=4, help="served requests checked against run_pass alone")
    ap.add_argument("--tuning", default="", help='JSON of engine launch knobs, e.g. {"gate_tile": 256}')
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default launch shapes")
    ap.add_argument("--tune-positions", type=int, default=1 << 24, help="seed positions the autotuner samples")
    ap.add_argument("--rate", type=float, default=50.0, help="config 5: Poisson arrival rate, requests/s")
    ap.add_argument("--requests", type=int, default=32, help="config 5: requests per timed window")
    ap.add_argument("--sweep", default="2,5", help="config 5: extra arrival rates, one window each")
    ap.add_argument("--sweep-requests", type=int, default=12)
    ap.add_argument("--workers", type=int, default=2, help="config 5: serving worker threads")
    ap.add_argument("--max-batch", type=int, default=16, help="config 5: queries per batch at most")
    ap.add_argument("--budget-gb", type=float, default=40.0, help="config 5: admission budget")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if args.config == 5:
            if rank == 0:
                print(json.dumps({"impl": "reference", "metric": METRIC, "unit": UNIT,
                                  "unavailable": "the reference has no serving loop; its CPU path is timed on "
                                                 "configs 2-4"}), flush=True)
            return
        run_reference(args, rank)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    try:
        if args.config == 5:
            run_serving(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
