"""Python view of the B200 engine, shaped like the reference's ``Engine``
(src/gpu/mod.rs:817-2307) and its pass driver ``seed_and_filter_all``
(src/run.rs:266-495).  All work happens in libhspz_b200.so through the C ABI;
this module only marshals host buffers.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _native as N
from .hsp import PASS_RECORD, SEGMENT_PAIR
from .scoring import build_sub_mat
from .sequence import as_bytes

BATCH_RECORD = np.dtype([("query", "<u4"), ("interval", "<u4"), ("strand", "<u4"),
                         ("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])


@dataclass
class EngineConfig:
    """Run flags that parameterise the path (src/cli.rs:41-183) and the
    EngineConfig knobs (src/gpu/mod.rs:1005-1019)."""
    sub_mat: List[int] = field(default_factory=lambda: build_sub_mat("", 910))
    seed: str = "12of19"
    xdrop: int = 910
    hspthresh: int = 3000
    noentropy: bool = False
    transitions: bool = True
    step: int = 1
    max_hits: int = 16711680
    occ_cap: int = 0
    wga_chunk: int = 250_000
    interval: int = 10_000_000
    strand: str = "both"

    def to_c(self) -> N.ConfigC:
        c = N.ConfigC()
        if len(self.sub_mat) != 64:
            raise ValueError("sub_mat must have 64 entries")
        for i, v in enumerate(self.sub_mat):
            c.sub_mat[i] = int(v)
        c.seed = self.seed.encode()[:63]
        c.xdrop, c.hspthresh = int(self.xdrop), int(self.hspthresh)
        c.noentropy, c.transitions = int(bool(self.noentropy)), int(bool(self.transitions))
        c.step, c.max_hits, c.occ_cap = int(self.step), int(self.max_hits), int(self.occ_cap)
        c.wga_chunk, c.interval = int(self.wga_chunk), int(self.interval)
        strands = {"plus": 1, "minus": 2, "both": 3}
        if self.strand not in strands:
            raise ValueError(f"--strand must be plus, minus or both, got {self.strand}")
        c.strand = strands[self.strand]
        return c


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _take(ptr: C.c_void_p, n: int, dtype) -> np.ndarray:
    if not ptr.value or n == 0:
        if ptr.value:
            N.lib().hz_free(ptr)
        return np.zeros(0, dtype=dtype)
    raw = (C.c_uint8 * (n * dtype.itemsize)).from_address(ptr.value)
    arr = np.frombuffer(raw, dtype=dtype).copy()
    N.lib().hz_free(ptr)
    return arr


def shape_info(seed: str = "12of19"):
    """(width, care positions) of a seed pattern (Shape::parse, src/seed.rs:49-79)."""
    size, k = C.c_uint32(), C.c_uint32()
    N.check(N.lib().hz_shape_info(seed.encode(), C.byref(size), C.byref(k)))
    return size.value, k.value


class Engine:
    """One engine per device; owns the resident target and the query."""

    def __init__(self, config: Optional[EngineConfig] = None, device: int = 0):
        self.config = config or EngineConfig()
        self._h = C.c_void_p()
        N.check(N.lib().hz_engine_create(C.byref(self.config.to_c()), device, C.byref(self._h)))
        self.seed_size, self.kmer_size = shape_info(self.config.seed)

    def close(self):
        if self._h and self._h.value:
            N.lib().hz_engine_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- target -----------------------------------------------------------
    def load_tables(self, index_table: np.ndarray, pos_table: np.ndarray, ref_seq: np.ndarray):
        """Engine::new's host-built tables (src/gpu/mod.rs:1005-1041)."""
        it = np.ascontiguousarray(index_table, dtype=np.uint32)
        pt = np.ascontiguousarray(pos_table, dtype=np.uint32)
        rs = np.ascontiguousarray(ref_seq, dtype=np.uint8)
        N.check(N.lib().hz_engine_load_tables(self._h, _ptr(it), it.size, _ptr(pt), pt.size, _ptr(rs), rs.size))

    def load_target(self, ref_ascii):
        """Build the seed table on the device from the ASCII reference block."""
        a = np.ascontiguousarray(as_bytes(ref_ascii))
        N.check(N.lib().hz_engine_load_target(self._h, _ptr(a), a.size))

    def read_tables(self):
        il, pl = C.c_uint64(), C.c_uint64()
        N.check(N.lib().hz_engine_read_tables(self._h, None, C.byref(il), None, C.byref(pl)))
        it = np.zeros(il.value, dtype=np.uint32)
        pt = np.zeros(max(pl.value, 1), dtype=np.uint32)
        N.check(N.lib().hz_engine_read_tables(self._h, _ptr(it), C.byref(il), _ptr(pt), C.byref(pl)))
        return it, pt[: pl.value]

    # --- query ------------------------------------------------------------
    def swap_query(self, query: np.ndarray, query_rc: np.ndarray):
        """Engine::swap_query with both strands in the device alphabet."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        r = np.ascontiguousarray(query_rc, dtype=np.uint8)
        if q.size != r.size:
            raise ValueError("query and query_rc differ in length")
        N.check(N.lib().hz_swap_query(self._h, _ptr(q), _ptr(r), q.size))

    def swap_query_ascii(self, query_ascii):
        a = np.ascontiguousarray(as_bytes(query_ascii))
        N.check(N.lib().hz_swap_query_ascii(self._h, _ptr(a), a.size))

    # --- per call -----------------------------------------------------------
    def upload_seeds(self, slot: int, seeds: np.ndarray):
        s = np.ascontiguousarray(seeds, dtype=np.uint64)
        N.check(N.lib().hz_upload_seeds(self._h, slot, _ptr(s), s.size))

    def generate_seeds(self, slot: int, rev: bool, rng, transitions: Optional[bool] = None) -> int:
        t = self.config.transitions if transitions is None else transitions
        n = C.c_uint64()
        N.check(N.lib().hz_generate_seeds(self._h, slot, int(bool(rev)), int(rng[0]), int(rng[1]), int(bool(t)),
                                          C.byref(n)))
        return n.value

    def seed_and_filter(self, slot: int, rev: bool):
        """FilterOutput: (hsps deduped per MAX_HITS chunk in LASTZ order, stats)."""
        out, n, st = C.c_void_p(), C.c_uint64(), N.StatsC()
        N.check(N.lib().hz_seed_and_filter(self._h, slot, int(bool(rev)), C.byref(out), C.byref(n), C.byref(st)))
        return _take(out, n.value, SEGMENT_PAIR), st.as_dict()

    def run_pass(self):
        """seed_and_filter_all over the swapped-in query, plain per-chunk form."""
        out, n, st = C.c_void_p(), C.c_uint64(), N.StatsC()
        N.check(N.lib().hz_run_pass(self._h, C.byref(out), C.byref(n), C.byref(st)))
        return _take(out, n.value, PASS_RECORD), st.as_dict()

    # --- batched form ---------------------------------------------------------
    def stage_queries(self, queries):
        """Keep many ASCII query blocks resident (both strands encoded on the device)."""
        arrs = [np.ascontiguousarray(as_bytes(q)) for q in queries]
        qs = (N.QueryC * max(len(arrs), 1))()
        for i, a in enumerate(arrs):
            qs[i].ascii = a.ctypes.data if a.size else None
            qs[i].len = a.size
        N.check(N.lib().hz_stage_queries(self._h, qs, len(arrs)))
        self._staged = arrs  # keep alive until the copies are done (they are synchronous)

    def select_query(self, index: int):
        """Point the per-call entry points (run_pass, seed_and_filter, ...) at
        staged query `index` without uploading it again."""
        N.check(N.lib().hz_select_query(self._h, index))

    def run_batched(self):
        """Every call of every staged query through shared waves; records per
        query in the same order run_pass gives for that query alone."""
        out, n, st = C.c_void_p(), C.c_uint64(), N.StatsC()
        N.check(N.lib().hz_run_batched(self._h, C.byref(out), C.byref(n), C.byref(st)))
        return _take(out, n.value, BATCH_RECORD), st.as_dict()

    # --- profiling ----------------------------------------------------------
    def set_profiling(self, on: bool = True):
        N.check(N.lib().hz_engine_set_profiling(self._h, int(bool(on))))

    def profile(self):
        out = {}
        i = 0
        name = C.create_string_buffer(128)
        ms, n = C.c_double(), C.c_uint64()
        while N.lib().hz_engine_profile_entry(self._h, i, name, 128, C.byref(ms), C.byref(n)) == 0:
            out[name.value.decode()] = (ms.value, n.value)
            i += 1
        return out

    def profile_reset(self):
        N.check(N.lib().hz_engine_profile_reset(self._h))

    def set_stream(self, stream_handle: int):
        """Run on a caller-owned cudaStream_t (an int handle, e.g.
        torch.cuda.current_stream().cuda_stream); 0 restores the own stream."""
        N.check(N.lib().hz_engine_set_stream(self._h, C.c_void_p(stream_handle or None)))

    def set_tuning(self, **knobs):
        """Launch-shape knobs: gate_version, gate_sparse, gate_tile, gate_cap,
        gate_blocks_per_sm, wave_positions, wave_hits_cap, device_dedup, device_dedup_min,
        graph, plain_streams, tile_cap, cand_cap, raw_cap.  Results never
        depend on them."""
        for k, v in knobs.items():
            N.check(N.lib().hz_engine_set_tuning(self._h, k.encode(), int(v)))

    def autotune(self, sample_positions: int = 0) -> dict:
        """Time candidate launch shapes on a sample of the staged work and keep
        the fastest (results never depend on them)."""
        t = N.TuningC()
        N.check(N.lib().hz_engine_autotune(self._h, int(sample_positions), C.byref(t)))
        return t.as_dict()

    @property
    def launches(self) -> int:
        return int(N.lib().hz_engine_launches(self._h))

    # --- serving loop ---------------------------------------------------------
    def serve_start(self, budget_bytes: int, workers: int = 2, max_batch_queries: int = 0):
        """Start worker threads that take submitted query blocks as they
        arrive, batching those that fit the device memory budget."""
        cfg = N.ServeConfigC(budget_bytes=int(budget_bytes), workers=int(workers),
                             max_batch_queries=int(max_batch_queries))
        N.check(N.lib().hz_serve_start(self._h, C.byref(cfg)))

    def serve_submit(self, query_ascii) -> int:
        a = np.ascontiguousarray(as_bytes(query_ascii))
        t = C.c_uint64()
        N.check(N.lib().hz_serve_submit(self._h, _ptr(a) if a.size else None, a.size, C.byref(t)))
        return t.value

    def serve_poll(self, ticket: int, timeout_ms: int = -1):
        """(records like run_pass, timings) for a finished ticket; raises
        HzError (HZ_E_TIMEOUT while it is still queued or running)."""
        out, n, tm = C.c_void_p(), C.c_uint64(), N.ServeTimesC()
        N.check(N.lib().hz_serve_poll(self._h, int(ticket), int(timeout_ms), C.byref(out), C.byref(n),
                                      C.byref(tm)))
        return _take(out, n.value, PASS_RECORD), tm.as_dict()

    def serve_estimate(self, length: int) -> int:
        """Device working memory the serving loop expects a request of
        `length` bases to need now."""
        b = C.c_uint64()
        N.check(N.lib().hz_serve_estimate(self._h, int(length), C.byref(b)))
        return b.value

    def serve_stats(self):
        """(totals over finished batches, requests queued, requests running)."""
        st, q, r = N.StatsC(), C.c_uint64(), C.c_uint64()
        N.check(N.lib().hz_serve_stats(self._h, C.byref(st), C.byref(q), C.byref(r)))
        return st.as_dict(), q.value, r.value

    def serve_cancel(self, ticket: int):
        N.check(N.lib().hz_serve_cancel(self._h, int(ticket)))

    def serve_stop(self):
        N.check(N.lib().hz_serve_stop(self._h))


def dedup_and_order(h: np.ndarray) -> np.ndarray:
    """dedup_and_order (src/hsp.rs:94-126) through the library's host code."""
    a = np.ascontiguousarray(h, dtype=SEGMENT_PAIR).copy()
    k = C.c_uint64()
    N.check(N.lib().hz_dedup_and_order(_ptr(a), a.size, C.byref(k)))
    return a[: k.value]
