"""ctypes binding of the CPU oracle (oracle/hspz_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU legs of bench.py, always as the checker.  The product package never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libhspz_oracle.so")

HSP_DTYPE = np.dtype([("ref_start", "<u4"), ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])
OUT_DTYPE = np.dtype([("interval", "<u4"), ("strand", "<u4"), ("ref_start", "<u4"),
                      ("query_start", "<u4"), ("len", "<u4"), ("score", "<i4")])


class Shape(C.Structure):
    _fields_ = [("size", C.c_uint32), ("kmer_size", C.c_uint32),
                ("pos", C.c_uint32 * 32), ("transition", C.c_uint32 * 32)]


class Params(C.Structure):
    _fields_ = [("sub_mat", C.c_int32 * 64), ("xdrop", C.c_int32), ("hspthresh", C.c_int32),
                ("noentropy", C.c_uint32), ("max_hits", C.c_uint32), ("occ_cap", C.c_uint32),
                ("transitions", C.c_uint32), ("wga_chunk", C.c_uint32), ("interval", C.c_uint32),
                ("strand", C.c_uint32), ("threads", C.c_uint32)]


class Stats(C.Structure):
    _fields_ = [("seeds", C.c_uint64), ("hits", C.c_uint64), ("raw_hsps", C.c_uint64),
                ("hsps", C.c_uint64), ("cells", C.c_uint64), ("calls", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.hzo_encode.argtypes = [P, C.c_uint64, P]
        L.hzo_revcomp.argtypes = [P, C.c_uint64, P]
        L.hzo_shape_parse.argtypes = [C.c_char_p, C.POINTER(Shape)]
        L.hzo_seed_table_build.argtypes = [P, C.c_uint64, C.POINTER(Shape), C.c_uint32, P,
                                           C.POINTER(C.c_void_p), C.POINTER(C.c_uint64)]
        L.hzo_seed_and_filter.argtypes = [C.POINTER(Params), C.POINTER(Shape), P, C.c_uint64, P, P, P,
                                          C.c_uint64, C.c_uint32, C.c_uint32, C.POINTER(C.c_void_p),
                                          C.POINTER(C.c_uint64), C.POINTER(Stats)]
        L.hzo_seed_and_filter_all.argtypes = [C.POINTER(Params), C.POINTER(Shape), P, C.c_uint64, P, P,
                                              P, P, C.c_uint64, C.c_int64, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_uint64), C.POINTER(Stats)]
        L.hzo_dedup_and_order.argtypes = [P, C.c_uint64]
        L.hzo_dedup_and_order.restype = C.c_uint64
        L.hzo_extend_hit.argtypes = [P, C.c_uint32, P, C.c_uint32, C.POINTER(Params), C.c_uint32,
                                     C.c_uint32, P, C.POINTER(C.c_uint64), C.POINTER(C.c_int32)]
        L.hzo_ln_export.argtypes = [C.c_double]
        L.hzo_ln_export.restype = C.c_double
        L.hzo_batches.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, P]
        L.hzo_batches.restype = C.c_int64
        L.hzo_chunk_limits.argtypes = [P, C.c_uint64, C.c_uint32, P, C.c_uint32, C.POINTER(C.c_uint32)]
        L.hzo_free.argtypes = [P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def encode(ascii_bytes) -> np.ndarray:
    a = np.ascontiguousarray(np.frombuffer(bytes(ascii_bytes), dtype=np.uint8))
    out = np.empty_like(a)
    lib().hzo_encode(_ptr(a), a.size, _ptr(out))
    return out


def revcomp(ascii_bytes) -> np.ndarray:
    a = np.ascontiguousarray(np.frombuffer(bytes(ascii_bytes), dtype=np.uint8))
    out = np.empty_like(a)
    lib().hzo_revcomp(_ptr(a), a.size, _ptr(out))
    return out


def shape(spec: str = "12of19") -> Shape:
    s = Shape()
    if lib().hzo_shape_parse(spec.encode(), C.byref(s)) != 0:
        raise ValueError(f"bad seed shape {spec}")
    return s


def seed_table(codes: np.ndarray, sh: Shape, step: int = 1):
    codes = np.ascontiguousarray(codes, dtype=np.uint8)
    idx = np.zeros(1 << (2 * sh.kmer_size), dtype=np.uint32)
    p = C.c_void_p()
    n = C.c_uint64()
    rc = lib().hzo_seed_table_build(_ptr(codes), codes.size, C.byref(sh), step, _ptr(idx), C.byref(p),
                                    C.byref(n))
    if rc != 0:
        raise MemoryError("oracle seed table build failed")
    pos = np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint32)), shape=(max(n.value, 1),))[: n.value].copy()
    lib().hzo_free(p)
    return idx, pos


def params(sub_mat, xdrop=910, hspthresh=3000, noentropy=False, max_hits=16711680, occ_cap=0,
           transitions=True, wga_chunk=250000, interval=10000000, strand=3, threads=1) -> Params:
    p = Params()
    for i, v in enumerate(sub_mat):
        p.sub_mat[i] = int(v)
    p.xdrop, p.hspthresh, p.noentropy = xdrop, hspthresh, int(bool(noentropy))
    p.max_hits, p.occ_cap, p.transitions = max_hits, occ_cap, int(bool(transitions))
    p.wga_chunk, p.interval, p.strand, p.threads = wga_chunk, interval, strand, threads
    return p


def seed_and_filter(p: Params, sh: Shape, ref: np.ndarray, idx, pos, qry: np.ndarray, start: int, end: int):
    out = C.c_void_p()
    n = C.c_uint64()
    st = Stats()
    rc = lib().hzo_seed_and_filter(C.byref(p), C.byref(sh), _ptr(ref), ref.size, _ptr(idx), _ptr(pos),
                                   _ptr(qry), qry.size, start, end, C.byref(out), C.byref(n), C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle seed_and_filter failed: {rc}")
    arr = _take(out, n.value, HSP_DTYPE)
    return arr, st.as_dict()


def seed_and_filter_all(p: Params, sh: Shape, ref: np.ndarray, idx, pos, qf: np.ndarray, qr: np.ndarray,
                        max_batches: int = 0):
    out = C.c_void_p()
    n = C.c_uint64()
    st = Stats()
    rc = lib().hzo_seed_and_filter_all(C.byref(p), C.byref(sh), _ptr(ref), ref.size, _ptr(idx), _ptr(pos),
                                       _ptr(qf), _ptr(qr), qf.size, max_batches, C.byref(out), C.byref(n),
                                       C.byref(st))
    if rc != 0:
        raise RuntimeError(f"oracle seed_and_filter_all failed: {rc}")
    return _take(out, n.value, OUT_DTYPE), st.as_dict()


def dedup_and_order(h: np.ndarray) -> np.ndarray:
    a = np.ascontiguousarray(h, dtype=HSP_DTYPE).copy()
    k = lib().hzo_dedup_and_order(_ptr(a), a.size)
    return a[:k]


def extend_hit(p: Params, ref, qry, r: int, q: int):
    h = np.zeros(1, dtype=HSP_DTYPE)
    cells = C.c_uint64()
    total = C.c_int32()
    acc = lib().hzo_extend_hit(_ptr(ref), ref.size, _ptr(qry), qry.size, C.byref(p), r, q, _ptr(h),
                               C.byref(cells), C.byref(total))
    return bool(acc), h[0], cells.value, total.value


def ln(x: float) -> float:
    return lib().hzo_ln_export(x)


def chunk_limits(hit_num, max_hits: int):
    """The MAX_HITS chunk list (start_seed, last_seed, start_hit, end_hit)
    of one call's inclusive running hit counts; raises ValueError where the
    reference panics."""
    h = np.ascontiguousarray(hit_num, dtype=np.uint32)
    cap = int(h[-1]) // max(max_hits, 1) + 2
    out = np.zeros(4 * cap, dtype=np.uint32)
    n = C.c_uint32()
    rc = lib().hzo_chunk_limits(_ptr(h), h.size, max_hits, _ptr(out), cap, C.byref(n))
    if rc:
        raise ValueError(f"chunk_limits failed: {rc}")
    return [tuple(int(x) for x in out[4 * i: 4 * i + 4]) for i in range(n.value)]


def _take(ptr: C.c_void_p, n: int, dtype) -> np.ndarray:
    if not ptr.value:
        return np.zeros(0, dtype=dtype)
    raw = (C.c_uint8 * (n * dtype.itemsize)).from_address(ptr.value)
    arr = np.frombuffer(bytes(raw), dtype=dtype).copy()
    lib().hzo_free(ptr)
    return arr
