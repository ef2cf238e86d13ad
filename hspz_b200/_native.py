"""ctypes binding of libhspz_b200.so (the C ABI in include/hspz_b200.h).

The library is built in-tree (hspz_b200/_lib/) by ``hspz_b200.build``.  There
is no fallback: if the library or a usable sm_100 device is missing, the
calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libhspz_b200.so")

HZ_OK = 0
HZ_E_STATE = -1
HZ_E_CUDA = -5
HZ_E_OOM = -12
HZ_E_INVALID = -22
HZ_E_BUDGET = -28
HZ_E_TIMEOUT = -110


class HzError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"hspz_b200 error {code}: {msg}")
        self.code = code


class SegmentPairC(C.Structure):
    _fields_ = [("ref_start", C.c_uint32), ("query_start", C.c_uint32), ("len", C.c_uint32),
                ("score", C.c_int32)]


class PassRecordC(C.Structure):
    _fields_ = [("interval", C.c_uint32), ("strand", C.c_uint32), ("h", SegmentPairC)]


class ConfigC(C.Structure):
    _fields_ = [("sub_mat", C.c_int32 * 64), ("seed", C.c_char * 64), ("xdrop", C.c_int32),
                ("hspthresh", C.c_int32), ("noentropy", C.c_uint32), ("transitions", C.c_uint32),
                ("step", C.c_uint32), ("max_hits", C.c_uint32), ("occ_cap", C.c_uint32),
                ("wga_chunk", C.c_uint32), ("interval", C.c_uint32), ("strand", C.c_uint32)]


class StatsC(C.Structure):
    _fields_ = [("seeds", C.c_uint64), ("hits", C.c_uint64), ("raw_hsps", C.c_uint64), ("hsps", C.c_uint64),
                ("cells", C.c_uint64), ("calls", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class QueryC(C.Structure):
    _fields_ = [("ascii", C.c_void_p), ("len", C.c_uint64)]


class TuningC(C.Structure):
    _fields_ = [("gate_tile", C.c_int32), ("gate_cap", C.c_int32), ("gate_blocks_per_sm", C.c_int32),
                ("graph", C.c_int32), ("best_ms", C.c_double), ("start_ms", C.c_double),
                ("candidates", C.c_uint32), ("sample_calls", C.c_uint32), ("sample_positions", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class ServeConfigC(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("workers", C.c_uint32), ("max_batch_queries", C.c_uint32)]


class ServeTimesC(C.Structure):
    _fields_ = [("queued_ms", C.c_double), ("service_ms", C.c_double), ("total_ms", C.c_double),
                ("batch_queries", C.c_uint32), ("worker", C.c_uint32)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_lib = None

# (name, restype, argtypes) of every exported entry point.
P = C.c_void_p
U32, U64, I32 = C.c_uint32, C.c_uint64, C.c_int32
PU64 = C.POINTER(C.c_uint64)
SIGNATURES = {
    "hz_last_error": (C.c_char_p, []),
    "hz_free": (None, [P]),
    "hz_shape_info": (C.c_int, [C.c_char_p, C.POINTER(U32), C.POINTER(U32)]),
    "hz_engine_create": (C.c_int, [C.POINTER(ConfigC), C.c_int, C.POINTER(P)]),
    "hz_engine_destroy": (None, [P]),
    "hz_engine_load_tables": (C.c_int, [P, P, U64, P, U64, P, U64]),
    "hz_engine_load_target": (C.c_int, [P, P, U64]),
    "hz_engine_read_tables": (C.c_int, [P, P, PU64, P, PU64]),
    "hz_swap_query": (C.c_int, [P, P, P, U64]),
    "hz_swap_query_ascii": (C.c_int, [P, P, U64]),
    "hz_upload_seeds": (C.c_int, [P, U32, P, U64]),
    "hz_generate_seeds": (C.c_int, [P, U32, C.c_int, U32, U32, C.c_int, PU64]),
    "hz_seed_and_filter": (C.c_int, [P, U32, C.c_int, C.POINTER(P), PU64, C.POINTER(StatsC)]),
    "hz_run_pass": (C.c_int, [P, C.POINTER(P), PU64, C.POINTER(StatsC)]),
    "hz_dedup_and_order": (C.c_int, [P, U64, PU64]),
    "hz_render_records": (C.c_int, [P, U64, C.POINTER(C.c_char_p), U32, C.POINTER(C.c_char_p), U32, C.c_char,
                                    C.POINTER(P), PU64]),
    "hz_dedup_and_order_device_noalloc": (C.c_int, [P, U32, P, P, P]),
    "hz_stage_queries": (C.c_int, [P, C.POINTER(QueryC), U32]),
    "hz_select_query": (C.c_int, [P, U32]),
    "hz_run_batched": (C.c_int, [P, C.POINTER(P), PU64, C.POINTER(StatsC)]),
    "hz_engine_set_profiling": (C.c_int, [P, C.c_int]),
    "hz_engine_profile_entry": (C.c_int, [P, U32, C.c_char_p, U32, C.POINTER(C.c_double), PU64]),
    "hz_engine_profile_reset": (C.c_int, [P]),
    "hz_engine_launches": (U64, [P]),
    "hz_engine_set_stream": (C.c_int, [P, P]),
    "hz_engine_set_tuning": (C.c_int, [P, C.c_char_p, C.c_int64]),
    "hz_engine_autotune": (C.c_int, [P, U64, C.POINTER(TuningC)]),
    "hz_serve_start": (C.c_int, [P, C.POINTER(ServeConfigC)]),
    "hz_serve_submit": (C.c_int, [P, P, U64, PU64]),
    "hz_serve_poll": (C.c_int, [P, U64, C.c_int, C.POINTER(P), PU64, C.POINTER(ServeTimesC)]),
    "hz_serve_stats": (C.c_int, [P, C.POINTER(StatsC), PU64, PU64]),
    "hz_serve_estimate": (C.c_int, [P, C.c_uint64, PU64]),
    "hz_serve_cancel": (C.c_int, [P, U64]),
    "hz_serve_stop": (C.c_int, [P]),
}


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise HzError(HZ_E_STATE, f"{LIB_PATH} is not built; run hspz_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(rc: int):
    if rc != HZ_OK:
        raise HzError(rc, lib().hz_last_error().decode(errors="replace"))
