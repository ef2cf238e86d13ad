"""CPU-side checks of the C-ABI library: it loads, exports every entry point
include/hspz_b200.h declares, refuses to run without a device, and its host
code (Shape::parse, dedup_and_order) matches the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import oracle
from hspz_b200 import _native as N
from hspz_b200 import engine as E
from hspz_b200.build import build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def built():
    build()


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "hspz_b200.h")).read()
    return sorted(set(re.findall(r"\b(hz_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(N.LIB_PATH)
    names = declared_symbols()
    assert len(names) >= 15
    for n in names:
        assert hasattr(lib, n), f"{n} declared but not exported"
    assert set(names) == set(N.SIGNATURES), "ctypes signatures drifted from the header"


def test_no_device_means_a_loud_error():
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(N.HzError) as ei:
        E.Engine()
    assert ei.value.code == N.HZ_E_CUDA


def test_shape_info_matches_oracle():
    for spec in ["12of19", "14of22", "11011", "TTT0T00TT00T0T0TTTT", "110111"]:
        s = oracle.shape(spec)
        assert E.shape_info(spec) == (s.size, s.kmer_size)
    with pytest.raises(N.HzError):
        E.shape_info("101")
    with pytest.raises(N.HzError):
        E.shape_info("1" * 16)


def test_library_dedup_matches_oracle():
    rng = np.random.default_rng(11)
    for n in [0, 1, 2, 17, 300]:
        a = np.zeros(n, dtype=oracle.HSP_DTYPE)
        a["ref_start"] = rng.integers(0, 50, n)
        a["query_start"] = rng.integers(0, 50, n)
        a["len"] = rng.integers(0, 20, n)
        a["score"] = rng.integers(-3, 3, n)
        got = E.dedup_and_order(a)
        want = oracle.dedup_and_order(a)
        assert got.tobytes() == want.tobytes()
    # field extremes: coordinates near 2^32 (wrapping ends) and scores at both
    # ends of i32, which the library's sort keys flip for descending order
    for n in [64, 3000]:
        a = np.zeros(n, dtype=oracle.HSP_DTYPE)
        edge = np.array([0, 1, 2, 0xFFFFFFFD, 0xFFFFFFFE, 0xFFFFFFFF], dtype=np.uint64)
        a["ref_start"] = rng.choice(edge, n)
        a["query_start"] = rng.choice(edge, n)
        a["len"] = rng.choice(np.array([0, 1, 2, 0xFFFFFFFF], dtype=np.uint64), n)
        a["score"] = rng.choice(np.array([-2**31, -2**31 + 1, -1, 0, 1, 2**31 - 2, 2**31 - 1]), n)
        assert E.dedup_and_order(a).tobytes() == oracle.dedup_and_order(a).tobytes()
    # wrapping diagonal: query start beyond ref start sorts last (src/hsp.rs:298-303)
    a = np.array([(4, 10, 0, 0), (10, 4, 0, 0)], dtype=oracle.HSP_DTYPE)
    assert E.dedup_and_order(a).tolist() == [(10, 4, 0, 0), (4, 10, 0, 0)]


def test_noalloc_dedup_refuses_bad_buffers_before_touching_a_device():
    """The allocation-free dedup checks its arguments on the host first, so
    these refusals need no GPU: too many records, null, misaligned and
    overlapping buffers (it reads d_in while writing d_out, so an in-place
    call would corrupt its own input)."""
    lib = N.lib()
    f = lib.hz_dedup_and_order_device_noalloc
    P = C.c_void_p
    n = 1000
    cases = [
        ((1 << 18) + 1, P(0x100000), P(0x900000), P(0x80), "fixed scratch"),
        (n, None, P(0x900000), P(0x80), "null device pointer"),
        (n, P(0x100002), P(0x900000), P(0x80), "4-byte aligned"),
        (n, P(0x100000), P(0x100000), P(0x80), "must not overlap"),            # in place
        (n, P(0x100000), P(0x100000 + 16 * n - 16), P(0x80), "must not overlap"),  # last record shared
        (n, P(0x100000), P(0x900000), P(0x100000 + 64), "must not overlap"),   # count inside d_in
        (n, P(0x100000), P(0x900000), P(0x900000 + 16 * n - 4), "must not overlap"),  # count inside d_out
    ]
    for count, d_in, d_out, d_n, msg in cases:
        assert f(d_in, count, d_out, d_n, None) == N.HZ_E_INVALID
        assert msg.encode() in lib.hz_last_error()
