"""The allocation-free device dedup entry point.

Some callers cannot allocate device memory: a host program whose own
allocator already owns the device, or a serving loop that admits work
against a fixed memory budget.  hz_dedup_and_order_device_noalloc serves them
with a scratch array built into the library.  Here the caller's buffers come
from PyTorch (standing in for such a host), and the results are checked
against the host entry point hz_dedup_and_order on the same records,
exactly, on two calls in a row that share the scratch array.  This file is
named to run last, so that a failure here leaves every other test already run.
"""
import ctypes as C

import numpy as np
import pytest

from hspz_b200 import _native as N
from hspz_b200 import engine as E
from hspz_b200.build import build
from hspz_b200.hsp import SEGMENT_PAIR

pytestmark = pytest.mark.gpu


def hsp_set(seed: int, n: int) -> np.ndarray:
    """Records with many duplicates and nested segments on shared diagonals,
    the shapes dedup has to resolve."""
    rng = np.random.default_rng(seed)
    a = np.zeros(n, dtype=SEGMENT_PAIR)
    diag = rng.integers(0, 400, n)
    a["query_start"] = rng.integers(0, 5000, n)
    a["ref_start"] = a["query_start"] + diag
    a["len"] = rng.integers(0, 300, n)
    a["score"] = rng.integers(3000, 9000, n)
    dup = rng.integers(0, n, n // 3)
    a[dup[: len(dup) // 2]] = a[dup[len(dup) // 2:]]
    return a


def test_noalloc_dedup_equals_host_entry_point_on_two_calls():
    import torch

    build()
    lib = N.lib()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    for seed, n in ((1, 60_000), (2, 45_000)):  # the second call reuses the scratch of the first
        recs = hsp_set(seed, n)
        want = E.dedup_and_order(recs)
        d_in = torch.from_numpy(recs.view(np.uint8).copy()).to(dev)
        d_out = torch.full((n * SEGMENT_PAIR.itemsize,), 0xAB, dtype=torch.uint8, device=dev)
        d_n = torch.zeros(1, dtype=torch.int32, device=dev)
        N.check(lib.hz_dedup_and_order_device_noalloc(C.c_void_p(d_in.data_ptr()), n, C.c_void_p(d_out.data_ptr()),
                                                      C.c_void_p(d_n.data_ptr()), C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize(dev)
        k = int(d_n.item())
        got = np.frombuffer(d_out[: k * SEGMENT_PAIR.itemsize].cpu().numpy().tobytes(), dtype=SEGMENT_PAIR)
        assert k == want.size and 0 < k < n
        assert got.tobytes() == want.tobytes()


def test_noalloc_dedup_refuses_more_than_its_scratch_holds():
    build()
    lib = N.lib()
    rc = lib.hz_dedup_and_order_device_noalloc(C.c_void_p(256), (1 << 18) + 1, C.c_void_p(256), C.c_void_p(256),
                                                None)
    assert rc == N.HZ_E_INVALID
    assert b"fixed scratch" in lib.hz_last_error()
