"""The uint32 device sort that allocates nothing (hpcs_sort_u32_dev_noalloc), called through
the C ABI, must give the same bits as the regular context-based entry point
(hpcs_sort_u32_dev): integer keys, so the tolerance is exact equality.  It is meant for callers
that cannot allocate GPU memory -- their framework owns every device allocation, or
cudaMalloc/cudaFree are not allowed where they call -- and takes all its scratch from a fixed
array compiled into the library, so it is limited to HPCS_NOALLOC_MAX_KEYS keys.

This file is collected last so that a failure here cannot hide the other tests."""
import ctypes as C

import numpy as np
import pytest

from hpcsharp_b200 import datagen, native
from tests.gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

NOALLOC_MAX_KEYS = 1 << 20


def _entry():
    lib = native.load()
    fn = lib.hpcs_sort_u32_dev_noalloc
    fn.argtypes = [C.c_void_p, C.c_int64, C.c_void_p]
    fn.restype = C.c_int
    return lib, fn


def _inputs(kind: str, n: int, seed: int) -> np.ndarray:
    a = datagen.u32_uniform(n, seed=seed)
    if kind == "below_2_24":
        return a & np.uint32(0x00FFFFFF)  # top digit all zero: three passes run, an odd number
    if kind == "constant":
        return np.full(n, 0xDEADBEEF, dtype=np.uint32)  # every pass skipped
    return a


# (keys, n, seed) of consecutive calls: the scratch keeps each call's contents for the next
CALLS = [("uniform", NOALLOC_MAX_KEYS, 101), ("uniform", 777_777, 202), ("below_2_24", 999_999, 303),
         ("constant", 65_537, 404), ("uniform", 4_099, 505)]


def test_no_alloc_sort_matches_context_sort_and_numpy():
    """Several calls in a row, each compared bit for bit with the context-based sort and with
    numpy's sort: whole digit passes, an odd number of executed passes (the result comes back
    from the scratch array) and all passes skipped."""
    import torch

    lib, fn = _entry()
    ctx = native.Context(0)
    try:
        stream = torch.cuda.current_stream().cuda_stream
        for kind, n, seed in CALLS:
            a = _inputs(kind, n, seed)
            t_noalloc = to_dev(a)
            t_regular = to_dev(a)
            rc = fn(t_noalloc.data_ptr(), n, stream)
            assert rc == native.HPCS_OK, lib.hpcs_last_error_message()
            ctx.sort_dev(t_regular, dtype="u32", stream=stream)
            torch.cuda.synchronize()
            ctx.synchronize()
            got = from_dev(t_noalloc, np.uint32)
            np.testing.assert_array_equal(got, from_dev(t_regular, np.uint32))
            np.testing.assert_array_equal(got, np.sort(a))
    finally:
        ctx.close()


def test_no_alloc_sort_rejects_too_many_keys():
    import torch

    lib, fn = _entry()
    t = torch.zeros(NOALLOC_MAX_KEYS + 1, dtype=torch.int32, device="cuda")
    rc = fn(t.data_ptr(), NOALLOC_MAX_KEYS + 1, torch.cuda.current_stream().cuda_stream)
    assert rc == native.HPCS_ERR_RANGE
    assert b"HPCS_NOALLOC_MAX_KEYS" in lib.hpcs_last_error_message()
    assert fn(None, 10, None) == native.HPCS_ERR_NULL


def test_no_alloc_sort_refuses_a_stream_under_capture():
    """The call synchronises with its stream, so on a stream being captured into a CUDA graph it
    returns HPCS_ERR_UNSUPPORTED and enqueues nothing (the capture stays valid)."""
    import torch

    lib, fn = _entry()
    a = datagen.u32_uniform(10_000, seed=9)
    t = to_dev(a)
    s = torch.cuda.Stream()
    assert fn(t.data_ptr(), a.size, s.cuda_stream) == native.HPCS_OK  # set-up outside any capture
    torch.cuda.synchronize()
    u = to_dev(a)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        rc = fn(u.data_ptr(), a.size, s.cuda_stream)
        u.add_(0)  # the capture holds at least this kernel
    assert rc == native.HPCS_ERR_UNSUPPORTED
    assert b"captured" in lib.hpcs_last_error_message()
    g.replay()
    torch.cuda.synchronize()
    np.testing.assert_array_equal(from_dev(u, np.uint32), a)  # nothing was sorted
    np.testing.assert_array_equal(from_dev(t, np.uint32), np.sort(a))
