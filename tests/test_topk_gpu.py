"""GPU radix top-k against the oracle's SelectTopK restatement (SelectionTopKRadix.cs):
a[k] is the k-th smallest and a[k..] the multiset of the n-k largest, bit for bit; the prefix
here holds the k smallest; the k-largest form equals the tail of the oracle's sort."""
import json
import os

import numpy as np
import pytest

from hpcsharp_b200 import algorithm, datagen, native
from tests.gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

U = {4: np.uint32, 8: np.uint64}


def bits(a):
    return a.view(U[a.dtype.itemsize])


def oracle_sorted(orc, a):
    s = a.copy()
    orc.sort_radix_lsd(s)
    return s


def sorted_bits(orc, a):
    return bits(oracle_sorted(orc, a))


CASES = [(1, 0), (2, 0), (2, 1), (1000, 0), (1000, 999), (4097, 2048), (100_003, 50_000),
         (1_000_003, 999_990), (1_000_003, 10), (3_000_001, 1_500_000)]


@pytest.mark.parametrize("n,k", CASES)
@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_select_topk_contract(ctx, orc, dt, n, k):
    a = datagen.by_name(dt, n, seed=n * 7 + k)
    srt = sorted_bits(orc, a)
    ref = a.copy()
    if dt in ("u32", "i32", "f32", "u64"):  # the oracle's SelectTopK restatement
        assert orc.select_topk(ref, k) == 0
        assert bits(ref)[k] == srt[k]
    got = a.copy()
    ctx.select_topk(got, k)
    g = bits(got)
    assert g[k] == srt[k]
    np.testing.assert_array_equal(np.sort(g[k:]), np.sort(srt[k:]))   # multiset of the n-k largest
    np.testing.assert_array_equal(np.sort(g[:k]), np.sort(srt[:k]))   # and the k smallest before it
    if dt in ("u32", "i32", "f32", "u64"):
        np.testing.assert_array_equal(np.sort(g[k:]), np.sort(bits(ref)[k:]))


@pytest.mark.parametrize("kind", ["constant", "mod7", "two_values"])
def test_select_topk_duplicates(ctx, orc, kind):
    n = 200_001
    base = datagen.u32_uniform(n, seed=3)
    a = {"constant": np.full(n, 5, np.uint32), "mod7": base % np.uint32(7),
         "two_values": (base & np.uint32(1)) * np.uint32(0x01000001)}[kind]
    srt = np.sort(a)
    for k in (0, 1, n // 3, n - 1):
        got = a.copy()
        ctx.select_topk(got, k)
        assert got[k] == srt[k]
        np.testing.assert_array_equal(np.sort(got[k:]), srt[k:])


@pytest.mark.parametrize("poison", ["max", "zero"])
def test_sampled_window_falls_back(ctx, orc, poison):
    """The select and the k largest read a strided sample (8192 keys at stride n // 8192) to
    choose the keys worth keeping.  Keys planted at exactly the sample positions make the sample
    lie about the distribution; the selection must then take its fallback path (all keys, two
    reads) and still return the exact result."""
    n = 1_000_003
    a = datagen.u32_uniform(n, seed=11)
    stride = n // 8192
    a[np.arange(8192, dtype=np.int64) * stride] = np.uint32(0xFFFFFFFF if poison == "max" else 0)
    srt = np.sort(a)
    for k in (0, 17, n // 2, n - 5):
        got = a.copy()
        ctx.select_topk(got, k)
        assert got[k] == srt[k]
        np.testing.assert_array_equal(np.sort(got[k:]), srt[k:])
    for k in (10, 5000, 100_000):
        np.testing.assert_array_equal(ctx.topk_largest(a, k), srt[n - k:])


@pytest.mark.parametrize("k", [0, 1, 10, 1000, 100_000])
@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64"])
def test_topk_largest(ctx, orc, dt, k):
    n = 1_234_567
    a = datagen.by_name(dt, n, seed=k + 1)
    srt = sorted_bits(orc, a)
    out = ctx.topk_largest(a, k)
    np.testing.assert_array_equal(bits(out), srt[n - k:])


def test_topk_largest_device(ctx, orc):
    import torch

    n, k = 2_000_003, 1000
    a = datagen.f32_normal_special(n, seed=9)
    t = to_dev(a)
    out = torch.empty(k, dtype=torch.int32, device="cuda")
    ctx.topk_largest_dev(t, k, out, dtype="f32", stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    np.testing.assert_array_equal(bits(from_dev(out, np.float32)), sorted_bits(orc, a)[n - k:])


def test_select_topk_device_in_place(ctx, orc):
    import torch

    n, k = 1_000_003, 333_333
    a = datagen.u64_uniform(n, seed=4)
    t = to_dev(a)
    ctx.select_topk_dev(t, k, dtype="u64", stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    got = from_dev(t, np.uint64)
    srt = sorted_bits(orc, a)
    assert got[k] == srt[k]
    np.testing.assert_array_equal(np.sort(got[k:]), srt[k:])


def test_reference_wrapper_and_errors(ctx, orc):
    a = datagen.u32_uniform(100_000, seed=2)
    b = a.copy()
    algorithm.SelectTopK(b, 99_990)
    np.testing.assert_array_equal(np.sort(b[99_990:]), np.sort(a)[99_990:])
    c = a.copy()
    algorithm.SelectTopK(c, 1000, 50_000, 30_000)  # (start, length, k): k indexes the array
    sub = np.sort(a[1000:51_000])
    assert c[30_000] == sub[29_000]
    np.testing.assert_array_equal(np.sort(c[30_000:51_000]), sub[29_000:])
    np.testing.assert_array_equal(c[:1000], a[:1000])
    with pytest.raises(native.ArgumentOutOfRangeException):
        algorithm.SelectTopK(a.copy(), 100_000)  # k == Length
    with pytest.raises(native.ArgumentNullException):
        algorithm.SelectTopK(None, 1)
    lib = native.load()
    assert lib.hpcs_select_topk_u32(ctx.handle, a.ctypes.data, 0, 0) == native.HPCS_ERR_RANGE
    assert lib.hpcs_select_topk_u32(ctx.handle, a.ctypes.data, 10, -1) == native.HPCS_ERR_RANGE


def test_topk_golden(ctx):
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))["topk"][0]
    import hashlib

    a = datagen.by_name(g["dtype"], g["n"], g["seed"])
    b = a.copy()
    ctx.select_topk(b, g["k"])
    assert int(b[g["k"]]) == g["kth_value"]
    top = np.sort(b[g["k"]:])
    assert hashlib.sha256(top.view(np.uint8).tobytes()).hexdigest() == g["top_sorted_sha256"]


@pytest.mark.parametrize("dt", ["u32", "u64", "i32", "f32"])
def test_select_radix_contract(dt):
    """SelectRadix(a, k) returns the k-th smallest key and leaves it at a[k] (larger keys
    after it); SelectRadix(a, start, length, k) does so within the subarray with k indexing
    the whole array; SelectRadix(a, [k...]) leaves every a[k_i] at the k_i-th smallest."""
    a0 = datagen.by_name(dt, 300_007, seed=77)
    srt = a0.copy()
    native.default_context().sort(srt)
    for k in (0, 1, 150_000, 300_006):
        a = a0.copy()
        v = algorithm.SelectRadix(a, k)
        assert v.tobytes() == srt[k].tobytes() and a[k].tobytes() == srt[k].tobytes()
    a = a0.copy()
    v = algorithm.SelectRadix(a, 1000, 50_000, 20_000)
    sub = a0[1000:51_000].copy()
    native.default_context().sort(sub)
    assert v.tobytes() == sub[19_000].tobytes()
    assert np.array_equal(a[:1000], a0[:1000]) and np.array_equal(a[51_000:], a0[51_000:])
    a = a0.copy()
    ks = np.array([3, 99, 12_345, 299_000])
    assert algorithm.SelectRadix(a, ks) is None
    for k in ks:
        assert a[k].tobytes() == srt[k].tobytes()
    with pytest.raises(native.ArgumentOutOfRangeException):
        algorithm.SelectRadix(a0.copy(), a0.size)
