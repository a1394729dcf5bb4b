"""Full-size workloads (the plain-sort-at-scale and pairs configurations): 256 Mi u32 uniform,
i32 normal(0, 2^20) and f32 normal(0,1) with specials; 128 Mi u64 uniform and AND-of-3;
200 M u64 Zipf(1.1) keys + u32 index items; 100 M f64 normal(0,1) keys + index items.

Each output is compared byte for byte with the oracle's SortRadixPar / SortRadix<T>(items,
keys) restatement run on the same seeded input on the host cores, and also checked through
size-independent properties on the GPU: the output is in the reference's key order, it is a
permutation of the input (order-independent checksums), and for key+index pairs every item
points at its key in the input and equal keys keep their input order (stability)."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native
from tests.gpu_util import checksum_dev, from_dev, is_sorted_dev, ordered_i64, to_dev

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def assert_same_bytes(got: np.ndarray, want: np.ndarray) -> None:
    assert got.shape == want.shape and got.dtype.itemsize == want.dtype.itemsize
    gu = got.view(np.uint32 if got.dtype.itemsize == 4 else np.uint64)
    wu = want.view(gu.dtype)
    if not np.array_equal(gu, wu):
        bad = np.flatnonzero(gu != wu)
        raise AssertionError(f"{bad.size} keys differ from the oracle, first at {bad[:5]}")


PLAIN = [
    ("u32", 1 << 28, lambda n: datagen.u32_uniform(n, 1)),
    ("i32", 1 << 28, lambda n: datagen.i32_normal(n, 1)),
    ("f32", 1 << 28, lambda n: datagen.f32_normal_special(n, 1)),
    ("u64", 1 << 27, lambda n: datagen.u64_uniform(n, 1)),
    ("u64", 1 << 27, lambda n: datagen.u64_and3(n, 1)),
]


@pytest.mark.parametrize("dt,n,gen", PLAIN, ids=["u32_256M", "i32_normal_256M", "f32_specials_256M",
                                                 "u64_uniform_128M", "u64_and3_128M"])
def test_plain_sort_at_scale(ctx, orc, dt, n, gen):
    import torch

    a = gen(n)
    t = to_dev(a)
    before = checksum_dev(t)
    ctx.sort_dev(t, dtype=dt, stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    assert is_sorted_dev(t, dt)
    assert checksum_dev(t) == before
    got = from_dev(t, a.dtype)
    del t
    torch.cuda.empty_cache()
    orc.sort_radix_par(a)  # in place: now the reference's result
    assert_same_bytes(got, a)


PAIRS = [
    ("u64", 200_000_000, lambda n: datagen.u64_zipf(n, 1)),
    ("f64", 100_000_000, lambda n: datagen.f64_normal(n, 1)),
]


@pytest.mark.parametrize("dt,n,gen", PAIRS, ids=["u64_zipf_200M_pairs", "f64_normal_100M_pairs"])
def test_pairs_at_scale(ctx, orc, dt, n, gen):
    import torch

    a = gen(n)
    keys = to_dev(a)
    orig = keys.clone()
    items = torch.arange(n, dtype=torch.int32, device="cuda")
    ctx.sort_pairs_dev(keys, items, dtype=dt, stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    assert is_sorted_dev(keys, dt)
    idx = items.to(torch.int64)
    # items are a permutation of 0..n-1 and each points at its key in the input
    assert int(idx.min()) == 0 and int(idx.max()) == n - 1
    assert int(idx.sum()) == n * (n - 1) // 2
    assert torch.equal(orig[idx], keys)
    # stability: equal keys keep increasing input positions
    o = ordered_i64(keys, dt)
    same = o[1:] == o[:-1]
    assert bool((idx[1:][same] > idx[:-1][same]).all())
    if dt == "u64":
        assert int(same.sum()) > n // 2  # Zipf duplicates are heavy
    got_keys = from_dev(keys, a.dtype)
    got_items = from_dev(items, np.uint32)
    del keys, orig, items, idx, o, same
    torch.cuda.empty_cache()
    want_items = np.arange(n, dtype=np.uint32)
    orc.sort_pairs(a, want_items)  # in place: the reference's keys and stable permutation
    assert_same_bytes(got_keys, a)
    assert_same_bytes(got_items, want_items)


def test_sort_beyond_2_to_30_keys(ctx):
    """A .NET array may hold up to 2^31 - 1 keys; the chunked passes use 32-bit positions, so a
    plain sort and a pairs sort of more than 2^30 keys work (sorted, a permutation, stable)."""
    import torch

    n = (1 << 30) + 4097
    a = datagen.u32_uniform(n, 5)
    t = to_dev(a)
    del a
    before = checksum_dev(t)
    ctx.sort_dev(t, dtype="u32", stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    assert is_sorted_dev(t, "u32")
    assert checksum_dev(t) == before
    # pairs: keys with heavy duplicates, items = input positions
    keys = (t[:n] & 0xFFFF).contiguous()  # a sorted-then-masked permutation: many equal keys
    orig = keys.clone()
    del t
    items = torch.arange(n, dtype=torch.int32, device="cuda")
    ctx.sort_pairs_dev(keys, items, dtype="u32", stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    assert is_sorted_dev(keys, "u32")
    idx = items.to(torch.int64)
    assert int(idx.sum()) == n * (n - 1) // 2
    assert torch.equal(orig[idx], keys)
    same = keys[1:] == keys[:-1]
    assert bool((idx[1:][same] > idx[:-1][same]).all())
    del keys, orig, items, idx, same
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dt,n,gen", PAIRS, ids=["u64_zipf_200M_pairs", "f64_normal_100M_pairs"])
def test_pairs_at_scale_both_rank_modes(ctx, dt, n, gen):
    """The shipping context ranks with ordered shared atomics when its probe passed; the
    peer-mask mode is fully defined by PTX.  Both must give the identical keys and stable
    permutation on the full-size pairs configurations (heavy duplicates: many same-address
    atomics per warp instruction)."""
    import torch

    peer = native.Context(0, rank_mode=1)
    try:
        a = gen(n)
        out = {}
        for name, c in (("ctx", ctx), ("peer", peer)):
            keys = to_dev(a)
            items = torch.arange(n, dtype=torch.int32, device="cuda")
            c.sort_pairs_dev(keys, items, dtype=dt, stream=native.torch_stream())
            torch.cuda.synchronize()
            c.synchronize()
            out[name] = (keys, items)
        assert peer.rank_mode == 1
        assert torch.equal(out["ctx"][0], out["peer"][0])
        assert torch.equal(out["ctx"][1], out["peer"][1])
        del out
        torch.cuda.empty_cache()
    finally:
        peer.close()
