"""Batched segmented sort: every array of a mixed batch equals the oracle's sort of that array
alone (bit for bit), for all dtypes and lengths around the in-shared-memory / tiled threshold,
through the one-shot call and the graph-captured plan."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native
from tests.gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

LENGTHS = [0, 1, 2, 31, 32, 33, 255, 4095, 4096, 4097, 8191, 8192, 8193, 20_000, 65_536, 300_001]
DT = ["u32", "i32", "f32", "u64", "i64", "f64"]


def make_batch(seed, lengths=LENGTHS, dtypes=DT):
    rng = np.random.default_rng(seed)
    host = []
    for i, n in enumerate(lengths):
        dt = dtypes[rng.integers(len(dtypes))] if len(dtypes) > 1 else dtypes[0]
        host.append((datagen.by_name(dt, n, seed=seed * 1000 + i), dt))
    return host


def oracle_sorted(orc, a):
    s = a.copy()
    orc.sort_radix_lsd(s)
    return s


def check(host, devs, orc):
    for (a, dt), t in zip(host, devs):
        got = from_dev(t, a.dtype) if a.size else a
        want = oracle_sorted(orc, a)
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8)), (dt, a.size)


@pytest.mark.parametrize("dt", DT)
def test_single_dtype_batch(ctx, orc, dt):
    import torch

    host = make_batch(11, dtypes=[dt])
    devs = [to_dev(a) if a.size else torch.empty(0, device="cuda") for a, _ in host]
    ctx.sort_segmented_dev([(t, d) for t, (_, d) in zip(devs, host)],
                           stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    check(host, devs, orc)


def test_mixed_batch_many_small(ctx, orc):
    import torch

    rng = np.random.default_rng(5)
    lengths = list((32 * 2 ** rng.uniform(0, 13, size=700)).astype(np.int64))
    host = make_batch(7, lengths=lengths)
    devs = [to_dev(a) for a, _ in host]
    ctx.sort_segmented_dev([(t, d) for t, (_, d) in zip(devs, host)],
                           stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    check(host, devs, orc)


def test_plan_graph_replays(ctx, orc):
    import torch

    host = make_batch(21)
    devs = [to_dev(a) if a.size else torch.empty(0, device="cuda") for a, _ in host]
    plan = ctx.segplan([(t, d) for t, (_, d) in zip(devs, host)])
    try:
        s = native.torch_stream()
        plan.execute(s)
        torch.cuda.synchronize()
        ctx.synchronize()
        check(host, devs, orc)
        # new data in the same arrays, same graph
        host2 = [(datagen.by_name(d, a.size, seed=999 + i), d) for i, (a, d) in enumerate(host)]
        for t, (a, _) in zip(devs, host2):
            if a.size:
                t.copy_(to_dev(a))
        torch.cuda.synchronize()
        plan.execute(s)
        torch.cuda.synchronize()
        ctx.synchronize()
        check(host2, devs, orc)
    finally:
        plan.close()


def test_segmented_equals_plain_sort(ctx):
    """The batched result equals the plain per-array entry point's result."""
    import torch

    host = make_batch(33, lengths=[5000, 9000, 123_457, 1_000_003])
    a_dev = [to_dev(a) for a, _ in host]
    b_dev = [to_dev(a) for a, _ in host]
    s = native.torch_stream()
    ctx.sort_segmented_dev([(t, d) for t, (_, d) in zip(a_dev, host)], stream=s)
    for t, (_, d) in zip(b_dev, host):
        ctx.sort_dev(t, dtype=d, stream=s)
    torch.cuda.synchronize()
    ctx.synchronize()
    for x, y in zip(a_dev, b_dev):
        assert torch.equal(x, y)


def test_segment_errors(ctx):
    import ctypes as C

    lib = native.load()
    arr = (native.HpcsSegment * 1)()
    arr[0].keys = None
    arr[0].n = 10
    arr[0].dtype = 0
    assert lib.hpcs_sort_segmented_dev(ctx.handle, arr, 1, None) == native.HPCS_ERR_NULL
    arr[0].keys = 16
    arr[0].dtype = 9
    assert lib.hpcs_sort_segmented_dev(ctx.handle, arr, 1, None) == native.HPCS_ERR_UNSUPPORTED
    assert lib.hpcs_sort_segmented_dev(ctx.handle, None, 0, None) == native.HPCS_OK


@pytest.mark.parametrize("variant", list(range(11)))
def test_every_variant_matches_oracle(orc, variant):
    """Each kernel variant (warp level with 8- or 4-bit digits, block level with each tile
    shape), forced onto every length class it can hold, sorts every array of a mixed batch
    exactly as the oracle sorts it alone, through the one-shot call and a plan."""
    import torch

    limits = native.seg_class_limits()
    variants = native.seg_variants()
    assert len(variants) == 11
    c = native.Context(0)
    try:
        table = c.seg_tuning
        lengths = []
        for w in range(2):
            cap = variants[variant]["max_keys"][w]
            for cl, lim in enumerate(limits):
                if cap < 0 or (lim >= 0 and lim <= cap):
                    table[w][cl] = variant
        c.seg_tuning = table
        assert c.seg_tuning == table
        rng = np.random.default_rng(variant)
        cap4 = variants[variant]["max_keys"][0]
        top = cap4 if cap4 > 0 else 40_000
        lengths = [0, 1, 2, 3, 31, 32, 33, 64, 65] + list((2 ** rng.uniform(1, np.log2(top), size=120)).astype(np.int64))
        lengths += [top, top - 1]
        host = make_batch(30 + variant, lengths=lengths)
        devs = [to_dev(a) if a.size else torch.empty(0, device="cuda") for a, _ in host]
        segs = [(t, d) for t, (_, d) in zip(devs, host)]
        c.sort_segmented_dev(segs, stream=native.torch_stream())
        torch.cuda.synchronize()
        c.synchronize()
        check(host, devs, orc)
        # the same arrays again through a graph-captured plan
        for t, (a, _) in zip(devs, host):
            if a.size:
                t.copy_(to_dev(a))
        torch.cuda.synchronize()
        plan = c.segplan(segs)
        plan.execute()
        c.synchronize()
        check(host, devs, orc)
        plan.close()
    finally:
        c.close()


def test_tuning_rejects_a_variant_too_small(ctx):
    table = ctx.seg_tuning
    bad = [row[:] for row in table]
    bad[0][7] = 0  # a 128-key warp variant cannot hold the unbounded class
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.seg_tuning = bad
    assert ctx.seg_tuning == table


def test_builtin_table_is_the_tuned_record(ctx):
    import json
    import os

    from hpcsharp_b200 import autotune

    rec = json.load(open(os.path.join(os.path.dirname(autotune.__file__), "tune", "b200_148sm.json")))
    assert ctx.seg_tuning == rec["table"]


GRID_LENGTHS = [65_536, 100_003, 262_145, 16_384 * 8 * 3 - 1, 1_048_576 + 7, 2_500_001]
# (minimum length, tiles per CTA): the defaults (65,536 and 32), and 2^18 keys with 8-tile
# ranges, where every array of the grid level spans several CTAs
GRID_GEOMETRIES = [(0, 0), (262_144, 8)]


@pytest.mark.parametrize("geometry", GRID_GEOMETRIES, ids=["default", "min256k_tiles8"])
@pytest.mark.parametrize("use_plan", [False, True], ids=["one_shot", "plan_twice"])
def test_grid_level_arrays(ctx, orc, use_plan, geometry):
    """Arrays of at least the context's grid-level length, with aligned keys, go to the grid
    level (the plain sort's kernels per range of the array); unaligned ones of the same length
    stay on the block level.  Constant and low-byte-only arrays make passes the identity (an odd
    number runs: the copy back).  Every array must equal the oracle's sort of it alone."""
    import torch

    if geometry != (0, 0):
        ctx = native.Context(0, seg_grid_min_keys=geometry[0], seg_grid_tiles=geometry[1])

    host = []
    for i, n in enumerate(GRID_LENGTHS):
        for j, dt in enumerate(DT):
            a = datagen.by_name(dt, n, seed=40 + 10 * i + j)
            if (i + j) % 5 == 3:
                a = a.copy()
                a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)[:] &= 0xFF  # low byte only
            if (i + j) % 7 == 5:
                a = np.full_like(a, a[0])  # every pass the identity
            host.append((a, dt))
    offsets = [1 if k % 4 == 1 else 0 for k in range(len(host))]  # every fourth array unaligned
    devs = [to_dev(a, offset_elems=o) for (a, _), o in zip(host, offsets)]
    segs = [(t, d) for t, (_, d) in zip(devs, host)]
    if use_plan:
        plan = ctx.segplan(segs)
        try:
            for rep in range(2):
                if rep:  # restore the inputs: the second replay sorts them again
                    for t, (a, _), o in zip(devs, host, offsets):
                        t.copy_(to_dev(a))
                plan.execute(stream=native.torch_stream())
                torch.cuda.synchronize()
                ctx.synchronize()
                check(host, devs, orc)
        finally:
            plan.close()
    else:
        ctx.sort_segmented_dev(segs, stream=native.torch_stream())
        torch.cuda.synchronize()
        ctx.synchronize()
        check(host, devs, orc)
    if geometry != (0, 0):
        ctx.close()
