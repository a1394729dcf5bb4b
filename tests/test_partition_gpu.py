"""GPU parity of PartitionRadix and SelectRadix(Par) against the oracle, through the C ABI.

Reference: Algorithm.PartitionRadix(this uint[] a, [start, length,] k or int[] k, threshold)
(PartitionRadix.cs:135-210, the in-place MSD partition of :15-113) and
ParallelAlgorithm.SelectRadixPar(this uint[] a, [start, length,] k) (SelectionRadixParallel.cs:
254-283).  Neither is stable and the order inside each part is the algorithm's own, so parity is
the observable contract: a[k_i] is bit-identical to the oracle's a[k_i] (the key the sorted
subarray has there), each part between consecutive indices holds the same multiset of keys as
the oracle's part, and the keys outside the subarray are untouched."""
import numpy as np
import pytest

from hpcsharp_b200 import algorithm, datagen, native

pytestmark = pytest.mark.gpu

DTYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
UVIEW = {4: np.uint32, 8: np.uint64}


def _keys(dt: str, n: int, seed: int, dup: bool) -> np.ndarray:
    a = datagen.by_name(dt, n, seed=seed)
    if dup:  # heavy duplicates: every key drawn from 7 values (runs of equal keys around every k)
        vals = a[:7].copy()
        a = vals[np.random.default_rng(seed).integers(0, vals.size, size=n)]
    return a


def _parts(b: np.ndarray, start: int, length: int, ks) -> list:
    bounds = [start] + sorted(set(int(k) for k in ks)) + [start + length]
    u = b.view(UVIEW[b.dtype.itemsize])
    out = []
    for lo, hi in zip(bounds[:-1], bounds[1:]):
        lo2 = lo + 1 if lo != start else lo  # a[k] itself is compared on its own
        out.append(np.sort(u[lo2:hi]))
    return out


def assert_partition_parity(orc, a, got, start, length, ks):
    want = a.copy()
    orc.partition_radix(want, start, length, np.sort(np.unique(ks)))
    u = UVIEW[a.dtype.itemsize]
    np.testing.assert_array_equal(got[:start].view(u), a[:start].view(u))
    np.testing.assert_array_equal(got[start + length:].view(u), a[start + length:].view(u))
    for k in ks:
        assert got[k:k + 1].view(u)[0] == want[k:k + 1].view(u)[0], f"a[{k}] differs from the oracle"
    for p, q in zip(_parts(got, start, length, ks), _parts(want, start, length, ks)):
        np.testing.assert_array_equal(p, q)
    # and the contract itself: every part lies between the keys at its ends
    key = orc.order_key(got)
    bounds = [start] + sorted(set(int(k) for k in ks)) + [start + length]
    for i, (lo, hi) in enumerate(zip(bounds[:-1], bounds[1:])):
        seg = key[lo:hi]
        if seg.size and i > 0:
            assert seg.min() >= key[lo]
        if seg.size and hi < start + length:
            assert seg.max() <= key[hi]


CASES = [
    # (n, start, length or None for the rest, ks relative to start)
    (1, 0, None, [0]),
    (2, 0, None, [1]),
    (1000, 0, None, [0, 999]),
    (100_003, 0, None, [50_001]),
    (100_003, 17, 90_001, [0, 45_000, 90_000]),
    (1_000_003, 5, None, [3, 99, 12_345, 999_990]),
    (1_000_003, 0, None, [10, 20, 30, 40, 50, 999_000]),  # more than four indices: the sort path
    (333_333, 1000, 200_000, [150_000, 150_000, 7]),      # repeated and unordered indices
]


@pytest.mark.parametrize("dup", [False, True], ids=["distinct", "dups"])
@pytest.mark.parametrize("case", range(len(CASES)))
@pytest.mark.parametrize("dt", DTYPES)
def test_partition_radix_parity(ctx, orc, dt, case, dup):
    n, start, length, rel = CASES[case]
    length = n - start if length is None else length
    ks = [start + r for r in rel]
    a = _keys(dt, n, seed=11 * case + (3 if dup else 0), dup=dup)
    got = a.copy()
    ctx.partition_radix(got, start, length, ks)
    assert_partition_parity(orc, a, got, start, length, ks)


@pytest.mark.parametrize("dt", DTYPES)
def test_select_radix_par_value(ctx, orc, dt):
    """SelectRadixPar returns the k-th smallest key of the subarray (k absolute) and leaves it at
    a[k]: the oracle's partition puts the same key there."""
    a0 = _keys(dt, 777_777, seed=5, dup=False)
    u = UVIEW[a0.dtype.itemsize]
    for start, length, k in ((0, 777_777, 0), (0, 777_777, 777_776), (0, 777_777, 388_888), (123, 500_000, 300_000)):
        a = a0.copy()
        v = algorithm.SelectRadixPar(a, k) if (start, length) == (0, a0.size) else algorithm.SelectRadixPar(
            a, start, length, k)
        want = a0.copy()
        orc.partition_radix(want, start, length, [k])
        assert np.array([v]).view(u)[0] == want[k:k + 1].view(u)[0]
        assert a[k:k + 1].view(u)[0] == want[k:k + 1].view(u)[0]
        assert_partition_parity(orc, a0, a, start, length, [k])


def test_partition_radix_python_mirror_forms(ctx, orc):
    """The reference's overloads: (a, k), (a, k[]), (a, start, length, k), (a, start, length, k[])."""
    a0 = _keys("u32", 200_003, seed=9, dup=False)
    for args in ((100_000,), ([5, 100_000, 200_000],), (10, 150_000, 70_000), (10, 150_000, [10, 150_009])):
        a = a0.copy()
        assert algorithm.PartitionRadix(a, *args) is None
        if len(args) == 1:
            start, length, k = 0, a0.size, args[0]
        else:
            start, length, k = args
        assert_partition_parity(orc, a0, a, start, length, list(np.atleast_1d(k)))


def test_partition_radix_errors(ctx):
    lib = native.load()
    a = np.arange(100, dtype=np.uint32)
    ks = np.array([5], dtype=np.int64)
    # ArgumentNullException: array, k
    assert lib.hpcs_partition_radix_u32(ctx.handle, None, 0, 10, ks.ctypes.data, 1) == native.HPCS_ERR_NULL
    assert lib.hpcs_partition_radix_u32(ctx.handle, a.ctypes.data, 0, 10, None, 1) == native.HPCS_ERR_NULL
    # ArgumentOutOfRangeException: start < 0, length <= 0, k outside the subarray
    assert lib.hpcs_partition_radix_u32(ctx.handle, a.ctypes.data, -1, 10, ks.ctypes.data, 1) == native.HPCS_ERR_RANGE
    assert lib.hpcs_partition_radix_u32(ctx.handle, a.ctypes.data, 0, 0, ks.ctypes.data, 1) == native.HPCS_ERR_RANGE
    bad = np.array([10], dtype=np.int64)
    assert lib.hpcs_partition_radix_u32(ctx.handle, a.ctypes.data, 0, 10, bad.ctypes.data, 1) == native.HPCS_ERR_RANGE
    # no indices: nothing happens
    b = a[::-1].copy()
    assert lib.hpcs_partition_radix_u32(ctx.handle, b.ctypes.data, 0, 100, None, 0) == native.HPCS_OK
    np.testing.assert_array_equal(b, a[::-1])
    out = np.zeros(1, dtype=np.uint32)
    assert lib.hpcs_select_radix_u32(ctx.handle, a.ctypes.data, 0, 10, 5, None) == native.HPCS_ERR_NULL
    assert lib.hpcs_select_radix_u32(ctx.handle, a.ctypes.data, 0, 10, 10, out.ctypes.data) == native.HPCS_ERR_RANGE
    with pytest.raises(native.ArgumentOutOfRangeException):
        algorithm.PartitionRadix(a.copy(), 100)
    with pytest.raises(native.ArgumentNullException):
        algorithm.PartitionRadix(None, 1)
    with pytest.raises(native.ArgumentOutOfRangeException):
        algorithm.SelectRadixPar(a.copy(), 5, 10, 3)
