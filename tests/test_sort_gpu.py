"""GPU parity of the plain LSD sort against the oracle (bit-exact), through the C ABI.

Sizes straddle the 4096/8192-key tile boundaries and the 16-byte bulk-copy tail; the
distributions include the adversarial ones (constant, presorted, reversed, single-bin
digits, AND-of-3 low entropy, heavy duplicates) and the float specials."""
import numpy as np
import pytest

from hpcsharp_b200 import algorithm, datagen, native
from tests.gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

DTYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
SIZES = [1, 2, 3, 5, 17, 255, 256, 257, 4095, 4096, 4097, 8191, 8192, 8193, 65539, 1_000_003]


def oracle_sorted(orc, a):
    s = a.copy()
    orc.sort_radix_lsd(s)
    return s


def assert_same_bits(x, y):
    assert x.dtype == y.dtype and x.shape == y.shape
    if not np.array_equal(x.view(np.uint8), y.view(np.uint8)):
        bad = np.flatnonzero(x.view(SIGNED_U[x.dtype.itemsize]) != y.view(SIGNED_U[y.dtype.itemsize]))
        raise AssertionError(f"{bad.size} mismatches, first at {bad[:5]}")


SIGNED_U = {4: np.uint32, 8: np.uint64}


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", DTYPES)
def test_host_sort_parity(ctx, orc, dt, n):
    a = datagen.by_name(dt, n, seed=1000 + n)
    want = oracle_sorted(orc, a)
    got = a.copy()
    ctx.sort(got)
    assert_same_bits(got, want)


def test_known_answer_program_cs(ctx):
    # HPCsharpExamples/HPCsharpExamples/Program.cs:15-34
    for dt in (np.uint32, np.int32, np.uint64, np.int64, np.float32, np.float64):
        a = np.array([21, 43, 16, 5, 54, 3], dtype=dt)
        ctx.sort(a)
        assert a.tolist() == [3, 5, 16, 21, 43, 54]


@pytest.mark.parametrize("seedfn", ["pcg32", "xorshift64s"])
def test_config1_10m_u32(ctx, orc, seedfn):
    """10,000,000 uint32 uniform from a seeded PCG32 / xorshift64* stream: equal to the
    restated SortRadix (serial and parallel) and to std::sort (the Array.Sort stand-in)."""
    n = 10_000_000
    a = datagen.u32_pcg32_stream(n, 1) if seedfn == "pcg32" else datagen.u32_xorshift64s(n, 1)
    serial = oracle_sorted(orc, a)
    par = a.copy()
    orc.sort_radix_par(par)
    std = a.copy()
    orc.std_sort(std)
    got = a.copy()
    algorithm.SortRadixPar(got)
    assert_same_bits(got, serial)
    assert_same_bits(got, par)
    assert_same_bits(got, std)


def _adversarial(dt, n, kind):
    npdt = native.NP_OF[dt]
    w = np.dtype(npdt).itemsize
    u = np.uint32 if w == 4 else np.uint64
    if kind == "constant":
        return np.full(n, 7, dtype=u).view(npdt)
    if kind == "zeros":
        return np.zeros(n, dtype=npdt)
    base = datagen.by_name(dt, n, seed=77)
    if kind == "sorted":
        s = base.copy()
        s.sort(kind="stable")
        return s
    if kind == "reversed":
        s = base.copy()
        s.sort(kind="stable")
        return s[::-1].copy()
    if kind == "single_bin_byte1":
        b = base.view(u).copy()
        b &= ~u(0xFF00)
        b |= u(0x3400)
        return b.view(npdt)
    if kind == "two_values":
        b = (base.view(u) & u(1)).astype(u) * u(0x01000001)
        return b.view(npdt)
    if kind == "dups_mod_1000":
        return (base.view(u) % u(1000)).astype(u).view(npdt)
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["constant", "zeros", "sorted", "reversed", "single_bin_byte1", "two_values",
                                  "dups_mod_1000"])
@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64"])
def test_adversarial_distributions(ctx, orc, dt, kind):
    a = _adversarial(dt, 300_001, kind)
    want = oracle_sorted(orc, a)
    got = a.copy()
    ctx.sort(got)
    assert_same_bits(got, want)


def test_low_entropy_u64_and3(ctx, orc):
    a = datagen.u64_and3(2_000_003, seed=3)
    want = oracle_sorted(orc, a)
    got = a.copy()
    ctx.sort(got)
    assert_same_bits(got, want)


@pytest.mark.parametrize("skip", [True, False])
def test_skip_trivial_passes_same_result(orc, skip):
    c = native.Context(0, skip_trivial_passes=skip)
    try:
        for kind in ("single_bin_byte1", "constant", "two_values"):
            a = _adversarial("u32", 123_457, kind)
            want = oracle_sorted(orc, a)
            got = a.copy()
            c.sort(got)
            assert_same_bits(got, want)
    finally:
        c.close()


@pytest.mark.parametrize("offset", [0, 1, 3])
@pytest.mark.parametrize("dt", DTYPES)
def test_device_sort_parity(ctx, orc, dt, offset):
    import torch

    a = datagen.by_name(dt, 777_777, seed=21)
    want = oracle_sorted(orc, a)
    t = to_dev(a, offset)
    ctx.sort_dev(t, dtype=dt, stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    assert_same_bits(from_dev(t, a.dtype), want)


def test_repeated_calls_reuse_scratch(ctx, orc):
    # shrinking and growing sizes on one context
    for n in (5_000_000, 1000, 3_000_001, 8192, 1):
        a = datagen.u32_uniform(n, seed=n)
        want = oracle_sorted(orc, a)
        got = a.copy()
        ctx.sort(got)
        assert_same_bits(got, want)


def test_argument_errors(ctx):
    lib = native.load()
    a = np.zeros(10, dtype=np.uint32)
    assert lib.hpcs_sort_u32(ctx.handle, None, 10) == native.HPCS_ERR_NULL
    assert lib.hpcs_sort_u32(ctx.handle, a.ctypes.data, -1) == native.HPCS_ERR_RANGE
    assert lib.hpcs_sort_u32(ctx.handle, a.ctypes.data, 0) == native.HPCS_OK
    assert lib.hpcs_sort_u32(ctx.handle, a.ctypes.data, (1 << 31)) == native.HPCS_ERR_RANGE
    # select / top-k keep the 2^30 - 1 limit (checked before any copy)
    assert lib.hpcs_select_topk_u32(ctx.handle, a.ctypes.data, (1 << 30), 0) == native.HPCS_ERR_RANGE
    with pytest.raises(native.ArgumentNullException):
        algorithm.SortRadixPar(None)


def test_subrange_sort_in_place(ctx, orc):
    a = datagen.u32_uniform(100_000, seed=4)
    b = a.copy()
    algorithm.SortRadixLsd(b, 1000, 50_000)
    want = a.copy()
    want[1000:51_000] = oracle_sorted(orc, a[1000:51_000].copy())
    assert_same_bits(b, want)


def test_pool_budget_is_enforced(orc):
    c = native.Context(0, pool_bytes=1 << 20)
    try:
        a = datagen.u32_uniform(1_000_000, seed=1)
        with pytest.raises(native.HpcsError) as e:
            c.sort(a)
        assert e.value.status == native.HPCS_ERR_OOM
        small = datagen.u32_uniform(10_000, seed=2)
        want = oracle_sorted(orc, small)
        c.sort(small)
        assert_same_bits(small, want)
    finally:
        c.close()


@pytest.mark.parametrize("scheme", ["chunked", "lookback"])
def test_device_wait_is_bounded(orc, scheme):
    """Look-back passes: a unit that never publishes (host-set test hook) makes every later
    unit's look-back run out after the spin limit.  Chunked passes: the hooked tile waits on
    a flag that nothing sets.  Either way the call returns HPCS_ERR_DEVICE_TIMEOUT and the
    context stays usable."""
    n = 600_000  # several look-back units after the poisoned one, whatever the unit size
    c = native.Context(0, spin_limit_ns=20_000_000, poison_tile=1, pass_scheme=scheme)
    try:
        a = datagen.u32_uniform(n, seed=1)
        with pytest.raises(native.DeviceTimeoutError):
            c.sort(a)
    finally:
        c.close()
    c2 = native.Context(0)
    try:
        a = datagen.u32_uniform(n, seed=1)
        want = oracle_sorted(orc, a)
        c2.sort(a)
        assert_same_bits(a, want)
    finally:
        c2.close()


def test_rank_probe_selects_a_mode(ctx):
    # 0 = ordered shared atomics (lane order verified on this GPU), 1 = peer-mask ranking
    assert ctx.rank_mode in (0, 1)


@pytest.mark.parametrize("dt", DTYPES)
def test_peer_mask_ranking_parity(orc, dt):
    """The fully defined peer-mask ranking gives the same bits as the oracle."""
    c = native.Context(0, rank_mode=1)
    try:
        assert c.rank_mode == 1
        for n in (4097, 300_001):
            a = datagen.by_name(dt, n, seed=55 + n)
            want = oracle_sorted(orc, a)
            got = a.copy()
            c.sort(got)
            assert_same_bits(got, want)
        keys = _adversarial(dt if dt in ("u32", "i32", "f32", "u64") else "u64", 100_003, "dups_mod_1000")
        want = oracle_sorted(orc, keys)
        got = keys.copy()
        c.sort(got)
        assert_same_bits(got, want)
    finally:
        c.close()


def test_known_answer_user_defined_class_sort():
    """HPCsharpExamples/HPCsharpExamples/SortOfUserDefinedClass.cs:87-104: SortRadix(element =>
    element.Key) of the example's (Key, Index) objects, stable: the two 18s keep their order."""
    items = [(16, 0), (12, 1), (18, 2), (18, 3), (10, 4), (2, 5)]
    want = [(2, 5), (10, 4), (12, 1), (16, 0), (18, 2), (18, 3)]
    assert algorithm.SortRadixLsd(items, lambda t: t[0]) == want
    assert algorithm.SortRadixFaster(items, lambda t: t[0]) == want


@pytest.mark.parametrize("wide", [False, True])
def test_user_defined_type_sort_by_key(wide):
    """SortRadixLsd(items, getKey) / SortRadixFaster: stable ascending by the extracted key, a
    new list, equal to Python's stable sort by the same key."""
    rng = np.random.default_rng(9)
    n = 200_003
    hi = (1 << 40) if wide else 1000
    items = [(int(k), i) for i, k in enumerate(rng.integers(0, hi, size=n, dtype=np.uint64))]
    want = sorted(items, key=lambda t: t[0])
    assert algorithm.SortRadixLsd(items, lambda t: t[0]) == want
    assert algorithm.SortRadixFaster(items, lambda t: t[0]) == want
    assert algorithm.SortRadixLsd([], lambda t: t) == []


@pytest.mark.parametrize("dt", ["f32", "f64", "i32"])
def test_sort_radix_msd_alias(ctx, orc, dt):
    a = datagen.by_name(dt, 100_003, seed=5)
    want = oracle_sorted(orc, a)
    got = algorithm.SortRadixMsd(a.copy())
    assert_same_bits(got, want)


@pytest.mark.parametrize("dt", [np.uint8, np.int8, np.uint16, np.int16])
@pytest.mark.parametrize("n", [1, 15, 16, 17, 4099, 1_000_003, 40_000_001])
def test_counting_sort_8_16_bit(ctx, dt, n):
    """SortCountingInPlace / SortCounting for byte, sbyte, ushort and short keys: equal to a
    stable sort by value (uniform and skewed values, ragged 16-byte tails)."""
    rng = np.random.default_rng(n)
    info = np.iinfo(dt)
    a = rng.integers(info.min, int(info.max) + 1, size=n, dtype=np.int64).astype(dt)
    if n > 1000:
        a[: n // 3] = dt(7)  # one value holds a third of the keys
        rng.shuffle(a)
    want = np.sort(a, kind="stable")
    got = algorithm.SortCounting(a)
    assert np.array_equal(got, want)
    b = a.copy()
    algorithm.SortCountingInPlace(b)
    assert np.array_equal(b, want)


@pytest.mark.parametrize("dt", [np.uint8, np.int16])
def test_counting_sort_one_value_and_two_runs(ctx, dt):
    """Runs that span every fill range of the output: all keys equal, and two values only."""
    n = 3_000_017
    for a in (np.full(n, 5, dtype=dt), np.where(np.arange(n) % 3 == 0, dt(-1 if dt == np.int16 else 200), dt(4))):
        want = np.sort(a, kind="stable")
        b = a.copy()
        algorithm.SortCountingInPlace(b)
        assert np.array_equal(b, want)


def test_counting_sort_device_unaligned(ctx):
    import torch

    a = np.random.default_rng(3).integers(0, 65536, size=100_003, dtype=np.int64).astype(np.uint16)
    t = torch.from_numpy(a.view(np.int16).copy()).cuda()
    big = torch.zeros(a.size + 3, dtype=torch.int16, device="cuda")
    big[3:].copy_(t)
    lib = native.load()
    native.check(lib.hpcs_sort_u16_dev(ctx.handle, big.data_ptr() + 6, a.size, native.torch_stream()))
    torch.cuda.synchronize()
    ctx.synchronize()
    assert np.array_equal(big[3:].cpu().numpy().view(np.uint16), np.sort(a))


SMALL_SORT_SIZES = [4096 * 31 + 1, 131_072, 131_073]  # 32 CTAs (one partial), the maximum, one past it


@pytest.mark.parametrize("rank_mode", [0, 1], ids=["ordered_atomic", "peer_mask"])
@pytest.mark.parametrize("n", SMALL_SORT_SIZES)
@pytest.mark.parametrize("dt", ["u32", "f32", "i64"])
def test_small_sort_limits(orc, dt, n, rank_mode):
    """Keys-only sorts of up to 128 Ki keys run all their passes in one cooperative launch
    (one 4096-key slice per CTA, a grid barrier between the count and the scatter of each pass);
    one key more takes the large-array kernels.  Both sides of the limit, both ranking modes,
    bit-exact against the oracle, with duplicates so that stability across slices matters."""
    a = datagen.by_name(dt, n, seed=77 + n)
    a[::3] = a[0]  # a run of equal keys spread over every slice
    want = oracle_sorted(orc, a)
    c = native.Context(0, rank_mode=rank_mode)
    try:
        got = a.copy()
        c.sort(got)
        assert_same_bits(got, want)
    finally:
        c.close()


@pytest.mark.parametrize("rank_mode", [0, 1], ids=["ordered_atomic", "peer_mask"])
@pytest.mark.parametrize("n", SMALL_SORT_SIZES)
def test_small_pairs_sort_limits(orc, n, rank_mode):
    """Key + index pairs of up to 128 Ki keys take the one-launch sort too: the permutation must
    equal the oracle's stable pairs sort on both sides of the limit, in both ranking modes."""
    keys = datagen.u64_zipf(n, seed=5 + n)
    items = np.arange(n, dtype=np.uint32)
    k2, i2 = keys.copy(), items.copy()
    orc.sort_pairs(k2, i2)
    c = native.Context(0, rank_mode=rank_mode)
    try:
        c.sort_pairs(keys, items)
        np.testing.assert_array_equal(keys, k2)
        np.testing.assert_array_equal(items, i2)
    finally:
        c.close()
