"""CPU tests of the oracle itself (no GPU): the reference's known answer, independent STL
cross-checks, fidelity of the parallel restatements to the serial ones, the float order
on hand-written bit patterns, pairs stability, histograms and the top-k contract."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen

SIZES = [0, 1, 2, 63, 64, 65, 65535, 65536, 65537, 1_000_000]


def test_known_answer_program_cs(orc):
    # HPCsharpExamples/HPCsharpExamples/Program.cs:15-34 sorts {21,43,16,5,54,3}
    for dt in (np.uint32, np.int32, np.uint64, np.int64):
        a = np.array([21, 43, 16, 5, 54, 3], dtype=dt)
        orc.sort_radix_lsd(a)
        assert a.tolist() == [3, 5, 16, 21, 43, 54]
        b = np.array([21, 43, 16, 5, 54, 3], dtype=dt)
        orc.sort_radix_par(b)
        assert b.tolist() == [3, 5, 16, 21, 43, 54]


# HPCsharpExamples/HPCsharpExamples/SortOfUserDefinedClass.cs:87-104: userArray.SortRadix(element
# => element.Key), commented "(stable)", on (Key, Index) = (16,0) (12,1) (18,2) (18,3) (10,4) (2,5);
# the stable order it prints is (2:5) (10:4) (12:1) (16:0) (18:2) (18:3).
UDT_EXAMPLE = [(16, 0), (12, 1), (18, 2), (18, 3), (10, 4), (2, 5)]
UDT_EXAMPLE_SORTED = [(2, 5), (10, 4), (12, 1), (16, 0), (18, 2), (18, 3)]


def test_known_answer_user_defined_class_sort(orc):
    """The key + index pairs sort (the reference's SortRadix by key, RadixSortLsd.cs:1183-1237)
    on the example's keys, with the index as the item: stable, so the two 18s keep their order."""
    for kdt in (np.uint32, np.uint64):
        keys = np.array([k for k, _ in UDT_EXAMPLE], dtype=kdt)
        items = np.array([i for _, i in UDT_EXAMPLE], dtype=np.uint32)
        orc.sort_pairs(keys, items)
        assert list(zip(keys.tolist(), items.tolist())) == UDT_EXAMPLE_SORTED


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", ["u32", "i32", "u64", "i64"])
def test_integer_lsd_matches_std_sort(orc, dt, n):
    a = datagen.by_name(dt, n, seed=11)
    ref = a.copy()
    orc.std_sort(ref)
    s = a.copy()
    orc.sort_radix_lsd(s)
    np.testing.assert_array_equal(s, ref)
    p = a.copy()
    orc.sort_radix_par(p, threads=4)
    np.testing.assert_array_equal(p, ref)


@pytest.mark.parametrize("n", [0, 1, 65537, 1_000_000])
def test_u32_par_quanta_equal_serial(orc, n):
    a = datagen.u32_uniform(n, seed=5)
    s = a.copy()
    orc.sort_radix_lsd(s)
    for q in (1024, 64 * 1024):
        p = a.copy()
        orc.sort_radix_par_u32_full(p, threads=3, quantum=q)
        np.testing.assert_array_equal(p, s)


@pytest.mark.parametrize("dt", ["f32", "f64"])
def test_float_lsd_matches_stable_transformed(orc, dt):
    a = datagen.by_name(dt, 300_000, seed=3)
    s = a.copy()
    orc.sort_radix_lsd(s)
    r = a.copy()
    orc.stable_sort_transformed(r)
    np.testing.assert_array_equal(s.view(np.uint8), r.view(np.uint8))
    p = a.copy()
    orc.sort_radix_par(p, threads=4)
    np.testing.assert_array_equal(p.view(np.uint8), s.view(np.uint8))
    # numeric order agrees with numpy except for the relative order of -0/+0
    fin = s[np.isfinite(s) | np.isinf(s)]
    assert np.all(fin[:-1] <= fin[1:])


def test_float_order_of_special_bit_patterns(orc):
    # Histogram.cs:1210-1248: sign 0 -> flip the sign bit; sign 1 -> flip every bit
    order = [0xFFC00000, 0xFF800000, 0xBF800000, 0x80000001, 0x80000000,
             0x00000000, 0x00000001, 0x3F800000, 0x7F800000, 0x7FC00000]
    # -NaN, -inf, -1, -min subnormal, -0, +0, +min subnormal, 1, +inf, +NaN
    rng = np.random.default_rng(0)
    a = np.array(order, dtype=np.uint32)[rng.permutation(len(order))].view(np.float32)
    orc.sort_radix_lsd(a)
    assert a.view(np.uint32).tolist() == order
    order64 = [0xFFF8000000000000, 0xFFF0000000000000, 0xBFF0000000000000, 0x8000000000000001,
               0x8000000000000000, 0x0, 0x1, 0x3FF0000000000000, 0x7FF0000000000000, 0x7FF8000000000000]
    b = np.array(order64, dtype=np.uint64)[rng.permutation(len(order64))].view(np.float64)
    orc.sort_radix_lsd(b)
    assert b.view(np.uint64).tolist() == order64


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_pairs_are_stable_argsort(orc, dt):
    n = 200_000
    keys = datagen.by_name(dt, n, seed=9)
    if dt in ("u32", "u64"):
        keys = keys % np.array(1000, dtype=keys.dtype)  # heavy duplicates
    perm = orc.stable_argsort(keys.copy())
    k = keys.copy()
    items = np.arange(n, dtype=np.uint32)
    orc.sort_pairs(k, items)
    np.testing.assert_array_equal(items, perm)
    np.testing.assert_array_equal(k.view(np.uint8), keys[perm].view(np.uint8))


def test_pairs_zipf_u64(orc):
    keys = datagen.u64_zipf(300_000, seed=2)
    assert np.unique(keys).size < keys.size // 3  # duplicates are heavy
    perm = orc.stable_argsort(keys.copy())
    k = keys.copy()
    items = np.arange(keys.size, dtype=np.uint32)
    orc.sort_pairs(k, items)
    np.testing.assert_array_equal(items, perm)


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_histogram_byte_components(orc, dt):
    a = datagen.by_name(dt, 100_003, seed=4)
    l, r = 17, a.size - 5
    h = orc.histogram_byte_components(a, l, r)
    hp = orc.histogram_byte_components(a, l, r, parallel=True)
    np.testing.assert_array_equal(h, hp)
    key = orc.order_key(a[l:r + 1])
    for d in range(a.dtype.itemsize):
        want = np.bincount(((key >> np.array(8 * d, dtype=key.dtype)) & np.array(0xFF, dtype=key.dtype))
                           .astype(np.int64), minlength=256)
        np.testing.assert_array_equal(h[d], want)
    # l > r gives zeros (HistogramParallel.cs:170-176)
    assert not orc.histogram_byte_components(a, 10, 9).any()


def test_signed_histogram_flips_top_byte(orc):
    a = np.array([-1, 0, 1, -2**31, 2**31 - 1], dtype=np.int32)
    h = orc.histogram_byte_components(a, 0, a.size - 1)
    # top byte ^ 128: -1 -> 0x7F, 0 -> 0x80, 1 -> 0x80, INT_MIN -> 0x00, INT_MAX -> 0xFF
    assert h[3][0x7F] == 1 and h[3][0x80] == 2 and h[3][0x00] == 1 and h[3][0xFF] == 1


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64"])
@pytest.mark.parametrize("n,k", [(1, 0), (2, 1), (1000, 0), (1000, 999), (100_000, 50_000), (100_000, 99_990),
                                 (65_536, 12_345)])
def test_select_topk_contract(orc, dt, n, k):
    a = datagen.by_name(dt, n, seed=n + k)
    srt = a.copy()
    orc.stable_sort_transformed(srt)
    b = a.copy()
    assert orc.select_topk(b, k) == 0
    # SelectionTopKRadix.cs contract: a[k] is the k-th smallest, a[k..] the n-k largest
    assert b[k:k + 1].view(np.uint8).tobytes() == srt[k:k + 1].view(np.uint8).tobytes()
    top = b[k:].copy()
    orc.stable_sort_transformed(top)
    np.testing.assert_array_equal(top.view(np.uint8), srt[k:].view(np.uint8))


def test_select_topk_duplicates(orc):
    a = (datagen.u32_uniform(50_000, seed=8) % np.uint32(7)).astype(np.uint32)
    srt = np.sort(a)
    for k in (0, 1, 7000, 49_999):
        b = a.copy()
        assert orc.select_topk(b, k) == 0
        assert b[k] == srt[k]
        np.testing.assert_array_equal(np.sort(b[k:]), srt[k:])


@pytest.mark.parametrize("n", [0, 1, 65535, 65536, 65537, 3_000_017])
def test_oracle_key_stream_equals_product_generator(orc, n):
    """The CPU baseline generates its keys inside the oracle; they must be the very keys the GPU
    benchmark sorts (same SHA-256), so both arms run the same configuration."""
    import hashlib

    a = orc.gen_u32_uniform(n, seed=1, threads=3)
    b = datagen.u32_uniform(n, 1)
    assert hashlib.sha256(a.tobytes()).hexdigest() == hashlib.sha256(b.tobytes()).hexdigest()


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_workspace_sort_radix_par_equals_serial(orc, dt):
    """SortRadixPar on a workspace made once (scratch allocated outside the sort) gives the
    serial restatement's result, on two calls in a row of different sizes."""
    ws = orc.RadixParWorkspace(400_000, np.dtype(datagen.by_name(dt, 1).dtype).itemsize)
    try:
        for n, seed in ((400_000, 3), (123_457, 4)):
            a = datagen.by_name(dt, n, seed=seed)
            s = a.copy()
            orc.sort_radix_lsd(s)
            w = a.copy()
            ws.sort(w, threads=3)
            np.testing.assert_array_equal(w.view(np.uint8), s.view(np.uint8))
        with pytest.raises(ValueError):
            ws.sort(datagen.by_name(dt, 400_001, seed=1))
    finally:
        ws.close()
