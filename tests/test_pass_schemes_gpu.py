"""The two digit-pass schemes give the oracle's bits: chunked passes (per-range counts
forwarded from the previous pass) and single-pass decoupled look-back, each forced for every
size (the automatic choice picks between them by key type and n).  Sizes
put the chunked geometry at its edges: one tile, one range per SM exactly, one tile more
than there are SMs (ranges of two tiles, half the SMs idle), many tiles per range with a
short last range, and ragged 16-byte tails."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native

pytestmark = pytest.mark.gpu

SMS = 148
TILE = {"u32": 16384, "i32": 16384, "f32": 16384, "u64": 8192, "i64": 8192, "f64": 8192}


def _sizes(dt):
    t = TILE[dt]
    return [t - 1, t, t + 3, SMS * t, SMS * t + 1, 37 * SMS * t - 5, 5_000_011]


@pytest.fixture(scope="module", params=["chunked", "lookback"])
def sctx(request):
    c = native.Context(0, pass_scheme=request.param)
    yield c
    c.close()


def _oracle(orc, a):
    s = a.copy()
    orc.sort_radix_lsd(s)
    return s


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_scheme_parity_plain(sctx, orc, dt):
    for n in _sizes(dt):
        a = datagen.by_name(dt, n, seed=7 + n)
        got = a.copy()
        sctx.sort(got)
        assert np.array_equal(got.view(np.uint8), _oracle(orc, a).view(np.uint8)), (dt, n)


@pytest.mark.parametrize("dt", ["u32", "f32", "u64", "f64"])
def test_scheme_parity_pairs(sctx, orc, dt):
    for n in (4097, SMS * 8192 + 7, 3_000_017):
        keys = datagen.by_name(dt, n, seed=11 + n)
        if dt in ("u32", "u64"):
            keys = keys % np.array(1000, dtype=keys.dtype)  # heavy duplicates: stability shows
        items = np.arange(n, dtype=np.uint32)
        ko, io = keys.copy(), items.copy()
        orc.sort_pairs(ko, io)
        kg, ig = keys.copy(), items.copy()
        sctx.sort_pairs(kg, ig)
        assert np.array_equal(kg.view(np.uint8), ko.view(np.uint8)), (dt, n)
        assert np.array_equal(ig, io), (dt, n)


@pytest.mark.parametrize("kind", ["constant", "byte1_only", "top_byte_only"])
def test_scheme_skipped_passes(sctx, orc, kind):
    """Skipped passes between executed ones: the forwarded counts must be those of the next
    executed digit."""
    n = 2_000_003
    rng = np.random.default_rng(5)
    if kind == "constant":
        a = np.full(n, 0xDEADBEEF, dtype=np.uint32)
    elif kind == "byte1_only":
        a = (rng.integers(0, 256, n, dtype=np.uint32) << np.uint32(8)) | np.uint32(0x7F0000AA)
    else:
        a = (rng.integers(0, 256, n, dtype=np.uint32) << np.uint32(24)) | rng.integers(0, 256, n, dtype=np.uint32)
    got = a.copy()
    sctx.sort(got)
    assert np.array_equal(got, _oracle(orc, a))


@pytest.mark.parametrize("dist", ["zipf", "few_values", "f32_normal", "and3_u64", "and3_u32"])
def test_scheme_skewed_digits(sctx, orc, dist):
    """Digits with frequent values: equal lanes' atomics are grouped (ranks by popcount)
    and the next pass's most frequent value is derived by subtraction; the bits and the
    stable order of equal keys still match the oracle."""
    n = 3_000_017
    if dist == "zipf":
        keys = datagen.u64_zipf(n, seed=3)
    elif dist == "few_values":
        rng = np.random.default_rng(8)
        keys = rng.choice(np.array([7, 0xFF00FF, 1 << 40, 3], dtype=np.uint64), size=n, p=[0.6, 0.2, 0.15, 0.05])
    elif dist == "and3_u64":  # 0 holds ~34% of every byte: one dominant value, not two
        keys = datagen.u64_and3(n, seed=5)
    elif dist == "and3_u32":
        rng = np.random.default_rng(9)
        keys = rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
        for _ in range(2):
            keys &= rng.integers(0, 1 << 32, n, dtype=np.uint64).astype(np.uint32)
    else:
        keys = datagen.f32_normal(n, seed=4)
    got = keys.copy()
    sctx.sort(got)
    assert np.array_equal(got.view(np.uint8), _oracle(orc, keys).view(np.uint8))
    items = np.arange(n, dtype=np.uint32)
    ko, io = keys.copy(), items.copy()
    orc.sort_pairs(ko, io)
    kg, ig = keys.copy(), items.copy()
    sctx.sort_pairs(kg, ig)
    assert np.array_equal(kg.view(np.uint8), ko.view(np.uint8))
    assert np.array_equal(ig, io)


@pytest.mark.parametrize("dist", ["normal_specials", "uniform01", "bits"])
def test_auto_scheme_float_keys_choose_on_device(orc, dist):
    """4-byte float keys past the chunked threshold under the automatic scheme: the histogram
    kernel picks look-back passes (normal keys: several frequent sign-and-exponent bytes) or
    chunked passes (uniform(0,1): two bytes hold most keys; uniform bits: no frequent value),
    and launches of the other kind return at once.  Every choice gives the oracle's bits."""
    import torch

    from tests.gpu_util import from_dev, to_dev

    n = 52_000_003  # above the 48 Mi-key chunked threshold, ragged
    rng = np.random.default_rng(11)
    if dist == "normal_specials":
        a = rng.standard_normal(n).astype(np.float32)
        a[::97] = -0.0
        a[::101] = 0.0
        a[::103] = np.inf
        a[::107] = -np.inf
        a[::109] = np.float32("nan")
        a[::113] = np.float32(1e-40)  # subnormal
    elif dist == "uniform01":
        a = rng.random(n, dtype=np.float32)
    else:
        a = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32).view(np.float32)
    c = native.Context(0)
    try:
        t = to_dev(a)
        c.sort_dev(t, dtype="f32", stream=native.torch_stream())
        torch.cuda.synchronize()
        got = from_dev(t, np.float32)
        c.synchronize()
    finally:
        c.close()
    want = _oracle(orc, a)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
