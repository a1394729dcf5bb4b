"""The wide-digit passes (three passes of up to 11-bit digits for 32-bit keys, each after a
counting read of its input) give the oracle's bits: the 8-bit SortRadix/SortRadixPar restatement
for keys, SortRadix<T>(items, keys) for pairs (same keys and the same stable permutation).

The scheme is forced for every size.  Sizes put the range geometry at its edges: fewer keys than
a 16-byte vector, one tile, one range per SM exactly, one tile more than there are SMs, many
tiles per range with a short last range, and ragged tails; inputs include passes that are the
identity (one digit value for every key), heavy duplicates and the float specials."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native
from tests.gpu_util import from_dev, to_dev

pytestmark = pytest.mark.gpu

SMS = 148
TILE = 16384
PAIR_TILE = 8192
SIZES = [2, 3, 5, 17, TILE - 1, TILE, TILE + 3, SMS * TILE, SMS * TILE + 1, 9 * SMS * TILE - 5, 5_000_011]


@pytest.fixture(scope="module")
def wctx():
    c = native.Context(0, pass_scheme="wide")
    yield c
    c.close()


def _oracle(orc, a):
    s = a.copy()
    orc.sort_radix_lsd(s)
    return s


def _same(x, y):
    return np.array_equal(x.view(np.uint8), y.view(np.uint8))


@pytest.mark.parametrize("dt", ["u32", "i32", "f32"])
def test_wide_parity_plain(wctx, orc, dt):
    for n in SIZES:
        a = datagen.by_name(dt, n, seed=17 + n)
        got = a.copy()
        wctx.sort(got)
        assert _same(got, _oracle(orc, a)), (dt, n)


@pytest.mark.parametrize("kind", ["constant", "low_11_only", "top_10_only", "two_values", "and3", "heavy_dups"])
def test_wide_parity_skewed(wctx, orc, kind):
    n = 3_000_017
    a = datagen.u32_uniform(n, seed=5)
    if kind == "constant":
        a[:] = 0xCAFEBABE  # every pass is the identity: the result stays in the caller's buffer
    elif kind == "low_11_only":
        a &= np.uint32(0x7FF)  # two identity passes: an odd number runs, the copy-back is taken
    elif kind == "top_10_only":
        a &= np.uint32(0xFFC00000)
    elif kind == "two_values":
        a = np.where(a & 1, np.uint32(0x12345678), np.uint32(0x9ABCDEF0)).astype(np.uint32)
    elif kind == "and3":
        a = a & datagen.u32_uniform(n, seed=6) & datagen.u32_uniform(n, seed=7)
    else:
        a = a % np.uint32(1000)
    got = a.copy()
    wctx.sort(got)
    assert _same(got, _oracle(orc, a)), kind


@pytest.mark.parametrize("dt", ["u32", "i32", "f32"])
def test_wide_parity_pairs(wctx, orc, dt):
    for n in (5, 4097, SMS * PAIR_TILE + 7, 3_000_017):
        keys = datagen.by_name(dt, n, seed=11 + n)
        if dt == "u32":
            keys = keys % np.array(1000, dtype=keys.dtype)  # heavy duplicates: stability shows
        items = np.arange(n, dtype=np.uint32)
        ko, io = keys.copy(), items.copy()
        orc.sort_pairs(ko, io)
        kg, ig = keys.copy(), items.copy()
        wctx.sort_pairs(kg, ig)
        assert _same(kg, ko), (dt, n)
        assert np.array_equal(ig, io), (dt, n)


@pytest.mark.parametrize("offset", [0, 1, 3])
def test_wide_device_pointers(wctx, orc, offset):
    import torch

    n = 2_000_003
    a = datagen.u32_uniform(n, seed=41 + offset)
    t = to_dev(a, offset_elems=offset)
    wctx.sort_dev(t, dtype="u32", stream=native.torch_stream())
    torch.cuda.synchronize()
    wctx.synchronize()
    assert _same(from_dev(t, np.uint32), _oracle(orc, a))


def test_auto_scheme_takes_wide_passes_for_large_u32(ctx):
    """The automatic scheme sorts 2^25 and more 32-bit keys with the wide passes: three pass
    launches per sort instead of four."""
    import torch

    n = 1 << 25
    a = datagen.u32_uniform(n, seed=3)
    t = to_dev(a)
    ctx.profile(True)
    ctx.profile_read()
    ctx.sort_dev(t, dtype="u32", stream=native.torch_stream())
    prof = ctx.profile_read()
    ctx.profile(False)
    torch.cuda.synchronize()
    if ctx.rank_mode == 0:
        assert prof["onesweep"][0] == 3
    s = from_dev(t, np.uint32)
    assert np.array_equal(s, np.sort(a))
