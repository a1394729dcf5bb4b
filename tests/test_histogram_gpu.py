"""GPU parity of the exported fused byte histogram (hpcs_histogram_byte_components_<t> and the
device form hpcs_histogram_byte_components_dev) against the oracle, through the C ABI.

The reference calls: ParallelAlgorithm.HistogramByteComponentsPar (HistogramParallel.cs:214 u32,
:416 i32, :547 u64, :617 i64) and the serial Algorithm.HistogramByteComponents (Histogram.cs:
261-296 u32, :957-990 u64, :992-1017 i32, :1019-1052 i64).  They count a[l..r] with both bounds
inclusive into counts[P][256], digit d = byte d, and a signed key's top byte flipped
(`count3[((uint)x >> 24) ^ 128]`, Histogram.cs:1014; `>> 56`, :1049).  l > r counts nothing
(HistogramParallel.cs:177-183).  Every case is compared with the oracle's serial and
divide-and-conquer parallel restatements and with an independent numpy bincount."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native
from tests.gpu_util import to_dev

pytestmark = pytest.mark.gpu

DTYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def numpy_histogram(a: np.ndarray, l: int, r: int, dt: str) -> np.ndarray:
    """counts[P][256] by numpy: the reference's digit rule written independently of the oracle."""
    P = a.dtype.itemsize
    u = a.view(np.uint32 if P == 4 else np.uint64)[l:r + 1] if r >= l else a.view(np.uint32 if P == 4 else np.uint64)[:0]
    if dt.startswith("f"):
        top = np.uint64(1) << np.uint64(8 * P - 1)
        allones = np.uint64((1 << (8 * P)) - 1)
        w = u.astype(np.uint64)
        neg = (w & top) != 0
        w = np.where(neg, w ^ allones, w ^ top)  # Histogram.cs:1210-1288
    else:
        w = u.astype(np.uint64)
    out = np.zeros((P, 256), dtype=np.uint32)
    for d in range(P):
        byte = ((w >> np.uint64(8 * d)) & np.uint64(0xFF)).astype(np.int64)
        if d == P - 1 and dt.startswith("i"):
            byte ^= 128
        out[d] = np.bincount(byte, minlength=256).astype(np.uint32)
    return out


def _keys(dt: str, n: int, seed: int) -> np.ndarray:
    if dt == "i64":
        # both signs in every byte position, including the extremes
        a = datagen.i64_uniform(n, seed)
        if n >= 4:
            a[:4] = [np.iinfo(np.int64).min, -1, 0, np.iinfo(np.int64).max]
        return a
    a = datagen.by_name(dt, n, seed=seed)
    if dt == "i32" and n >= 4:
        a[:4] = [np.iinfo(np.int32).min, -1, 0, np.iinfo(np.int32).max]
    return a


RANGES = [
    # (n, l, r): whole array, ragged inner ranges around the 16-byte vector and tile edges,
    # one element, and empty ranges (l == r + 1, l > r + 1)
    (1, 0, 0),
    (17, 0, 16),
    (1000, 3, 996),
    (4099, 1, 4097),
    (65_537, 0, 65_536),
    (100_003, 5, 99_990),
    (1_000_003, 0, 1_000_002),
    (1_000_003, 123_457, 876_543),
    (3_000_001, 7, 2_999_999),
    (50, 20, 20),
    (50, 20, 19),
    (50, 30, 10),
]


@pytest.mark.parametrize("n,l,r", RANGES, ids=[f"n{n}_l{l}_r{r}" for n, l, r in RANGES])
@pytest.mark.parametrize("dt", DTYPES)
def test_histogram_host_parity(ctx, orc, dt, n, l, r):
    a = _keys(dt, n, seed=n + 7 * l + 3)
    got = ctx.histogram(a, l, r)
    want = orc.histogram_byte_components(a, l, r)
    want_par = orc.histogram_byte_components(a, l, r, parallel=True)
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(got, want_par)
    np.testing.assert_array_equal(got, numpy_histogram(a, l, r, dt))
    assert int(got.sum()) == got.shape[0] * max(0, r - l + 1)


@pytest.mark.parametrize("dt", ["i32", "i64"])
def test_signed_top_digit_flip(ctx, dt):
    """The top byte of a signed key is flipped: -1 counts in bin 0x7F, 0 in bin 0x80, the
    minimum in bin 0x00 and the maximum in bin 0xFF (Histogram.cs:1014, :1049)."""
    npdt = native.NP_OF[dt]
    info = np.iinfo(npdt)
    a = np.array([-1, 0, info.min, info.max, -1], dtype=npdt)
    c = ctx.histogram(a, 0, a.size - 1)
    top = c[-1]
    assert top[0x7F] == 2 and top[0x80] == 1 and top[0x00] == 1 and top[0xFF] == 1
    assert int(top.sum()) == 5
    # the lower bytes are not flipped: -1 has 0xFF bytes, the minimum 0x00 bytes
    assert c[0][0xFF] == 3 and c[0][0x00] == 2


@pytest.mark.parametrize("offset", [0, 1, 3])
@pytest.mark.parametrize("dt", DTYPES)
def test_histogram_device_parity(ctx, orc, dt, offset):
    """The device form on aligned and unaligned device pointers (the unaligned ones are staged
    through aligned scratch first)."""
    import torch

    n = 2_000_003
    a = _keys(dt, n, seed=31 + offset)
    t = to_dev(a, offset_elems=offset)
    counts = torch.full((a.dtype.itemsize * 256,), 0x5A5A5A5A, dtype=torch.int32, device="cuda")
    ctx.histogram_dev(t, counts, dtype=dt, stream=native.torch_stream())
    torch.cuda.synchronize()
    ctx.synchronize()
    got = counts.cpu().numpy().view(np.uint32).reshape(a.dtype.itemsize, 256)
    np.testing.assert_array_equal(got, orc.histogram_byte_components(a, 0, n - 1))


def test_histogram_device_empty_zeroes_counts(ctx):
    import torch

    lib = native.load()
    keys = torch.zeros(16, dtype=torch.int32, device="cuda")  # a valid pointer, zero keys counted
    counts = torch.full((4 * 256,), 9, dtype=torch.int32, device="cuda")
    rc = lib.hpcs_histogram_byte_components_dev(ctx.handle, native.DTYPES["u32"], keys.data_ptr(), 0,
                                                counts.data_ptr(), native.torch_stream())
    assert rc == native.HPCS_OK
    torch.cuda.synchronize()
    ctx.synchronize()
    assert int(counts.abs().sum()) == 0


def test_histogram_errors(ctx):
    lib = native.load()
    a = np.arange(10, dtype=np.uint32)
    counts = np.zeros((4, 256), dtype=np.uint32)
    # l < 0: ArgumentOutOfRangeException
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.histogram(a, -1, 5)
    # NULL array / NULL counts: ArgumentNullException
    assert lib.hpcs_histogram_byte_components_u32(ctx.handle, None, 0, 5, counts.ctypes.data) == native.HPCS_ERR_NULL
    assert lib.hpcs_histogram_byte_components_u32(ctx.handle, a.ctypes.data, 0, 5, None) == native.HPCS_ERR_NULL
    # more than HPCS_MAX_KEYS keys
    assert lib.hpcs_histogram_byte_components_u32(ctx.handle, a.ctypes.data, 0, 1 << 31,
                                                  counts.ctypes.data) == native.HPCS_ERR_RANGE
    # an empty range zeroes the caller's counts
    counts[:] = 3
    assert lib.hpcs_histogram_byte_components_u32(ctx.handle, a.ctypes.data, 6, 5,
                                                  counts.ctypes.data) == native.HPCS_OK
    assert not counts.any()
