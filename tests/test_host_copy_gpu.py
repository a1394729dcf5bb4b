"""Host-array entry points on pageable memory (what a fixed .NET array is): the library copies
such arrays in chunks through its pinned buffers with several host threads.  The results must be
the same bits as with one plain cudaMemcpyAsync per array and as the oracle's, for sizes around the
chunk boundaries, keys-only and pairs, and when the array is pinned (no staging)."""
import numpy as np
import pytest

from hpcsharp_b200 import datagen, native

pytestmark = pytest.mark.gpu

CHUNK_KEYS = (16 << 20) // 4  # 16 MiB chunks of u32 keys


@pytest.fixture(scope="module")
def plain_ctx():
    c = native.Context(0, staged_host_copies=False)
    yield c
    c.close()


# sizes whose last chunk is empty, tiny, just under a chunk, and over 1 MiB but not a multiple of the
# copy threads' 64-byte pieces (every byte of every chunk must be copied)
@pytest.mark.parametrize("n", [2 * CHUNK_KEYS, 2 * CHUNK_KEYS + 1, 5 * CHUNK_KEYS - 3, 9 * CHUNK_KEYS + 12345,
                               3 * CHUNK_KEYS + 3_222_785])
def test_staged_sort_matches_plain_copy_and_oracle(ctx, plain_ctx, orc, n):
    a = datagen.u32_uniform(n, seed=n % 1000)
    staged = a.copy()
    ctx.sort(staged)
    plain = a.copy()
    plain_ctx.sort(plain)
    np.testing.assert_array_equal(staged, plain)
    want = a.copy()
    orc.sort_radix_par(want)
    np.testing.assert_array_equal(staged, want)


def test_staged_pairs_and_u64(ctx, orc):
    n = 3 * CHUNK_KEYS + 77
    keys = datagen.u64_zipf(n, seed=2)
    items = np.arange(n, dtype=np.uint32)
    k2, i2 = keys.copy(), items.copy()
    orc.sort_pairs(k2, i2)
    ctx.sort_pairs(keys, items)
    np.testing.assert_array_equal(keys, k2)
    np.testing.assert_array_equal(items, i2)


def test_staged_16_bit_counting_sort(ctx):
    """A 16-bit array whose byte count is not a multiple of 4 (odd n): the last chunk's last bytes."""
    n = 40_000_001
    a = np.random.default_rng(3).integers(0, 1 << 16, size=n, dtype=np.int64).astype(np.uint16)
    got = a.copy()
    ctx.sort(got)
    np.testing.assert_array_equal(got, np.sort(a))


def test_pinned_host_array_is_not_staged(ctx, orc):
    import torch

    n = 3 * CHUNK_KEYS
    pinned = torch.empty(n, dtype=torch.int32, pin_memory=True).numpy().view(np.uint32)
    pinned[:] = datagen.u32_uniform(n, seed=4)
    want = pinned.copy()
    orc.sort_radix_par(want)
    ctx.sort(pinned)
    np.testing.assert_array_equal(pinned, want)
