"""GPU parity of the sharded sort: the partition kernel (hpcs_shard_partition_dev) against
the numpy partition in the oracle's key order, bit for bit, and the whole sharded sort with
the library's kernels on every rank -- two and three gloo ranks sharing cuda:0 (collectives
staged through host memory; the ranks' kernels never wait on one another) and one NCCL
rank -- against the oracle's stable sort of the whole array."""
import datetime
import os

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from tests.shard_util import NP_OF, collect, part_of

pytestmark = pytest.mark.gpu

VIEW = {4: np.int32, 8: np.int64}
LIMIT_S = 600


def _keys(dt: str, n: int, rng, dup: bool) -> np.ndarray:
    npdt = NP_OF[dt]
    if dup:
        vals = rng.integers(-3, 4, size=n)
        return vals.astype(npdt) if dt[0] != "u" else (vals + 3).astype(npdt)
    if dt[0] == "f":
        a = rng.standard_normal(n).astype(npdt)
        a[::29] = -0.0
        a[::31] = 0.0
        a[::37] = np.nan
        return a
    bits = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * 2 + rng.integers(0, 2, size=n, dtype=np.uint64)
    return bits.astype(np.uint32).view(npdt) if npdt().itemsize == 4 else bits.view(npdt)


def _splitters(a: np.ndarray, gpos0: int, parts: int, rng):
    """parts-1 ascending (key, position) splitters drawn from the keys and positions near the
    shard, ties in key included."""
    if parts == 1 or a.size == 0:
        return a[:0].copy(), np.zeros(0, dtype=np.int64)
    idx = rng.integers(0, a.size, size=parts - 1)
    sk = a[idx].copy()
    sg = gpos0 + rng.integers(-5, a.size + 5, size=parts - 1).astype(np.int64)
    sg = np.maximum(sg, 0)
    order = np.lexsort((sg, oracle.order_key(sk)))
    return sk[order], sg[order]


@pytest.mark.parametrize("dt", ["u32", "i32", "f32", "u64", "i64", "f64"])
@pytest.mark.parametrize("n,parts,dup,items", [
    (1, 2, False, True), (1000, 3, False, False), (2049, 8, True, True), (100_003, 64, False, True),
    (100_003, 2, True, False), (3_000_017, 8, False, True), (3_000_017, 5, True, True), (70_001, 1, False, True),
])
def test_partition_matches_oracle(ctx, dt, n, parts, dup, items):
    import torch

    from hpcsharp_b200 import native
    from tests.gpu_util import to_dev

    rng = np.random.default_rng(n * 131 + parts * 7 + (dt == "f32"))
    a = _keys(dt, n, rng, dup)
    gpos0 = int(rng.integers(0, 1 << 31))
    sk, sg = _splitters(a, gpos0, parts, rng)
    it = rng.integers(0, 1 << 32, size=n, dtype=np.uint64).astype(np.uint32)
    keys = to_dev(a)
    k_out = torch.empty_like(keys)
    i_in = torch.from_numpy(it.view(np.int32)).cuda() if items else None
    i_out = torch.empty_like(i_in) if items else None
    counts = torch.full((parts,), -1, dtype=torch.int64, device="cuda")
    spk = to_dev(sk) if parts > 1 else None
    spg = torch.from_numpy(sg).cuda() if parts > 1 else None
    ctx.shard_partition_dev(keys, i_in, gpos0, spk, spg, parts, k_out, i_out, counts, dtype=dt,
                            stream=native.torch_stream())
    torch.cuda.synchronize()
    part = part_of(a, gpos0, sk, sg, parts)
    perm = np.argsort(part, kind="stable")
    want_counts = np.bincount(part, minlength=parts)
    assert counts.cpu().numpy().tolist() == want_counts.tolist()
    got = k_out.cpu().numpy().view(VIEW[a.dtype.itemsize])
    assert np.array_equal(got, a[perm].view(VIEW[a.dtype.itemsize]))
    if items:
        assert np.array_equal(i_out.cpu().numpy().view(np.uint32), it[perm])


def test_partition_rejects_bad_arguments(ctx):
    import torch

    from hpcsharp_b200 import native

    k = torch.zeros(16, dtype=torch.int32, device="cuda")
    o = torch.empty_like(k)
    c = torch.zeros(4, dtype=torch.int64, device="cuda")
    sg = torch.zeros(3, dtype=torch.int64, device="cuda")
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.shard_partition_dev(k, None, 0, k[:3], sg, 65, o, None, c, dtype="u32")
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.shard_partition_dev(k, None, 0, k[:3], sg, 0, o, None, c, dtype="u32")
    with pytest.raises(native.ArgumentNullException):
        ctx.shard_partition_dev(k, None, 0, None, None, 4, o, None, c, dtype="u32")
    with pytest.raises(native.ArgumentNullException):
        ctx.shard_partition_dev(k, k, 0, k[:3], sg, 4, o, None, c, dtype="u32")
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.shard_partition_dev(k, None, -1, k[:3], sg, 4, o, None, c, dtype="u32")
    with pytest.raises(native.ArgumentOutOfRangeException):
        ctx.shard_partition_dev(k, None, 0, k[:3], sg, 4, k, None, c, dtype="u32")


CASES = {  # name: (dtype, shard sizes)
    "u32": ("u32", [400_000, 0, 700_001]),
    "f32": ("f32", [300_007, 500_000]),
    "i64_dup": ("i64", [250_000, 260_000]),
    "f64": ("f64", [123_457, 200_000]),
}


def _global(name: str, world: int):
    """(dtype, shard sizes of `world` ranks, global array); with fewer ranks than the case
    lists, the last rank takes the remaining shards."""
    dt, sizes = CASES[name]
    rng = np.random.default_rng(len(name) * 1009 + sizes[0])
    a = _keys(dt, sum(sizes), rng, dup=name.endswith("_dup"))
    return dt, sizes[:world - 1] + [sum(sizes[world - 1:])], a


def _rank(rank, world, port, backend, names, q):
    import torch
    import torch.distributed as dist

    from hpcsharp_b200 import native, sharded

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device("cuda:0") if backend == "nccl" else None)
    ctx = native.Context(0)
    try:
        out = {}
        for name in names:
            dt, sizes, a = _global(name, world)
            lo = sum(sizes[:rank])
            shard = a[lo: lo + sizes[rank]]
            keys = torch.from_numpy(shard.view(VIEW[shard.dtype.itemsize]).copy()).cuda()
            items = torch.arange(lo, lo + sizes[rank], dtype=torch.int32, device="cuda")
            ops = sharded.DeviceOps(ctx, dt)
            for balance in (True, False):
                k, i = sharded.sort_sharded(keys, items, ops=ops, balance=balance)
                k2, _ = sharded.sort_sharded(keys, None, ops=ops, balance=balance)
                torch.cuda.synchronize()
                out[(name, balance)] = (k.cpu().numpy(), i.cpu().numpy(), k2.cpu().numpy())
        ctx.synchronize()
        q.put((rank, out))
    finally:
        ctx.close()
        dist.destroy_process_group()


def _run(world, backend, names):
    c = mp.get_context("spawn")
    q = c.Queue()
    port = 29700 + (os.getpid() + 13 * world) % 1000
    procs = [c.Process(target=_rank, args=(r, world, port, backend, names, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    res = collect(q, procs, limit_s=LIMIT_S)
    for name in names:
        dt, sizes, a = _global(name, world)
        perm = np.argsort(oracle.order_key(a), kind="stable")
        want = a[perm].view(VIEW[a.dtype.itemsize])
        for balance in (True, False):
            outs = [res[r][(name, balance)] for r in range(world)]
            assert np.array_equal(np.concatenate([o[0] for o in outs]), want), (name, balance)
            assert np.array_equal(np.concatenate([o[1] for o in outs]).astype(np.int64), perm), (name, balance)
            assert np.array_equal(np.concatenate([o[2] for o in outs]), want), (name, balance)
            if balance:
                assert [o[0].size for o in outs] == sizes
            else:  # sampled splitters: every part within 10% of an even share
                n = sum(sizes)
                assert all(abs(o[0].size - n / world) < 0.1 * n for o in outs), [o[0].size for o in outs]


def test_sharded_sort_two_gloo_ranks_on_one_gpu():
    _run(2, "gloo", ["f32", "i64_dup", "f64"])


def test_sharded_sort_three_gloo_ranks_on_one_gpu():
    _run(3, "gloo", ["u32"])


def test_sharded_sort_one_nccl_rank():
    _run(1, "nccl", ["u32", "f64"])
