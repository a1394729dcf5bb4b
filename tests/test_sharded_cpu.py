"""The sharded sort's host logic on CPU: sizes, splitter sampling, partition sizes, the two
all-to-all exchanges and the rebalance, run by 2 and 3 gloo ranks with the per-rank kernels
replaced by numpy stand-ins (stable sorts and a stable partition in the oracle's key order).
The concatenated outputs must equal the oracle's stable sort of the concatenated shards,
keys and item payloads (global positions) both."""
import datetime
import os
import zlib

import numpy as np
import torch.multiprocessing as mp

import oracle
from hpcsharp_b200 import sharded
from tests.shard_util import NumpyOps, collect


def make_case(name: str):
    """(dtype, shard sizes, global array) of a named case."""
    rng = np.random.default_rng(zlib.crc32(name.encode()))
    if name == "u32_ragged":
        sizes, dt = [3000, 0, 4100], "u32"
        a = rng.integers(0, 1 << 32, size=sum(sizes), dtype=np.uint64).astype(np.uint32)
    elif name == "f32_specials":
        sizes, dt = [2500, 1700], "f32"
        a = rng.standard_normal(sum(sizes)).astype(np.float32)
        a[::7] = -0.0
        a[::11] = 0.0
        a[::13] = np.inf
        a[::17] = -np.inf
        a[::19] = np.float32("nan")
        a[::23] = -np.float32("nan")
    elif name == "i64_all_equal":
        sizes, dt = [5000, 3000], "i64"
        a = np.full(sum(sizes), -42, dtype=np.int64)
    elif name == "u64_tiny_shards":
        sizes, dt = [5, 1, 9], "u64"
        a = rng.integers(0, 4, size=sum(sizes), dtype=np.uint64)
    elif name == "i32_few_values":
        sizes, dt = [4000, 4000, 3000], "i32"
        a = rng.integers(-3, 3, size=sum(sizes)).astype(np.int32)
    elif name == "empty":
        sizes, dt = [0, 0, 0], "u32"
        a = np.zeros(0, dtype=np.uint32)
    else:
        raise KeyError(name)
    return dt, sizes, a[: sum(sizes)]


LIMIT_S = 240
CASES_2 = ["f32_specials", "i64_all_equal"]
CASES_3 = ["u32_ragged", "u64_tiny_shards", "i32_few_values", "empty"]


def _rank(rank, world, port, cases, q):
    import torch
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out = {}
        for name in cases:
            dt, sizes, a = make_case(name)
            lo = sum(sizes[:rank])
            shard = a[lo: lo + sizes[rank]].copy()
            view = np.int32 if shard.dtype.itemsize == 4 else np.int64
            keys = torch.from_numpy(shard.view(view).copy())
            items = torch.arange(lo, lo + sizes[rank], dtype=torch.int32)
            ops = NumpyOps(dt)
            for balance in (True, False):
                k, i = sharded.sort_sharded(keys, items, ops=ops, samples=64, seed=3, balance=balance)
                k2, _ = sharded.sort_sharded(keys, None, ops=ops, samples=64, seed=3, balance=balance)
                out[(name, balance)] = (k.numpy().copy(), i.numpy().copy(), k2.numpy().copy())
            assert torch.equal(keys, torch.from_numpy(shard.view(view)))  # the input is not modified
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _run(world, cases):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() + 7 * world) % 1000
    procs = [ctx.Process(target=_rank, args=(r, world, port, cases, q), daemon=True) for r in range(world)]
    for p in procs:
        p.start()
    return collect(q, procs, limit_s=LIMIT_S)


def _check(res, world, cases):
    for name in cases:
        dt, sizes, a = make_case(name)
        perm = np.argsort(oracle.order_key(a), kind="stable")
        want_k = a[perm]
        for balance in (True, False):
            outs = [res[r][(name, balance)] for r in range(world)]
            got_k = np.concatenate([o[0] for o in outs]).view(a.dtype)
            got_i = np.concatenate([o[1] for o in outs]).astype(np.int64)
            got_k2 = np.concatenate([o[2] for o in outs]).view(a.dtype)
            assert np.array_equal(got_k.view(np.uint8), want_k.view(np.uint8)), (name, balance)
            assert np.array_equal(got_i, perm), (name, balance)
            assert np.array_equal(got_k2.view(np.uint8), want_k.view(np.uint8)), (name, balance)
            if balance:
                assert [o[0].size for o in outs] == sizes, name
            elif name == "i64_all_equal":  # equal keys are split by position: parts near n/world
                n = sum(sizes)
                assert all(abs(o[0].size - n / world) < 0.2 * n for o in outs)


def test_two_gloo_ranks_sort_like_one_array():
    _check(_run(2, CASES_2), 2, CASES_2)


def test_three_gloo_ranks_sort_like_one_array():
    _check(_run(3, CASES_3), 3, CASES_3)


def test_rebalance_sizes_move_contiguous_pieces():
    held, target = [5, 0, 7, 3], [4, 4, 4, 3]
    sends = [sharded.rebalance_sizes(held, target, r)[0] for r in range(4)]
    recvs = [sharded.rebalance_sizes(held, target, r)[1] for r in range(4)]
    assert sends == [[4, 1, 0, 0], [0, 0, 0, 0], [0, 3, 4, 0], [0, 0, 0, 3]]
    assert recvs == [[4, 0, 0, 0], [1, 0, 3, 0], [0, 0, 4, 0], [0, 0, 0, 3]]
    for r in range(4):  # what r sends to d is what d receives from r
        assert all(sends[r][d] == recvs[d][r] for d in range(4))


def test_sample_positions_are_stratified_and_ascending():
    p = sharded.sample_positions(1000, 10, seed=1, rank=0)
    assert p.size == 10 and np.all(np.diff(p) > 0)
    assert np.all(p // 100 == np.arange(10))
    assert sharded.sample_positions(5, 5, 0, 1).tolist() == [0, 1, 2, 3, 4]
    assert sharded.sample_positions(7, 0, 0, 0).size == 0
    assert sharded.splitter_indices(100, 4) == [25, 50, 75]
    assert sharded.splitter_indices(3, 4) == [0, 1, 2]
