"""Serving loop: sort and top-k requests of mixed size and dtype submitted at random times
from several threads; every result equals (bit for bit) the same request run alone through
the plain entry point, and the oracle's result; admission under a tight HBM budget still
completes everything."""
import threading
import time

import numpy as np
import pytest

from hpcsharp_b200 import datagen, native

pytestmark = pytest.mark.gpu

DT = ["u32", "i32", "f32", "u64"]


def make_requests(seed, count, lo=1000, hi=3_000_000):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        dt = DT[rng.integers(len(DT))]
        op = "sort" if rng.random() < 0.7 else "topk"
        k = int(min(n, [10, 1000, 100_000][rng.integers(3)])) if op == "topk" else 0
        keys = datagen.by_name(dt, n, seed=seed * 10_000 + i)
        out = np.empty(n if op == "sort" else k, dtype=keys.dtype)
        reqs.append((op, keys, out, k))
    return reqs


def alone(ctx, op, keys, k):
    if op == "sort":
        a = keys.copy()
        ctx.sort(a)
        return a
    return ctx.topk_largest(keys, k)


def bits(a):
    return a.view(np.uint8)


def run_mixed(server, reqs, threads=3, jitter_s=0.002, seed=0):
    tickets = [None] * len(reqs)

    def client(ix):
        rng = np.random.default_rng(seed + ix)
        for i in range(ix, len(reqs), threads):
            op, keys, out, k = reqs[i]
            time.sleep(rng.uniform(0, jitter_s))
            tickets[i] = server.submit(op, keys, out, k)

    ths = [threading.Thread(target=client, args=(t,)) for t in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    return [server.wait(t) for t in tickets]


def test_each_result_same_alone_and_in_the_mix(ctx, orc):
    reqs = make_requests(3, 60)
    server = native.Server(0, slots=4, hbm_budget_bytes=4 << 30, coalesce_max_keys=1 << 16)
    try:
        infos = run_mixed(server, reqs)
    finally:
        server.close()
    assert any(i["coalesced"] for i in infos) and not all(i["coalesced"] for i in infos)
    for (op, keys, out, k), info in zip(reqs, infos):
        ref = alone(ctx, op, keys, k)
        assert np.array_equal(bits(out), bits(ref)), (op, keys.dtype, keys.size, k)
        s = keys.copy()
        orc.sort_radix_lsd(s)
        want = s if op == "sort" else s[s.size - k:]
        assert np.array_equal(bits(out), bits(want))
        assert info["submit_ns"] <= info["admit_ns"] <= info["done_ns"]


def test_tight_budget_admits_by_free_memory(ctx):
    # the budget holds only a few of the larger requests at once: they must wait and still finish
    reqs = make_requests(5, 24, lo=200_000, hi=2_000_000)
    server = native.Server(0, slots=4, hbm_budget_bytes=48 << 20, coalesce_max_keys=1 << 15)
    try:
        infos = run_mixed(server, reqs, threads=2, jitter_s=0.0)
        st = server.stats()
    finally:
        server.close()
    assert st["completed"] == len(reqs) and st["arena_peak"] <= 48 << 20
    for (op, keys, out, k) in reqs:
        assert np.array_equal(bits(out), bits(alone(ctx, op, keys, k)))


def test_request_larger_than_budget_is_refused():
    server = native.Server(0, slots=1, hbm_budget_bytes=1 << 20)
    try:
        keys = datagen.u32_uniform(1_000_000, seed=1)
        out = np.empty_like(keys)
        with pytest.raises(native.HpcsError) as e:
            server.submit("sort", keys, out)
        assert e.value.status == native.HPCS_ERR_OOM
        with pytest.raises(native.ArgumentOutOfRangeException):
            server.submit("topk", keys[:100], out[:10], k=101)
    finally:
        server.close()
