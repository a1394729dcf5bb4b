"""The multi-rank (replicas) timing logic of bench.py on CPU: two gloo ranks agree on the
slowest rank's time and the job throughput counts both ranks' keys."""
import os

import pytest
import torch.multiprocessing as mp


def _rank(rank, world, port, q):
    import torch.distributed as dist

    from hpcsharp_b200 import replicas

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = 10.0 + 5.0 * rank  # rank 1 is slower
        m = replicas.max_over_ranks(mine)
        v = replicas.weak_scaling_gkeys(1 << 28, 4, world, m)
        q.put((rank, m, v))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [15.0, 15.0]
    want = (1 << 28) * 4 * 2 / (15.0 / 1e3) / 1e9
    assert all(abs(r[2] - want) < 1e-9 for r in res)


def test_single_process_is_identity():
    from hpcsharp_b200 import replicas

    assert replicas.max_over_ranks(3.5) == 3.5
    assert replicas.weak_scaling_gkeys(1000, 2, 1, 1.0) == pytest.approx(2e-3)
