"""Numpy stand-ins of the sharded sort's per-rank kernels (stable sorts and the stable
partition by (key order, global position) splitters), in the oracle's key order: the host
logic runs on them on CPU, and the GPU partition is checked against them.  Also the
collection of results from rank processes."""
import queue
import time

import numpy as np

import oracle

NP_OF = {"u32": np.uint32, "i32": np.int32, "f32": np.float32, "u64": np.uint64, "i64": np.int64,
         "f64": np.float64}


class NumpyOps:
    """Numpy stand-ins of DeviceOps on CPU tensors holding the keys' bytes."""

    def __init__(self, dtype: str):
        self.dtype = dtype
        self.np = NP_OF[dtype]

    def _order(self, t) -> np.ndarray:
        return oracle.order_key(t.numpy().view(self.np))

    def sort(self, keys) -> None:
        perm = np.argsort(self._order(keys), kind="stable")
        keys.copy_(keys[perm])

    def sort_pairs(self, keys, items) -> None:
        perm = np.argsort(self._order(keys), kind="stable")
        keys.copy_(keys[perm])
        items.copy_(items[perm])

    def partition(self, keys, items, gpos0, split_keys, split_gpos, parts):
        import torch

        part = part_of(keys.numpy().view(self.np), gpos0,
                       split_keys.numpy().view(self.np) if parts > 1 else None,
                       split_gpos.numpy() if parts > 1 else None, parts)
        perm = np.argsort(part, kind="stable")
        counts = torch.from_numpy(np.bincount(part, minlength=parts).astype(np.int64))
        return keys[perm].clone(), (items[perm].clone() if items is not None else None), counts


def part_of(keys: np.ndarray, gpos0: int, split_keys, split_gpos, parts: int) -> np.ndarray:
    """Part of each key: the number of splitters at or below (key, gpos0 + index) in (key
    order, global position) order."""
    ok = oracle.order_key(keys)
    g = gpos0 + np.arange(keys.size, dtype=np.int64)
    part = np.zeros(keys.size, dtype=np.int64)
    if parts > 1:
        sk = oracle.order_key(split_keys)
        for j in range(parts - 1):
            part += (sk[j] < ok) | ((sk[j] == ok) & (split_gpos[j] <= g))
    return part


def collect(q, procs, limit_s: float) -> dict:
    """{rank: result} from the rank processes; fails as soon as one of them exits without a
    result instead of waiting out the limit."""
    res, t0 = {}, time.monotonic()
    while len(res) < len(procs):
        try:
            r, out = q.get(timeout=2)
            res[r] = out
        except queue.Empty:
            dead = [p.exitcode for p in procs if p.exitcode not in (None, 0)]
            assert not dead, f"a rank process failed (exit codes {dead})"
            assert time.monotonic() - t0 < limit_s, "rank processes ran out of time"
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return res
