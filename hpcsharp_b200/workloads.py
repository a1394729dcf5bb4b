"""Synthetic workloads of the batched and served forms (seeded, reproducible).

Batched set: `count` arrays with lengths log-uniform over [lo, hi] (ln n uniform), the dtype of
each array drawn uniformly from `dtypes`, values from the per-dtype generators of
hpcsharp_b200.datagen.  The literal 65,536-array set averages (hi-lo)/ln(hi/lo) ~ 100,848 keys
per array (~6.6 G keys); `target_total` rescales every length by target_total / sum (floor,
minimum lo) to reach the stated ~250 M keys.  Arrays of one dtype are packed into one pool,
each starting on a 16-byte boundary.
"""
from __future__ import annotations

import numpy as np

from . import datagen

BATCH_DTYPES = ("u32", "i32", "f32", "u64")
ALIGN_BYTES = 16


def batched_lengths(count: int = 65_536, lo: int = 32, hi: int = 1 << 20, seed: int = 4,
                    target_total: int | None = 250_000_000):
    rng = np.random.default_rng(seed)
    n = np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), size=count))).astype(np.int64)
    n = np.clip(n, lo, hi)
    if target_total:
        n = np.maximum(lo, np.floor(n * (target_total / n.sum()))).astype(np.int64)
    dt_idx = rng.integers(0, len(BATCH_DTYPES), size=count)
    return n, [BATCH_DTYPES[i] for i in dt_idx]


class BatchedSet:
    """Host pools (one numpy array per dtype) and each array's (dtype, offset, n)."""

    def __init__(self, lengths, dtypes, seed: int = 1):
        self.items = []  # (dtype, offset_in_pool_elems, n)
        sizes = {}
        for n, dt in zip(lengths, dtypes):
            w = np.dtype(datagen_dtype(dt)).itemsize
            step = ALIGN_BYTES // w
            off = sizes.get(dt, 0)
            self.items.append((dt, off, int(n)))
            sizes[dt] = off + (int(n) + step - 1) // step * step
        self.pools = {dt: datagen.by_name(dt, size, seed=seed + i) for i, (dt, size) in enumerate(sorted(sizes.items()))}
        self.total_keys = int(sum(int(n) for n in lengths))
        self.total_bytes = int(sum(int(n) * np.dtype(datagen_dtype(dt)).itemsize for n, dt in zip(lengths, dtypes)))

    def segment(self, i):
        dt, off, n = self.items[i]
        return self.pools[dt][off:off + n]


def datagen_dtype(dt: str):
    return {"u32": np.uint32, "i32": np.int32, "f32": np.float32, "u64": np.uint64, "i64": np.int64,
            "f64": np.float64}[dt]


SERVE_DTYPES = ("u32", "i32", "f32", "u64")


def serving_trace(count: int = 120, lo: int = 1 << 10, hi: int = 1 << 26, seed: int = 9):
    """Requests of the serving workload: 70% sort / 30% top-k (k from {10, 1000, 100000},
    redrawn until k <= n), n log-uniform over [lo, hi], dtype uniform over SERVE_DTYPES.
    Returns a list of (op, dtype, n, k) and unit-rate exponential inter-arrival gaps (divide
    by the arrival rate)."""
    rng = np.random.default_rng(seed)
    reqs = []
    for _ in range(count):
        n = int(np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi)))))
        dt = SERVE_DTYPES[rng.integers(len(SERVE_DTYPES))]
        if rng.random() < 0.7:
            reqs.append(("sort", dt, n, 0))
        else:
            ks = [k for k in (10, 1000, 100_000) if k <= n]
            reqs.append(("topk", dt, n, int(ks[rng.integers(len(ks))])))
    gaps = rng.exponential(1.0, size=count)
    return reqs, gaps
