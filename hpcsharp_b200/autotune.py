"""Autotuner of the batched segmented sort.

For each key width (4-byte keys timed as u32, 8-byte keys as u64) and each length class of the
segmented sort, it times every kernel variant that can hold the class's longest array on a
synthetic batch of that class (lengths log-uniform over the class, uniform keys, the batch
restored before every run, CUDA events around the graph-captured plan) and keeps the fastest.
The variants differ in level (one warp or one CTA per array), tile shape (threads x keys per
thread) and digit width (4 or 8 bits per pass for the warp level).

The result is a JSON record keyed by the GPU (name, SM count, driver and runtime versions):
the chosen table and every measurement.  `apply(ctx, record)` installs a table on a context;
the library's built-in table is the record committed for B200 (hpcsharp_b200/tune/).

    python -m hpcsharp_b200.autotune --out hpcsharp_b200/tune/b200.json
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys

import numpy as np

from . import native

WIDTH_DTYPE = {0: "u32", 1: "u64"}
MAX_LEN = 1 << 20  # longest array of the unbounded class in the tuning batches


def class_bounds() -> list[tuple[int, int]]:
    """(shortest, longest) array length of each class as tuned."""
    limits = native.seg_class_limits()
    out, lo = [], 2
    for lim in limits:
        hi = MAX_LEN if lim < 0 else lim
        out.append((lo, hi))
        lo = hi + 1
    return out


def batch_lengths(lo: int, hi: int, total_keys: int, min_arrays: int, seed: int,
                  max_arrays: int = 1 << 18) -> np.ndarray:
    """Lengths log-uniform over [lo, hi] until total_keys keys (min_arrays..max_arrays arrays)."""
    rng = np.random.default_rng(seed)
    mean = (hi - lo) / max(1e-9, np.log(hi / lo)) if hi > lo else lo
    count = min(max_arrays, max(min_arrays, int(total_keys / mean)))
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi + 1), size=count))).clip(lo, hi).astype(np.int64)


def _fits(variant: dict, w: int, hi: int) -> bool:
    cap = variant["max_keys"][w]
    return cap < 0 or hi <= cap


def time_variant(ctx: "native.Context", w: int, c: int, v: int, lengths: np.ndarray, reps: int = 5,
                 seed: int = 1) -> float:
    """Median ms of the plan over `lengths` arrays of width w with class c forced to variant v."""
    import torch

    dt = WIDTH_DTYPE[w]
    tdt = torch.int32 if w == 0 else torch.int64
    align = 4 if w == 0 else 2  # elements per 16 bytes
    offs = np.zeros(len(lengths) + 1, dtype=np.int64)
    offs[1:] = np.cumsum((lengths + align - 1) // align * align)
    g = torch.Generator(device=f"cuda:{ctx.device}").manual_seed(seed)
    info = torch.iinfo(tdt)
    pristine = torch.randint(info.min, info.max, (int(offs[-1]),), dtype=tdt, device=f"cuda:{ctx.device}",
                             generator=g)
    pool = pristine.clone()
    segs = [((pool.data_ptr() + int(o) * pool.element_size(), int(n)), dt) for o, n in zip(offs[:-1], lengths)]
    table = ctx.seg_tuning
    saved = [row[:] for row in table]
    table[w][c] = v
    ctx.seg_tuning = table
    try:
        plan = ctx.segplan(segs)
        s = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{ctx.device}")
        times = []
        for r in range(reps + 2):
            with torch.cuda.stream(s):
                pool.copy_(pristine)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            plan.execute()
            b.record(s)
            ctx.synchronize()
            if r >= 2:
                times.append(a.elapsed_time(b))
        plan.close()
    finally:
        ctx.seg_tuning = saved
    return statistics.median(times)


def device_key(ctx: "native.Context") -> dict:
    import torch

    p = torch.cuda.get_device_properties(ctx.device)
    drv = None
    try:
        import pynvml  # nvidia_ml_py

        pynvml.nvmlInit()
        drv = pynvml.nvmlSystemGetDriverVersion()
        drv = drv.decode() if isinstance(drv, bytes) else drv
    except Exception:
        pass
    return {"name": p.name, "sms": p.multi_processor_count, "driver": drv, "cuda_runtime": torch.version.cuda}


def tune(ctx: "native.Context | None" = None, total_keys: int = 24 << 20, reps: int = 5,
         log=print) -> dict:
    own = ctx is None
    ctx = ctx or native.Context(0)
    try:
        variants = native.seg_variants()
        bounds = class_bounds()
        table = ctx.seg_tuning
        measurements = []
        for w in (0, 1):
            for c, (lo, hi) in enumerate(bounds):
                lengths = batch_lengths(lo, hi, total_keys // (1 + w), min_arrays=4 * 148, seed=100 * w + c)
                keys = int(lengths.sum())
                best = None
                for v, var in enumerate(variants):
                    if not _fits(var, w, hi):
                        continue
                    ms = time_variant(ctx, w, c, v, lengths, reps=reps)
                    rate = keys / (ms / 1e3) / 1e9
                    measurements.append({"width_bytes": 4 << w, "class": c, "lengths": [lo, hi],
                                         "arrays": len(lengths), "keys": keys, "variant": v,
                                         "ms": round(ms, 4), "gkeys_s": round(rate, 3)})
                    log(f"{4 << w}-byte keys class {c} [{lo}, {hi}] x{len(lengths)}: variant {v} "
                        f"({var['kind']} {var['threads']}x{var['keys_per_thread']}, {var['digit_bits']}-bit) "
                        f"{ms:.3f} ms = {rate:.2f} Gkeys/s")
                    if best is None or ms < best[0]:
                        best = (ms, v)
                table[w][c] = best[1]
        return {"device": device_key(ctx), "class_limits": native.seg_class_limits(), "variants": variants,
                "table": table, "measurements": measurements,
                "method": f"median of {reps} runs after 2 warm-ups, batch restored before each run, "
                          f"~{total_keys >> 20} Mi 4-byte or {total_keys >> 21} Mi 8-byte uniform keys per class"}
    finally:
        if own:
            ctx.close()


def save(record: dict, path: str) -> None:
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    with open(path, "w") as f:
        json.dump(record, f, indent=1)


def load(path: str) -> dict:
    with open(path) as f:
        return json.load(f)


def apply(ctx: "native.Context", record: dict) -> None:
    """Install a tuned table on a context (raises if a variant cannot hold its class)."""
    ctx.seg_tuning = record["table"]


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=None, help="JSON record to write")
    ap.add_argument("--keys", type=int, default=24 << 20, help="4-byte keys per class batch")
    ap.add_argument("--reps", type=int, default=5)
    a = ap.parse_args(argv)
    rec = tune(total_keys=a.keys, reps=a.reps)
    print(json.dumps({"device": rec["device"], "table": rec["table"]}))
    if a.out:
        save(rec, a.out)
    return 0


if __name__ == "__main__":
    sys.exit(main())
