"""Generates tests/golden/golden.json: SHA-256 digests of the oracle's outputs for seeded
inputs (the reference's own test suite has no radix-sort vectors; these pin the CPU
restatement between runs and pin the GPU results against it).

Run from the repository root:  python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from hpcsharp_b200 import datagen  # noqa: E402

CASES = [
    # (name, dtype, generator, n, seed)
    ("c1_u32_pcg32_10m", "u32", "pcg32_stream", 10_000_000, 1),
    ("c1_u32_xorshift_10m", "u32", "xorshift64s", 10_000_000, 1),
    ("u32_uniform_1m", "u32", "by_name", 1_000_003, 7),
    ("i32_normal_1m", "i32", "by_name", 1_000_003, 7),
    ("f32_specials_1m", "f32", "by_name", 1_000_003, 7),
    ("u64_uniform_1m", "u64", "by_name", 1_000_003, 7),
    ("u64_and3_1m", "u64", "and3", 1_000_003, 7),
    ("i64_uniform_1m", "i64", "by_name", 1_000_003, 7),
    ("f64_normal_1m", "f64", "by_name", 1_000_003, 7),
]
PAIR_CASES = [
    ("pairs_u64_zipf_1m", "u64", "zipf", 1_000_003, 11),
    ("pairs_f64_normal_1m", "f64", "by_name", 1_000_003, 11),
]
TOPK_CASES = [("topk_u32_1m", "u32", 1_000_003, 5, 1_000_003 - 1000)]


def gen(dtype, kind, n, seed):
    if kind == "pcg32_stream":
        return datagen.u32_pcg32_stream(n, seed)
    if kind == "xorshift64s":
        return datagen.u32_xorshift64s(n, seed)
    if kind == "and3":
        return datagen.u64_and3(n, seed)
    if kind == "zipf":
        return datagen.u64_zipf(n, seed)
    return datagen.by_name(dtype, n, seed)


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    return h.hexdigest()


def main():
    out = {"cases": [], "pairs": [], "topk": []}
    for name, dt, kind, n, seed in CASES:
        a = gen(dt, kind, n, seed)
        s = a.copy()
        oracle.sort_radix_lsd(s)
        out["cases"].append({"name": name, "dtype": dt, "gen": kind, "n": n, "seed": seed,
                             "input_sha256": digest(a), "sorted_sha256": digest(s)})
    for name, dt, kind, n, seed in PAIR_CASES:
        k = gen(dt, kind, n, seed)
        items = np.arange(n, dtype=np.uint32)
        k2, i2 = k.copy(), items.copy()
        oracle.sort_pairs(k2, i2)
        out["pairs"].append({"name": name, "dtype": dt, "gen": kind, "n": n, "seed": seed,
                             "input_sha256": digest(k), "keys_sha256": digest(k2), "items_sha256": digest(i2)})
    for name, dt, n, seed, k in TOPK_CASES:
        a = datagen.by_name(dt, n, seed)
        b = a.copy()
        assert oracle.select_topk(b, k) == 0
        top = np.sort(b[k:])
        out["topk"].append({"name": name, "dtype": dt, "n": n, "seed": seed, "k": k,
                            "kth_value": int(b[k]), "top_sorted_sha256": digest(top)})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", path)


if __name__ == "__main__":
    main()
