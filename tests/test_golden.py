"""Committed fixtures (tests/golden/golden.json, made by make_golden.py): the generators and
the oracle must reproduce them on CPU, and the GPU library must produce the same digests."""
import hashlib
import json
import os

import numpy as np
import pytest

from hpcsharp_b200 import datagen

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = json.load(open(os.path.join(HERE, "golden", "golden.json")))


def digest(*arrays):
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).view(np.uint8).tobytes())
    return h.hexdigest()


def gen(case):
    kind, dt, n, seed = case.get("gen", "by_name"), case["dtype"], case["n"], case["seed"]
    if kind == "pcg32_stream":
        return datagen.u32_pcg32_stream(n, seed)
    if kind == "xorshift64s":
        return datagen.u32_xorshift64s(n, seed)
    if kind == "and3":
        return datagen.u64_and3(n, seed)
    if kind == "zipf":
        return datagen.u64_zipf(n, seed)
    return datagen.by_name(dt, n, seed)


@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: c["name"])
def test_oracle_reproduces_golden(orc, case):
    a = gen(case)
    assert digest(a) == case["input_sha256"]
    orc.sort_radix_lsd(a)
    assert digest(a) == case["sorted_sha256"]


@pytest.mark.parametrize("case", GOLDEN["pairs"], ids=lambda c: c["name"])
def test_oracle_pairs_reproduce_golden(orc, case):
    k = gen(case)
    assert digest(k) == case["input_sha256"]
    items = np.arange(case["n"], dtype=np.uint32)
    orc.sort_pairs(k, items)
    assert digest(k) == case["keys_sha256"] and digest(items) == case["items_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN["cases"], ids=lambda c: c["name"])
def test_gpu_matches_golden(ctx, case):
    a = gen(case)
    ctx.sort(a)
    assert digest(a) == case["sorted_sha256"]


@pytest.mark.gpu
@pytest.mark.parametrize("case", GOLDEN["pairs"], ids=lambda c: c["name"])
def test_gpu_pairs_match_golden(ctx, case):
    k = gen(case)
    items = np.arange(case["n"], dtype=np.uint32)
    ctx.sort_pairs(k, items)
    assert digest(k) == case["keys_sha256"] and digest(items) == case["items_sha256"]
