"""The committed autotuner record agrees with the library's built-in table, names variants
that exist and hold their classes, and the tuner's batch generator stays inside each class."""
import json
import os

import numpy as np

from hpcsharp_b200 import autotune, native

REC = os.path.join(os.path.dirname(autotune.__file__), "tune", "b200_148sm.json")


def test_record_is_consistent():
    rec = json.load(open(REC))
    assert rec["device"]["sms"] == 148 and "B200" in rec["device"]["name"]
    vs = native.seg_variants()
    limits = native.seg_class_limits()
    assert rec["class_limits"] == limits
    for w in range(2):
        for c, v in enumerate(rec["table"][w]):
            cap = vs[v]["max_keys"][w]
            assert cap < 0 or (limits[c] >= 0 and limits[c] <= cap)
            # the chosen variant is the fastest measured for (width, class)
            ms = {m["variant"]: m["ms"] for m in rec["measurements"]
                  if m["width_bytes"] == 4 << w and m["class"] == c}
            assert min(ms, key=ms.get) == v


def test_batch_lengths_stay_in_class():
    for c, (lo, hi) in enumerate(autotune.class_bounds()):
        n = autotune.batch_lengths(lo, hi, 1 << 20, min_arrays=64, seed=c)
        assert n.min() >= lo and n.max() <= hi and n.size >= 64
