"""CPU-only checks of the C ABI: the library builds and loads, exports every function that
include/*.h declares, and rejects bad arguments without touching a GPU."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from hpcsharp_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = []
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"\b(hpcs_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_library_builds_and_loads():
    build.build_all()
    lib = native.load()
    assert lib.hpcs_abi_version() == 1


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(native.LIB_PATH)
    names = declared_functions()
    assert len(names) >= 39
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_status_strings_and_defaults():
    lib = native.load()
    assert lib.hpcs_status_string(0) == b"HPCS_OK"
    assert lib.hpcs_status_string(5) == b"HPCS_ERR_DEVICE_TIMEOUT"
    cfg = native.default_config()
    assert cfg.skip_trivial_passes == 1 and cfg.poison_tile == -1 and cfg.spin_limit_ns > 0
    # the remaining settings default to the library's choices (0 = built-in value)
    assert cfg.pass_scheme == 0 and cfg.staged_host_copies == 1
    assert cfg.seg_grid_min_keys == 0 and cfg.seg_grid_tiles == 0 and list(cfg.reserved) == [0, 0, 0]


def test_null_context_and_arrays_are_rejected_without_gpu():
    lib = native.load()
    a = np.zeros(4, dtype=np.uint32)
    assert lib.hpcs_sort_u32(None, a.ctypes.data, 4) == native.HPCS_ERR_NULL
    assert lib.hpcs_sort_pairs_u64(None, None, None, 4) == native.HPCS_ERR_NULL
    assert lib.hpcs_ctx_synchronize(None) == native.HPCS_ERR_NULL
    assert b"NULL" in lib.hpcs_last_error_message()


def test_ctx_create_reports_missing_device():
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(native.HpcsError) as e:
        native.Context(0)
    assert e.value.status == native.HPCS_ERR_NO_DEVICE


def test_segmented_variants_and_classes_without_gpu():
    """The segmented sort's variant list and length classes are host-side facts: warp-level
    variants hold 32 x keys-per-thread 4-byte keys (half for 8-byte keys), block-level ones
    any length; the classes rise and the last is unbounded."""
    vs = native.seg_variants()
    assert len(vs) == 11
    for v in vs:
        if v["kind"] == "warp":
            assert v["max_keys"] == [32 * v["keys_per_thread"], 16 * v["keys_per_thread"]]
            assert v["digit_bits"] in (4, 8) and v["threads"] == 256
        else:
            assert v["max_keys"] == [-1, -1] and v["digit_bits"] == 8
    limits = native.seg_class_limits()
    assert limits[-1] == -1 and all(a < b for a, b in zip(limits[:-2], limits[1:-1]))
    assert native.load().hpcs_seg_class_limit(99) == -2
    assert native.load().hpcs_ctx_set_seg_tuning(None, None) == native.HPCS_ERR_NULL
