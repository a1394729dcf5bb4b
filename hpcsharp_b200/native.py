"""ctypes bindings of libhpcs_gpu.so (the C ABI declared in include/hpcs_gpu.h).

This module is plumbing for Python callers (tests, benchmarks, the serving demo); the
compute path is the CUDA library.  There is no CPU fallback: if the library or a CUDA
device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
# HPCS_GPU_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("HPCS_GPU_LIB") or os.path.join(_PKG, "libhpcs_gpu.so")

HPCS_OK = 0
HPCS_ERR_NULL = 1
HPCS_ERR_RANGE = 2
HPCS_ERR_OOM = 3
HPCS_ERR_CUDA = 4
HPCS_ERR_DEVICE_TIMEOUT = 5
HPCS_ERR_UNSUPPORTED = 6
HPCS_ERR_NO_DEVICE = 7
HPCS_ERR_BUSY = 8

DTYPES = {"u32": 0, "i32": 1, "f32": 2, "u64": 3, "i64": 4, "f64": 5}
NP_OF = {"u32": np.uint32, "i32": np.int32, "f32": np.float32, "u64": np.uint64, "i64": np.int64, "f64": np.float64}
CT_OF = {"u32": C.c_uint32, "i32": C.c_int32, "f32": C.c_float, "u64": C.c_uint64, "i64": C.c_int64,
         "f64": C.c_double}


# 8- and 16-bit keys: sorted by the counting sort (plain sorts only)
COUNT_NP_OF = {"u8": np.uint8, "i8": np.int8, "u16": np.uint16, "i16": np.int16}


def dtype_name(arr_dtype, counting: bool = False) -> str:
    dt = np.dtype(arr_dtype)
    for k, v in NP_OF.items():
        if np.dtype(v) == dt:
            return k
    if counting:
        for k, v in COUNT_NP_OF.items():
            if np.dtype(v) == dt:
                return k
    raise TypeError(f"unsupported key dtype {dt}")


class HpcsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{_status_name(status)}: {message}")
        self.status = status


class ArgumentNullException(HpcsError, ValueError):
    """Raised for HPCS_ERR_NULL (the reference throws ArgumentNullException)."""


class ArgumentOutOfRangeException(HpcsError, IndexError):
    """Raised for HPCS_ERR_RANGE (the reference throws ArgumentOutOfRangeException)."""


class DeviceTimeoutError(HpcsError):
    """A bounded device-side wait ran out (HPCS_ERR_DEVICE_TIMEOUT)."""


class HpcsConfig(C.Structure):
    _fields_ = [
        ("pool_bytes", C.c_int64),
        ("skip_trivial_passes", C.c_int32),
        ("rank_mode", C.c_int32),
        ("spin_limit_ns", C.c_int64),
        ("poison_tile", C.c_int32),
        ("pass_scheme", C.c_int32),
        ("staged_host_copies", C.c_int32),
        ("seg_grid_min_keys", C.c_int32),
        ("seg_grid_tiles", C.c_int32),
        ("reserved", C.c_int32 * 3),
    ]


PASS_SCHEMES = {"auto": 0, "lookback": 1, "chunked": 2}
KCLASS = {"histogram": 0, "onesweep": 1, "finalize": 2, "topk": 3, "segmented": 4, "shard": 5, "lookback": 6}


class HpcsSegment(C.Structure):
    _fields_ = [("keys", C.c_void_p), ("n", C.c_int64), ("dtype", C.c_int32), ("reserved", C.c_int32)]


SEG_CLASSES = 8


class HpcsSegTuning(C.Structure):
    _fields_ = [("variant", (C.c_int32 * SEG_CLASSES) * 2)]


class HpcsSegVariantInfo(C.Structure):
    _fields_ = [("kind", C.c_int32), ("threads", C.c_int32), ("keys_per_thread", C.c_int32),
                ("digit_bits", C.c_int32), ("max_keys", C.c_int64 * 2)]


class HpcsRequest(C.Structure):
    _fields_ = [("op", C.c_int32), ("dtype", C.c_int32), ("input", C.c_void_p), ("output", C.c_void_p),
                ("n", C.c_int64), ("k", C.c_int64)]


class HpcsRequestInfo(C.Structure):
    _fields_ = [("status", C.c_int32), ("coalesced", C.c_int32), ("submit_ns", C.c_int64),
                ("admit_ns", C.c_int64), ("done_ns", C.c_int64)]


class HpcsServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("slots", C.c_int32), ("hbm_budget_bytes", C.c_int64),
                ("coalesce_max_keys", C.c_int64), ("coalesce_max_requests", C.c_int32), ("reserved", C.c_int32 * 5)]


class HpcsServerCounters(C.Structure):
    _fields_ = [(f, C.c_int64) for f in ("completed", "keys", "batches", "coalesced", "pending", "arena_bytes",
                                         "arena_used", "arena_peak")]


class HpcsProfile(C.Structure):
    _fields_ = [("launches", C.c_int64 * 8), ("total_ms", C.c_double * 8)]


_lib = None
_lib_lock = threading.Lock()


def _status_name(status: int) -> str:
    names = {0: "HPCS_OK", 1: "HPCS_ERR_NULL", 2: "HPCS_ERR_RANGE", 3: "HPCS_ERR_OOM", 4: "HPCS_ERR_CUDA",
             5: "HPCS_ERR_DEVICE_TIMEOUT", 6: "HPCS_ERR_UNSUPPORTED", 7: "HPCS_ERR_NO_DEVICE", 8: "HPCS_ERR_BUSY"}
    return names.get(status, f"status {status}")


def _declare(lib) -> None:
    P, I64, I32, U32P = C.c_void_p, C.c_int64, C.c_int, C.POINTER(C.c_uint32)
    lib.hpcs_config_default.argtypes = [C.POINTER(HpcsConfig)]
    lib.hpcs_config_default.restype = None
    lib.hpcs_ctx_create.argtypes = [I32, C.POINTER(HpcsConfig), C.POINTER(P)]
    lib.hpcs_ctx_destroy.argtypes = [P]
    lib.hpcs_ctx_synchronize.argtypes = [P]
    lib.hpcs_ctx_stream.argtypes = [P]
    lib.hpcs_ctx_stream.restype = P
    lib.hpcs_ctx_rank_mode.argtypes = [P]
    lib.hpcs_last_error_message.restype = C.c_char_p
    lib.hpcs_status_string.argtypes = [I32]
    lib.hpcs_status_string.restype = C.c_char_p
    for t in DTYPES:
        getattr(lib, f"hpcs_sort_{t}").argtypes = [P, P, I64]
        getattr(lib, f"hpcs_sort_{t}_dev").argtypes = [P, P, I64, P]
        getattr(lib, f"hpcs_sort_pairs_{t}").argtypes = [P, P, P, I64]
        getattr(lib, f"hpcs_sort_pairs_{t}_dev").argtypes = [P, P, P, I64, P]
        getattr(lib, f"hpcs_histogram_byte_components_{t}").argtypes = [P, P, I64, I64, P]
        getattr(lib, f"hpcs_select_topk_{t}").argtypes = [P, P, I64, I64]
        getattr(lib, f"hpcs_select_topk_{t}_dev").argtypes = [P, P, I64, I64, P]
        getattr(lib, f"hpcs_topk_largest_{t}").argtypes = [P, P, I64, I64, P]
        getattr(lib, f"hpcs_topk_largest_{t}_dev").argtypes = [P, P, I64, I64, P, P]
        getattr(lib, f"hpcs_partition_radix_{t}").argtypes = [P, P, I64, I64, P, I64]
        getattr(lib, f"hpcs_select_radix_{t}").argtypes = [P, P, I64, I64, I64, P]
    lib.hpcs_histogram_byte_components_dev.argtypes = [P, I32, P, I64, P, P]
    lib.hpcs_shard_partition_dev.argtypes = [P, I32, P, P, I64, I64, P, P, I32, P, P, P, P]
    for t in COUNT_NP_OF:
        getattr(lib, f"hpcs_sort_{t}").argtypes = [P, P, I64]
        getattr(lib, f"hpcs_sort_{t}_dev").argtypes = [P, P, I64, P]
    lib.hpcs_ctx_profile_enable.argtypes = [P, I32]
    lib.hpcs_ctx_profile_read.argtypes = [P, C.POINTER(HpcsProfile)]
    lib.hpcs_ctx_trace_tiles.argtypes = [P, P, I32, I32]
    lib.hpcs_sort_segmented_dev.argtypes = [P, C.POINTER(HpcsSegment), I64, P]
    lib.hpcs_segplan_create.argtypes = [P, C.POINTER(HpcsSegment), I64, C.POINTER(P)]
    lib.hpcs_segplan_execute.argtypes = [P, P]
    lib.hpcs_segplan_destroy.argtypes = [P]
    lib.hpcs_seg_variants.argtypes = [C.POINTER(HpcsSegVariantInfo), I32]
    lib.hpcs_seg_class_limit.argtypes = [I32]
    lib.hpcs_seg_class_limit.restype = I64
    lib.hpcs_ctx_get_seg_tuning.argtypes = [P, C.POINTER(HpcsSegTuning)]
    lib.hpcs_ctx_set_seg_tuning.argtypes = [P, C.POINTER(HpcsSegTuning)]
    lib.hpcs_server_config_default.argtypes = [C.POINTER(HpcsServerConfig)]
    lib.hpcs_server_config_default.restype = None
    lib.hpcs_server_create.argtypes = [C.POINTER(HpcsServerConfig), C.POINTER(P)]
    lib.hpcs_server_submit.argtypes = [P, C.POINTER(HpcsRequest), C.POINTER(C.c_uint64)]
    lib.hpcs_server_wait.argtypes = [P, C.c_uint64, I64, C.POINTER(HpcsRequestInfo)]
    lib.hpcs_server_stats.argtypes = [P, C.POINTER(HpcsServerCounters)]
    lib.hpcs_server_destroy.argtypes = [P]


def load():
    """Load libhpcs_gpu.so (raises if it was not built)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(f"{LIB_PATH} is missing; run `python -m hpcsharp_b200.build`")
            lib = C.CDLL(LIB_PATH)
            _declare(lib)
            _lib = lib
    return _lib


def check(status: int) -> None:
    if status == HPCS_OK:
        return
    msg = load().hpcs_last_error_message().decode(errors="replace")
    if status == HPCS_ERR_NULL:
        raise ArgumentNullException(status, msg)
    if status == HPCS_ERR_RANGE:
        raise ArgumentOutOfRangeException(status, msg)
    if status == HPCS_ERR_DEVICE_TIMEOUT:
        raise DeviceTimeoutError(status, msg)
    raise HpcsError(status, msg)


def seg_variants() -> list[dict]:
    """The segmented sort's kernel variants (index = variant id)."""
    lib = load()
    arr = (HpcsSegVariantInfo * 64)()
    n = lib.hpcs_seg_variants(arr, 64)
    return [{"kind": "warp" if arr[i].kind == 0 else "block", "threads": arr[i].threads,
             "keys_per_thread": arr[i].keys_per_thread, "digit_bits": arr[i].digit_bits,
             "max_keys": [arr[i].max_keys[0], arr[i].max_keys[1]]} for i in range(n)]


def seg_class_limits() -> list[int]:
    """Upper length limit of each length class of the segmented sort (-1: unbounded)."""
    lib = load()
    return [int(lib.hpcs_seg_class_limit(c)) for c in range(SEG_CLASSES)]


def default_config() -> HpcsConfig:
    cfg = HpcsConfig()
    load().hpcs_config_default(C.byref(cfg))
    return cfg


def _ptr(a) -> int | None:
    """Address of a numpy array (host) or a torch tensor (device)."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags.c_contiguous:
            raise ValueError("array must be C-contiguous")
        return a.ctypes.data
    if hasattr(a, "data_ptr"):
        if not a.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return a.data_ptr()
    raise TypeError(f"unsupported array type {type(a)}")


class Context:
    """One hpcs_ctx: a CUDA stream plus grow-only scratch on one device."""

    def __init__(self, device: int = 0, *, pool_bytes: int = 0, skip_trivial_passes: bool = True,
                 spin_limit_ns: int = 2_000_000_000, poison_tile: int = -1, rank_mode: int = 0,
                 pass_scheme: str = "auto", staged_host_copies: bool = True, seg_grid_min_keys: int = 0,
                 seg_grid_tiles: int = 0):
        self.lib = load()
        cfg = default_config()
        cfg.staged_host_copies = 1 if staged_host_copies else 0
        cfg.seg_grid_min_keys = seg_grid_min_keys
        cfg.seg_grid_tiles = seg_grid_tiles
        cfg.pool_bytes = pool_bytes
        cfg.skip_trivial_passes = 1 if skip_trivial_passes else 0
        cfg.spin_limit_ns = spin_limit_ns
        cfg.poison_tile = poison_tile
        cfg.rank_mode = rank_mode
        cfg.pass_scheme = PASS_SCHEMES[pass_scheme]
        h = C.c_void_p()
        check(self.lib.hpcs_ctx_create(device, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.device = device

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.hpcs_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def rank_mode(self) -> int:
        """0: ordered shared atomics (lane order verified on this GPU); 1: peer-mask ranking."""
        return int(self.lib.hpcs_ctx_rank_mode(self.handle))

    @property
    def stream(self) -> int:
        return self.lib.hpcs_ctx_stream(self.handle) or 0

    def synchronize(self) -> None:
        check(self.lib.hpcs_ctx_synchronize(self.handle))

    def profile(self, enable: bool = True) -> None:
        """Record a CUDA event pair around every kernel this context launches."""
        check(self.lib.hpcs_ctx_profile_enable(self.handle, 1 if enable else 0))

    def profile_read(self) -> dict:
        """{kernel class: (launches, total ms)} since the last read (waits for the GPU)."""
        p = HpcsProfile()
        check(self.lib.hpcs_ctx_profile_read(self.handle, C.byref(p)))
        return {k: (int(p.launches[v]), float(p.total_ms[v])) for k, v in KCLASS.items()}

    def trace_tiles(self, buf, capacity_tiles: int, digit_pass: int) -> None:
        """Attach a device buffer (int64, 7 words per tile) for the onesweep tile trace."""
        check(self.lib.hpcs_ctx_trace_tiles(self.handle, _ptr(buf) if buf is not None else None,
                                            capacity_tiles, digit_pass))

    # ---- host arrays (synchronous, in place) ----
    def sort(self, a: np.ndarray) -> np.ndarray:
        t = dtype_name(a.dtype, counting=True)
        check(getattr(self.lib, f"hpcs_sort_{t}")(self.handle, _ptr(a), a.size))
        return a

    def sort_pairs(self, keys: np.ndarray, items: np.ndarray):
        t = dtype_name(keys.dtype)
        if items is not None and items.dtype.itemsize != 4:
            raise TypeError("items must be 4-byte")
        if items is not None and items.size != keys.size:
            raise ArgumentOutOfRangeException(HPCS_ERR_RANGE, "keys and items differ in length")
        check(getattr(self.lib, f"hpcs_sort_pairs_{t}")(self.handle, _ptr(keys), _ptr(items), keys.size))
        return keys, items

    def histogram(self, a: np.ndarray, l: int, r: int) -> np.ndarray:
        t = dtype_name(a.dtype)
        P = a.dtype.itemsize
        counts = np.zeros((P, 256), dtype=np.uint32)
        check(getattr(self.lib, f"hpcs_histogram_byte_components_{t}")(self.handle, _ptr(a), l, r, _ptr(counts)))
        return counts

    def select_topk(self, a: np.ndarray, k: int) -> np.ndarray:
        """SelectTopK(a, k) in place: a[k] = k-th smallest, a[k:] = the n-k largest."""
        t = dtype_name(a.dtype)
        check(getattr(self.lib, f"hpcs_select_topk_{t}")(self.handle, _ptr(a), a.size, k))
        return a

    def partition_radix(self, a: np.ndarray, start: int, length: int, ks) -> np.ndarray:
        """PartitionRadix over a[start, start + length) by the absolute indices ks, in place."""
        t = dtype_name(a.dtype)
        kk = np.ascontiguousarray(np.atleast_1d(np.asarray(ks, dtype=np.int64)))
        check(getattr(self.lib, f"hpcs_partition_radix_{t}")(self.handle, _ptr(a), start, length,
                                                               kk.ctypes.data if kk.size else None, kk.size))
        return a

    def select_radix(self, a: np.ndarray, start: int, length: int, k: int):
        """SelectRadix(Par): the k-th smallest key of a[start, start + length) (k absolute), left at a[k]."""
        t = dtype_name(a.dtype)
        out = np.zeros(1, dtype=a.dtype)
        check(getattr(self.lib, f"hpcs_select_radix_{t}")(self.handle, _ptr(a), start, length, k, _ptr(out)))
        return out[0]

    def topk_largest(self, a: np.ndarray, k: int) -> np.ndarray:
        """The k largest keys of a, ascending."""
        t = dtype_name(a.dtype)
        out = np.empty(k, dtype=a.dtype)
        if k:
            check(getattr(self.lib, f"hpcs_topk_largest_{t}")(self.handle, _ptr(a), a.size, k, _ptr(out)))
        return out

    # ---- device tensors (asynchronous on `stream`, default: the context's stream) ----
    def sort_dev(self, t, dtype: str | None = None, stream: int | None = None) -> None:
        name = dtype or _torch_dtype_name(t)
        check(getattr(self.lib, f"hpcs_sort_{name}_dev")(self.handle, _ptr(t), t.numel(), stream))

    def sort_pairs_dev(self, keys, items, dtype: str | None = None, stream: int | None = None) -> None:
        name = dtype or _torch_dtype_name(keys)
        check(getattr(self.lib, f"hpcs_sort_pairs_{name}_dev")(self.handle, _ptr(keys), _ptr(items), keys.numel(),
                                                                stream))

    def select_topk_dev(self, t, k: int, dtype: str | None = None, stream: int | None = None) -> None:
        name = dtype or _torch_dtype_name(t)
        check(getattr(self.lib, f"hpcs_select_topk_{name}_dev")(self.handle, _ptr(t), t.numel(), k, stream))

    def topk_largest_dev(self, t, k: int, out, dtype: str | None = None, stream: int | None = None) -> None:
        name = dtype or _torch_dtype_name(t)
        check(getattr(self.lib, f"hpcs_topk_largest_{name}_dev")(self.handle, _ptr(t), t.numel(), k, _ptr(out),
                                                                 stream))

    def sort_segmented_dev(self, segments, stream: int | None = None) -> None:
        """segments: list of (device tensor or (ptr, n), dtype name).  Sorted in place."""
        arr = make_segments(segments)
        check(self.lib.hpcs_sort_segmented_dev(self.handle, arr, len(arr), stream))

    def segplan(self, segments) -> "SegPlan":
        return SegPlan(self, segments)

    @property
    def seg_tuning(self) -> list[list[int]]:
        """Variant per [4-byte keys, 8-byte keys][length class] of the segmented sort."""
        t = HpcsSegTuning()
        check(self.lib.hpcs_ctx_get_seg_tuning(self.handle, C.byref(t)))
        return [[int(t.variant[w][c]) for c in range(SEG_CLASSES)] for w in range(2)]

    @seg_tuning.setter
    def seg_tuning(self, table) -> None:
        t = HpcsSegTuning()
        for w in range(2):
            for c in range(SEG_CLASSES):
                t.variant[w][c] = int(table[w][c])
        check(self.lib.hpcs_ctx_set_seg_tuning(self.handle, C.byref(t)))

    def histogram_dev(self, t, counts, dtype: str | None = None, stream: int | None = None) -> None:
        name = dtype or _torch_dtype_name(t)
        check(self.lib.hpcs_histogram_byte_components_dev(self.handle, DTYPES[name], _ptr(t), t.numel(),
                                                          _ptr(counts), stream))


    def shard_partition_dev(self, keys, items, gpos0: int, split_keys, split_gpos, parts: int, keys_out,
                            items_out, counts_out, dtype: str | None = None, stream: int | None = None) -> None:
        """Stable partition of a shard into `parts` parts by (key, global position) splitters
        (hpcs_shard_partition_dev); counts_out receives the parts' sizes (int64)."""
        name = dtype or _torch_dtype_name(keys)
        check(self.lib.hpcs_shard_partition_dev(self.handle, DTYPES[name], _ptr(keys), _ptr(items), keys.numel(),
                                                gpos0, _ptr(split_keys), _ptr(split_gpos), parts, _ptr(keys_out),
                                                _ptr(items_out), _ptr(counts_out), stream))


def make_segments(segments):
    arr = (HpcsSegment * len(segments))()
    for i, (t, dt) in enumerate(segments):
        if isinstance(t, tuple):
            ptr, n = t
        else:
            ptr, n = _ptr(t), t.numel()
        arr[i].keys = ptr
        arr[i].n = n
        arr[i].dtype = DTYPES[dt]
    return arr


class SegPlan:
    """A batched segmented sort captured once (device-resident descriptors + CUDA graph)."""

    def __init__(self, ctx: "Context", segments):
        self.ctx = ctx
        arr = make_segments(segments)
        h = C.c_void_p()
        check(ctx.lib.hpcs_segplan_create(ctx.handle, arr, len(arr), C.byref(h)))
        self.handle = h

    def execute(self, stream: int | None = None) -> None:
        check(self.ctx.lib.hpcs_segplan_execute(self.handle, stream))

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.ctx.lib.hpcs_segplan_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def torch_stream(device=None) -> int:
    """The stream argument of the *_dev calls that runs them on torch's current stream of
    `device`.  Torch's default stream has the handle 0, which the C ABI reads as the context's
    own stream, so it is passed as cudaStreamLegacy (1)."""
    import torch

    h = torch.cuda.current_stream(device).cuda_stream
    return h if h else 1


def _torch_dtype_name(t) -> str:
    import torch

    m = {torch.int32: "i32", torch.float32: "f32", torch.int64: "i64", torch.float64: "f64"}
    if hasattr(torch, "uint32"):
        m[torch.uint32] = "u32"
    if hasattr(torch, "uint64"):
        m[torch.uint64] = "u64"
    if t.dtype not in m:
        raise TypeError(f"unsupported tensor dtype {t.dtype}; pass dtype=")
    return m[t.dtype]


OPS = {"sort": 0, "topk": 1}


class Server:
    """Continuous-batching sort / top-k server (hpcs_server_* in the C ABI)."""

    def __init__(self, device: int = 0, *, slots: int = 4, hbm_budget_bytes: int = 16 << 30,
                 coalesce_max_keys: int = 1 << 17, coalesce_max_requests: int = 4096):
        self.lib = load()
        cfg = HpcsServerConfig()
        self.lib.hpcs_server_config_default(C.byref(cfg))
        cfg.device, cfg.slots, cfg.hbm_budget_bytes = device, slots, hbm_budget_bytes
        cfg.coalesce_max_keys, cfg.coalesce_max_requests = coalesce_max_keys, coalesce_max_requests
        h = C.c_void_p()
        check(self.lib.hpcs_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h

    def submit(self, op: str, keys: np.ndarray, out: np.ndarray, k: int = 0) -> int:
        """Queues a request; keys/out must stay alive until wait() returns for its ticket."""
        r = HpcsRequest()
        r.op, r.dtype = OPS[op], DTYPES[dtype_name(keys.dtype)]
        r.input, r.output, r.n, r.k = keys.ctypes.data, out.ctypes.data, keys.size, k
        t = C.c_uint64()
        check(self.lib.hpcs_server_submit(self.handle, C.byref(r), C.byref(t)))
        return t.value

    def wait(self, ticket: int, timeout_ns: int = 0) -> dict:
        info = HpcsRequestInfo()
        status = self.lib.hpcs_server_wait(self.handle, ticket, timeout_ns, C.byref(info))
        check(status)
        return {"coalesced": bool(info.coalesced), "submit_ns": info.submit_ns, "admit_ns": info.admit_ns,
                "done_ns": info.done_ns}

    def stats(self) -> dict:
        c = HpcsServerCounters()
        check(self.lib.hpcs_server_stats(self.handle, C.byref(c)))
        return {f: getattr(c, f) for f, _ in HpcsServerCounters._fields_}

    def close(self) -> None:
        if getattr(self, "handle", None):
            self.lib.hpcs_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Context | None = None


def default_context() -> Context:
    """Per-process context on device 0, created on first use."""
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx
