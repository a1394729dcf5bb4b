"""ctypes front end of the CPU oracle (liboracle.so, built from oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the CPU-baseline
leg of bench.py, as the checker and the timed CPU baseline.  Never part of the product path.

Every function operates in place on numpy arrays, like the reference's extension methods.
kind: 0 unsigned, 1 signed (top byte ^ 0x80), 2 float (sign 0: flip sign bit, sign 1:
flip all bits).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lib = None

KIND = {"u32": 0, "i32": 1, "f32": 2, "u64": 0, "i64": 1, "f64": 2}
WIDTH = {"u32": 32, "i32": 32, "f32": 32, "u64": 64, "i64": 64, "f64": 64}


def build() -> str:
    src = os.path.join(HERE, "oracle.cpp")
    if not os.path.exists(LIB_PATH) or os.path.getmtime(src) > os.path.getmtime(LIB_PATH):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P, I64, I = C.c_void_p, C.c_int64, C.c_int
        for t in ("u32", "i32", "f32", "u64", "i64", "f64"):
            getattr(L, f"orc_sort_radix_lsd_{t}").argtypes = [P, I64]
        for t in ("u32", "f32", "f64"):
            getattr(L, f"orc_sort_radix_par_{t}").argtypes = [P, I64, I64, I]
        L.orc_sort_radix_par_u64_full.argtypes = [P, I64, I64, I]
        for t in ("i32", "u64", "i64"):
            getattr(L, f"orc_sort_radix_par_{t}").argtypes = [P, I64, I]
        L.orc_sort_pairs_k32_v32.argtypes = [P, P, I64, I]
        L.orc_sort_pairs_k64_v32.argtypes = [P, P, I64, I]
        for w in ("k32", "k64"):
            getattr(L, f"orc_histogram_byte_components_{w}").argtypes = [P, I64, I64, I, P]
            getattr(L, f"orc_histogram_byte_components_par_{w}").argtypes = [P, I64, I64, I, P, I]
            getattr(L, f"orc_select_topk_{w}").argtypes = [P, I64, I64, I]
            getattr(L, f"orc_select_topk_{w}").restype = I
            getattr(L, f"orc_stable_sort_transformed_{w}").argtypes = [P, I64, I]
            getattr(L, f"orc_stable_argsort_{w}").argtypes = [P, I64, I, P]
        for t in ("u32", "i32", "u64", "i64"):
            getattr(L, f"orc_std_sort_{t}").argtypes = [P, I64]
        L.orc_hardware_threads.restype = I
        L.orc_radix_par_ws_create.argtypes = [I64, I64, I]
        L.orc_radix_par_ws_create.restype = P
        L.orc_radix_par_ws_destroy.argtypes = [P]
        L.orc_sort_radix_par_ws_k32.argtypes = [P, P, I64, I, I]
        L.orc_sort_radix_par_ws_k64.argtypes = [P, P, I64, I, I]
        L.orc_gen_u32_uniform.argtypes = [P, I64, C.c_uint64, I]
        for w in ("k32", "k64"):
            getattr(L, f"orc_partition_radix_{w}").argtypes = [P, I64, I64, P, I64, I, I64]
        _lib = L
    return _lib


def _name(a: np.ndarray) -> str:
    m = {np.dtype(np.uint32): "u32", np.dtype(np.int32): "i32", np.dtype(np.float32): "f32",
         np.dtype(np.uint64): "u64", np.dtype(np.int64): "i64", np.dtype(np.float64): "f64"}
    return m[a.dtype]


def _w(a):
    return "k32" if a.dtype.itemsize == 4 else "k64"


def sort_radix_lsd(a: np.ndarray) -> np.ndarray:
    """Serial SortRadixLsd restatement (RadixSortLsd.cs:127-532), in place."""
    getattr(lib(), f"orc_sort_radix_lsd_{_name(a)}")(a.ctypes.data, a.size)
    return a


def sort_radix_par(a: np.ndarray, threads: int = 0, quantum: int = 64 * 1024) -> np.ndarray:
    """SortRadixPar restatement (RadixSortLsdParallel.cs): fully parallel for u32 (and the
    float keys), partially parallel (parallel histogram, serial scatter) for i32/u64/i64."""
    t = _name(a)
    th = threads if threads > 0 else hardware_threads()
    L = lib()
    if t in ("u32", "f32", "f64"):
        getattr(L, f"orc_sort_radix_par_{t}")(a.ctypes.data, a.size, quantum, th)
    else:
        getattr(L, f"orc_sort_radix_par_{t}")(a.ctypes.data, a.size, th)
    return a


class RadixParWorkspace:
    """Scratch of SortRadixPar made once: the output array and the per-quantum buffers, counts
    and starts that the reference allocates at the top of each call (RadixSortLsdParallel.cs:
    151-170).  sort() then runs the fully parallel restatement without allocating, so a timed
    loop measures the sort alone."""

    def __init__(self, n: int, itemsize: int = 4, quantum: int = 64 * 1024):
        self.n, self.itemsize = int(n), int(itemsize)
        self.handle = lib().orc_radix_par_ws_create(self.n, quantum, self.itemsize)
        if not self.handle:
            raise MemoryError("workspace creation failed")

    def sort(self, a: np.ndarray, threads: int = 0) -> np.ndarray:
        """Fully parallel SortRadixPar of a (any of the six key types) in place."""
        if a.dtype.itemsize != self.itemsize or a.size > self.n or not a.flags.c_contiguous:
            raise ValueError("array does not fit the workspace")
        th = threads if threads > 0 else hardware_threads()
        fn = lib().orc_sort_radix_par_ws_k32 if self.itemsize == 4 else lib().orc_sort_radix_par_ws_k64
        if fn(self.handle, a.ctypes.data, a.size, KIND[_name(a)], th) != 0:
            raise RuntimeError("SortRadixPar workspace call failed")
        return a

    def close(self) -> None:
        if self.handle:
            lib().orc_radix_par_ws_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def gen_u32_uniform(n: int, seed: int = 1, threads: int = 0) -> np.ndarray:
    """The benchmark's uniform uint32 keys (PCG32 per 64 Ki chunk), generated here so that a CPU
    baseline loads no library of the product; equal to hpcsharp_b200.datagen.u32_uniform."""
    a = np.empty(int(n), dtype=np.uint32)
    lib().orc_gen_u32_uniform(a.ctypes.data, a.size, seed, threads if threads > 0 else hardware_threads())
    return a


def sort_radix_par_u32_full(a: np.ndarray, threads: int = 0, quantum: int = 64 * 1024):
    lib().orc_sort_radix_par_u32(a.ctypes.data, a.size, quantum, threads if threads > 0 else hardware_threads())
    return a


def sort_pairs(keys: np.ndarray, items: np.ndarray):
    """SortRadix<T>(items, keys) restatement (RadixSortLsd.cs:1183-1299), both in place."""
    assert items.dtype.itemsize == 4 and items.size == keys.size
    fn = lib().orc_sort_pairs_k32_v32 if keys.dtype.itemsize == 4 else lib().orc_sort_pairs_k64_v32
    fn(keys.ctypes.data, items.ctypes.data, keys.size, KIND[_name(keys)])
    return keys, items


def histogram_byte_components(a: np.ndarray, l: int, r: int, parallel: bool = False) -> np.ndarray:
    """counts[P][256] of a[l..r] (Histogram.cs:261-1052 / HistogramParallel.cs)."""
    P = a.dtype.itemsize
    out = np.zeros((P, 256), dtype=np.uint32)
    if parallel:
        getattr(lib(), f"orc_histogram_byte_components_par_{_w(a)}")(a.ctypes.data, l, r, KIND[_name(a)],
                                                                      out.ctypes.data, hardware_threads())
    else:
        getattr(lib(), f"orc_histogram_byte_components_{_w(a)}")(a.ctypes.data, l, r, KIND[_name(a)],
                                                                  out.ctypes.data)
    return out


def select_topk(a: np.ndarray, k: int) -> int:
    """SelectTopK(a, k) restatement (SelectionTopKRadix.cs:96-171), in place."""
    return getattr(lib(), f"orc_select_topk_{_w(a)}")(a.ctypes.data, a.size, k, KIND[_name(a)])


def partition_radix(a: np.ndarray, start: int, length: int, ks, threshold: int = 1024) -> np.ndarray:
    """PartitionRadix(a, start, length, k or k[], threshold) restatement (PartitionRadix.cs:15-210),
    in place; ks are absolute indices in ascending order."""
    kk = np.ascontiguousarray(np.atleast_1d(np.asarray(ks, dtype=np.int64)))
    getattr(lib(), f"orc_partition_radix_{_w(a)}")(a.ctypes.data, start, length, kk.ctypes.data, kk.size,
                                                   KIND[_name(a)], threshold)
    return a


def stable_sort_transformed(a: np.ndarray) -> np.ndarray:
    getattr(lib(), f"orc_stable_sort_transformed_{_w(a)}")(a.ctypes.data, a.size, KIND[_name(a)])
    return a


def stable_argsort(a: np.ndarray) -> np.ndarray:
    perm = np.empty(a.size, dtype=np.uint32)
    getattr(lib(), f"orc_stable_argsort_{_w(a)}")(a.ctypes.data, a.size, KIND[_name(a)], perm.ctypes.data)
    return perm


def std_sort(a: np.ndarray) -> np.ndarray:
    """std::sort (introsort): the Array.Sort stand-in for integer keys."""
    getattr(lib(), f"orc_std_sort_{_name(a)}")(a.ctypes.data, a.size)
    return a


def hardware_threads() -> int:
    return int(lib().orc_hardware_threads())


def order_key(a: np.ndarray) -> np.ndarray:
    """The reference's order transform as numpy unsigned integers (for test assertions)."""
    t = _name(a)
    if a.dtype.itemsize == 4:
        u = a.view(np.uint32)
        top = np.uint32(0x80000000)
        allones = np.uint32(0xFFFFFFFF)
    else:
        u = a.view(np.uint64)
        top = np.uint64(0x8000000000000000)
        allones = np.uint64(0xFFFFFFFFFFFFFFFF)
    if KIND[t] == 1:
        return u ^ top
    if KIND[t] == 2:
        neg = (u & top) != 0
        return np.where(neg, u ^ allones, u ^ top)
    return u.copy()
