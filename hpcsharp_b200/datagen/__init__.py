"""Seeded synthetic key generators (numpy front end of libhpcs_gen.so).

Deterministic for a seed and independent of the thread count; see gen.cpp for the
streams.  Used by the tests and the benchmark to build the sort workloads.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_PKG = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
_LIB_PATH = os.path.join(_PKG, "libhpcs_gen.so")
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            from .. import build

            build.build_gen()
        lib = C.CDLL(_LIB_PATH)
        P, I64, U64, I32, D = C.c_void_p, C.c_int64, C.c_uint64, C.c_int, C.c_double
        lib.hg_u32_uniform.argtypes = [P, I64, U64, I32]
        lib.hg_u32_pcg32_stream.argtypes = [P, I64, U64]
        lib.hg_u32_xorshift64s.argtypes = [P, I64, U64]
        lib.hg_u64_uniform.argtypes = [P, I64, U64, I32]
        lib.hg_u64_and3.argtypes = [P, I64, U64, I32]
        lib.hg_i32_normal.argtypes = [P, I64, U64, D, I32]
        lib.hg_f32_normal_special.argtypes = [P, I64, U64, D, I32]
        lib.hg_f32_normal.argtypes = [P, I64, U64, I32]
        lib.hg_f64_normal.argtypes = [P, I64, U64, I32]
        lib.hg_u64_zipf.argtypes = [P, I64, U64, D, I64, I32]
        lib.hg_iota_u32.argtypes = [P, I64, I32]
        _lib = lib
    return _lib


def _empty(n, dt, out):
    if out is None:
        return np.empty(int(n), dtype=dt)
    assert out.dtype == np.dtype(dt) and out.size == n and out.flags.c_contiguous
    return out


def u32_uniform(n, seed=1, threads=0, out=None):
    a = _empty(n, np.uint32, out)
    _load().hg_u32_uniform(a.ctypes.data, a.size, seed, threads)
    return a


def u32_pcg32_stream(n, seed=1):
    a = np.empty(int(n), dtype=np.uint32)
    _load().hg_u32_pcg32_stream(a.ctypes.data, a.size, seed)
    return a


def u32_xorshift64s(n, seed=1):
    a = np.empty(int(n), dtype=np.uint32)
    _load().hg_u32_xorshift64s(a.ctypes.data, a.size, seed)
    return a


def u64_uniform(n, seed=1, threads=0, out=None):
    a = _empty(n, np.uint64, out)
    _load().hg_u64_uniform(a.ctypes.data, a.size, seed, threads)
    return a


def u64_and3(n, seed=1, threads=0, out=None):
    a = _empty(n, np.uint64, out)
    _load().hg_u64_and3(a.ctypes.data, a.size, seed, threads)
    return a


def i32_normal(n, seed=1, sigma=float(1 << 20), threads=0, out=None):
    a = _empty(n, np.int32, out)
    _load().hg_i32_normal(a.ctypes.data, a.size, seed, sigma, threads)
    return a


def f32_normal_special(n, seed=1, special_frac=0.001, threads=0, out=None):
    a = _empty(n, np.float32, out)
    _load().hg_f32_normal_special(a.ctypes.data, a.size, seed, special_frac, threads)
    return a


def f32_normal(n, seed=1, threads=0, out=None):
    a = _empty(n, np.float32, out)
    _load().hg_f32_normal(a.ctypes.data, a.size, seed, threads)
    return a


def f64_normal(n, seed=1, threads=0, out=None):
    a = _empty(n, np.float64, out)
    _load().hg_f64_normal(a.ctypes.data, a.size, seed, threads)
    return a


def u64_zipf(n, seed=1, s=1.1, nvalues=1_000_000, threads=0, out=None):
    a = _empty(n, np.uint64, out)
    _load().hg_u64_zipf(a.ctypes.data, a.size, seed, s, nvalues, threads)
    return a


def iota_u32(n, threads=0, out=None):
    a = _empty(n, np.uint32, out)
    _load().hg_iota_u32(a.ctypes.data, a.size, threads)
    return a


def i64_uniform(n, seed=1, threads=0):
    return u64_uniform(n, seed, threads).view(np.int64)


def by_name(dtype: str, n: int, seed: int = 1, threads: int = 0) -> np.ndarray:
    """The default distribution of each key dtype used by the plain-sort workloads:
    u32 uniform; i32 normal(0, 2^20); f32 normal(0,1) with +/-0, +/-inf, subnormals;
    u64 uniform; i64 uniform; f64 normal(0,1)."""
    if dtype == "u32":
        return u32_uniform(n, seed, threads)
    if dtype == "i32":
        return i32_normal(n, seed, threads=threads)
    if dtype == "f32":
        return f32_normal_special(n, seed, threads=threads)
    if dtype == "u64":
        return u64_uniform(n, seed, threads)
    if dtype == "i64":
        return i64_uniform(n, seed, threads)
    if dtype == "f64":
        return f64_normal(n, seed, threads)
    raise ValueError(dtype)
