"""Build recipe for the native parts of hpcsharp_b200.

Outputs (all in-tree, git-ignored, shipped with the tree):
  hpcsharp_b200/libhpcs_gpu.so   CUDA kernels + C ABI (include/hpcs_gpu.h), sm_100a only
  hpcsharp_b200/libhpcs_gen.so   seeded synthetic key generators (host C++)

nvcc cross-compiles for sm_100a without a GPU.  Run: python -m hpcsharp_b200.build
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
    "-Xptxas", "-warn-spills",
    "--expt-relaxed-constexpr",
]
OBJ_DIR = os.path.join(ROOT, "_build")

GPU_SOURCES = ["capi.cu", "noalloc.cu", "segmented_host.cu", "serve.cu"]


def _gpu_deps() -> list[str]:
    """Every header of csrc/ (any of them can change the library)."""
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cuh"))


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _stale(target: str, sources: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def _run(cmd: list[str]) -> None:
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        sys.stderr.write(res.stdout + res.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    if res.stderr.strip():
        sys.stderr.write(res.stderr)


def build_gpu(force: bool = False, verbose_ptxas: bool = False, out: str | None = None,
              defines: list[str] | None = None) -> str:
    """Compile libhpcs_gpu.so; `defines` (e.g. ["HPCS_K32_KPT=12"]) build a tuning variant."""
    out = out or os.path.join(PKG, "libhpcs_gpu.so")
    srcs = [os.path.join(CSRC, s) for s in GPU_SOURCES]
    deps = srcs + _gpu_deps() + [os.path.join(ROOT, "include", "hpcs_gpu.h")]
    if force or _stale(out, deps):
        from concurrent.futures import ThreadPoolExecutor

        flags = list(NVCC_FLAGS)
        if verbose_ptxas:
            flags += ["-Xptxas", "-v"]
        for d in defines or []:
            flags += ["-D" + d]
        # one object per translation unit, compiled concurrently, then one link
        tag = os.path.splitext(os.path.basename(out))[0]
        os.makedirs(OBJ_DIR, exist_ok=True)
        objs = [os.path.join(OBJ_DIR, f"{tag}.{os.path.splitext(os.path.basename(src))[0]}.o") for src in srcs]
        with ThreadPoolExecutor(max_workers=len(srcs)) as pool:
            list(pool.map(lambda so: _run([_nvcc(), *flags, "-c", "-o", so[1], so[0]]), zip(srcs, objs)))
        _run([_nvcc(), "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", out, *objs])
    return out


def build_gen(force: bool = False) -> str:
    out = os.path.join(PKG, "libhpcs_gen.so")
    src = os.path.join(PKG, "datagen", "gen.cpp")
    if force or _stale(out, [src]):
        _run(["g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-pthread", "-o", out, src])
    return out


def build_all(force: bool = False) -> None:
    build_gen(force)
    build_gpu(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", os.path.join(PKG, "libhpcs_gpu.so"), os.path.join(PKG, "libhpcs_gen.so"))
