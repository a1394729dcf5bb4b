"""The C++ host mirror (include/hpcsharp_gpu.hpp) compiles against the C ABI (CPU), and its
usage program passes on a GPU."""
import os
import subprocess

import pytest

from hpcsharp_b200 import build, native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "mirror_test.cpp")
EXE = os.path.join(ROOT, "tests", "cpp", "mirror_test")


def compile_mirror():
    build.build_gpu()
    libdir = os.path.dirname(native.LIB_PATH)
    cmd = ["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"), SRC, "-o", EXE,
           f"-L{libdir}", "-l:libhpcs_gpu.so", f"-Wl,-rpath,{libdir}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return EXE


def test_mirror_compiles_and_links():
    assert os.path.exists(compile_mirror())


@pytest.mark.gpu
def test_mirror_program_passes_on_gpu():
    exe = compile_mirror()
    r = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "mirror_test: ok" in r.stdout
