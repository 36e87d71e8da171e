"""The drop-in API from C and C++: tests/c_api/check_c_api.c is compiled as C99 and
tests/c_api/check_cpp_api.cpp as C++11 (the C++ layer of the header, as OneFFT's
tests/test_cpp.cpp uses it) against include/onefft.h, each linked to libonefft_cuda.so the way a
OneFFT caller would link (cc / c++ ... -lonefft_cuda); tests/c_api/check_cuda_api.c is a C99
caller of the device-pointer additions (include/onefft_cuda.h) that allocates its buffers with
the CUDA runtime. Compiling and linking needs no GPU; running the programs' checks does.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_api", "check_c_api.c")
SRC_CPP = os.path.join(ROOT, "tests", "c_api", "check_cpp_api.cpp")


SRC_CUDA = os.path.join(ROOT, "tests", "c_api", "check_cuda_api.c")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(out_dir: str, src: str, compilers: tuple[str, ...], std: str, name: str, extra=()) -> str:
    import onefft_b200
    if not os.path.exists(onefft_b200.LIB_PATH):
        from onefft_b200 import build
        build.build()
    cc = next((c for c in map(shutil.which, compilers) if c), None)
    if cc is None:
        pytest.skip(f"no compiler among {compilers}")
    exe = os.path.join(out_dir, name)
    libdir = os.path.dirname(onefft_b200.LIB_PATH)
    cmd = [cc, f"-std={std}", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), src,
           "-L", libdir, "-lonefft_cuda", f"-Wl,-rpath,{libdir}", *extra, "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def build_c_program(out_dir: str) -> str:
    return _build(out_dir, SRC, ("cc", "gcc"), "c99", "check_c_api")


def build_cpp_program(out_dir: str) -> str:
    return _build(out_dir, SRC_CPP, ("c++", "g++"), "c++11", "check_cpp_api")


def build_cuda_program(out_dir: str) -> str:
    inc, lib = os.path.join(CUDA_HOME, "include"), os.path.join(CUDA_HOME, "lib64")
    if not os.path.exists(os.path.join(inc, "cuda_runtime_api.h")):
        pytest.skip("no CUDA runtime headers")
    return _build(out_dir, SRC_CUDA, ("cc", "gcc"), "c99", "check_cuda_api",
                  ("-I", inc, "-L", lib, "-lcudart", f"-Wl,-rpath,{lib}"))


def test_c_program_compiles_and_links(tmp_path):
    """include/onefft.h is valid C99 and every function the program calls resolves in the library."""
    exe = build_c_program(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_c_program_checks_pass(tmp_path):
    exe = build_c_program(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout


def test_cpp_program_compiles_and_links(tmp_path):
    """The header's C++ layer compiles as C++11 and links against the library."""
    exe = build_cpp_program(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cpp_program_checks_pass(tmp_path):
    exe = build_cpp_program(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout


def test_cuda_api_program_compiles_and_links(tmp_path):
    """include/onefft_cuda.h is valid C99 and its device entry points resolve in the library."""
    exe = build_cuda_program(str(tmp_path))
    assert os.path.exists(exe)


@pytest.mark.gpu
def test_cuda_api_program_checks_pass(tmp_path):
    exe = build_cuda_program(str(tmp_path))
    r = subprocess.run([exe], capture_output=True, text=True, timeout=600)
    print(r.stdout)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "all checks passed" in r.stdout
