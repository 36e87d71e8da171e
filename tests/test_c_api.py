"""The drop-in API from C: tests/c_api/check_c_api.c is compiled as C99 against include/onefft.h
and linked to libonefft_cuda.so the way a OneFFT caller would link (cc ... -lonefft_cuda).
Compiling and linking needs no GPU; running the program's checks does.
"""
from __future__ import annotations

import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_api", "check_c_api.c")


def build_c_program(out_dir: str) -> str:
    import onefft_b200
    if not os.path.exists(onefft_b200.LIB_PATH):
        from onefft_b200 import build
        build.build()
    cc = shutil.which("cc") or shutil.which("gcc")
    if cc is None:
        pytest.skip("no C compiler")
    exe = os.path.join(out_dir, "check_c_api")
    libdir = os.path.dirname(onefft_b200.LIB_PATH)
    cmd = [cc, "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", libdir, "-lonefft_cuda", f"-Wl,-rpath,{libdir}", "-lm", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


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
