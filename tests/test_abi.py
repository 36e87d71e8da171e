"""CPU tests of the C-ABI boundary: the library loads, exports every symbol that include/*.h
declares, and rejects invalid sizes the way OneFFT does (tests/test_onefft.c:170-182) before any
device work — these calls touch no GPU.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols() -> set[str]:
    names = set()
    for h in ("onefft.h", "onefft_cuda.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names |= set(re.findall(r"^ONEFFT_API [^;]*?\b(onefft_\w+)\(", src, flags=re.M))
    return names


def exported_symbols(path: str) -> set[str]:
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


@pytest.fixture(scope="module")
def cuda_lib():
    import onefft_b200
    if not os.path.exists(onefft_b200.LIB_PATH):
        from onefft_b200 import build
        build.build()
    return onefft_b200.lib()


def test_header_declares_reference_api():
    names = declared_symbols()
    reference_api = {"onefft_forward", "onefft_inverse", "onefft_cache_prepare", "onefft_cache_clear",
                     "onefft_plan_create", "onefft_plan_destroy", "onefft_plan_forward", "onefft_plan_inverse",
                     "onefft_plan_size", "onefft_implementation"}
    assert reference_api <= names


def test_library_exports_every_declared_symbol(cuda_lib):
    import onefft_b200
    exported = exported_symbols(onefft_b200.LIB_PATH)
    missing = declared_symbols() - exported
    assert not missing, missing
    # the Python mirror types exactly the declared set
    assert set(onefft_b200.C_SYMBOLS) == declared_symbols()
    for name in declared_symbols():
        assert hasattr(cuda_lib, name)


def test_library_links_no_torch_and_no_cufft():
    import onefft_b200
    deps = subprocess.run(["ldd", onefft_b200.LIB_PATH], capture_output=True, text=True).stdout
    assert "torch" not in deps and "cufft" not in deps


def test_implementation_string(cuda_lib):
    assert cuda_lib.onefft_implementation() == b"cuda sm_100a"


def test_invalid_sizes_rejected_without_device(cuda_lib):
    """Same list as tests/test_onefft.c:171; validation happens before any CUDA call."""
    invalid = [0, 3, 5, 6, 7, 12, 1000, 1023, 1025, 2**64 - 1, 2**31]
    for n in invalid:
        assert cuda_lib.onefft_plan_create(n) is None
    cuda_lib.onefft_plan_destroy(None)  # must be accepted
    x = np.zeros(6, np.float32)
    out = np.full(6, 7.0, np.float32)
    assert cuda_lib.onefft_forward(x.ctypes.data, out.ctypes.data, 3) == -1
    assert cuda_lib.onefft_inverse(x.ctypes.data, out.ctypes.data, 0) == -1
    assert (out == 7.0).all()
    assert cuda_lib.onefft_cache_prepare(12) == -1 and cuda_lib.onefft_cache_prepare(0) == -1
    assert b"power of two" in cuda_lib.onefft_last_error()
    split = (ctypes.c_int * 2)(4, 4)
    assert cuda_lib.onefft_plan_create_split(1000, 2, split) is None
    bad = (ctypes.c_int * 2)(3, 5)  # pass shorter than 16
    assert cuda_lib.onefft_plan_create_split(256, 2, bad) is None
    assert cuda_lib.onefft_plan_size(None) == 0


def test_device_calls_reject_bad_arguments_without_device(cuda_lib):
    # NULL plan is rejected on the host
    assert cuda_lib.onefft_dev_forward_batched(None, 0, 0, 1, None) == -2
    assert cuda_lib.onefft_plan_forward_batched(None, 0, 0, 1) == -2


def test_uneven_descriptors_validated_on_host(cuda_lib):
    """Invalid uneven-batch descriptors are rejected before any device work."""
    import onefft_b200 as ofb
    bad = [
        ([17], [0], [0]),          # size beyond 2^16
        ([4], [2], [0]),           # direction not 0/1
        ([4], [0], [-1]),          # negative offset
        ([4, 4], [0, 1], [0, 15]),  # overlapping transforms
    ]
    for log2n, inv, off in bad:
        d = np.empty(len(log2n), ofb.DESC_DTYPE)
        d["log2n"], d["inverse"], d["offset"] = log2n, inv, off
        assert cuda_lib.onefft_uneven_create(d.ctypes.data, d.size) is None
        assert cuda_lib.onefft_last_error()
    assert cuda_lib.onefft_uneven_create(None, 3) is None
    # split choices outside the compiled candidates (0 .. 2 per size 2^13 .. 2^16)
    d = np.empty(1, ofb.DESC_DTYPE)
    d["log2n"], d["inverse"], d["offset"] = 14, 0, 0
    for m, bad_choice in ((13, 3), (16, -1)):
        choice = (ctypes.c_int * 17)()
        choice[m] = bad_choice
        assert cuda_lib.onefft_uneven_create_split(d.ctypes.data, 1, choice) is None
        assert b"split choice" in cuda_lib.onefft_last_error()
    with pytest.raises(ValueError):
        ofb.UnevenBatch([17], [0], [0], split={13: 1})
    cuda_lib.onefft_uneven_destroy(None)
    assert cuda_lib.onefft_uneven_span(None) == 0
    assert cuda_lib.onefft_uneven_execute(None, 0, 0, None) == -2


def test_column_transform_shapes_validated_on_host(cuda_lib):
    """onefft_columns_create rejects shapes outside its contract before any device work."""
    import onefft_b200 as ofb
    for args in [(8, 16), (1 << 25, 16), (256, 8), (256, 24), (256, 16, 512), (256, 16, 3), (256, 16, 1, 128),
                 (256, 16, 1, 1 << 41), (256, 16, 1, 1 << 12, 1), (256, 16, 1, 0, 3), (1 << 20, 1 << 12)]:
        with pytest.raises(ValueError):
            ofb.Columns(*args)
    assert cuda_lib.onefft_columns_execute(None, 0, 0, 0, None) == -2
    cuda_lib.onefft_columns_destroy(None)


def test_python_mirror_raises_on_invalid_size(cuda_lib):
    import onefft_b200
    with pytest.raises(ValueError):
        onefft_b200.forward(np.zeros(6, np.float32))
    with pytest.raises(ValueError):
        onefft_b200.Plan(12)


def test_batched_width_rule_matches_autotuner(cuda_lib):
    """One-pass plans accept exactly the transforms-per-block widths the autotuner times
    (onefft_b200.autotune.batched_log_c_candidates, plus -1 for the tuned one); any other width
    is rejected as an invalid split before device work (an accepted width goes on to build the
    plan, which without a device fails with a CUDA error instead)."""
    from onefft_b200.autotune import batched_log_c_candidates
    for log2n in range(4, 15):
        ok = set(batched_log_c_candidates(log2n)) | {-1}
        for c in range(-3, 17):
            lens = (ctypes.c_int * 1)(log2n)
            cols = (ctypes.c_int * 1)(c)
            h = cuda_lib.onefft_plan_create_tiles(1 << log2n, 1, lens, cols, 0, 0)
            rejected = h is None and b"invalid pass split" in cuda_lib.onefft_last_error()
            if h:
                cuda_lib.onefft_plan_destroy(h)
            assert rejected == (c not in ok), (log2n, c)


def test_autotuner_candidates_are_valid_splits(cuda_lib):
    """Every multi-pass shape the autotuner times (onefft_b200.autotune.candidates) passes the
    library's split validation; a shape the library rejects would be timed as an error."""
    from onefft_b200.autotune import candidates
    for m in (15, 20, 24, 27, 30):
        for lens, cols, chunk in candidates(m):
            k = len(lens)
            h = cuda_lib.onefft_plan_create_tiles(1 << m, k, (ctypes.c_int * k)(*lens), (ctypes.c_int * k)(*cols),
                                                  3, chunk)
            if h:
                cuda_lib.onefft_plan_destroy(h)
            else:
                assert b"invalid pass split" not in cuda_lib.onefft_last_error(), (m, lens, cols, chunk)


def test_fused_candidates_are_valid_shapes(cuda_lib):
    """Every fused shape the autotuner times (onefft_b200.autotune.fused_candidates: the first two
    passes as one persistent kernel) passes the library's validation."""
    from onefft_b200.autotune import fused_candidates
    for m in (22, 24, 27, 30):
        for lens, cols, chunk, lag in fused_candidates(m):
            opts = 2 | 4 | (lag << 8)  # ONEFFT_OPT_TMA | ONEFFT_OPT_FUSED | ONEFFT_OPT_LAG(lag)
            h = cuda_lib.onefft_plan_create_tiles(1 << m, 3, (ctypes.c_int * 3)(*lens), (ctypes.c_int * 3)(*cols),
                                                  opts, chunk)
            if h:
                cuda_lib.onefft_plan_destroy(h)
            else:
                assert b"invalid pass split" not in cuda_lib.onefft_last_error(), (m, lens, cols, chunk, lag)
