"""Shared fixtures of the onefft_b200 test suite.

Markers: ``gpu`` tests need a CUDA device (a B200) and call the product through its C ABI
(``libonefft_cuda.so`` via ctypes); everything else runs on the CPU: the oracle against the
reference's golden vectors, the host-side logic, and that the C library loads and exports every
symbol its headers declare.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); calls the CUDA library through its C ABI")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    if not os.path.exists(O.ORACLE_SO):
        O.build()
    return O


@pytest.fixture(scope="session")
def ref_errors():
    with open(os.path.join(GOLDEN, "ref_errors.json")) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def ref_small():
    with np.load(os.path.join(GOLDEN, "ref_small.npz")) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def uniform_inputs(oracle):
    """Per-size xorshift inputs in the reference test's order (tests/test_onefft.c:122)."""
    st = oracle.SEED_TESTS
    out = {}
    for l in range(21):
        x, st = oracle.gen_uniform(2 * (1 << l), st)
        out[l] = x
    return out


@pytest.fixture(scope="session")
def ofb():
    """The product's Python mirror with the CUDA library loaded; needs a GPU."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import onefft_b200
    onefft_b200.lib()
    return onefft_b200
