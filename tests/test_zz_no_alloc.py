"""GPU test of onefft_uneven_execute_noalloc through the C ABI.

This entry point exists for callers that cannot let a library allocate device memory: real-time
threads that must never block in the allocator or meet an out-of-memory error once running, and
applications that give all device memory to their own arena or budget. It runs the same
persistent kernel as onefft_uneven_execute, with its twiddle tables, descriptors and work queue
in one fixed device array instead of a batch object's allocation.

The test checks two calls in a row, each with a different descriptor list, against the existing
entry point (onefft_uneven_create + onefft_uneven_execute) on the same inputs. Both run the same
kernel (the tuned in-block splits) with tables built by the same kernels, so every transform
must equal the existing result bit for bit (and so lie within the reference's error bound of
it); the second call also shows that the array left behind by the first does not leak into it.
It also checks the stated limit. The file is named to be collected last, and it needs nothing
from the other test files.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAX_COUNT = 4096


def torch():
    import torch as t
    return t


def make_batch(oracle, ofb, count, seed, lo, hi):
    rng = np.random.default_rng(seed)
    desc = np.empty(count, ofb.DESC_DTYPE)
    desc["log2n"] = rng.integers(lo, hi + 1, count)
    desc["inverse"] = rng.random(count) < 0.5
    sizes = (1 << desc["log2n"].astype(np.int64)) + (seed % 3)  # some gaps between transforms
    desc["offset"] = np.concatenate([[seed % 5], seed % 5 + np.cumsum(sizes)[:-1]])
    order = rng.permutation(count)  # descriptors in no particular order
    desc = np.ascontiguousarray(desc[order])
    span = int((desc["offset"] + (1 << desc["log2n"].astype(np.int64))).max())
    x, _ = oracle.gen_uniform(2 * span, seed)
    return desc, x


def test_noalloc_matches_existing_entry_point_on_two_calls(ofb, oracle):
    T = torch()
    L = ofb.lib()
    stream = T.cuda.current_stream().cuda_stream
    for count, seed, lo, hi in ((3000, 7, 0, 16), (1200, 8, 3, 16)):
        desc, x = make_batch(oracle, ofb, count, seed, lo, hi)
        d_in = T.from_numpy(x).cuda()
        want = T.zeros_like(d_in)
        existing = ofb.UnevenBatch(desc)
        existing.execute(d_in.data_ptr(), want.data_ptr(), stream)
        got = T.full_like(d_in, float("nan"))
        rc = L.onefft_uneven_execute_noalloc(desc.ctypes.data, count, d_in.data_ptr(), got.data_ptr(), stream)
        assert rc == 0, ofb.last_error()
        T.cuda.synchronize()
        existing.destroy()
        g, w = got.cpu().numpy(), want.cpu().numpy()
        for m, off in zip(desc["log2n"].tolist(), desc["offset"].tolist()):
            n = 1 << m
            a, b = g[2 * off:2 * (off + n)], w[2 * off:2 * (off + n)]
            assert oracle.rel_rms(a, b.astype(np.float64)) <= oracle.tolerance(m), (seed, m, off)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (seed, m, off)
        print(f"no-alloc call with {count} transforms: all identical to the existing entry point")


def test_noalloc_rejects_more_than_the_limit(ofb):
    T = torch()
    L = ofb.lib()
    desc = np.zeros(MAX_COUNT + 1, ofb.DESC_DTYPE)
    desc["log2n"] = 4
    desc["offset"] = np.arange(MAX_COUNT + 1) * 16
    buf = T.zeros(2 * 16 * (MAX_COUNT + 1) * 2, device="cuda")
    half = buf.numel() // 2
    rc = L.onefft_uneven_execute_noalloc(desc.ctypes.data, desc.size, buf.data_ptr(), buf.data_ptr() + 4 * half, None)
    assert rc == -2
    assert "4096" in ofb.last_error()
