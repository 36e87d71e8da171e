"""GPU tests of the uneven batch (one persistent launch over many sizes) through the C ABI.

The reference has no batch API: its callers loop over onefft_plan_forward/_inverse per transform
(OneFFT include/onefft.h:102-106). The uneven batch must therefore give the per-transform plain
path's results: bit for bit for every size whose split is the same, and within the reference's
error bound for 2^13 and 2^14 (one kernel on the plain path, two in-block passes here).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def torch():
    import torch as t
    return t


def make_batch(oracle, count, seed, lo=4, hi=16, gap=0):
    rng = np.random.default_rng(seed)
    log2n = rng.integers(lo, hi + 1, count).astype(np.int32)
    inverse = (rng.random(count) < 0.5).astype(np.int32)
    sizes = (1 << log2n.astype(np.int64)) + gap
    offset = np.concatenate([[0], np.cumsum(sizes)[:-1]]).astype(np.int64)
    span = int(offset[-1] + (1 << int(log2n[-1])))
    x, _ = oracle.gen_uniform(2 * span, seed & 0xFFFFFFFF or 1)
    return log2n, inverse, offset, span, x


def plain_path(ofb, T, log2n, inverse, offset, d_in):
    """Each transform through onefft_dev_*_batched with batch 1 (the plain per-transform path)."""
    out = T.zeros_like(d_in)
    plans = {}
    base_in, base_out = d_in.data_ptr(), out.data_ptr()
    for m, inv, off in zip(log2n.tolist(), inverse.tolist(), offset.tolist()):
        p = plans.get(m) or plans.setdefault(m, ofb.Plan(1 << m))
        (p.dev_inverse if inv else p.dev_forward)(base_in + 8 * off, base_out + 8 * off, 1)
    T.cuda.synchronize()
    for p in plans.values():
        p.destroy()
    return out


def compare(oracle, log2n, offset, got, want, tol_sizes=(13, 14)):
    g = got.cpu().numpy()
    w = want.cpu().numpy()
    worst = 0.0
    for m, off in zip(log2n.tolist(), offset.tolist()):
        n = 1 << m
        a = g[2 * off:2 * (off + n)]
        b = w[2 * off:2 * (off + n)]
        if m in tol_sizes:
            d = oracle.rel_rms(a, b.astype(np.float64))
            worst = max(worst, d)
            assert d < 2 * oracle.tolerance(m), (m, off, d)
        else:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (m, off)
    return worst


def test_uneven_config3_full(ofb, oracle):
    """20000 transforms, log2 n uniform in 4..16, packed back to back, half inverse."""
    T = torch()
    log2n, inverse, offset, span, x = make_batch(oracle, 20000, 0xC0F3)
    batch = ofb.UnevenBatch(log2n, inverse, offset)
    assert batch.span == span
    d_in = T.from_numpy(x).cuda()
    d_out = T.full_like(d_in, float("nan"))
    batch.execute(d_in.data_ptr(), d_out.data_ptr())
    T.cuda.synchronize()
    assert batch.status() == 0
    want = plain_path(ofb, T, log2n, inverse, offset, d_in)
    worst = compare(oracle, log2n, offset, d_out, want)
    print(f"uneven 20000: bitwise equal to the plain path except 2^13/2^14 (worst rel diff {worst:.3g})")
    # sampled transforms against FP64 and the reference library
    rng = np.random.default_rng(3)
    g = d_out.cpu().numpy()
    for i in rng.choice(len(log2n), 24, replace=False):
        m, off, inv = int(log2n[i]), int(offset[i]), bool(inverse[i])
        n = 1 << m
        xi = x[2 * off:2 * (off + n)]
        want64 = oracle.fft64(xi, inv) if n <= 4096 else oracle.fft64_numpy(xi, inv)
        err = oracle.rel_rms(g[2 * off:2 * (off + n)], want64)
        assert err < oracle.tolerance(m)
        if oracle.have_reference():
            assert err <= 2 * oracle.rel_rms(oracle.ref_fft(xi, inv), want64)
    # replay with other buffers: the graph's pointers are patched, the counter re-zeroed
    d_out2 = T.zeros_like(d_in)
    batch.execute(d_in.data_ptr(), d_out2.data_ptr())
    batch.execute(d_in.data_ptr(), d_out2.data_ptr())
    T.cuda.synchronize()
    assert batch.status() == 0
    assert T.equal(d_out2, d_out)
    batch.destroy()


def test_uneven_all_sizes_and_gaps(ofb, oracle):
    """Every size 2^0 .. 2^16, several of each (partial groups), with gaps between transforms
    that must stay untouched."""
    T = torch()
    rng = np.random.default_rng(11)
    log2n = np.repeat(np.arange(0, 17), [700, 300, 129, 65, 33, 17, 9, 5, 3, 3, 2, 2, 2, 3, 2, 2, 2]).astype(np.int32)
    rng.shuffle(log2n)
    inverse = (rng.random(log2n.size) < 0.5).astype(np.int32)
    sizes = (1 << log2n.astype(np.int64)) + 3
    offset = np.concatenate([[5], 5 + np.cumsum(sizes)[:-1]]).astype(np.int64)
    span = int(offset[-1] + (1 << int(log2n[-1])) + 7)
    x, _ = oracle.gen_uniform(2 * span, 99)
    batch = ofb.UnevenBatch(log2n, inverse, offset)
    d_in = T.from_numpy(x).cuda()
    sentinel = 12345.0
    d_out = T.full_like(d_in, sentinel)
    batch.execute(d_in.data_ptr(), d_out.data_ptr())
    T.cuda.synchronize()
    assert batch.status() == 0
    want = plain_path(ofb, T, log2n, inverse, offset, d_in)
    compare(oracle, log2n, offset, d_out, want)
    covered = np.zeros(span, bool)
    for m, off in zip(log2n.tolist(), offset.tolist()):
        covered[off:off + (1 << m)] = True
    g = d_out.cpu().numpy().reshape(-1, 2)
    assert (g[~covered[:g.shape[0]]] == sentinel).all(), "wrote outside the transforms"
    batch.destroy()


def test_uneven_in_block_passes_repeatable(ofb, oracle):
    """Many 2^13 .. 2^16 transforms, each run by one block as two passes of tile after tile, at
    8-byte (not 16-byte) aligned offsets: ten executions equal the first bit for bit and the
    2^15 / 2^16 results equal the plain path's. A block that reused a tile's shared memory
    before its slowest warp had read it would show up as a run that differs."""
    T = torch()
    rng = np.random.default_rng(23)
    log2n = rng.integers(13, 17, 600).astype(np.int32)
    inverse = (rng.random(log2n.size) < 0.5).astype(np.int32)
    sizes = (1 << log2n.astype(np.int64)) + 1
    offset = np.concatenate([[1], 1 + np.cumsum(sizes)[:-1]]).astype(np.int64)
    span = int(offset[-1] + (1 << int(log2n[-1])))
    x, _ = oracle.gen_uniform(2 * span, 23)
    batch = ofb.UnevenBatch(log2n, inverse, offset)
    d_in = T.from_numpy(x).cuda()
    first = T.zeros_like(d_in)
    batch.execute(d_in.data_ptr(), first.data_ptr())
    again = T.zeros_like(d_in)
    for _ in range(10):
        batch.execute(d_in.data_ptr(), again.data_ptr())
        T.cuda.synchronize()
        assert T.equal(again, first)
    big = log2n >= 15
    want = plain_path(ofb, T, log2n[big], inverse[big], offset[big], d_in)
    compare(oracle, log2n[big], offset[big], first, want)
    batch.destroy()


@pytest.mark.parametrize("choice", [0, 1, 2])
def test_uneven_split_choices(ofb, oracle, choice):
    """Every compiled in-block split of 2^13 .. 2^16 (onefft_uneven_create_split), at 8-byte
    aligned offsets: within twice the size's error bound of the plain path, within the bound of
    FP64 on sampled transforms, and two executions equal bit for bit."""
    T = torch()
    rng = np.random.default_rng(40 + choice)
    log2n = rng.integers(13, 17, 200).astype(np.int32)
    inverse = (rng.random(log2n.size) < 0.5).astype(np.int32)
    sizes = (1 << log2n.astype(np.int64)) + 1
    offset = np.concatenate([[1], 1 + np.cumsum(sizes)[:-1]]).astype(np.int64)
    span = int(offset[-1] + (1 << int(log2n[-1])))
    x, _ = oracle.gen_uniform(2 * span, 41 + choice)
    batch = ofb.UnevenBatch(log2n, inverse, offset, split={m: choice for m in range(13, 17)})
    d_in = T.from_numpy(x).cuda()
    got = T.zeros_like(d_in)
    batch.execute(d_in.data_ptr(), got.data_ptr())
    again = T.zeros_like(d_in)
    batch.execute(d_in.data_ptr(), again.data_ptr())
    T.cuda.synchronize()
    assert T.equal(again, got)
    want = plain_path(ofb, T, log2n, inverse, offset, d_in)
    compare(oracle, log2n, offset, got, want, tol_sizes=(13, 14, 15, 16))
    g = got.cpu().numpy()
    for i in rng.choice(len(log2n), 8, replace=False):
        m, off, inv = int(log2n[i]), int(offset[i]), bool(inverse[i])
        n = 1 << m
        want64 = oracle.fft64_numpy(x[2 * off:2 * (off + n)], inv)
        assert oracle.rel_rms(g[2 * off:2 * (off + n)], want64) < oracle.tolerance(m)
    batch.destroy()


def test_uneven_rejects_bad_arguments(ofb):
    T = torch()
    L = ofb.lib()
    with pytest.raises(ValueError):
        ofb.UnevenBatch([4, 4], [0, 0], [0, 8])  # overlap
    with pytest.raises(ValueError):
        ofb.UnevenBatch([17], [0], [0])
    b = ofb.UnevenBatch([4, 5], [0, 1], [0, 16])
    buf = T.zeros(2 * 64, device="cuda")
    assert L.onefft_uneven_execute(b._h, buf.data_ptr() + 4, buf.data_ptr() + 512, None) == -2
    assert L.onefft_uneven_execute(b._h, buf.data_ptr(), buf.data_ptr() + 64, None) == -2  # overlap
    b.destroy()
    for bad in (-1, 3):
        with pytest.raises(ValueError):
            ofb.UnevenBatch([14], [0], [0], split={14: bad})
