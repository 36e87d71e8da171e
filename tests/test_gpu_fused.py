"""GPU tests of the fused first two passes (k_pass01_fused, ONEFFT_OPT_FUSED) through the C ABI.

A three-pass transform n = A B C can run its passes 0 and 1 as one persistent kernel that takes
tiles chunk by chunk (a pass-1 tile waits, bounded, until every pass-0 tile of its chunk has
published). The tile arithmetic is the separate passes', so:
  - results equal the same split run as separate TMA-staged passes bit for bit, for every
    compiled tile pair, several chunk sizes and lags, both directions, a batch of two, and lie
    within the reference bound of the FP64 oracle;
  - concurrent use is safe: four host threads sharing one plan, and one thread enqueueing on more
    streams than the plan has counter slots without synchronising, all give the same bits;
  - inside a stream capture the plan falls back to separate launches (same bits on replay);
  - an expired wait is reported (onefft_plan_status) and the plan recovers.
"""
from __future__ import annotations

import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def torch():
    import torch as t
    return t


def plan_fused(ofb, n, split, cols, chunk, lag=1, l2_keep=False):
    return ofb.Plan(n, split=split, cols=cols, chunk=chunk, tma=True, fuse_lag=lag, l2_keep=l2_keep)


# (split, tile widths, chunk bits, lag): one or more per compiled tile pair
CASES = [
    ((8, 7, 5), (3, 4, 4), 3, 1),
    ((8, 7, 5), (3, 4, 4), 4, 2),
    ((8, 8, 6), (3, 3, 3), 3, 1),
    ((8, 8, 6), (4, 4, 4), 4, 3),
    ((8, 9, 5), (4, 3, 3), 4, 1),
    ((8, 9, 6), (4, 3, 3), 5, 1),
    ((9, 9, 4), (3, 3, 4), 3, 1),
    ((10, 10, 4), (3, 3, 4), 3, 1),
    ((10, 11, 4), (3, 2, 4), 3, 1),
]


@pytest.mark.parametrize("split,cols,chunk,lag", CASES)
def test_fused_equals_separate_passes(ofb, oracle, split, cols, chunk, lag):
    T = torch()
    m = sum(split)
    n = 1 << m
    batch = 2
    g = T.Generator(device="cuda").manual_seed(m * 16 + chunk)
    x = T.randn(2 * n * batch, device="cuda", generator=g)
    fused = plan_fused(ofb, n, split, cols, chunk, lag, l2_keep=(lag == 2))
    plain = ofb.Plan(n, split=split, cols=cols, tma=True)
    a, b = T.empty_like(x), T.empty_like(x)
    for inv in (False, True):
        (fused.dev_inverse if inv else fused.dev_forward)(x.data_ptr(), a.data_ptr(), batch)
        (plain.dev_inverse if inv else plain.dev_forward)(x.data_ptr(), b.data_ptr(), batch)
        T.cuda.synchronize()
        assert fused.status() == 0 and plain.status() == 0
        assert T.equal(a, b), (split, cols, chunk, lag, inv)
        xs = x[:2 * n].cpu().numpy()
        err = oracle.rel_rms(a[:2 * n].cpu().numpy(), oracle.fft64_numpy(xs, inv))
        assert err < oracle.tolerance(m), err
    # a second run on the same plan (counters were reset by the first) gives the same bits
    fused.dev_forward(x.data_ptr(), a.data_ptr(), batch)
    plain.dev_forward(x.data_ptr(), b.data_ptr(), batch)
    T.cuda.synchronize()
    assert T.equal(a, b)
    fused.destroy()
    plain.destroy()


def test_fused_concurrent_threads_and_streams(ofb):
    T = torch()
    split, cols, chunk = (8, 8, 6), (3, 3, 3), 3
    n = 1 << sum(split)
    x = T.randn(2 * n, device="cuda", generator=T.Generator(device="cuda").manual_seed(7))
    plan = plan_fused(ofb, n, split, cols, chunk)
    want = T.empty_like(x)
    plan.dev_forward(x.data_ptr(), want.data_ptr(), 1)
    T.cuda.synchronize()
    # one thread, more streams than the plan's four counter slots, no synchronisation between
    streams = [T.cuda.Stream() for _ in range(7)]
    outs = [T.empty_like(x) for _ in streams]
    T.cuda.synchronize()
    for rep in range(3):
        for s, o in zip(streams, outs):
            plan.dev_forward(x.data_ptr(), o.data_ptr(), 1, s.cuda_stream)
    T.cuda.synchronize()
    assert plan.status() == 0
    for o in outs:
        assert T.equal(o, want)
    # four host threads sharing the plan through the host-pointer path
    xh = x.cpu().numpy()
    wh = want.cpu().numpy()
    errors = []

    def worker():
        try:
            for _ in range(5):
                y = plan.forward(xh)
                if not np.array_equal(y, wh):
                    errors.append("differs")
        except Exception as e:  # reported below
            errors.append(repr(e))

    threads = [threading.Thread(target=worker) for _ in range(4)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    plan.destroy()


def test_fused_under_stream_capture(ofb):
    T = torch()
    split, cols, chunk = (8, 9, 5), (4, 3, 3), 4
    n = 1 << sum(split)
    x = T.randn(2 * n, device="cuda", generator=T.Generator(device="cuda").manual_seed(9))
    plan = plan_fused(ofb, n, split, cols, chunk)
    want = T.empty_like(x)
    plan.dev_forward(x.data_ptr(), want.data_ptr(), 1)
    T.cuda.synchronize()
    got = T.zeros_like(x)
    s = T.cuda.Stream()
    graph = T.cuda.CUDAGraph()
    with T.cuda.stream(s):
        with T.cuda.graph(graph, stream=s):
            plan.dev_forward(x.data_ptr(), got.data_ptr(), 1, s.cuda_stream)
    graph.replay()
    T.cuda.synchronize()
    assert T.equal(got, want)
    del graph
    plan.destroy()


def test_fused_expired_wait_reported(ofb):
    T = torch()
    L = ofb.lib()
    split, cols, chunk = (8, 7, 5), (3, 4, 4), 3
    n = 1 << sum(split)
    x = T.randn(2 * n, device="cuda", generator=T.Generator(device="cuda").manual_seed(11))
    plan = plan_fused(ofb, n, split, cols, chunk)
    want = T.empty_like(x)
    plan.dev_forward(x.data_ptr(), want.data_ptr(), 1)
    T.cuda.synchronize()
    got = T.empty_like(x)
    assert L.onefft_debug_expire_waits(1) == 0
    try:
        plan.dev_forward(x.data_ptr(), got.data_ptr(), 1)
        T.cuda.synchronize()
    finally:
        assert L.onefft_debug_expire_waits(0) == 0
    assert plan.status() == -1000
    # the counters were left zeroed: the next runs on every slot are correct
    for _ in range(5):
        plan.dev_forward(x.data_ptr(), got.data_ptr(), 1)
        T.cuda.synchronize()
        assert plan.status() == 0
        assert T.equal(got, want)
    plan.destroy()
