"""GPU tests of the weighted entry points: out_b = post * T(pre * in_b) with the weights applied
inside the kernels that read the input and write the output (onefft_dev_forward_weighted /
onefft_dev_inverse_weighted).

Each case is checked against the unweighted transform of the same plan with the products done
separately in torch (complex64): the only differences are the rounding of those products (FP32
products computed in a different order), so the relative RMS difference stays near FP32's
precision (bound 2e-6). Every kernel family that applies weights is covered: one thread per
transform (n <= 8), one kernel (16 .. 2^14), first and last passes through bulk tensor copies,
the plain pass kernels (8-byte aligned buffers), three passes with a middle pass (which applies
neither), and chunked first passes.
"""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu

TOL = 2e-6


def torch():
    import torch as t
    return t


def rel_rms(T, a, b):
    return ((a.double() - b.double()).norm() / b.double().norm()).item()


CASES = [  # (log2 n, plan options)
    (0, {}), (2, {}), (3, {}), (4, {}), (10, {}), (12, {}), (14, {}),
    (15, {}), (18, {}), (20, {}), (22, {}),
    (18, {"split": (6, 6, 6), "cols": (3, 3, 3), "tma": True}),
    (18, {"split": (6, 6, 6), "cols": (3, 3, 3), "chunk": 3}),
    (16, {"split": (8, 8), "cols": (3, 3)}),
]


@pytest.mark.parametrize("log2n,opts", CASES)
@pytest.mark.parametrize("aligned", [True, False])
def test_weighted_matches_separate_products(ofb, log2n, opts, aligned):
    T = torch()
    n = 1 << log2n
    batch = 3
    g = T.Generator(device="cuda").manual_seed(100 + log2n)
    plan = ofb.Plan(n, **opts)
    off = 0 if aligned else 2  # two floats = 8 bytes: the plain (non bulk-copy) kernels
    buf = T.randn(2 * n * batch + 2, device="cuda", generator=g)
    x = buf[off:off + 2 * n * batch]
    pre = T.randn(2 * n, device="cuda", generator=g)
    post = T.randn(2 * n, device="cuda", generator=g)
    xc = T.view_as_complex(x.view(batch, n, 2))
    pc = T.view_as_complex(pre.view(n, 2))
    qc = T.view_as_complex(post.view(n, 2))
    out_buf = T.empty(2 * n * batch + 2, device="cuda")
    out = out_buf[off:off + 2 * n * batch]
    for inverse in (False, True):
        for use_pre, use_post in ((True, False), (False, True), (True, True)):
            # separate: pre-multiply in torch, plain transform, post-multiply in torch
            src = (xc * pc) if use_pre else xc
            src = T.view_as_real(src.contiguous()).reshape(-1).contiguous()
            ref = T.empty_like(src)
            (plan.dev_inverse if inverse else plan.dev_forward)(src.data_ptr(), ref.data_ptr(), batch)
            refc = T.view_as_complex(ref.view(batch, n, 2))
            if use_post:
                refc = refc * qc
            want = T.view_as_real(refc).reshape(-1)
            out.fill_(float("nan"))
            plan.dev_weighted(x.data_ptr(), out.data_ptr(), batch, pre.data_ptr() if use_pre else None,
                              post.data_ptr() if use_post else None, inverse=inverse)
            T.cuda.synchronize()
            for b in range(batch):
                s = slice(2 * n * b, 2 * n * (b + 1))
                err = rel_rms(T, out[s], want[s])
                assert err < TOL, (log2n, opts, aligned, inverse, use_pre, use_post, b, err)
    plan.destroy()


def test_weighted_without_weights_equals_plain(ofb):
    """Both weights NULL: bit for bit the plain entry point."""
    T = torch()
    for log2n in (5, 12, 20):
        n = 1 << log2n
        plan = ofb.Plan(n)
        x = T.randn(4 * n, device="cuda")
        a, b = T.empty_like(x), T.empty_like(x)
        plan.dev_weighted(x.data_ptr(), a.data_ptr(), 2)
        plan.dev_forward(x.data_ptr(), b.data_ptr(), 2)
        T.cuda.synchronize()
        assert T.equal(a, b)
        plan.destroy()


def test_weighted_rejects_bad_weights(ofb):
    T = torch()
    L = ofb.lib()
    n = 1 << 10
    plan = ofb.Plan(n)
    x = T.randn(2 * n, device="cuda")
    out = T.empty(4 * n, device="cuda")
    w = T.randn(2 * n + 1, device="cuda")
    # weights inside the output, misaligned weights
    assert L.onefft_dev_forward_weighted(plan.handle, x.data_ptr(), out.data_ptr(), 1, out.data_ptr() + 8,
                                         None, None) == -2
    assert L.onefft_dev_forward_weighted(plan.handle, x.data_ptr(), out.data_ptr(), 1, None,
                                         w.data_ptr() + 4, None) == -2
    plan.destroy()
    tc = ofb.Plan(n, bf16x3=True)
    assert L.onefft_dev_forward_weighted(tc.handle, x.data_ptr(), out.data_ptr(), 1, w.data_ptr(), None,
                                         None) == -2
    tc.destroy()
