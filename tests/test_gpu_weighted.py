"""GPU tests of the weighted entry points: out_b = post * T(pre * in_b) with the weights applied
inside the kernels that read the input and write the output (onefft_dev_forward_weighted /
onefft_dev_inverse_weighted).

Each case is checked two ways:
  - against the FP64 oracle post * F64(pre * x) (numpy, complex128), with the parity rule: the
    relative RMS error at most 2x that of the reference library computing the same thing the way
    its callers would (pre * x in complex64, onefft_forward / onefft_inverse, * post in
    complex64), max-abs stated;
  - against the unweighted transform of the same plan with the products done separately in
    torch (complex64): the only differences are the rounding of those products (FP32 products
    computed in a different order), so the relative RMS difference stays near FP32's precision
    (bound 2e-6). Every kernel family that applies weights is covered: one thread per
transform (n <= 8), one kernel (16 .. 2^14), first and last passes through bulk tensor copies,
the plain pass kernels (8-byte aligned buffers), three passes with a middle pass (which applies
neither), and chunked first passes.
"""
from __future__ import annotations

import numpy as np
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


def _c64(a):
    return np.ascontiguousarray(a, np.float32).view(np.complex64)


@pytest.mark.parametrize("log2n,opts", CASES)
def test_weighted_against_fp64_oracle(ofb, oracle, log2n, opts):
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    T = torch()
    n = 1 << log2n
    batch = 2
    rng = np.random.default_rng(200 + log2n)
    x = rng.standard_normal(2 * n * batch).astype(np.float32)
    pre = rng.standard_normal(2 * n).astype(np.float32)
    post = rng.standard_normal(2 * n).astype(np.float32)
    plan = ofb.Plan(n, **opts)
    d_x, d_pre, d_post = (T.from_numpy(a).cuda() for a in (x, pre, post))
    d_out = T.empty_like(d_x)
    for inverse in (False, True):
        plan.dev_weighted(d_x.data_ptr(), d_out.data_ptr(), batch, d_pre.data_ptr(), d_post.data_ptr(),
                          inverse=inverse)
        T.cuda.synchronize()
        got = d_out.cpu().numpy()
        worst = worst_abs = 0.0
        for b in range(batch):
            xb = x[2 * n * b:2 * n * (b + 1)]
            # FP64 oracle: post * F64(pre * x), every product in FP64
            w = xb.astype(np.float64).view(np.complex128) * pre.astype(np.float64).view(np.complex128)
            f = np.fft.ifft(w) * n if inverse else np.fft.fft(w)
            want = np.ascontiguousarray(f * post.astype(np.float64).view(np.complex128)).view(np.float64)
            # the reference library doing the same with its callers' FP32 products
            src = np.ascontiguousarray(_c64(xb) * _c64(pre)).view(np.float32)
            ref = (_c64(oracle.ref_fft(src, inverse)) * _c64(post)).view(np.float32)
            gb = got[2 * n * b:2 * n * (b + 1)]
            err, ref_err = oracle.rel_rms(gb, want), oracle.rel_rms(ref, want)
            worst = max(worst, err / max(ref_err, 1e-30))
            worst_abs = max(worst_abs, oracle.max_abs(gb, want))
            assert err <= 2 * ref_err + 1e-12, (log2n, opts, inverse, b, err, ref_err)
        print(f"weighted n=2^{log2n} {opts} {'inv' if inverse else 'fwd'}: worst err/ref {worst:.3f} "
              f"max_abs {worst_abs:.3g}")
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
