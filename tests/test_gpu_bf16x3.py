"""GPU tests of the split-BF16 tensor-core variants (configuration: 256 transforms of n = 2^16 and
16 of n = 2^22, standard-normal values with 1 % of the entries scaled by 1e3).

The variants compute the radix-16 stages as BF16 split matrix products with FP32 accumulation:
hi/lo parts with three product terms (onefft_plan_create_bf16x3), or hi/mid/lo parts with six
(onefft_plan_create_bf16x6). Each must compute the DFT (error far below O(1): a wrong fragment
layout would show as O(1) error) and its error against FP64 is measured beside the FP32 path's;
the library accepts a variant only at sizes where it meets the FP32 path's bound (relative RMS at
most 2x OneFFT's), and a plan that requires acceptance is refused elsewhere.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def torch():
    import torch as t
    return t


def errors(oracle, got, x, n, rows):
    rel, mx = [], 0.0
    for r in rows:
        xi = x[2 * n * r:2 * n * (r + 1)]
        want = oracle.fft64_numpy(xi)
        g = got[2 * n * r:2 * n * (r + 1)]
        rel.append(oracle.rel_rms(g, want))
        mx = max(mx, oracle.max_abs(g, want))
    return max(rel), mx


VARIANTS = {3: {"bf16x3": True}, 6: {"bf16x6": True}}


@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("log2n,batch,rows", [(16, 256, range(0, 256, 37)), (22, 16, (0, 9))])
def test_bf16_split_vs_fp32_error(ofb, oracle, log2n, batch, rows, terms):
    T = torch()
    n = 1 << log2n
    x = np.concatenate([oracle.gen_wide(n, 0xC0F4 + log2n, b * n) for b in range(batch)])
    d_in = T.from_numpy(x).cuda()
    out_tc, out_32 = T.empty_like(d_in), T.empty_like(d_in)
    tc = ofb.Plan(n, **VARIANTS[terms])
    fp = ofb.Plan(n)
    tc.dev_forward(d_in.data_ptr(), out_tc.data_ptr(), batch)
    fp.dev_forward(d_in.data_ptr(), out_32.data_ptr(), batch)
    T.cuda.synchronize()
    e_tc, m_tc = errors(oracle, out_tc.cpu().numpy(), x, n, rows)
    e_32, m_32 = errors(oracle, out_32.cpu().numpy(), x, n, rows)
    ref = max(oracle.rel_rms(oracle.ref_fft(x[2 * n * r:2 * n * (r + 1)]),
                             oracle.fft64_numpy(x[2 * n * r:2 * n * (r + 1)])) for r in rows) \
        if oracle.have_reference() else e_32
    print(f"n=2^{log2n} x {batch}: split-BF16 {terms} terms rel RMS {e_tc:.3g} max-abs {m_tc:.3g}; "
          f"FP32 {e_32:.3g} / {m_32:.3g}; reference {ref:.3g}; bound 2x reference -> "
          f"{'meets it' if e_tc <= 2 * ref else 'misses it'}")
    assert e_32 <= 2 * ref
    assert e_tc < 1e-4  # the tensor-core stages compute the DFT, to BF16-split accuracy
    # acceptance follows the measurement: a size the library accepts meets the bound here, and a
    # size that misses it is refused when acceptance is required
    try:
        ofb.Plan(n, require_accepted=True, **VARIANTS[terms]).destroy()
        accepted = True
    except ValueError:
        accepted = False
    if accepted:
        assert e_tc <= 2 * ref, (terms, log2n, e_tc, ref)
    if e_tc > 2 * ref:
        assert not accepted
    if terms == 6:  # the configuration sizes meet the bound with six terms
        assert accepted
    tc.destroy()
    fp.destroy()


@pytest.mark.parametrize("terms", [3, 6])
@pytest.mark.parametrize("log2n", [4, 5, 8, 12, 13, 14, 15, 18])
def test_bf16_split_all_engines(ofb, oracle, log2n, terms):
    """Every tensor-core kernel shape (one-kernel sizes, two and three passes, inverse) computes
    the transform."""
    T = torch()
    n = 1 << log2n
    batch = max(1, (1 << 16) // n)
    x = oracle.gen_normal(2 * n * batch, 40 + log2n)
    d_in = T.from_numpy(x).cuda()
    out = T.empty_like(d_in)
    p = ofb.Plan(n, **VARIANTS[terms])
    for inv in (False, True):
        (p.dev_inverse if inv else p.dev_forward)(d_in.data_ptr(), out.data_ptr(), batch)
        T.cuda.synchronize()
        g = out.cpu().numpy()
        for r in (0, batch - 1):
            xi = x[2 * n * r:2 * n * (r + 1)]
            err = oracle.rel_rms(g[2 * n * r:2 * n * (r + 1)], oracle.fft64_numpy(xi, inv))
            assert err < 1e-4, (log2n, inv, r, err)
    p.destroy()
