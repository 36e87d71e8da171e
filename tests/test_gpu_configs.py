"""GPU parity at the full sizes of the benchmark configurations, through the C ABI.

  n=1024 single forward+inverse, uniform [-1,1): inverse(forward(x)) = 1024 x and the forward
      result against an FP64 direct DFT of every bin;
  16384 x n=4096 batched, standard normal: 64 sampled transforms against FP64 (each within 2x
      the reference library's error on the same transform), and the whole batch through
      size-independent properties (Parseval per transform, linearity);
  single n = 2^20, 2^22, 2^24 .. 2^27, forward and inverse, against the full FP64 FFT (numpy,
      complex128) within 2x the reference's error on the same input (tests/golden/ref_errors.json);
      at 2^27 also the round trip, Parseval and two direct-DFT bins.
The parity rule: relative RMS against the FP64 oracle at most 2x the reference's on the same
input (FP32 arithmetic, so this is the tolerance; no bitwise claim), max-abs stated.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED_C1 = 0xC0F1
SEED_C2 = 0xC0F2


def torch():
    import torch as t
    return t


def test_config1_n1024(ofb, oracle):
    n = 1024
    x, _ = oracle.gen_uniform(2 * n, SEED_C1)
    plan = ofb.Plan(n)
    y = plan.forward(x)
    back = plan.inverse(y)
    assert oracle.rel_rms(back, x.astype(np.float64) * n) < 2 * oracle.tolerance(10)
    want = oracle.dft_bins(x, np.arange(n))
    err = oracle.rel_rms(y, want)
    ref = oracle.rel_rms(oracle.ref_fft(x), want) if oracle.have_reference() else None
    print(f"config1 n=1024 rel_rms {err:.3g} (reference {ref}) max_abs {oracle.max_abs(y, want):.3g}")
    assert err < oracle.tolerance(10)
    if ref is not None:
        assert err <= 2 * ref
    plan.destroy()


def test_config2_batched_4096(ofb, oracle):
    T = torch()
    n, batch = 4096, 16384
    x = oracle.gen_normal(2 * n * batch, SEED_C2)
    plan = ofb.Plan(n)
    d_in = T.from_numpy(x).cuda()
    d_out = T.empty_like(d_in)
    rng = np.random.default_rng(5)
    sample = np.sort(rng.choice(batch, 64, replace=False))
    for inv in (False, True):
        (plan.dev_inverse if inv else plan.dev_forward)(d_in.data_ptr(), d_out.data_ptr(), batch)
        T.cuda.synchronize()
        out = d_out.view(batch, n, 2)
        worst = worst_ratio = 0.0
        for b in sample:
            xb = x[2 * n * b:2 * n * (b + 1)]
            want = oracle.fft64(xb, inv)
            got = out[b].cpu().numpy().reshape(-1)
            err = oracle.rel_rms(got, want)
            assert err < oracle.tolerance(12)
            if oracle.have_reference():
                ref = oracle.rel_rms(oracle.ref_fft(xb, inv), want)
                worst_ratio = max(worst_ratio, err / ref)
            worst = max(worst, oracle.max_abs(got, want))
        print(f"config2 4096x16384 {'inv' if inv else 'fwd'}: worst err/ref {worst_ratio:.3f} max_abs {worst:.3g}")
        assert worst_ratio <= 2.0
        # Parseval on every transform: sum |X|^2 = n sum |x|^2
        xin = d_in.view(batch, n, 2).double()
        e_in = (xin ** 2).sum(dim=(1, 2))
        e_out = (out.double() ** 2).sum(dim=(1, 2))
        rel = ((e_out - n * e_in).abs() / (n * e_in)).max().item()
        assert rel < 1e-5
    # linearity over the whole batch: F(a x + y) = a F(x) + F(y)
    y_in = T.roll(d_in, shifts=2 * n)  # another valid batch
    fa = T.empty_like(d_in)
    fb = T.empty_like(d_in)
    fab = T.empty_like(d_in)
    plan.dev_forward(d_in.data_ptr(), fa.data_ptr(), batch)
    plan.dev_forward(y_in.data_ptr(), fb.data_ptr(), batch)
    comb = (2.0 * d_in + y_in).contiguous()
    plan.dev_forward(comb.data_ptr(), fab.data_ptr(), batch)
    T.cuda.synchronize()
    num = (fab.double() - (2.0 * fa.double() + fb.double())).norm()
    den = fab.double().norm()
    assert (num / den).item() < 1e-6
    plan.destroy()


@pytest.mark.parametrize("log2n", [20, 22, 24, 25, 26])
def test_config2_single_large(ofb, oracle, ref_errors, log2n):
    T = torch()
    n = 1 << log2n
    x = oracle.gen_normal(2 * n, ref_errors["seed_normal"] + log2n)
    plan = ofb.Plan(n)
    d_in = T.from_numpy(x).cuda()
    d_out = T.empty_like(d_in)
    for inv in (False, True):
        d = "inverse" if inv else "forward"
        (plan.dev_inverse if inv else plan.dev_forward)(d_in.data_ptr(), d_out.data_ptr(), 1)
        T.cuda.synchronize()
        got = d_out.cpu().numpy()
        want = oracle.fft64_numpy(x, inv)
        err = oracle.rel_rms(got, want)
        ref = ref_errors["normal"][str(log2n)][d]["rel_rms"]
        print(f"config2 n=2^{log2n} {d}: rel_rms {err:.3g} reference {ref:.3g} max_abs {oracle.max_abs(got, want):.3g}")
        assert err <= 2 * ref
        assert err < oracle.tolerance(log2n)
    plan.destroy()


def test_config2_single_2p27(ofb, oracle, ref_errors):
    """The largest benchmark item (1 GiB per buffer) under the parity rule in both directions:
    relative RMS against numpy's FP64 FFT of the same input at most 2x the reference library's
    (tests/golden/ref_errors.json, the reference run on this input), max-abs stated; plus the
    round trip, Parseval and two FP64 direct-DFT bins."""
    T = torch()
    log2n = 27
    n = 1 << log2n
    x = oracle.gen_normal(2 * n, ref_errors["seed_normal"] + log2n)
    plan = ofb.Plan(n)
    assert len(plan.passes()) == 3 and sum(plan.passes()) == 27
    d_in = T.from_numpy(x).cuda()
    d_out = T.empty_like(d_in)
    d_back = T.empty_like(d_in)
    plan.dev_forward(d_in.data_ptr(), d_out.data_ptr(), 1)
    plan.dev_inverse(d_out.data_ptr(), d_back.data_ptr(), 1)
    T.cuda.synchronize()
    assert plan.status() == 0
    # round trip and Parseval on the device, in FP64
    xin = d_in.double()
    rt = ((d_back.double() - n * xin).norm() / (n * xin.norm())).item()
    assert rt < 2 * oracle.tolerance(log2n)
    pars = abs((d_out.double() ** 2).sum().item() - n * (xin ** 2).sum().item()) / (n * (xin ** 2).sum().item())
    assert pars < 1e-5
    del xin, d_back
    fwd = d_out.cpu().numpy()
    bins = [1, n // 3]
    want_bins = oracle.dft_bins(x, bins)
    sel = fwd.reshape(-1, 2)[bins].reshape(-1)
    assert np.abs(sel - want_bins).max() / np.abs(want_bins).max() < 2e-6
    for inv in (False, True):
        d = "inverse" if inv else "forward"
        if inv:
            plan.dev_inverse(d_in.data_ptr(), d_out.data_ptr(), 1)
            T.cuda.synchronize()
            got = d_out.cpu().numpy()
        else:
            got = fwd
        want = oracle.fft64_numpy(x, inv)
        err = oracle.rel_rms(got, want)
        ref = ref_errors["normal"][str(log2n)][d]["rel_rms"]
        print(f"config2 n=2^27 {d}: rel_rms {err:.3g} reference {ref:.3g} max_abs {oracle.max_abs(got, want):.3g} "
              f"(reference {ref_errors['normal'][str(log2n)][d]['max_abs']:.3g})")
        assert err <= 2 * ref
        assert err < oracle.tolerance(log2n)
        del want, got
    plan.destroy()


@pytest.mark.parametrize("log2n", [28, 29, 30])
def test_max_sizes_round_trip(ofb, oracle, log2n):
    """The largest sizes OneFFT accepts (2^28 .. 2^30; 2^30 complex values = 8 GiB per buffer),
    through size-independent properties computed on the device in FP64: the round trip
    inverse(forward(x)) = n x, Parseval (sum |X|^2 = n sum |x|^2) and linearity
    F(x + 2 x') = F(x) + 2 F(x') with x' a shifted copy; at 2^28 also two bins against the FP64
    direct DFT."""
    T = torch()
    n = 1 << log2n
    g = T.Generator(device="cuda").manual_seed(log2n)
    plan = ofb.Plan(n)
    x = T.randn(2 * n, device="cuda", generator=g)
    y = T.empty_like(x)
    z = T.empty_like(x)
    plan.dev_forward(x.data_ptr(), y.data_ptr(), 1)
    plan.dev_inverse(y.data_ptr(), z.data_ptr(), 1)
    T.cuda.synchronize()

    def sumsq(t):  # FP64 sum of squares, in chunks to bound the temporary
        return sum(float((c.double() ** 2).sum()) for c in t.split(1 << 28))

    def diffsq(a, b, scale):
        return sum(float(((ca.double() - scale * cb.double()) ** 2).sum()) for ca, cb in zip(a.split(1 << 28), b.split(1 << 28)))

    ex, ey = sumsq(x), sumsq(y)
    assert abs(ey - n * ex) / (n * ex) < 1e-5
    rt = (diffsq(z, x, float(n)) / (n * n * ex)) ** 0.5
    assert rt < 2 * oracle.tolerance(log2n), rt
    # linearity with a second input: x shifted by 12345 values
    x2 = T.roll(x, 2 * 12345)
    comb = x + 2 * x2
    del z
    y2 = T.empty_like(x)
    yc = T.empty_like(x)
    plan.dev_forward(x2.data_ptr(), y2.data_ptr(), 1)
    plan.dev_forward(comb.data_ptr(), yc.data_ptr(), 1)
    T.cuda.synchronize()
    lin = sum(float(((cc.double() - ca.double() - 2 * cb.double()) ** 2).sum())
              for ca, cb, cc in zip(y.split(1 << 28), y2.split(1 << 28), yc.split(1 << 28)))
    assert (lin / sumsq(yc)) ** 0.5 < 1e-5
    if log2n == 28:
        xs = x.cpu().numpy()
        bins = [1, n // 3]
        want = oracle.dft_bins(xs, bins)
        got = y.view(-1, 2)[bins].cpu().numpy().reshape(-1)
        assert np.abs(got - want).max() / np.abs(want).max() < 2e-6
    print(f"n=2^{log2n}: passes {plan.passes()}, round trip {rt:.3g}")
    plan.destroy()
