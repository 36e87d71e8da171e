"""GPU tests of the differentiable FFT layer (torch autograd over the C ABI, adjoint kernel).

Configuration: batch 512 of n = 8192 complex64 inputs, standard normal; loss = sum |W * FFT(x)|^2
with W a seeded real weight vector uniform in [0,1). The gradient from the adjoint kernel is
checked
  * against FP64 central finite differences of the loss along 32 random complex directions
    (directional derivative = Re <grad, v> in torch's conjugate-Wirtinger convention);
  * against the gradient computed with the reference CPU library: 2 onefft_inverse(W^2 *
    onefft_forward(x)) (the unnormalised inverse is F^H);
and the adjoint identity <F x, y> = <x, F^H y> is checked on the raw kernels.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, BATCH = 8192, 512


def torch():
    import torch as t
    return t


@pytest.fixture(scope="module")
def data(oracle):
    x = oracle.gen_normal(2 * N * BATCH, 0xC0F5).view(np.complex64).reshape(BATCH, N)
    w = np.random.default_rng(0xC0F5).random(N, dtype=np.float64).astype(np.float32)
    return x, w


def loss64(x64: np.ndarray, w: np.ndarray) -> float:
    y = np.fft.fft(x64, axis=-1)
    return float((np.abs(y) ** 2 * w.astype(np.float64) ** 2).sum())


def test_gradient_vs_fp64_finite_differences(ofb, data):
    T = torch()
    from onefft_b200 import torch_fft
    x, w = data
    xt = T.from_numpy(x.copy()).cuda().requires_grad_(True)
    wt = T.from_numpy(w).cuda()
    loss = torch_fft.weighted_power_loss(xt, wt)
    loss.backward()
    g = xt.grad.cpu().numpy().astype(np.complex128)
    x64 = x.astype(np.complex128)
    # loss value against FP64
    ref_loss = loss64(x64, w)
    assert abs(loss.item() - ref_loss) / ref_loss < 1e-5
    rng = np.random.default_rng(17)
    worst = 0.0
    for _ in range(32):
        v = (rng.standard_normal(x.shape) + 1j * rng.standard_normal(x.shape)) / np.sqrt(2 * x.size)
        h = 1e-3
        fd = (loss64(x64 + h * v, w) - loss64(x64 - h * v, w)) / (2 * h)
        an = float(np.real(np.vdot(g, v)))
        scale = np.linalg.norm(g) * np.linalg.norm(v)
        worst = max(worst, abs(fd - an) / scale)
    print(f"autograd: worst |fd - <g,v>| / (|g||v|) over 32 directions = {worst:.3g}")
    assert worst < 1e-5


def test_gradient_vs_reference_library(ofb, oracle, data):
    T = torch()
    from onefft_b200 import torch_fft
    x, w = data
    rows = range(0, BATCH, 64)  # 8 sampled transforms through the CPU library
    xt = T.from_numpy(x.copy()).cuda().requires_grad_(True)
    torch_fft.weighted_power_loss(xt, T.from_numpy(w).cuda()).backward()
    g = xt.grad.cpu().numpy()
    w2 = (w.astype(np.float32) ** 2)
    for r in rows:
        xr = x[r].view(np.float32)
        if oracle.have_reference():
            y = oracle.ref_fft(xr).view(np.complex64)
            gr = 2 * oracle.ref_fft((w2 * y).astype(np.complex64).view(np.float32), inverse=True).view(np.complex64)
        else:
            y = oracle.port_fft(xr).view(np.complex64)
            gr = 2 * oracle.port_fft((w2 * y).astype(np.complex64).view(np.float32), inverse=True).view(np.complex64)
        want = 2 * np.fft.ifft(w2.astype(np.float64) ** 1 * np.fft.fft(x[r].astype(np.complex128))) * N
        d_ours = np.linalg.norm(g[r] - want) / np.linalg.norm(want)
        d_ref = np.linalg.norm(gr - want) / np.linalg.norm(want)
        assert d_ours <= 2 * d_ref + 1e-9, (r, d_ours, d_ref)


def test_fused_loss_equals_unfused(ofb, data):
    """The one-kernel loss + gradient gives the unfused path's gradient bit for bit and its loss
    up to summation order."""
    T = torch()
    from onefft_b200 import torch_fft
    x, w = data
    wt = T.from_numpy(w).cuda()
    xa = T.from_numpy(x.copy()).cuda().requires_grad_(True)
    la = torch_fft.weighted_power_loss(xa, wt)
    la.backward()
    xb = T.from_numpy(x.copy()).cuda().requires_grad_(True)
    lb = torch_fft.weighted_power_loss_fused(xb, wt)
    lb.backward()
    assert abs(la.item() - lb.item()) / la.item() < 1e-5
    assert T.equal(T.view_as_real(xa.grad), T.view_as_real(xb.grad))
    # other sizes of the fused kernel (one-kernel range), loss against FP64
    for lg in (4, 7, 10, 13, 14):
        n = 1 << lg
        xs = T.randn(8, n, dtype=T.complex64, device="cuda")
        ws = T.rand(n, device="cuda")
        lf = torch_fft.weighted_power_loss_fused(xs, ws).item()
        l64 = (np.abs(np.fft.fft(xs.cpu().numpy().astype(np.complex128), axis=-1)) ** 2
               * ws.cpu().numpy().astype(np.float64) ** 2).sum()
        assert abs(lf - l64) / l64 < 1e-5, (lg, lf, l64)


def test_adjoint_identity_and_inverse_grad(ofb, oracle):
    T = torch()
    from onefft_b200 import torch_fft
    g = T.Generator(device="cuda").manual_seed(3)
    x = T.randn(64, 4096, dtype=T.complex64, device="cuda", generator=g)
    y = T.randn(64, 4096, dtype=T.complex64, device="cuda", generator=g)
    fx = torch_fft.fft(x)
    fhy = torch_fft._run("adjoint", y)
    lhs = T.vdot(fx.reshape(-1).to(T.complex128), y.reshape(-1).to(T.complex128))
    rhs = T.vdot(x.reshape(-1).to(T.complex128), fhy.reshape(-1).to(T.complex128))
    assert abs(lhs - rhs).item() / abs(lhs).item() < 1e-6
    # ifft's gradient is the forward transform: d/dx sum |ifft(x)|^2 = 2 F (ifft x)
    xr = x.clone().requires_grad_(True)
    z = torch_fft.ifft(xr)
    T.view_as_real(z).square().sum().backward()
    want = 2 * torch_fft.fft(torch_fft.ifft(x))
    assert (T.linalg.vector_norm(xr.grad - want) / T.linalg.vector_norm(want)).item() < 1e-6
    with pytest.raises(RuntimeError):
        torch_fft.fft(x.cpu())
