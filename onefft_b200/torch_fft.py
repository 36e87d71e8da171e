"""Differentiable FFT for torch tensors over the C ABI of libonefft_cuda.so.

``fft(x)`` / ``ifft(x)`` transform the last dimension of a contiguous complex64 CUDA tensor
(unnormalised, OneFFT's convention) with ``onefft_dev_forward_batched`` /
``onefft_dev_inverse_batched`` on the current torch stream. Their backward is the hand-written
adjoint kernel ``onefft_dev_adjoint_batched``: for y = F x the vector-Jacobian product torch needs
(conjugate-Wirtinger convention) is F^H g = conj(F) g, the unnormalised inverse, which the kernel
computes as the forward transform with real and imaginary parts exchanged on load and store —
the conjugation of the upstream gradient is fused into those loads and stores. The adjoint of
the inverse is the forward transform.

``weighted_power_loss(x, w)`` is the loss of the differentiable-layer benchmark configuration,
sum |w * fft(x)|^2, built from these pieces; its gradient is 2 F^H (w^2 * F x).

No CPU path exists: CPU tensors raise. The transforms only enqueue work; a failure that a
multi-pass kernel finds while running (an expired bounded wait) is reported by ``check()`` after
the caller synchronises.
"""
from __future__ import annotations

import threading

import torch

from . import lib, last_error, Plan

_plans: dict[tuple[int, int], Plan] = {}
_plans_lock = threading.Lock()


def _plan(n: int, device: int) -> Plan:
    key = (n, device)
    p = _plans.get(key)
    if p is None:
        with _plans_lock:
            p = _plans.get(key)
            if p is None:
                with torch.cuda.device(device):
                    p = Plan(n)
                _plans[key] = p
    return p


def check() -> None:
    """Raises if a kernel of any plan this module used recorded a failure since the last check
    (onefft_plan_status); call after synchronising the streams the transforms ran on."""
    with _plans_lock:
        plans = list(_plans.values())
    for p in plans:
        p.check()


def _check(x: torch.Tensor) -> torch.Tensor:
    if not x.is_cuda:
        raise RuntimeError("onefft_b200 transforms CUDA tensors only (there is no CPU path)")
    if x.dtype != torch.complex64:
        raise TypeError("expected a complex64 tensor")
    return x.contiguous()


def _run(kind: str, x: torch.Tensor) -> torch.Tensor:
    x = _check(x)
    n = x.shape[-1]
    batch = x.numel() // n if n else 0
    y = torch.empty_like(x)
    if batch == 0:
        return y
    plan = _plan(n, x.device.index)
    stream = torch.cuda.current_stream(x.device).cuda_stream
    f = {"forward": lib().onefft_dev_forward_batched, "inverse": lib().onefft_dev_inverse_batched,
         "adjoint": lib().onefft_dev_adjoint_batched}[kind]
    with torch.cuda.device(x.device):
        rc = f(plan.handle, x.data_ptr(), y.data_ptr(), batch, stream)
    if rc != 0:
        raise RuntimeError(f"onefft {kind} failed ({rc}): {last_error()}")
    return y


class _FFT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return _run("forward", x)

    @staticmethod
    def backward(ctx, g):
        return _run("adjoint", g)


class _IFFT(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return _run("inverse", x)

    @staticmethod
    def backward(ctx, g):
        # the adjoint of the unnormalised inverse is the unnormalised forward transform
        return _run("forward", g)


def fft(x: torch.Tensor) -> torch.Tensor:
    """Unnormalised forward FFT over the last dimension (power-of-two length)."""
    return _FFT.apply(x)


def ifft(x: torch.Tensor) -> torch.Tensor:
    """Unnormalised inverse FFT over the last dimension (ifft(fft(x)) = n x)."""
    return _IFFT.apply(x)


def weighted_power_loss(x: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    """sum over the batch and frequencies of |w * fft(x)|^2, w real of length n."""
    y = fft(x)
    return (torch.view_as_real(y).square().sum(-1) * w.square()).sum()


class _FusedPowerLoss(torch.autograd.Function):
    """Loss and gradient from one kernel pass (onefft_dev_weighted_power_loss): the gradient is
    computed with the loss and kept until backward."""

    @staticmethod
    def forward(ctx, x, w):
        x = _check(x)
        w = w.detach().to(torch.float32).contiguous()
        n = x.shape[-1]
        batch = x.numel() // n
        plan = _plan(n, x.device.index)
        grad = torch.empty_like(x) if x.requires_grad else None
        loss = torch.empty((), dtype=torch.float64, device=x.device)
        stream = torch.cuda.current_stream(x.device).cuda_stream
        with torch.cuda.device(x.device):
            rc = lib().onefft_dev_weighted_power_loss(plan.handle, x.data_ptr(), w.data_ptr(),
                                                       grad.data_ptr() if grad is not None else None, batch,
                                                       loss.data_ptr(), stream)
        if rc != 0:
            raise RuntimeError(f"onefft fused loss failed ({rc}): {last_error()}")
        ctx.save_for_backward(grad if grad is not None else torch.empty(0))
        return loss.to(torch.float32)

    @staticmethod
    def backward(ctx, g):
        (grad,) = ctx.saved_tensors
        return grad * g.to(grad.real.dtype), None


def weighted_power_loss_fused(x: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    """Same value and gradient as weighted_power_loss, from a single fused kernel."""
    return _FusedPowerLoss.apply(x, w)
