"""GPU tests of the failure path of the multi-pass kernels, with no GPU fault.

OneFFT reports failure by its return value with `out` untouched (include/onefft.h:73-75). Here a
multi-pass kernel waits for each tile copy with a bounded wait; when the wait runs out, the kernel
records the failure in its plan's error word, lets the copy land, leaves the tile unwritten and
returns. The test hook onefft_debug_expire_waits(1) makes every first wait count as expired, so
this path runs for real on the device (nothing hangs and nothing faults: each copy still
completes before its block exits). Checked:
  - host-pointer calls return the error (-1000 for the batched call, -1 for onefft_forward) and
    leave `out` untouched;
  - device-pointer callers see it through onefft_plan_status(), which then reads 0 again;
  - with the hook off, the next calls on the same plan are correct.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ERR_CUDA_BASE = -1000


def test_expired_wait_reported_and_recovered(ofb, oracle):
    import torch
    L = ofb.lib()
    n = 1 << 20  # two TMA-staged passes in the tuned table
    plan = ofb.Plan(n)
    x, _ = oracle.gen_uniform(2 * n, 0xFA11)
    want = oracle.fft64_numpy(x)
    out = np.full(2 * n, 7.0, np.float32)
    assert L.onefft_debug_expire_waits(1) == 0
    try:
        rc_batched = L.onefft_plan_forward_batched(plan.handle, x.ctypes.data, out.ctypes.data, 1)
        msg = ofb.last_error()
        rc_cached = L.onefft_forward(x.ctypes.data, out.ctypes.data, n)
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.zeros_like(d_in)
        plan.dev_forward(d_in.data_ptr(), d_out.data_ptr(), 1)
        torch.cuda.synchronize()
    finally:
        assert L.onefft_debug_expire_waits(0) == 0
    assert rc_batched == ERR_CUDA_BASE, msg
    assert "did not complete" in msg
    assert rc_cached == -1
    assert (out == 7.0).all(), "output written after a failed transform"
    assert plan.status() == ERR_CUDA_BASE
    assert "did not complete" in ofb.last_error()
    assert plan.status() == 0  # reading cleared it
    # the same plan (and the cached one) work again
    y = plan.forward(x)
    assert oracle.rel_rms(y, want) < oracle.tolerance(20)
    assert L.onefft_forward(x.ctypes.data, out.ctypes.data, n) == 0
    assert np.array_equal(out, y)
    plan.dev_forward(d_in.data_ptr(), d_out.data_ptr(), 1)
    torch.cuda.synchronize()
    assert plan.status() == 0
    assert np.array_equal(d_out.cpu().numpy(), y)
    plan.destroy()


@pytest.mark.parametrize("ln", [10, 20])
def test_column_transform_expired_wait_reported(ofb, oracle, ln):
    """The column transform's tile copies (one pass at 2^10, two at 2^20) take the same failure
    path: nothing written, onefft_columns_status() reports it once, the next call is correct."""
    import torch
    L = ofb.lib()
    n, cols = 1 << ln, 64
    c = ofb.Columns(n, cols, 4, n * 256, 3 * cols)
    x = torch.from_numpy(oracle.gen_normal(2 * n * cols, 0xC01).view(np.complex64)).cuda()
    y = torch.full_like(x, 7.0)
    s = torch.cuda.current_stream().cuda_stream
    assert L.onefft_debug_expire_waits(1) == 0
    try:
        c.execute(x.data_ptr(), y.data_ptr(), 0, s)
        torch.cuda.synchronize()
    finally:
        assert L.onefft_debug_expire_waits(0) == 0
    assert (y == 7.0).all(), "output written after a failed column transform"
    assert c.status() == ERR_CUDA_BASE
    assert "did not complete" in ofb.last_error()
    assert c.status() == 0
    c.execute(x.data_ptr(), y.data_ptr(), 0, s)
    torch.cuda.synchronize()
    assert c.status() == 0
    want = oracle.columns_fp64(x.cpu().numpy(), n, cols, 4, n * 256, 3 * cols)
    got = y.cpu().numpy()
    assert np.linalg.norm(got - want) / np.linalg.norm(want) < oracle.tolerance(ln + 8)
    c.destroy()
