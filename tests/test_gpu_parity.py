"""GPU parity tests through the C ABI — the reference's test program, re-aimed at the B200 path.

Mirrors OneFFT tests/test_onefft.c check by check, for every size 2^0 .. 2^20:
  * forward and inverse against the FP64 FFT (tests/test_onefft.c:121-132): relative RMS within
    the reference's bound 4e-7 + 1e-7 log2 n AND at most 2x the reference library's own error on
    the same input (the parity rule), max-abs error recorded;
  * guard bands of 64 sentinels around every buffer, input unmodified, input misaligned by one
    float and output by three (tests/test_onefft.c:73-97, 118-119);
  * round trip inverse(forward(x)) = n x (tests/test_onefft.c:134-140);
  * impulse and constant known answers (tests/test_onefft.c:142-164);
  * invalid sizes (tests/test_onefft.c:170-182), cache == plan bitwise (:185-205), four threads
    sharing a plan and racing the cache (:207-259), the C++-layer round trip (test_cpp.cpp).
Plus what the GPU form adds: every pass kernel exercised at small sizes through forced pass
splits, device-pointer batches equal to one-at-a-time transforms bit for bit, the device FP64
twiddle rule equal to the CPU rule, and the allocation-failure contract.
"""
from __future__ import annotations

import ctypes
import math
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GUARD = 64
SENTINEL = np.float32(12345.0)


class Guarded:
    """2n floats at `misalign` floats past a 64-float sentinel band, with a band after."""

    def __init__(self, count: int, misalign: int):
        self.base = np.full(count + 2 * GUARD + 16, SENTINEL, np.float32)
        self.off = GUARD + misalign
        self.count = count
        self.data = self.base[self.off:self.off + count]

    @property
    def ptr(self) -> int:
        return self.base.ctypes.data + 4 * self.off

    def intact(self) -> bool:
        return bool((self.base[:self.off] == SENTINEL).all() and
                    (self.base[self.off + self.count:self.off + self.count + GUARD] == SENTINEL).all())


def fp64(oracle, x, inv):
    return oracle.fft64(x, inv) if x.size <= 2 * 4096 else oracle.fft64_numpy(x, inv)


MAX_ABS = {}


@pytest.mark.parametrize("log2n", list(range(0, 21)))
def test_size(ofb, oracle, uniform_inputs, ref_errors, log2n):
    n = 1 << log2n
    L = ofb.lib()
    plan = ofb.Plan(n)
    x = uniform_inputs[log2n]
    inb, outb, back = Guarded(2 * n, 1), Guarded(2 * n, 3), Guarded(2 * n, 0)
    inb.data[:] = x
    for inv in (0, 1):
        d = "inverse" if inv else "forward"
        outb.data[:] = 0
        (L.onefft_plan_inverse if inv else L.onefft_plan_forward)(plan.handle, inb.ptr, outb.ptr)
        assert ofb.last_error() == ""
        want = fp64(oracle, x, inv)
        err = oracle.rel_rms(outb.data, want)
        ref = ref_errors["uniform"][str(log2n)][d]["rel_rms"]
        MAX_ABS[(log2n, d)] = oracle.max_abs(outb.data, want)
        assert err < oracle.tolerance(log2n), (n, d, err)
        assert err <= 2 * ref + 1e-12, (n, d, err, ref)
        assert outb.intact(), "wrote outside of the output"
        assert inb.intact() and np.array_equal(inb.data, x), "input modified"
    # round trip
    L.onefft_plan_forward(plan.handle, inb.ptr, outb.ptr)
    L.onefft_plan_inverse(plan.handle, outb.ptr, back.ptr)
    want = x.astype(np.float64) * n
    assert oracle.rel_rms(back.data, want) < 2 * oracle.tolerance(log2n)
    assert back.intact()
    # impulse at j = 1 + (n/3) mod (n-1)
    j = 1 + (n // 3) % (n - 1) if n > 1 else 0
    imp = np.zeros(2 * n, np.float32)
    imp[2 * j] = 1.0
    y = plan.forward(imp).reshape(-1, 2).astype(np.float64)
    k = np.arange(n, dtype=np.uint64)
    ang = -2 * math.pi * ((np.uint64(j) * k) % np.uint64(n)).astype(np.float64) / n
    assert np.hypot(y[:, 0] - np.cos(ang), y[:, 1] - np.sin(ang)).max() < 4e-6
    # constant
    c = np.tile(np.array([0.5, -0.25], np.float32), n)
    y = plan.forward(c).reshape(-1, 2).astype(np.float64)
    worst = math.hypot(y[0, 0] - 0.5 * n, y[0, 1] + 0.25 * n) / n
    if n > 1:
        worst = max(worst, float(np.hypot(y[1:, 0], y[1:, 1]).max()) / n)
    assert worst < 1e-6
    plan.destroy()


def test_golden_vectors(ofb, oracle, ref_small):
    """GPU outputs against the reference's committed outputs (n <= 2^11): both within the
    reference bound of the FP64 oracle, and within the bound of each other."""
    for l in range(12):
        x = ref_small[f"in_{l}"]
        for d, inv in (("forward", False), ("inverse", True)):
            got = ofb.inverse(x) if inv else ofb.forward(x)
            gold = ref_small[f"out_{d}_{l}"]
            want = oracle.fft64(x, inv)
            assert oracle.rel_rms(got, want) <= 2 * oracle.rel_rms(gold, want) + 1e-12
            assert oracle.rel_rms(got, gold.astype(np.float64)) < 2 * oracle.tolerance(l)


def test_invalid_sizes(ofb):
    L = ofb.lib()
    for n in (0, 3, 5, 6, 7, 12, 1000, 1023, 1025, 2**64 - 1, 2**31):
        assert L.onefft_plan_create(n) is None
    L.onefft_plan_destroy(None)
    x = np.zeros(6, np.float32)
    out = np.full(6, 7.0, np.float32)
    assert L.onefft_forward(x.ctypes.data, out.ctypes.data, 3) == -1
    assert L.onefft_inverse(x.ctypes.data, out.ctypes.data, 0) == -1
    assert out[0] == 7 and out[5] == 7
    assert L.onefft_cache_prepare(12) == -1 and L.onefft_cache_prepare(0) == -1


def test_cache_equals_plan_bitwise(ofb, oracle):
    L = ofb.lib()
    st = 0x1234
    for l in range(0, 13):
        n = 1 << l
        x, st = oracle.gen_uniform(2 * n, st)
        plan = ofb.Plan(n)
        assert plan.size() == n
        if n == 64:
            ofb.cache_prepare(n)
        for inv in (False, True):
            want = plan.inverse(x) if inv else plan.forward(x)
            got = np.empty_like(x)
            f = L.onefft_inverse if inv else L.onefft_forward
            assert f(x.ctypes.data, got.ctypes.data, n) == 0
            assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), (n, inv)
        plan.destroy()
    ofb.cache_clear()
    ofb.cache_clear()


def test_threads_share_plan_and_race_cache(ofb, oracle):
    n = 4096
    L = ofb.lib()
    ofb.cache_clear()
    plan = ofb.Plan(n)
    x, _ = oracle.gen_uniform(2 * n, 77)
    expected = [plan.forward(x), plan.inverse(x)]
    mismatches = [0] * 4

    def worker(t):
        out = np.empty_like(x)
        for rnd in range(100):
            inv = (rnd + t) & 1
            if rnd & 2:
                f = L.onefft_inverse if inv else L.onefft_forward
                if f(x.ctypes.data, out.ctypes.data, n) != 0:
                    mismatches[t] += 1
            else:
                (L.onefft_plan_inverse if inv else L.onefft_plan_forward)(plan.handle, x.ctypes.data, out.ctypes.data)
            if not np.array_equal(out.view(np.uint32), expected[inv].view(np.uint32)):
                mismatches[t] += 1

    ts = [threading.Thread(target=worker, args=(t,)) for t in range(4)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert mismatches == [0, 0, 0, 0]
    plan.destroy()
    ofb.cache_clear()


def test_cpp_layer_round_trip(ofb):
    """tests/test_cpp.cpp:10-36 on the same data shape: round trip < 1e-5, moved plan equal."""
    n = 256
    i = np.arange(n, dtype=np.float32)
    z = (np.sin(np.float32(0.3) * i) + 1j * np.cos(np.float32(1.7) * i)).astype(np.complex64)
    with ofb.Plan(n) as plan:
        spec = plan.forward(z).view(np.complex64)
        back = plan.inverse(spec).view(np.complex64)
        assert np.abs(back / n - z).max() < 1e-5
        again = ofb.forward(z).view(np.complex64)
        assert np.array_equal(again, spec)
        assert np.array_equal(ofb.inverse(spec).view(np.complex64), back)


SPLITS = [
    (1 << 8, (4, 4)), (1 << 9, (5, 4)), (1 << 9, (4, 5)), (1 << 10, (6, 4)), (1 << 11, (7, 4)),
    (1 << 12, (8, 4)), (1 << 13, (9, 4)), (1 << 14, (10, 4)), (1 << 15, (11, 4)), (1 << 16, (12, 4)),
    (1 << 16, (4, 12)), (1 << 16, (8, 8)), (1 << 12, (4, 4, 4)), (1 << 13, (5, 4, 4)), (1 << 15, (4, 5, 6)),
    (1 << 17, (6, 6, 5)), (1 << 18, (6, 6, 6)), (1 << 20, (10, 10)), (1 << 13, (13,)), (1 << 14, (14,)),
]


SHAPES = [  # (n, split, tile widths, chunk)
    (1 << 12, (4, 4, 4), (2, 3, 2), 2), (1 << 15, (4, 5, 6), (4, 4, 4), 4), (1 << 18, (6, 6, 6), (3, 3, 3), 3),
    (1 << 16, (8, 8), (2, 2), 0), (1 << 16, (8, 8), (3, 4), 0), (1 << 20, (10, 10), (4, 3), 0),
    (1 << 21, (7, 7, 7), (4, 4, 4), 5), (1 << 24, (8, 8, 8), (4, 4, 4), 6), (1 << 22, (12, 5, 5), (2, 4, 4), 3),
]


TMA_SHAPES = [  # (n, split, tile widths, chunk) run through the bulk-tensor-copy kernels
    (1 << 12, (6, 6), (4, 4), 0), (1 << 16, (8, 8), (2, 3), 0), (1 << 18, (9, 9), (4, 3), 0),
    (1 << 20, (10, 10), (1, 2), 0), (1 << 22, (11, 11), (2, 1), 0), (1 << 24, (12, 12), (1, 1), 0),
    (1 << 24, (12, 12), (2, 2), 0), (1 << 20, (12, 8), (2, 3), 0),
    (1 << 21, (7, 7, 7), (4, 3, 4), 5), (1 << 24, (8, 8, 8), (4, 4, 4), 0), (1 << 23, (9, 7, 7), (3, 4, 3), 0),
]


@pytest.mark.parametrize("n,split,cols,chunk,tma", [(n, s, None, 0, False) for n, s in SPLITS] +
                         [s + (False,) for s in SHAPES] + [s + (True,) for s in TMA_SHAPES])
def test_pass_splits(ofb, oracle, n, split, cols, chunk, tma):
    """Every pass kernel (all tile lengths 2^4..2^12, widths 2..16, first/middle/last, chunked
    first passes, plain and TMA-staged) against FP64; TMA results equal the plain kernels'."""
    log2n = n.bit_length() - 1
    x = oracle.gen_normal(2 * n, 1000 + log2n)
    plan = ofb.Plan(n, split=split, cols=cols, chunk=chunk, tma=tma)
    if tma:
        import torch
        plain = ofb.Plan(n, split=split, cols=cols, chunk=chunk)
        d = torch.from_numpy(x).cuda()
        a, b = torch.empty_like(d), torch.empty_like(d)
        for inv in (False, True):
            (plan.dev_inverse if inv else plan.dev_forward)(d.data_ptr(), a.data_ptr(), 1)
            (plain.dev_inverse if inv else plain.dev_forward)(d.data_ptr(), b.data_ptr(), 1)
            torch.cuda.synchronize()
            assert torch.equal(a, b), (n, split, inv)
        # batched through the TMA kernels too (the batch is the copies' outermost dimension)
        xb = torch.from_numpy(oracle.gen_normal(6 * n, 77)).cuda()
        ya, yb = torch.empty_like(xb), torch.empty_like(xb)
        plan.dev_forward(xb.data_ptr(), ya.data_ptr(), 3)
        plain.dev_forward(xb.data_ptr(), yb.data_ptr(), 3)
        torch.cuda.synchronize()
        assert torch.equal(ya, yb)
        plain.destroy()
    assert plan.passes() == split
    default = ofb.Plan(n)
    for inv in (False, True):
        got = plan.inverse(x) if inv else plan.forward(x)
        want = fp64(oracle, x, inv)
        err = oracle.rel_rms(got, want)
        assert err < oracle.tolerance(log2n), (n, split, inv, err)
        if oracle.have_reference():
            ref = oracle.rel_rms(oracle.ref_fft(x, inv), want)
            assert err <= 2 * ref, (n, split, inv, err, ref)
    plan.destroy()
    default.destroy()


def _torch():
    import torch
    return torch


@pytest.mark.parametrize("log2n,batch", [(0, 1000), (3, 333), (4, 257), (8, 100), (10, 37), (12, 65), (13, 9),
                                          (14, 3), (15, 3), (17, 2), (21, 2)])
def test_device_batched_equals_single_bitwise(ofb, oracle, log2n, batch):
    torch = _torch()
    n = 1 << log2n
    x = oracle.gen_normal(2 * n * batch, 31 + log2n)
    plan = ofb.Plan(n)
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.full_like(d_in, float("nan"))
    for inv in (False, True):
        f = plan.dev_inverse if inv else plan.dev_forward
        f(d_in.data_ptr(), d_out.data_ptr(), batch, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        for b in sorted({0, batch // 2, batch - 1}):
            one = (plan.inverse if inv else plan.forward)(x[2 * n * b:2 * n * (b + 1)])
            assert np.array_equal(got[2 * n * b:2 * n * (b + 1)].view(np.uint32), one.view(np.uint32)), (b, inv)
    # host-pointer batched path (pipelined chunks) gives the same bits
    host = plan.forward(x, batch=batch)
    plan.dev_forward(d_in.data_ptr(), d_out.data_ptr(), batch)
    torch.cuda.synchronize()
    assert np.array_equal(host.view(np.uint32), d_out.cpu().numpy().view(np.uint32))
    plan.destroy()


@pytest.mark.parametrize("log2n", list(range(4, 15)))
def test_transforms_per_block_same_bits(ofb, oracle, log2n):
    """Every compiled number of transforms per block of a one-kernel size (the autotuner's
    choices) gives the default plan's results bit for bit, both directions, with a batch that
    leaves the last block partly empty; invalid widths are rejected."""
    from onefft_b200.autotune import batched_log_c_candidates
    torch = _torch()
    n = 1 << log2n
    batch = 2 * (1 << max(0, 13 - log2n)) + 3
    x = oracle.gen_normal(2 * n * batch, 57 + log2n)
    d_in = torch.from_numpy(x).cuda()
    want = torch.empty_like(d_in)
    default = ofb.Plan(n, split=(log2n,), cols=(max(0, 12 - log2n),))
    for inv in (False, True):
        (default.dev_inverse if inv else default.dev_forward)(d_in.data_ptr(), want.data_ptr(), batch)
        for c in batched_log_c_candidates(log2n):
            plan = ofb.Plan(n, split=(log2n,), cols=(c,))
            got = torch.full_like(d_in, float("nan"))
            (plan.dev_inverse if inv else plan.dev_forward)(d_in.data_ptr(), got.data_ptr(), batch)
            torch.cuda.synchronize()
            assert torch.equal(got, want), (log2n, c, inv)
            plan.destroy()
    default.destroy()
    for bad in (max(0, 12 - log2n) + 2, 14 - log2n, -2 if log2n < 12 else 2):
        if bad not in batched_log_c_candidates(log2n) and bad != -1:
            with pytest.raises(ValueError):
                ofb.Plan(n, split=(log2n,), cols=(bad,))


def test_device_pointer_contract(ofb):
    torch = _torch()
    L = ofb.lib()
    plan = ofb.Plan(1024)
    buf = torch.zeros(4 * 2048 + 16, dtype=torch.float32, device="cuda")
    base = buf.data_ptr()
    # misaligned by one float: rejected before any launch
    assert L.onefft_dev_forward_batched(plan.handle, base + 4, base + 2048 * 8, 1, None) == -2
    # overlapping input and output
    assert L.onefft_dev_forward_batched(plan.handle, base, base + 1024, 1, None) == -2
    # batch 0 is a no-op
    assert L.onefft_dev_forward_batched(plan.handle, base, base + 2048 * 8, 0, None) == 0
    # host API on device pointers works in place of staging
    x = torch.randn(2048, device="cuda")
    y = torch.empty_like(x)
    L.onefft_plan_forward(plan.handle, x.data_ptr(), y.data_ptr())
    assert ofb.last_error() == ""
    want = plan.forward(x.cpu().numpy())
    assert np.array_equal(y.cpu().numpy().view(np.uint32), want.view(np.uint32))
    plan.destroy()


def test_device_twiddle_rule_matches_cpu(ofb, oracle):
    """The FP64 rule evaluated on the device, rounded to FP32, equals the CPU restatement of
    OneFFT's rule (src/onefft.c:115-141) on whole tables."""
    L = ofb.lib()
    for l in (3, 10, 16, 20):
        n = 1 << l
        dev = np.empty(2 * n, np.float32)
        assert L.onefft_debug_twiddles(l, n, dev.ctypes.data) == 0
        cpu = oracle.twiddle_table(l, n)
        diff = dev.view(np.int32).astype(np.int64) - cpu.view(np.int32).astype(np.int64)
        # identical except where libm and CUDA's FP64 sin/cos round across a float boundary
        assert np.abs(diff).max() <= 1
        assert (diff != 0).mean() < 1e-5, (l, (diff != 0).sum())


def test_allocation_failure_leaves_output_untouched(ofb):
    L = ofb.lib()
    ofb.cache_clear()
    n = 1 << 12
    x = np.ones(2 * n, np.float32)
    out = np.full(2 * n, 7.0, np.float32)
    L.onefft_debug_fail_alloc(1)  # the plan's table allocation fails
    assert L.onefft_forward(x.ctypes.data, out.ctypes.data, n) == -1
    assert (out == 7.0).all()
    L.onefft_debug_fail_alloc(0)
    assert L.onefft_forward(x.ctypes.data, out.ctypes.data, n) == 0  # recovers once memory is back
    ofb.cache_clear()
    # staging allocation failure in a fresh thread (its own staging buffers)
    res = {}

    def worker():
        plan = L.onefft_plan_create(1 << 22)
        big_in = np.ones(2 << 22, np.float32)
        big_out = np.full(2 << 22, 7.0, np.float32)
        L.onefft_debug_fail_alloc(1)
        res["rc"] = L.onefft_plan_forward_batched(plan, big_in.ctypes.data, big_out.ctypes.data, 1)
        L.onefft_debug_fail_alloc(0)
        res["untouched"] = bool((big_out == 7.0).all())
        L.onefft_plan_destroy(plan)

    t = threading.Thread(target=worker)
    t.start()
    t.join()
    assert res["rc"] == -1 and res["untouched"]


def test_max_abs_report(ofb):
    """Prints the per-size max-abs errors gathered by test_size (the parity rule states them per size)."""
    for (l, d), v in sorted(MAX_ABS.items()):
        print(f"n=2^{l} {d}: max-abs {v:.3g}")


@pytest.mark.parametrize("log2n", [12, 13])
@pytest.mark.parametrize("batch", [5, 3001])
def test_pipelined_one_kernel_equals_default(ofb, log2n, batch):
    """The persistent double-buffered one-kernel form (ONEFFT_COLS_PIPELINED: the next
    transform's values arrive by one bulk copy while the current one computes) gives the default
    kernel's bits, for batches smaller than its grid and several times larger, both directions;
    8-byte aligned buffers take the default kernel instead (same bits again)."""
    import torch as T
    n = 1 << log2n
    pipe = ofb.Plan(n, split=(log2n,), cols=(15,))
    ref = ofb.Plan(n)
    g = T.Generator(device="cuda").manual_seed(log2n * 7 + batch)
    buf = T.randn(2 * n * batch + 2, device="cuda", generator=g)
    for off in (0, 2):  # 16-byte aligned, then 8-byte aligned
        x = buf[off:off + 2 * n * batch]
        a, b = T.empty_like(x), T.empty_like(x)
        for inv in (False, True):
            (pipe.dev_inverse if inv else pipe.dev_forward)(x.data_ptr(), a.data_ptr(), batch)
            (ref.dev_inverse if inv else ref.dev_forward)(x.data_ptr(), b.data_ptr(), batch)
            T.cuda.synchronize()
            assert pipe.status() == 0
            assert T.equal(a, b), (log2n, batch, off, inv)
    pipe.destroy()
    ref.destroy()
