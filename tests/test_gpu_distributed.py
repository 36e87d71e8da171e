"""GPU tests of the column transform (onefft_columns_*) and of the distributed four-step built on
it. Every GPU call here has one device, so the ranks of the multi-rank cases run one after
another in one process with the all-to-all done by indexing (the same exchange that
test_multigpu_gloo.py runs through gloo on the CPU); a one-rank case runs dist_fft itself.
"""
from __future__ import annotations

import numpy as np
import pytest

from test_multigpu_gloo import emulate_ranks

pytestmark = pytest.mark.gpu


def _run_columns(x: np.ndarray, n, cols, blocks=1, big_n=0, col0=0, flags=0) -> np.ndarray:
    import torch

    from onefft_b200 import Columns
    c = Columns(n, cols, blocks, big_n, col0)
    d_in = torch.from_numpy(np.ascontiguousarray(x, np.complex64)).cuda()
    d_out = torch.full_like(d_in, float("nan"))
    c.execute(d_in.data_ptr(), d_out.data_ptr(), flags, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    c.destroy()
    return d_out.cpu().numpy()


def _rel_rms(got, want) -> float:
    return float(np.linalg.norm(got - want) / np.linalg.norm(want))


# (log2 n, cols, blocks, log2 big_n (0 = none), col0, flags): one kernel (n <= 2^12) and two,
# the all-to-all send layout (blocks > 1), the larger transform's twiddle with a column offset
# (exponents beyond 2^32 at big_n = 2^36), both swap flags
COLUMN_CASES = [
    (4, 16, 1, 0, 0, 0),
    (8, 16, 1, 0, 0, 0),
    (12, 64, 4, 20, 64, 1),
    (10, 32, 32, 16, 32, 2),
    (13, 32, 8, 22, 96, 2),
    (16, 16, 2, 22, 48, 3),
    (18, 16, 4, 30, 112, 0),
    (20, 16, 16, 36, 1 << 10, 1),
    (22, 16, 1, 0, 0, 0),
]


@pytest.mark.parametrize("ln,cols,blocks,lbig,col0,flags", COLUMN_CASES)
def test_columns_against_fp64(ofb, oracle, ln, cols, blocks, lbig, col0, flags):
    n = 1 << ln
    big_n = (1 << lbig) if lbig else 0
    x = oracle.gen_normal(2 * n * cols, 0xC0 + ln).view(np.complex64)
    got = _run_columns(x, n, cols, blocks, big_n, col0, flags)
    want = oracle.columns_fp64(x, n, cols, blocks, big_n, col0, flags)
    assert np.isfinite(got).all()  # every output written
    err = _rel_rms(got, want)
    print(f"columns n=2^{ln} cols={cols} blocks={blocks} big_n=2^{lbig} col0={col0} flags={flags}: rel RMS {err:.3g}")
    assert err < oracle.tolerance(lbig or ln)


@pytest.mark.parametrize("ln", [8, 12, 13, 16, 20, 24])
def test_columns_equal_plain_plan_bitwise(ofb, ln):
    """Without the larger transform's twiddle and with one block, column b's results are the
    plain transform of column b, bit for bit, when the plain plan runs the same pass split (one
    kernel up to 2^12; (ceil(m/2), floor(m/2)) beyond)."""
    import torch

    from onefft_b200 import Columns
    n, cols = 1 << ln, 16 if ln > 20 else 32
    g = torch.Generator(device="cuda").manual_seed(ln)
    x = torch.randn(n, cols, dtype=torch.complex64, device="cuda", generator=g)
    out = torch.empty(cols, n, dtype=torch.complex64, device="cuda")
    c = Columns(n, cols)
    c.execute(x.data_ptr(), out.data_ptr(), 0, torch.cuda.current_stream().cuda_stream)
    xt = x.t().contiguous()
    ref = torch.empty_like(xt)
    if ln <= 12:
        plan = ofb.Plan(n, split=(ln,), cols=(-1,))
    else:
        a, b = (ln + 1) // 2, ln // 2
        plan = ofb.Plan(n, split=(a, b), cols=(ofb_pass_log_c(a), ofb_pass_log_c(b)), l2_keep=False)
    plan.dev_forward(xt.data_ptr(), ref.data_ptr(), cols, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    c.destroy()
    assert torch.equal(out, ref)


def ofb_pass_log_c(log_l: int) -> int:
    """The default tile width of a pass of length 2^log_l (pass_log_c in fft_kernels.cu)."""
    return 4 if log_l <= 9 else 3 if log_l == 10 else 2


@pytest.mark.parametrize("world,n1,n2", [(4, 1 << 10, 1 << 12), (8, 1 << 13, 1 << 12), (2, 1 << 14, 1 << 11)])
def test_distributed_ranks_emulated_on_gpu(ofb, oracle, ref_errors, world, n1, n2):
    """P ranks' column transforms on this library's kernels, run one after another, with the
    exchange done by indexing: the n1 n2-point transform in both directions, within the parity
    rule (at most 2x the reference library's rel-RMS on normal inputs of the same size)."""
    import torch

    from onefft_b200.distributed import clear_cache, gpu_columns

    def columns(v, n, cols, blocks, big_n, col0, flags):
        t = torch.from_numpy(np.ascontiguousarray(v, np.complex64)).cuda()
        return gpu_columns(t, n, cols, blocks, big_n, col0, flags).cpu().numpy()

    n = n1 * n2
    x = oracle.gen_normal(2 * n, 0xD15 + world).view(np.complex64)
    for inverse in (False, True):
        got = emulate_ranks(x, n1, n2, world, columns, inverse)
        want = oracle.fft64_numpy(x.view(np.float32), inverse).view(np.complex128).reshape(n2, n1).T
        err = _rel_rms(got, want)
        print(f"distributed four-step, {world} ranks emulated, n=2^{n.bit_length() - 1} "
              f"{'inverse' if inverse else 'forward'}: rel RMS {err:.3g}")
        assert err < oracle.tolerance(n.bit_length() - 1)
        ref = ref_errors["normal"].get(str(n.bit_length() - 1))
        if ref:
            assert err <= 2 * ref["inverse" if inverse else "forward"]["rel_rms"]
    clear_cache()


def test_dist_fft_single_rank_on_gpu(ofb, oracle):
    import torch

    from onefft_b200.distributed import clear_cache, dist_fft
    n1, n2 = 2048, 4096
    n = n1 * n2
    x = oracle.gen_normal(2 * n, 0xD15).view(np.complex64)
    cols = torch.from_numpy(x.reshape(n1, n2).copy()).cuda()
    for inverse in (False, True):
        out = dist_fft(cols, n1, n2, inverse=inverse).cpu().numpy()  # (n1, n2): [k1][k2] = X[k1 + n1 k2]
        got = np.ascontiguousarray(out.T).reshape(-1)  # natural order X[k1 + n1 k2]
        want = oracle.fft64_numpy(x.view(np.float32), inverse)
        err = oracle.rel_rms(got.view(np.float32), want)
        print(f"distributed four-step on one rank, n=2^23 {'inverse' if inverse else 'forward'}: rel RMS {err:.3g}")
        assert err < oracle.tolerance(23)
    clear_cache()


@pytest.mark.parametrize("ln", [10, 16])
def test_columns_misaligned_input_same_bits(ofb, ln):
    """An input 8 bytes off a 16-byte boundary takes the per-thread-load kernel for the first pass
    instead of the bulk tensor copy: the same bits."""
    import torch

    from onefft_b200 import Columns
    n, cols = 1 << ln, 32
    c = Columns(n, cols, 4, n * 256, 5 * cols)
    g = torch.Generator(device="cuda").manual_seed(ln)
    buf = torch.randn(n * cols + 1, dtype=torch.complex64, device="cuda", generator=g)
    x_odd = buf[1:]  # 8 bytes past the allocation's 256-byte boundary
    x_even = x_odd.clone()
    assert x_odd.data_ptr() % 16 == 8 and x_even.data_ptr() % 16 == 0
    a, b = torch.empty_like(x_even), torch.empty_like(x_even)
    s = torch.cuda.current_stream().cuda_stream
    c.execute(x_even.data_ptr(), a.data_ptr(), 0, s)
    c.execute(x_odd.data_ptr(), b.data_ptr(), 0, s)
    torch.cuda.synchronize()
    c.check()
    c.destroy()
    assert torch.equal(a, b)


def test_dist_fft_through_nccl_one_rank(ofb, oracle):
    """dist_fft with an NCCL process group of one rank: the exchange runs through NCCL's
    all_to_all on the GPU (a copy to itself), the result is the transform."""
    import socket

    import torch
    import torch.distributed as dist

    from onefft_b200.distributed import clear_cache, dist_fft
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        n1, n2 = 1024, 2048
        x = oracle.gen_normal(2 * n1 * n2, 0xCC1).view(np.complex64)
        cols = torch.from_numpy(x.reshape(n1, n2).copy()).cuda()
        out = dist_fft(cols, n1, n2).cpu().numpy()
        torch.cuda.synchronize()
    finally:
        dist.destroy_process_group()
        clear_cache()
    got = np.ascontiguousarray(out.T).reshape(-1)
    want = oracle.fft64_numpy(x.view(np.float32))
    assert oracle.rel_rms(got.view(np.float32), want) < oracle.tolerance(21)
