"""One transform too large for one GPU, split over P ranks with a single all-to-all.

n = N1 N2, x viewed as an N1 x N2 row-major matrix (x[N2 j1 + j2]), X[k1 + N1 k2] the result.

    input on rank r  : columns j2 in [r N2/P, (r+1) N2/P) of x, all rows     shape (N1, N2/P)
    1. local          : N1-point transforms down each column, times w_n^(j2 k1)
    2. all-to-all     : rank r sends rows k1 in rank s's block to rank s
    3. local          : N2-point transforms along each row k1 of the rank's block
    output on rank r : rows k1 in [r N1/P, (r+1) N1/P), all k2              shape (N1/P, N2)
                       element [k1 - r N1/P][k2] = X[k1 + N1 k2]

Input and output are both block-distributed (by columns in, by rows out), which is what lets the
transform cross the network once; callers that need natural order on one rank gather the blocks.
On GPUs the local transforms are this library's batched kernels and the exchange is NCCL's
all_to_all over NVLink (no collective inside the kernels); `fft_last_dim` lets the CPU tests run
the same exchange logic with gloo and a CPU stand-in for the kernels.
"""
from __future__ import annotations

import math

import torch


def twiddles(n1: int, n2: int, j2_first: int, j2_count: int, device) -> torch.Tensor:
    """w_n^(j2 k1) for k1 < N1 and the rank's columns j2, complex64, angle reduced modulo n in
    integers and evaluated in FP64 before the single rounding."""
    n = n1 * n2
    k1 = torch.arange(n1, dtype=torch.int64, device=device).unsqueeze(1)
    j2 = torch.arange(j2_first, j2_first + j2_count, dtype=torch.int64, device=device).unsqueeze(0)
    t = (k1 * j2) % n
    ang = (-2.0 * math.pi / n) * t.to(torch.float64)
    return torch.polar(torch.ones_like(ang), ang).to(torch.complex64)


def dist_fft(x_cols: torch.Tensor, n1: int, n2: int, group=None, fft_last_dim=None) -> torch.Tensor:
    """Forward transform of the whole n1 * n2 array; x_cols is this rank's (n1, n2/P) column block
    (complex64). Returns this rank's (n1/P, n2) row block of the result."""
    import torch.distributed as dist
    world = dist.get_world_size(group) if group is not None or dist.is_initialized() else 1
    rank = dist.get_rank(group) if world > 1 else 0
    if n1 % world or n2 % world:
        raise ValueError("N1 and N2 must be multiples of the number of ranks")
    c2, r1 = n2 // world, n1 // world
    if tuple(x_cols.shape) != (n1, c2):
        raise ValueError(f"expected the rank's column block of shape {(n1, c2)}")
    if fft_last_dim is None:
        from .torch_fft import fft as fft_last_dim
    # 1. N1-point transforms down the columns (as rows of the transposed block), then twiddles
    y = fft_last_dim(x_cols.transpose(0, 1).contiguous())  # (c2, n1): y[j2_local][k1]
    y = y * twiddles(n1, n2, rank * c2, c2, y.device).transpose(0, 1)
    # 2. one all-to-all: the block for rank s is rows k1 in [s r1, (s+1) r1)
    send = y.reshape(c2, world, r1).permute(1, 0, 2).contiguous()  # (world, c2, r1)
    if world > 1:
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=group)
    else:
        recv = send
    # recv[s][j2_local][k1_local]: columns j2 = s c2 + j2_local of this rank's rows
    rows = recv.permute(2, 0, 1).reshape(r1, n2).contiguous()  # (r1, n2): [k1_local][j2]
    # 3. N2-point transforms along each row
    return fft_last_dim(rows)
