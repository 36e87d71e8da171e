"""One transform too large for one GPU, split over P ranks with a single all-to-all.

n = N1 N2, x viewed as an N1 x N2 row-major matrix (x[N2 j1 + j2]), X[k1 + N1 k2] the result.

    input on rank r  : columns j2 in [r N2/P, (r+1) N2/P) of x, all rows     shape (N1, N2/P)
    1. local          : N1-point transforms down each column, times w_n^(j2 k1), written straight
                        into the all-to-all send layout [s][j2 - r N2/P][k1 - s N1/P]
    2. all-to-all     : rank r sends rows k1 in rank s's block to rank s
    3. local          : N2-point transforms down the columns of the received N2 x N1/P matrix
                        (element [j2][k1 - r N1/P]), written row-wise
    output on rank r : rows k1 in [r N1/P, (r+1) N1/P), all k2              shape (N1/P, N2)
                       element [k1 - r N1/P][k2] = X[k1 + N1 k2]

Input and output are both block-distributed (by columns in, by rows out), which is what lets the
transform cross the network once; callers that need natural order on one rank gather the blocks.
Steps 1 and 3 are each one call of the library's column transform (onefft_columns_execute: one
or two pass kernels, with the twiddle and the layout change done by the kernels that read and
write the data, so each local step moves the rank's block through HBM once per pass), and the
exchange is NCCL's all_to_all over NVLink. The inverse is swap(F(swap(x))): step 1 exchanges
re/im as it reads, step 3 as it writes. `columns` lets the CPU tests run the same exchange logic
with gloo and a CPU stand-in for the column transform.
"""
from __future__ import annotations

import torch

SWAP_IN, SWAP_OUT = 1, 2

_cache: dict = {}


def gpu_columns(x: torch.Tensor, n: int, cols: int, blocks: int, big_n: int, col0: int, flags: int) -> torch.Tensor:
    """The column transform of the n x cols matrix x (complex64 on a CUDA device) on the current
    stream: returns the n * cols results in the column layout of onefft_columns_execute. The
    column-transform objects (tables and, for n > 2^12, an n * cols work buffer) are kept per
    device and shape, so calls with the same shape must not run concurrently on different streams
    (they would share the work buffer); clear_cache() frees them."""
    from . import Columns
    if x.dtype != torch.complex64 or not x.is_contiguous():
        raise ValueError("expected a contiguous complex64 tensor")
    if x.numel() != n * cols:
        raise ValueError(f"expected {n} x {cols} values, got {x.numel()}")
    key = (x.device.index, n, cols, blocks, big_n, col0)
    c = _cache.get(key)
    if c is None:
        with torch.cuda.device(x.device):
            c = _cache[key] = Columns(n, cols, blocks, big_n, col0)
    out = torch.empty(n * cols, dtype=torch.complex64, device=x.device)
    c.execute(x.data_ptr(), out.data_ptr(), flags, torch.cuda.current_stream(x.device).cuda_stream)
    return out


def clear_cache() -> None:
    """Frees the column-transform objects gpu_columns keeps (after the streams that used them are done)."""
    for c in _cache.values():
        c.destroy()
    _cache.clear()


def dist_fft(x_cols: torch.Tensor, n1: int, n2: int, group=None, inverse: bool = False, columns=None) -> torch.Tensor:
    """Forward (or, with inverse, unnormalised inverse) transform of the whole n1 * n2 array;
    x_cols is this rank's (n1, n2/P) column block (complex64). Returns this rank's (n1/P, n2) row
    block of the result. columns(x, n, cols, blocks, big_n, col0, flags): the column transform
    (default gpu_columns, this library's kernels)."""
    import torch.distributed as dist
    grouped = group is not None or (dist.is_available() and dist.is_initialized())
    world = dist.get_world_size(group) if grouped else 1
    rank = dist.get_rank(group) if grouped else 0
    if n1 % world or n2 % world:
        raise ValueError("N1 and N2 must be multiples of the number of ranks")
    c2, r1 = n2 // world, n1 // world
    if tuple(x_cols.shape) != (n1, c2):
        raise ValueError(f"expected the rank's column block of shape {(n1, c2)}")
    col = columns if columns is not None else gpu_columns
    # 1. n1-point transforms down the columns, twiddle w_n^(j2 k1), send layout [s][j2 local][k1 local]
    send = col(x_cols.reshape(-1), n1, c2, world, n1 * n2, rank * c2, SWAP_IN if inverse else 0)
    # 2. one all-to-all: block s goes to rank s (through the process group whenever there is one,
    # a one-rank group included)
    if grouped:
        recv = torch.empty_like(send)
        dist.all_to_all_single(recv, send, group=group)
    else:
        recv = send
    # recv[s][j2 local][k1 local] is element (j2 = s c2 + j2 local, k1 local) of an n2 x r1 matrix
    # 3. n2-point transforms down its columns, row-wise: [k1 local][k2]
    out = col(recv, n2, r1, 1, 0, 0, SWAP_OUT if inverse else 0)
    return out.view(r1, n2)
