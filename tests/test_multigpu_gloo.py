"""Multi-rank host logic on the CPU (gloo, world size 2): the shards of a batch and of an uneven
batch cover every transform exactly once, ranks agree on the slowest rank's time, and transforms
computed rank by rank then gathered equal the single-process result. The transform here is the
oracle's CPU restatement standing in for the GPU kernel: what is tested is the sharding, not the
FFT.
"""
from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank: int, world: int, port: int, q):
    import torch
    import torch.distributed as dist

    import oracle
    from onefft_b200.shard import max_over_ranks, shard_batch, shard_uneven

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # uniform batch: contiguous ranges
        n, batch = 64, 37
        x, _ = oracle.gen_uniform(2 * n * batch, 5)
        first, count = shard_batch(batch, world, rank)
        mine = np.concatenate([oracle.port_fft(x[2 * n * b:2 * n * (b + 1)]) for b in range(first, first + count)])
        parts = [None] * world
        dist.all_gather_object(parts, (first, count, mine))
        # uneven batch: balanced by work
        rng = np.random.default_rng(1)
        log2n = rng.integers(0, 12, 200)
        shards = shard_uneven(log2n, world)
        t = max_over_ranks(0.5 + rank)
        q.put((rank, parts, [s.tolist() for s in shards], t))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_reduce(oracle):
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    n, batch = 64, 37
    x, _ = oracle.gen_uniform(2 * n * batch, 5)
    whole = np.concatenate([oracle.port_fft(x[2 * n * b:2 * n * (b + 1)]) for b in range(batch)])
    for rank, parts, shards, t in results:
        assert t == pytest.approx(1.5)  # the slowest rank's time, on every rank
        parts = sorted(parts, key=lambda p: p[0])
        assert sum(p[1] for p in parts) == batch
        assert [p[0] for p in parts] == [0, parts[0][1]]
        assert np.array_equal(np.concatenate([p[2] for p in parts]), whole)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(200))
    # both ranks computed the same uneven split
    assert results[0][2] == results[1][2]


def cpu_columns(x, n, cols, blocks, big_n, col0, flags):
    """CPU stand-in for the column-transform kernels: the oracle's FP64 statement of the same
    contract, back to complex64."""
    import torch

    import oracle
    return torch.from_numpy(oracle.columns_fp64(x.numpy(), n, cols, blocks, big_n, col0, flags).astype(np.complex64))


def dist_worker(rank: int, world: int, port: int, n1: int, n2: int, inverse: bool, q):
    import torch
    import torch.distributed as dist

    from onefft_b200.distributed import dist_fft

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(42)
        x = (rng.standard_normal(n1 * n2) + 1j * rng.standard_normal(n1 * n2)).astype(np.complex64)
        c2 = n2 // world
        cols = torch.from_numpy(np.ascontiguousarray(x.reshape(n1, n2)[:, rank * c2:(rank + 1) * c2]))
        out = dist_fft(cols, n1, n2, inverse=inverse, columns=cpu_columns)
        q.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,inverse", [(2, False), (4, False), (2, True)])
def test_distributed_four_step_one_all_to_all(world, inverse):
    n1, n2 = 64, 128
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=dist_worker, args=(r, world, port, n1, n2, inverse, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(42)
    x = (rng.standard_normal(n1 * n2) + 1j * rng.standard_normal(n1 * n2)).astype(np.complex64)
    z = x.astype(np.complex128)
    want = np.fft.ifft(z) * z.size if inverse else np.fft.fft(z)
    r1 = n1 // world
    for rank, blk in res.items():
        # block element [k1 - rank r1][k2] = X[k1 + n1 k2]
        k1 = np.arange(rank * r1, (rank + 1) * r1)[:, None]
        k2 = np.arange(n2)[None, :]
        ref = want[k1 + n1 * k2]
        assert np.linalg.norm(blk - ref) / np.linalg.norm(ref) < 1e-6


def emulate_ranks(x, n1, n2, world, columns, inverse=False):
    """The distributed four-step's data path with the exchange done by indexing, all ranks in one
    process: returns the (n1, n2) array of row blocks, [k1][k2] = X[k1 + n1 k2]."""
    c2, r1 = n2 // world, n1 // world
    m = x.reshape(n1, n2)
    sends = [columns(np.ascontiguousarray(m[:, r * c2:(r + 1) * c2]).reshape(-1), n1, c2, world, n1 * n2, r * c2,
                     1 if inverse else 0).reshape(world, c2 * r1) for r in range(world)]
    rows = []
    for r in range(world):
        recv = np.concatenate([sends[s][r] for s in range(world)])  # rank s's block for rank r
        rows.append(columns(recv, n2, r1, 1, 0, 0, 2 if inverse else 0).reshape(r1, n2))
    return np.concatenate(rows)


@pytest.mark.parametrize("world,n1,n2", [(1, 16, 32), (2, 64, 32), (4, 32, 128), (8, 128, 64)])
def test_column_contract_composes_to_the_transform(oracle, world, n1, n2):
    """The two column-transform steps and the exchange, on the oracle's FP64 statement of the
    column contract, give the n1 n2-point transform (forward and inverse)."""
    rng = np.random.default_rng(7)
    x = rng.standard_normal(n1 * n2) + 1j * rng.standard_normal(n1 * n2)
    for inverse in (False, True):
        got = emulate_ranks(x, n1, n2, world, oracle.columns_fp64, inverse)
        want = np.fft.ifft(x) * x.size if inverse else np.fft.fft(x)
        ref = want.reshape(n2, n1).T  # [k1][k2] = X[k1 + n1 k2]
        assert np.abs(got - ref).max() < 1e-9 * np.abs(ref).max()


def test_shard_balance():
    from onefft_b200.shard import shard_batch, shard_uneven, transform_cost
    assert [shard_batch(10, 3, r) for r in range(3)] == [(0, 4), (4, 3), (7, 3)]
    rng = np.random.default_rng(0)
    log2n = rng.integers(4, 17, 20000)
    for world in (2, 4, 8):
        shards = shard_uneven(log2n, world)
        loads = [transform_cost(log2n[s]).sum() for s in shards]
        assert max(loads) / min(loads) < 1.01
    with pytest.raises(ValueError):
        shard_batch(4, 2, 2)
