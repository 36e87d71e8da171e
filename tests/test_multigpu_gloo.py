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


def _numpy_fft_last_dim(t):
    """CPU stand-in for the GPU kernels: FP64 FFT along the last dimension, back to complex64."""
    import torch
    return torch.from_numpy(np.fft.fft(t.numpy().astype(np.complex128), axis=-1).astype(np.complex64))


def dist_worker(rank: int, world: int, port: int, n1: int, n2: int, q):
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
        out = dist_fft(cols, n1, n2, fft_last_dim=_numpy_fft_last_dim)
        q.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 4])
def test_distributed_four_step_one_all_to_all(world):
    n1, n2 = 64, 128
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=dist_worker, args=(r, world, port, n1, n2, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.default_rng(42)
    x = (rng.standard_normal(n1 * n2) + 1j * rng.standard_normal(n1 * n2)).astype(np.complex64)
    want = np.fft.fft(x.astype(np.complex128))
    r1 = n1 // world
    for rank, blk in res.items():
        # block element [k1 - rank r1][k2] = X[k1 + n1 k2]
        k1 = np.arange(rank * r1, (rank + 1) * r1)[:, None]
        k2 = np.arange(n2)[None, :]
        ref = want[k1 + n1 * k2]
        assert np.linalg.norm(blk - ref) / np.linalg.norm(ref) < 1e-6


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
