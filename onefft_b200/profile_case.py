"""Runs one transform shape a few times, for an external profiler (ncu) to capture.

    python -m onefft_b200.profile_case --log2n 24 [--split 8,8,8 --cols 4,4,4] [--batch 1] [--reps 3]
    python -m onefft_b200.profile_case --log2n 25 --split 8,7,10 --cols 4,4,3 --tma
    python -m onefft_b200.profile_case --log2n 12 --batch 4096            # the batched kernel
    python -m onefft_b200.profile_case --uneven 2000                      # the uneven-batch kernel
    python -m onefft_b200.profile_case --log2n 13 --batch 512 --loss      # fused loss + gradient
    python -m onefft_b200.profile_case --log2n 16 --batch 256 --bf16x3    # split-BF16 tensor cores
    python -m onefft_b200.profile_case --log2n 24 --split 8,8,8 --cols 4,4,4 --tma --chunk 4 --fuse-lag 1
                                                                          # fused passes 0+1
    python -m onefft_b200.profile_case --log2n 12 --columns 32768,8,30,3  # column transform:
                               # n = 2^12, cols, blocks, log2 big_n, rank (col0 = rank cols: rank 3 of 2^30 / 8)

Inputs are seeded standard-normal values on the device; the plan (and its table kernels) is
built before the timed transforms, so `ncu -k regex:k_pass -s <n>` can skip to them.
"""
from __future__ import annotations

import argparse

import numpy as np
import torch

import onefft_b200 as ofb


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--log2n", type=int, default=12)
    ap.add_argument("--split", default="")
    ap.add_argument("--cols", default="")
    ap.add_argument("--batch", type=int, default=1)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--inverse", action="store_true")
    ap.add_argument("--chunk", type=int, default=0, help="three passes: log2 last-digit columns per chunk")
    ap.add_argument("--tma", action="store_true", help="with --split: TMA-staged passes")
    ap.add_argument("--loss", action="store_true", help="the fused weighted-power loss and gradient")
    ap.add_argument("--bf16x3", action="store_true", help="the split-BF16 tensor-core plan (three terms)")
    ap.add_argument("--bf16x6", action="store_true", help="the split-BF16 tensor-core plan (six terms)")
    ap.add_argument("--fuse-lag", type=int, default=0, help="with --chunk and --tma: fused passes 0+1")
    ap.add_argument("--no-l2-keep", action="store_true", help="with --split: no L2 eviction hints")
    ap.add_argument("--uneven", type=int, default=0, help="run an uneven batch of this many transforms")
    ap.add_argument("--columns", default="", help="cols,blocks,log2 big_n,rank: the column transform of "
                                                  "an n x cols matrix with col0 = rank cols (onefft_columns_execute)")
    args = ap.parse_args()
    g = torch.Generator(device="cuda").manual_seed(7)
    if args.columns:
        cols, blocks, lbig, rank = (int(v) for v in args.columns.split(","))
        n = 1 << args.log2n
        c = ofb.Columns(n, cols, blocks, (1 << lbig) if lbig else 0, rank * cols)
        x = torch.randn(n * cols, dtype=torch.complex64, device="cuda", generator=g)
        y = torch.empty_like(x)
        for _ in range(args.reps):
            c.execute(x.data_ptr(), y.data_ptr(), ofb.SWAP_IN | ofb.SWAP_OUT if args.inverse else 0)
        torch.cuda.synchronize()
        print(f"columns n=2^{args.log2n} x {cols}, blocks {blocks}, big_n 2^{lbig}: {args.reps} runs")
        return
    if args.uneven:
        rng = np.random.default_rng(7)
        log2n = rng.integers(4, 17, args.uneven).astype(np.int32)
        inv = (rng.random(args.uneven) < 0.5).astype(np.int32)
        off = np.concatenate([[0], np.cumsum(1 << log2n.astype(np.int64))[:-1]])
        b = ofb.UnevenBatch(log2n, inv, off)
        x = torch.randn(2 * b.span, device="cuda", generator=g)
        y = torch.empty_like(x)
        for _ in range(args.reps):
            b.execute(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        print(f"uneven batch of {args.uneven} transforms, {b.span} values: {args.reps} runs")
        return
    n = 1 << args.log2n
    split = tuple(int(v) for v in args.split.split(",")) if args.split else None
    cols = tuple(int(v) for v in args.cols.split(",")) if args.cols else None
    if args.bf16x3 or args.bf16x6:
        plan = ofb.Plan(n, bf16x3=args.bf16x3, bf16x6=args.bf16x6)
    else:
        plan = ofb.Plan(n, split=split, cols=cols, chunk=args.chunk, tma=args.tma, fuse_lag=args.fuse_lag,
                        l2_keep=not args.no_l2_keep)
    if args.loss:
        x = torch.randn(2 * n * args.batch, device="cuda", generator=g)
        w = torch.rand(n, device="cuda", generator=g)
        grad = torch.empty_like(x)
        loss = torch.zeros(1, dtype=torch.float64, device="cuda")
        for _ in range(args.reps):
            rc = ofb.lib().onefft_dev_weighted_power_loss(plan.handle, x.data_ptr(), w.data_ptr(), grad.data_ptr(),
                                                          args.batch, loss.data_ptr(), None)
            if rc:
                raise RuntimeError(ofb.last_error())
        torch.cuda.synchronize()
        print(f"fused loss n=2^{args.log2n} x {args.batch}: {args.reps} runs, loss {loss.item():.6g}")
        return
    x = torch.randn(2 * n * args.batch, device="cuda", generator=g)
    y = torch.empty_like(x)
    f = plan.dev_inverse if args.inverse else plan.dev_forward
    for _ in range(args.reps):
        f(x.data_ptr(), y.data_ptr(), args.batch)
    torch.cuda.synchronize()
    print(f"n=2^{args.log2n} x {args.batch}, passes {plan.passes()}: {args.reps} runs")


if __name__ == "__main__":
    main()
