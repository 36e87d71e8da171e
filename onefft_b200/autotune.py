"""Autotuner of the pass split and tile widths per transform size.

    python -m onefft_b200.autotune [--min 15] [--max 27] [--out tuned.json]

For every log2 n in range it enumerates candidate shapes — two or three passes with lengths
2^4 .. 2^12, tile widths of 4, 8 or 16 columns per block, L2 evict-last stores on or off — builds
each as a plan (onefft_plan_create_tiles), checks its forward result against the default plan,
times the forward transform with CUDA events (L2 flushed before every repetition), and prints
the fastest shape per size as the C table used by onefft_api.cu (tuned_shape) plus a JSON record.

    python -m onefft_b200.autotune --uneven

tunes the uneven batch instead: the in-block two-pass split of each size 2^13 .. 2^16 among the
compiled candidates (uneven.h kUnevenSplits), printed as uneven.h's kUnevenTunedSplit.

    python -m onefft_b200.autotune --batched

tunes the one-kernel sizes 2^4 .. 2^14: whole transforms per thread block (the default 4096 / n,
half or twice that), printed as onefft_api.cu's kBatchedTunedLogC.

    python -m onefft_b200.autotune --fused [--min 22] [--max 30]

times, for the three-pass sizes, the first two passes fused into one persistent kernel
(fft_tma.cu k_pass01_fused): every compiled tile pair, chunk size of the last digit and lag of
pass 1 behind pass 0, with and without the L2 hints, against the current table's shape; each
result must equal the separate passes bit for bit. The L2 is flushed before each repetition by
reading a 512 MiB buffer (clean lines, so no write-backs land in the timed region). Prints the
table rows with the fuse_lag field.
"""
from __future__ import annotations

import argparse
import itertools
import json
import sys

import torch

import onefft_b200 as ofb


def tile_ok(l: int, c: int) -> bool:
    return 4 <= l <= 12 and c <= 4 and l + c <= 14 and (c >= 2 or (c == 1 and l >= 10))


def tma_ok(l: int, c: int) -> bool:
    """Tile shapes with a bulk-tensor-copy kernel (fft_tma.cu, pass_tma_supported)."""
    return 6 <= l <= 12 and 1 <= c <= 4 and l + c <= 14 and (l, c) in {
        (12, 2), (12, 1), (11, 1), (11, 2), (10, 1), (10, 2), (10, 3), (9, 2), (9, 3), (9, 4), (8, 2), (8, 3), (8, 4),
        (7, 3), (7, 4), (6, 4)}


def pass_log_c_default(log_l: int) -> int:
    """The library's default tile width of a pass (pass_log_c in fft_kernels.cu)."""
    return 4 if log_l <= 9 else 3 if log_l == 10 else 2


def candidates(m: int):
    """(log2 lengths, log2 tile widths, log2 chunk) shapes worth timing for 2^m."""
    out = []
    # two passes
    for l0 in range(4, 13):
        l1 = m - l0
        if 4 <= l1 <= 12:
            for c0 in (1, 2, 3, 4):
                for c1 in (1, 2, 3, 4):
                    if tile_ok(l0, c0) and tile_ok(l1, c1) and l0 + c0 >= 11 and l1 + c1 >= 11:
                        out.append(((l0, l1), (c0, c1), 0))
    # three passes, balanced lengths; passes 0+1 whole or in L2-sized chunks of the last digit
    for ls in itertools.product(range(5, 13), repeat=3):
        if sum(ls) != m or max(ls) - min(ls) > 3:
            continue
        for cs in itertools.product((2, 3, 4), repeat=3):
            if all(tile_ok(l, c) and l + c >= 11 for l, c in zip(ls, cs)) and cs[0] <= ls[2]:
                out.append((ls, cs, 0))
                for mib in (16, 32, 64):
                    g = (mib << 20).bit_length() - 1 - 3 - ls[0] - ls[1]  # 8 bytes per value
                    if cs[0] <= g < ls[2]:
                        out.append((ls, cs, g))
    return out


# Tile pairs (L0, C0, L1, C1) of the fused passes 0+1 (fft_tma.cu, pass01_fused_supported).
FUSED_PAIRS = {(8, 4, 9, 3), (8, 3, 8, 3), (8, 4, 8, 4), (8, 3, 7, 4), (9, 3, 9, 3), (10, 3, 10, 3),
               (10, 3, 11, 2)}


def fused_candidates(m: int):
    """(lengths, widths, chunk bits, lag) of fused three-pass shapes for 2^m."""
    out = []
    for l0, c0, l1, c1 in sorted(FUSED_PAIRS):
        l2 = m - l0 - l1
        if not 4 <= l2 <= 12:
            continue
        for c2 in (2, 3, 4):
            if not tile_ok(l2, c2) or l2 + c2 < 11 or c0 > l2:
                continue
            for g in range(c0, l2 + 1):
                chunks = 1 << (l2 - g)
                for lag in (1, 2, 3):
                    if lag <= chunks:
                        out.append(((l0, l1, l2), (c0, c1, c2), g, lag))
    return out


def tune_fused(lo: int, hi: int, reps: int) -> dict:
    flush = torch.ones(1 << 27, dtype=torch.float32, device="cuda")  # read to evict the L2

    def timed(plan, x, y):
        stream = torch.cuda.current_stream()
        ts = []
        for r in range(reps + 2):
            flush.max()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            plan.dev_forward(x.data_ptr(), y.data_ptr(), 1, stream.cuda_stream)
            e1.record(stream)
            torch.cuda.synchronize()
            if r >= 2:
                ts.append(e0.elapsed_time(e1) * 1e3)
        ts.sort()
        return ts[len(ts) // 2]

    results = {}
    for m in range(lo, hi + 1):
        n = 1 << m
        x = torch.randn(2 * n, device="cuda")
        y = torch.empty_like(x)
        ref = torch.empty_like(x)
        base = ofb.Plan(n)
        base_us = timed(base, x, y)
        rows = []
        separate = {}
        for ls, cs, g, lag in fused_candidates(m):
            if (ls, cs) not in separate:
                p = ofb.Plan(n, split=ls, cols=cs, tma=True)
                p.dev_forward(x.data_ptr(), ref.data_ptr(), 1)
                torch.cuda.synchronize()
                separate[(ls, cs)] = ref.clone()
                p.destroy()
            for keep in (False, True):
                try:
                    p = ofb.Plan(n, split=ls, cols=cs, chunk=g, tma=True, fuse_lag=lag, l2_keep=keep)
                except ValueError:
                    continue
                y.fill_(float("nan"))
                p.dev_forward(x.data_ptr(), y.data_ptr(), 1)
                torch.cuda.synchronize()
                if p.status() != 0 or not torch.equal(y, separate[(ls, cs)]):
                    raise RuntimeError(f"2^{m} {ls} {cs} chunk {g} lag {lag}: fused result differs")
                us = timed(p, x, y)
                p.destroy()
                rows.append({"len": ls, "cols": cs, "chunk": g, "lag": lag, "l2_keep": keep, "us": us})
        rows.sort(key=lambda r: r["us"])
        best = rows[0] if rows else None
        results[m] = {"base_us": base_us, "best": best, "top": rows[:8]}
        if best:
            print(f"m={m}: fused best {best['len']} cols {best['cols']} chunk {best['chunk']} lag {best['lag']} "
                  f"keep={best['l2_keep']} {best['us']:.1f} us; current table {base_us:.1f} us", flush=True)
        base.destroy()
        del x, y, ref, separate
        torch.cuda.empty_cache()
    print("// fused shapes: {npass, {len}, {cols}, l2_keep, chunk, tma, fuse_lag}")
    for m, r in results.items():
        b = r["best"]
        if b and b["us"] < r["base_us"]:
            ls, cs = b["len"], b["cols"]
            print(f"    /* {m} */ {{3, {{{ls[0]}, {ls[1]}, {ls[2]}}}, {{{cs[0]}, {cs[1]}, {cs[2]}}}, "
                  f"{int(b['l2_keep'])}, {b['chunk']}, 1, {b['lag']}}},  // {b['us']:.1f} us (was {r['base_us']:.1f})")
    return results


def time_plan(plan, x, y, reps: int, flush) -> float:
    stream = torch.cuda.current_stream()
    ts = []
    for r in range(reps + 2):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.dev_forward(x.data_ptr(), y.data_ptr(), 1, stream.cuda_stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if r >= 2:
            ts.append(e0.elapsed_time(e1) * 1e3)
    ts.sort()
    return ts[len(ts) // 2]


# ONEFFT_COLS_PIPELINED: the persistent double-buffered one-kernel form of 2^12 and 2^13
PIPELINED = 15


def batched_log_c_candidates(l: int) -> list[int]:
    """Transforms per block (log2) compiled for the one-kernel size 2^l (fft_kernels.cu,
    batched_log_c_supported): the default 4096 / n, half and twice that up to 8192 values; at 2^12
    and 2^13 also the pipelined form (fft_tma.cu, batched_pipe_supported)."""
    b = max(0, 12 - l)
    out = [c for c in (b - 1, b, b + 1) if c == b or (c >= 0 and l + c <= 13)]
    return out + ([PIPELINED] if l in (12, 13) else [])


def tune_batched(reps: int = 9) -> dict:
    """Transforms per block of the one-kernel sizes 2^4 .. 2^14: for each size a batch of
    2^25 / n transforms (256 MiB), forward, with every compiled width; each result must equal the
    default's bit for bit. Prints the fastest width per size as onefft_api.cu's
    kBatchedTunedLogC."""
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    out = {}
    for l in range(4, 15):
        n = 1 << l
        batch = (1 << 25) // n
        x = torch.randn(2 * n * batch, device="cuda")
        ref = torch.empty_like(x)
        y = torch.empty_like(x)
        p0 = ofb.Plan(n, split=(l,), cols=(max(0, 12 - l),))
        p0.dev_forward(x.data_ptr(), ref.data_ptr(), batch)
        p0.destroy()
        times = {}
        for c in batched_log_c_candidates(l):
            plan = ofb.Plan(n, split=(l,), cols=(c,))
            y.fill_(float("nan"))
            plan.dev_forward(x.data_ptr(), y.data_ptr(), batch)
            torch.cuda.synchronize()
            if not torch.equal(y, ref):
                raise RuntimeError(f"2^{l} with 2^{c} transforms per block differs from the default")
            ts = []
            for r in range(reps + 2):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                plan.dev_forward(x.data_ptr(), y.data_ptr(), batch)
                e1.record()
                torch.cuda.synchronize()
                if r >= 2:
                    ts.append(e0.elapsed_time(e1) * 1e3)
            plan.destroy()
            ts.sort()
            times[c] = ts[len(ts) // 2]
        best = min(times, key=times.get)
        out[l] = {"log_c": best, "us": times}
        label = lambda c: "pipelined" if c == PIPELINED else f"{1 << c}/block"  # noqa: E731
        print(f"batched 2^{l} x {batch}: " + ", ".join(f"{label(c)} {t:.1f} us" for c, t in times.items()) +
              f" -> {label(best)}", flush=True)
        del x, ref, y
        torch.cuda.empty_cache()
    table = [-1] * 15
    for l, r in out.items():
        table[l] = r["log_c"]
    print("static const int kBatchedTunedLogC[kMaxSingleLog2 + 1] = {" + ", ".join(str(v) for v in table) + "};")
    return out


def tune_uneven(reps: int = 9) -> dict:
    """In-block split per size 2^13 .. 2^16 of the uneven batch: for each size, 2^25 / n
    transforms of that size (256 MiB, half of them inverse) executed with every compiled split
    (onefft_uneven_create_split); prints the fastest choice per size as the table
    kUnevenTunedSplit of uneven.h. Choice 0 everywhere runs in the kernel compiled with those
    splits inlined, any other combination in the kernel that calls the split chosen at run time,
    so an alternative must win despite its call overhead; the tuned combination then gets a
    kernel of its own with its splits inlined."""
    import numpy as np
    out = {}
    for m in range(13, 17):
        n = 1 << m
        count = (1 << 25) // n
        rng = np.random.default_rng(m)
        log2n = np.full(count, m, np.int32)
        inverse = (rng.random(count) < 0.5).astype(np.int32)
        offset = np.arange(count, dtype=np.int64) * n
        x = torch.randn(2 * n * count, device="cuda")
        y = torch.empty_like(x)
        times = []
        for choice in range(3):
            b = ofb.UnevenBatch(log2n, inverse, offset, split={m: choice})
            ts = []
            for r in range(reps + 2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                b.execute(x.data_ptr(), y.data_ptr())
                e1.record()
                torch.cuda.synchronize()
                if r >= 2:
                    ts.append(e0.elapsed_time(e1) * 1e3)
            b.destroy()
            ts.sort()
            times.append(ts[len(ts) // 2])
        best = int(np.argmin(times))
        out[m] = {"choice": best, "us": times}
        print(f"uneven 2^{m} x {count}: " + ", ".join(f"split {c}: {t:.1f} us" for c, t in enumerate(times)) +
              f" -> {best}", flush=True)
        del x, y
        torch.cuda.empty_cache()
    table = [0] * 17
    for m, r in out.items():
        table[m] = r["choice"]
    print("constexpr int kUnevenTunedSplit[4] = {" + ", ".join(str(table[m]) for m in range(13, 17)) + "};")
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--min", type=int, default=15)
    ap.add_argument("--max", type=int, default=27)
    ap.add_argument("--reps", type=int, default=7)
    ap.add_argument("--out", default=None)
    ap.add_argument("--max-candidates", type=int, default=1000)
    ap.add_argument("--tma-only", action="store_true", help="only TMA-staged variants, no chunked passes")
    ap.add_argument("--chunked-only", action="store_true", help="only TMA-staged variants with L2-resident chunks")
    ap.add_argument("--uneven", action="store_true", help="tune the uneven batch's in-block splits instead")
    ap.add_argument("--batched", action="store_true", help="tune the transforms per block of sizes 2^4 .. 2^14")
    ap.add_argument("--fused", action="store_true", help="tune the fused first two passes of three-pass sizes")
    ap.add_argument("--split", default="", help="time only this split (log2 lengths, e.g. 12,12) against the "
                                                 "default plan, with --cols tile widths (e.g. 2,2)")
    ap.add_argument("--cols", default="")
    args = ap.parse_args()
    if args.fused:
        res = tune_fused(max(args.min, 22), args.max, args.reps)
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)
        return
    if args.uneven or args.batched:
        res = tune_uneven() if args.uneven else tune_batched()
        if args.out:
            with open(args.out, "w") as f:
                json.dump(res, f, indent=1)
        return
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    results = {}
    for m in range(args.min, args.max + 1):
        n = 1 << m
        x = torch.randn(2 * n, device="cuda")
        y = torch.empty_like(x)
        ref = ofb.Plan(n)
        ref.dev_forward(x.data_ptr(), y.data_ptr())
        torch.cuda.synchronize()
        want = y.clone()
        scale = want.abs().max().item()
        best = None
        rows = []
        cands = candidates(m)[: args.max_candidates]
        if args.split:
            ls = tuple(int(v) for v in args.split.split(","))
            cs = tuple(int(v) for v in args.cols.split(",")) if args.cols else tuple(pass_log_c_default(l) for l in ls)
            cands = [(ls, cs, 0)]
        variants = [(ls, cs, g, keep, tma) for ls, cs, g in cands for keep in (True, False)
                    for tma in ((False, True) if any(tma_ok(l, c) for l, c in zip(ls, cs)) else (False,))]
        if args.tma_only:
            variants = [v for v in variants if v[4] and not v[2]]
        if args.chunked_only:
            variants = [v for v in variants if v[4] and v[2]]
        for ls, cs, g, keep, tma in variants:
            if True:
                try:
                    p = ofb.Plan(n, split=ls, cols=cs, l2_keep=keep, chunk=g, tma=tma)
                except ValueError:
                    continue
                y.zero_()
                p.dev_forward(x.data_ptr(), y.data_ptr())
                torch.cuda.synchronize()
                err = (y - want).abs().max().item() / scale
                if err > 1e-5:
                    print(f"m={m} {ls} {cs} chunk={g} keep={keep}: result differs ({err:.2e}), skipped",
                          file=sys.stderr)
                    p.destroy()
                    continue
                us = time_plan(p, x, y, args.reps, flush)
                p.destroy()
                rows.append({"len": ls, "cols": cs, "l2_keep": keep, "chunk": g, "tma": tma, "us": us,
                             "gbs_16n": 16 * n / us / 1e3})
                if best is None or us < best["us"]:
                    best = rows[-1]
        base_us = time_plan(ref, x, y, args.reps, flush)
        ref.destroy()
        results[m] = {"best": best, "default_us": base_us, "all": sorted(rows, key=lambda r: r["us"])[:10]}
        print(f"m={m}: best {best['len']} cols {best['cols']} chunk {best['chunk']} keep={best['l2_keep']} "
              f"tma={best['tma']} {best['us']:.1f} us ({best['gbs_16n']:.0f} GB/s of 16n); default {base_us:.1f} us",
              flush=True)
        del x, y, want
        torch.cuda.empty_cache()
    print("// tuned shapes: {npass, {len}, {cols}, l2_keep, chunk, tma} for log2 n =", args.min, "..", args.max)
    for m, r in results.items():
        b = r["best"]
        ls = list(b["len"]) + [0] * (3 - len(b["len"]))
        cs = list(b["cols"]) + [0] * (3 - len(b["cols"]))
        print(f"    /* {m} */ {{{len(b['len'])}, {{{ls[0]}, {ls[1]}, {ls[2]}}}, {{{cs[0]}, {cs[1]}, {cs[2]}}}, "
              f"{int(b['l2_keep'])}, {b['chunk']}, {int(b['tma'])}}},")
    if args.out:
        with open(args.out, "w") as f:
            json.dump(results, f, indent=1)


if __name__ == "__main__":
    main()
