"""Benchmark of the B200 FFT path on the batched + large-transform workload.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (per GPU): the batched FP32 complex FFT configuration — 16384 independent transforms of
n = 4096 (512 MiB interleaved complex64) plus single transforms of n = 2^20, 2^24 and 2^27 —
with standard-normal inputs from a seeded generator. One step runs every item forward (x -> y)
and then inverse (y -> z) through the C ABI's device-pointer entry point on the current torch
stream. Timing: CUDA events over exactly K steps, barrier + synchronize on both sides, max over
ranks; each item's buffers are larger than L2 except n = 2^20, which the 1.5 GiB of other traffic
in a step evicts between its uses.

Printed (rank 0, one JSON line):
  value         sum over items of 2 * 5 n log2(n) batch / step time, GFLOP/s (the reference's
                unit, 5 n log2 n per transform and direction), summed over ranks
  e2e           the same metric through the drop-in host-pointer calls (onefft_plan_forward /
                _inverse for the single transforms, onefft_plan_forward_batched / _inverse for
                the batch) on pinned host buffers: every step copies all inputs in and all
                outputs back inside the timed region; per item a forward and an inverse host
                thread, so step s+1's uploads overlap step s's downloads (full-duplex PCIe)
  roofline      the item with the largest share of device time, against the measured HBM copy
                bandwidth: algorithmic bytes 16 n per transform and direction over its time
  cpu_baseline  the reference library compiled from its own sources, on this host's cores, on
                the same workload: one shared plan per size, threads pull transforms (largest
                first) from an atomic counter and call onefft_plan_forward/_inverse
  detail        per item: microseconds per direction, GFLOP/s, GB/s of 16 n, passes, launches

With --impl reference only rank 0 runs: it times the reference CPU library on the same workload
with all host threads and prints the same metric with "impl": "reference". Multi-GPU (torchrun,
one process per GPU): every rank runs the whole workload on its own data (weak scaling, no
collective on the data path).

With --dist the step is instead ONE forward transform of 2^27 N values distributed over the N
ranks (2^27 per rank): each rank's column transform writes the all-to-all send layout, NCCL's
all_to_all_single exchanges the blocks, and a second column transform gives the rank's rows of
the result (onefft_b200/distributed.py); same timing rules, metric 5 N log2 N per step.
"""
from __future__ import annotations

import argparse
import concurrent.futures
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# (name, log2 n, batch)
ITEMS = [("batch 16384 x 2^12", 12, 16384), ("single 2^20", 20, 1), ("single 2^24", 24, 1), ("single 2^27", 27, 1)]
METRIC = "5n*log2(n)/t GFLOP/s, FP32 c2c FFT (batched 16384x4096 + single 2^20, 2^24, 2^27; fwd+inv)"
WORKLOAD = {"workload": "batched FP32 complex FFT: 16384 x n=4096 plus single n=2^20, 2^24, 2^27, "
                        "forward then inverse each, interleaved complex64 in HBM",
            "items": [{"n": 1 << l, "batch": b} for _, l, b in ITEMS],
            "input": "standard normal re/im (seeded torch generator)",
            "l2": "inputs larger than L2 except n=2^20 (8 MiB), evicted by the other 1.5 GiB of traffic per step"}


def flops(log2n: int, batch: int) -> float:
    return 5.0 * (1 << log2n) * log2n * batch


STEP_FLOPS = sum(2 * flops(l, b) for _, l, b in ITEMS)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-configs", action="store_true")
    ap.add_argument("--e2e-schedule", default="pairs", choices=["pairs", "offset", "chains"],
                    help="host threads of the end-to-end measurement (see the e2e section)")
    ap.add_argument("--e2e-chains", type=int, default=2, help="chains per item of --e2e-schedule chains")
    ap.add_argument("--dist", action="store_true",
                    help="instead of the benchmark step: ONE forward transform of 2^27 N values distributed over "
                         "the N ranks (distributed four-step: column transform, NCCL all-to-all, column transform)")
    return ap.parse_args()


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def ncu_traffic(key: str):
    """DRAM bytes per launch of a kernel from the committed ncu summary, or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "ncu_dram_bytes.json")) as f:
            return json.load(f).get(key)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            time.sleep(0.3)
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
                power.append(float(p[3]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# ---- CPU side: the reference library on the host cores -----------------------------------------


def cpu_workload_descriptors():
    """Descriptors (log2n, complex offset, inverse) of one step, largest transforms first, each
    direction in its own region (the CPU harness transforms in -> out at the same offset)."""
    descs = []
    off = 0
    for _, l, b in ITEMS:
        n = 1 << l
        for inv in (0, 1):
            for i in range(b):
                descs.append((l, off + i * n, inv))
            off += n * b
    descs.sort(key=lambda d: -d[0])
    log2n = np.array([d[0] for d in descs], np.int32)
    offset = np.array([d[1] for d in descs], np.int64)
    inverse = np.array([d[2] for d in descs], np.int32)
    return log2n, offset, inverse, off


def cpu_step_times(steps: int, warmup: int, samples_per_step: int = 1):
    import oracle
    oracle.build()
    kind = "reference" if oracle.have_reference() else "port"
    cores = oracle.cpu_cores(kind)
    log2n, offset, inverse, span = cpu_workload_descriptors()
    rng = np.random.default_rng(12345)
    x = rng.standard_normal(2 * span, dtype=np.float32)
    out = np.empty_like(x)
    for _ in range(warmup):
        oracle.cpu_bench_uneven(log2n, offset, inverse, cores, x, out, 1, kind=kind)
    times = [oracle.cpu_bench_uneven(log2n, offset, inverse, cores, x, out, samples_per_step, kind=kind)
             for _ in range(steps)]
    if min(times) <= 0:
        raise RuntimeError("CPU reference run failed")
    return times, cores, kind, oracle.cpu_impl(kind)


def run_reference(args, rank: int):
    """--impl reference: the reference CPU library on this host, rank 0 only."""
    if rank != 0:
        return
    # a step is ~1-1.5 s of host work: the requested 20 + 5 steps take about half a minute
    steps = max(1, args.steps)
    warmup = max(1, args.warmup)
    times, cores, kind, impl = cpu_step_times(steps, warmup)
    t = sum(times) / len(times)
    value = STEP_FLOPS / t / 1e9
    sample = (f"the whole step per timed step ({steps} steps after {warmup} warm-up; {impl} kernels, "
              f"{cores} threads, largest transforms first)")
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": steps,
            "warmup": warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": dict(WORKLOAD, parallelism="host threads"),
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---- GPU side ------------------------------------------------------------------------------------


def pcie_ceiling(torch, nbytes: int = 1 << 30) -> dict:
    """Host <-> device copy bandwidth of this GPU with pinned buffers, as context for the end-to-end
    number: one direction alone, and both at once on two streams (what a step of host calls can
    reach at best). GB/s, best of three."""
    h_up = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    h_down = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    d_up = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_down = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn):
        best = float("inf")
        for _ in range(3):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            fn()
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return best

    def up():
        with torch.cuda.stream(s1):
            d_up.copy_(h_up, non_blocking=True)

    def down():
        with torch.cuda.stream(s2):
            h_down.copy_(d_down, non_blocking=True)

    def both():
        up()
        down()

    t_up, t_down, t_both = timed(up), timed(down), timed(both)
    del h_up, h_down, d_up, d_down
    return {"h2d_gbs": nbytes / t_up / 1e9, "d2h_gbs": nbytes / t_down / 1e9, "both_ways_gbs": 2 * nbytes / t_both / 1e9,
            "note": "1 GiB pinned copies, best of 3; a step moves h2d_bytes_per_step each way"}


def _time(torch, stream, fn, reps: int = 5, warm: int = 2) -> float:
    """Average seconds of fn() on the device (CUDA events on `stream`)."""
    for _ in range(warm):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps


def config1_latency(torch, ofb, L, stream):
    """One n = 1024 forward + inverse (the latency-bound configuration), as the reference's
    bench/bench.c:151-167 times it: the minimum over samples of one call pair, through the
    drop-in host API on pageable and on pinned host buffers (copies, launch and synchronisation
    included), and through the device-pointer entry points with a stream synchronisation; the
    reference library on one host core beside it."""
    n, log2n = 1024, 10
    pair_flops = 2 * 5.0 * n * log2n
    rng = np.random.default_rng(0xC0F1)
    xh = rng.uniform(-1, 1, 2 * n).astype(np.float32)
    yh, zh = np.empty_like(xh), np.empty_like(xh)
    xp = torch.from_numpy(xh).pin_memory()
    yp, zp = torch.empty_like(xp).pin_memory(), torch.empty_like(xp).pin_memory()
    plan = ofb.Plan(n)
    xd = xp.cuda()
    yd, zd = torch.empty_like(xd), torch.empty_like(xd)
    sptr = stream.cuda_stream

    def sample(fn, reps=400, warm=50):
        for _ in range(warm):
            fn()
        best = float("inf")
        for _ in range(reps):
            t0 = time.perf_counter()
            fn()
            best = min(best, time.perf_counter() - t0)
        return best

    def host_pageable():
        L.onefft_forward(xh.ctypes.data, yh.ctypes.data, n)
        L.onefft_inverse(yh.ctypes.data, zh.ctypes.data, n)

    def host_pinned():
        L.onefft_forward(xp.data_ptr(), yp.data_ptr(), n)
        L.onefft_inverse(yp.data_ptr(), zp.data_ptr(), n)

    def device():
        plan.dev_forward(xd.data_ptr(), yd.data_ptr(), 1, sptr)
        plan.dev_inverse(yd.data_ptr(), zd.data_ptr(), 1, sptr)
        stream.synchronize()

    t_pg, t_pn, t_d = sample(host_pageable), sample(host_pinned), sample(device)
    ok = bool(np.allclose(zh, xh * n, rtol=0, atol=1e-3 * n))
    res = {"us_host_api_pageable": 1e6 * t_pg, "us_host_api_pinned": 1e6 * t_pn, "us_device_pointers": 1e6 * t_d,
           "gflops_host_api_pinned": pair_flops / t_pn / 1e9, "round_trip_ok": ok,
           "note": "min over 400 samples of one forward + inverse pair (wall clock, synchronous)"}
    try:
        import oracle
        if oracle.have_reference():
            batch = 4096
            xb = np.tile(xh, batch)
            ob = np.empty_like(xb)
            t_f = oracle.cpu_bench_batched(n, batch, 1, False, xb, ob, 5) / batch
            t_i = oracle.cpu_bench_batched(n, batch, 1, True, xb, ob, 5) / batch
            res["us_reference_cpu_1thread"] = 1e6 * (t_f + t_i)
            res["reference_impl"] = oracle.cpu_impl()
    except Exception as e:  # reported, not fatal
        res["reference_error"] = str(e)
    plan.destroy()
    return res


def other_configs(torch, ofb, L, stream, peak):
    """The latency-bound n = 1024 pair, the uneven batch, the split-BF16 variant and the
    differentiable layer, each against the plain FP32 GPU path on the same data (accuracy of each
    is checked by the test suite)."""
    sptr = stream.cuda_stream
    out = {"config1 n=1024 fwd+inv latency": config1_latency(torch, ofb, L, stream)}
    g = torch.Generator(device="cuda").manual_seed(99)
    # uneven batch: 20000 transforms, log2 n uniform in 4..16, packed, half inverse
    rng = np.random.default_rng(0xC0F3)
    log2n = rng.integers(4, 17, 20000).astype(np.int32)
    inv = (rng.random(20000) < 0.5).astype(np.int32)
    off = np.concatenate([[0], np.cumsum(1 << log2n.astype(np.int64))[:-1]])
    ub = ofb.UnevenBatch(log2n, inv, off)
    x = torch.rand(2 * ub.span, device="cuda", generator=g) * 2 - 1
    y = torch.empty_like(x)
    t_u = _time(torch, stream, lambda: ub.execute(x.data_ptr(), y.data_ptr(), sptr))
    if ub.status() != 0:
        raise RuntimeError(f"uneven batch failed on the device: {ofb.last_error()}")
    plans = {m: ofb.Plan(1 << m) for m in range(4, 17)}
    base_in, base_out = x.data_ptr(), y.data_ptr()
    calls = [((L.onefft_dev_inverse_batched if i else L.onefft_dev_forward_batched), plans[m].handle,
              base_in + 8 * o, base_out + 8 * o) for m, i, o in zip(log2n.tolist(), inv.tolist(), off.tolist())]

    def per_transform():
        for f, h, a, b in calls:
            f(h, a, b, 1, sptr)

    t_p = _time(torch, stream, per_transform, reps=2, warm=1)
    # the plain path at its best: the same transforms already grouped by size and direction into
    # contiguous batches (the grouping copy is not timed), one batched call per group
    groups = []
    for m in range(4, 17):
        for d in (0, 1):
            sel = np.nonzero((log2n == m) & (inv == d))[0]
            if sel.size == 0:
                continue
            idx = torch.from_numpy((off[sel][:, None] + np.arange(1 << m)[None, :]).reshape(-1)).cuda()
            gx = torch.view_as_real(torch.view_as_complex(x.view(-1, 2))[idx]).reshape(-1).contiguous()
            groups.append((plans[m], d, int(sel.size), gx, torch.empty_like(gx)))

    def grouped():
        for p, d, cnt, gx, gy in groups:
            (p.dev_inverse if d else p.dev_forward)(gx.data_ptr(), gy.data_ptr(), cnt, sptr)

    t_g = _time(torch, stream, grouped)
    flops = float(sum(5.0 * (1 << m) * m for m in log2n.tolist()))
    out["uneven 20000 x 2^(4..16)"] = {
        "us_persistent": 1e6 * t_u, "us_plain_grouped": 1e6 * t_g, "us_per_transform_calls": 1e6 * t_p,
        "speedup_vs_grouped": t_g / t_u, "speedup_vs_per_transform": t_p / t_u,
        "gflops": flops / t_u / 1e9, "gbs_16n": 16 * ub.span / t_u / 1e9, "frac_hbm": 16 * ub.span / t_u / 1e9 / peak,
        "note": "one persistent launch vs (a) the plain FP32 path on the same transforms grouped by size and "
                "direction into contiguous batches, one onefft_dev_*_batched call per group (grouping copy not "
                "timed), and (b) one onefft_dev_*_batched call per transform; results equal the plain path bit "
                "for bit except 2^13/2^14 (tests/test_gpu_uneven.py)"}
    ub.destroy()
    del x, y, groups
    # split-BF16 tensor-core variants (3 and 6 product terms) vs plain FP32 on the same batches;
    # "accepted" is the library's own decision (a plan that requires acceptance is built only at
    # sizes where the variant met the FP32 error bound, measured by tests/test_gpu_bf16x3.py)
    for lg, batch in ((16, 256), (22, 16)):
        n = 1 << lg
        x = torch.randn(2 * n * batch, device="cuda", generator=g)
        y = torch.empty_like(x)
        fp = ofb.Plan(n)
        t_fp = _time(torch, stream, lambda: fp.dev_forward(x.data_ptr(), y.data_ptr(), batch, sptr))
        rec = {"us_fp32": 1e6 * t_fp}
        for terms, kw in ((3, {"bf16x3": True}), (6, {"bf16x6": True})):
            tc = ofb.Plan(n, **kw)
            t_tc = _time(torch, stream, lambda: tc.dev_forward(x.data_ptr(), y.data_ptr(), batch, sptr))
            tc.destroy()
            try:
                ofb.Plan(n, require_accepted=True, **kw).destroy()
                accepted = True
            except ValueError:
                accepted = False
            rec[f"us_bf16x{terms}"] = 1e6 * t_tc
            rec[f"time_ratio_fp32_over_bf16x{terms}"] = t_fp / t_tc
            rec[f"bf16x{terms}_accepted"] = accepted
        rec["note"] = ("errors against FP64 per term count in tests/test_gpu_bf16x3.py; a speedup at equal error "
                       "exists only where a variant is accepted and its time ratio exceeds 1")
        out[f"split-BF16 {batch} x 2^{lg}"] = rec
        fp.destroy()
        del x, y
    # distributed four-step: one rank's two column-transform calls for N = 2^30 over 8 ranks
    # (n1 = 2^10, n2 = 2^20: a 2^10 x 2^17 column block, 2^27 values, per rank; n1 = 2^10 keeps
    # step 1 to one pass of 1024-value tiles of 8 columns, which run near the copy bound, where
    # 4096-value columns would run their one pass at ~60 % of it)
    P, n1, n2, rank = 8, 1 << 10, 1 << 20, 3
    c2, r1 = n2 // P, n1 // P
    s1 = ofb.Columns(n1, c2, P, n1 * n2, rank * c2)
    s3 = ofb.Columns(n2, r1)
    xb = torch.randn(n1 * c2, dtype=torch.complex64, device="cuda", generator=g)
    yb, zb = torch.empty_like(xb), torch.empty_like(xb)
    t1 = _time(torch, stream, lambda: s1.execute(xb.data_ptr(), yb.data_ptr(), 0, sptr))
    t3 = _time(torch, stream, lambda: s3.execute(yb.data_ptr(), zb.data_ptr(), 0, sptr))
    moved = 16.0 * n1 * c2  # bytes read + written per pass
    exch = 8.0 * n1 * c2 * (P - 1) / P
    out["distributed 2^30 over 8 ranks, one rank's local steps"] = {
        "us_step1_columns_2^10_one_pass": 1e6 * t1, "us_step3_columns_2^20_two_passes": 1e6 * t3,
        "us_local": 1e6 * (t1 + t3), "gbs_step1": moved / t1 / 1e9, "gbs_step3_per_pass": 2 * moved / t3 / 1e9,
        "bytes_sent_per_rank": exch, "us_exchange_projected_at_770GBs": 1e6 * exch / 770e9,
        "note": "measured on one GPU: one rank's two onefft_columns_execute calls (transforms, the 2^30-point "
                "twiddle and the all-to-all layout inside the kernels); the NCCL all-to-all between them needs "
                "8 GPUs and was not run, its time is projected from the 770 GB/s measured peer copy; "
                "correctness in tests/test_gpu_distributed.py"}
    s1.destroy()
    s3.destroy()
    del xb, yb, zb
    # differentiable layer: forward + backward of sum |W * FFT(x)|^2, batch 512 x 8192
    from onefft_b200 import torch_fft
    n, batch = 8192, 512
    xc = torch.randn(batch, n, dtype=torch.complex64, device="cuda", generator=g).requires_grad_(True)
    wv = torch.rand(n, device="cuda", generator=g)

    def step():
        xc.grad = None
        torch_fft.weighted_power_loss(xc, wv).backward()

    def fused_step():
        xc.grad = None
        torch_fft.weighted_power_loss_fused(xc, wv).backward()

    t_s = _time(torch, stream, step)
    t_fu = _time(torch, stream, fused_step)
    t_f = _time(torch, stream, lambda: torch_fft._run("forward", xc.detach()))
    out["autograd 512 x 8192"] = {"ms_fwd_bwd": 1e3 * t_s, "ms_fwd_bwd_fused": 1e3 * t_fu,
                                  "fused_speedup": t_s / t_fu, "us_forward_kernel": 1e6 * t_f,
                                  "note": "loss and gradient checked against FP64 finite differences and the "
                                          "reference library; the fused kernel's gradient equals the unfused "
                                          "one bit for bit (tests/test_gpu_autograd.py)"}
    for p in plans.values():
        p.destroy()
    return out


def run_dist(args, world: int, rank: int, local_rank: int):
    """One transform of N = 2^27 world values over the ranks (weak scaling: 2^27 values, 1 GiB, per
    rank): n1 = 2^10 rows, n2 = N / 2^10 columns; per step each rank runs its column transform into
    the all-to-all send layout, the all-to-all, and the column transform of what it received
    (onefft_b200.distributed.dist_fft). Timed on the device with CUDA events, max over ranks."""
    import datetime

    import torch

    import onefft_b200 as ofb
    from onefft_b200.distributed import clear_cache, gpu_columns
    from onefft_b200.shard import max_over_ranks

    import socket

    import torch.distributed as dist

    torch.cuda.set_device(local_rank)
    # the exchange always runs through NCCL: under torchrun over the job's ranks, alone as a
    # one-rank group (NCCL's all-to-all copying the blocks to this GPU itself)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    else:
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    n1 = 1 << 10
    n2 = (1 << 17) * world
    if n1 // world < 16 or n2 > 1 << 24:
        raise SystemExit("--dist supports 1 .. 64 ranks")
    c2, r1 = n2 // world, n1 // world
    g = torch.Generator(device="cuda").manual_seed(77 + rank)
    x = torch.randn(n1 * c2, dtype=torch.complex64, device="cuda", generator=g)
    recv = torch.empty_like(x)
    L = ofb.lib()

    def step():
        send = gpu_columns(x, n1, c2, world, n1 * n2, rank * c2, 0)
        dist.all_to_all_single(recv, send)
        return gpu_columns(recv, n2, r1, 1, 0, 0, 0)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = L.onefft_debug_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    dist.barrier()
    launches = int(L.onefft_debug_launch_count() - launches0)
    clk = clocks.stop()
    t = max_over_ranks(e0.elapsed_time(e1) / 1e3, device="cuda") / args.steps
    N = n1 * n2
    clear_cache()
    dist.destroy_process_group()
    if rank == 0:
        line = {"metric": "distributed transform GFLOP/s (5 N log2 N per step)", "value": 5.0 * N * math.log2(N) / t / 1e9,
                "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32", "data": "synthetic",
                "config": {"workload": f"one forward transform of 2^{int(math.log2(N))} values over {world} GPUs, "
                                       f"n1 = 2^10, n2 = 2^{int(math.log2(n2))}",
                           "inputs": "larger than L2", "parallelism": f"four-step, one all-to-all, {world} ranks"},
                "gpu_launches": launches, "clocks": clk, "mode": "dist"}
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.dist:
        run_dist(args, world, rank, local_rank)
        return

    import torch

    import onefft_b200 as ofb
    from onefft_b200.shard import max_over_ranks

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    L = ofb.lib()
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    work = []
    for name, l, b in ITEMS:
        n = 1 << l
        plan = ofb.Plan(n)
        x = torch.randn(2 * n * b, device="cuda", generator=gen, dtype=torch.float32)
        work.append({"name": name, "log2n": l, "batch": b, "plan": plan, "x": x, "y": torch.empty_like(x),
                     "z": torch.empty_like(x), "passes": plan.passes()})

    def launch(w, inverse):
        src, dst = (w["y"], w["z"]) if inverse else (w["x"], w["y"])
        f = L.onefft_dev_inverse_batched if inverse else L.onefft_dev_forward_batched
        rc = f(w["plan"].handle, src.data_ptr(), dst.data_ptr(), w["batch"], sptr)
        if rc != 0:
            raise RuntimeError(ofb.last_error())

    nev = 2 * len(work)
    events = [[torch.cuda.Event(enable_timing=True) for _ in range(nev + 1)] for _ in range(args.steps)]

    def step(ev=None):
        i = 0
        for w in work:
            for inv in (False, True):
                if ev:
                    ev[i].record(stream)
                launch(w, inv)
                i += 1
        if ev:
            ev[i].record(stream)

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = L.onefft_debug_launch_count()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    for k in range(args.steps):
        step(events[k])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = int(L.onefft_debug_launch_count() - launches0)
    clk = clocks.stop()
    for w in work:  # a kernel failure recorded during the timed steps voids the run
        w["plan"].check()
    t = events[0][0].elapsed_time(events[-1][-1]) / 1e3
    t = max_over_ranks(t, device="cuda")
    per_step = t / args.steps
    value = world * STEP_FLOPS / per_step / 1e9
    peak, peak_kind = measured_peaks()

    # per item and direction: average launch-group time over the K steps
    detail = {}
    share = []
    for wi, w in enumerate(work):
        n, b = 1 << w["log2n"], w["batch"]
        tt = []
        for d in range(2):
            s = sum(events[k][2 * wi + d].elapsed_time(events[k][2 * wi + d + 1]) for k in range(args.steps))
            tt.append(s / args.steps / 1e3)
        td = sum(tt) / 2
        share.append(sum(tt))
        detail[w["name"]] = {"us_forward": 1e6 * tt[0], "us_inverse": 1e6 * tt[1],
                             "gflops": flops(w["log2n"], b) / td / 1e9, "gbs_16n": 16 * n * b / td / 1e9,
                             "frac_hbm": 16 * n * b / td / 1e9 / peak, "passes": list(w["passes"]),
                             "launches_per_direction": len(w["passes"])}
    dom = int(np.argmax(share))
    w = work[dom]
    n, b = 1 << w["log2n"], w["batch"]
    td = share[dom] / 2
    achieved = 16 * n * b / td / 1e9
    kernel = "k_batched" if len(w["passes"]) == 1 else "k_pass x%d" % len(w["passes"])
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "kernel": f"{kernel} ({w['name']})",
                "traffic": ncu_traffic(w["name"]), "traffic_unit": "DRAM bytes per launch (ncu)",
                "algorithmic_bytes_per_launch": 16 * n * b / len(w["passes"]),
                "share_of_step": share[dom] / sum(share), "frac_of_8TBs_nominal": achieved / 8000.0}

    # ---- end to end through the drop-in host-pointer calls (pinned host buffers) ----
    e2e = None
    if not args.no_e2e:
        # Per item: pinned input, two pinned intermediates (step s writes hy[s % 2]) and the
        # pinned result. Each item has a forward host thread and an inverse host thread (the
        # library keeps per-thread streams and staging buffers): the inverse of step s follows
        # the forward of step s, which waits until the inverse of step s - 2 has released its
        # intermediate. So step s + 1's copies to the device overlap step s's copies back
        # (PCIe is full duplex) while every step still moves all of its inputs in and all of
        # its results out.
        host = []
        for w in work:
            hx = torch.empty(w["x"].numel(), dtype=torch.float32, pin_memory=True)
            hx.copy_(w["x"])
            hy = [torch.empty_like(hx, pin_memory=True) for _ in range(2)]
            host.append((w, hx, hy, torch.empty_like(hx, pin_memory=True)))
        pools = [(concurrent.futures.ThreadPoolExecutor(max_workers=1),
                  concurrent.futures.ThreadPoolExecutor(max_workers=1)) for _ in host]
        nchain = max(2, args.e2e_chains)
        chain_pools = [[concurrent.futures.ThreadPoolExecutor(max_workers=1) for _ in range(nchain)] for _ in host]

        def call(w, src, dst, inverse):
            h = w["plan"].handle
            if w["batch"] > 1:
                f = L.onefft_plan_inverse_batched if inverse else L.onefft_plan_forward_batched
                if f(h, src.data_ptr(), dst.data_ptr(), w["batch"]):
                    raise RuntimeError(ofb.last_error())
            else:
                (L.onefft_plan_inverse if inverse else L.onefft_plan_forward)(h, src.data_ptr(), dst.data_ptr())

        offset = args.e2e_schedule == "offset"

        def e2e_steps_run(k):
            futs = []
            for (w, hx, hy, hz), (pf, pi) in zip(host, pools):
                done_f = [threading.Event() for _ in range(k)]
                done_i = [threading.Event() for _ in range(k)]
                failed = []
                nb = len(hy)
                # "offset": the inverse thread starts half a call late (one copy of the item at
                # ~55 GB/s), so its uploads meet the forward thread's downloads and the other way
                # round; it stays behind because each of its calls starts when its previous ends
                half = 8.0 * (1 << w["log2n"]) * w["batch"] / 55e9 if offset else 0.0

                def fwd_thread(w=w, hx=hx, hy=hy, done_f=done_f, done_i=done_i, failed=failed, nb=nb):
                    try:
                        for s in range(k):
                            if s >= nb:
                                done_i[s - nb].wait()
                            if not failed:
                                call(w, hx, hy[s % nb], False)
                            done_f[s].set()
                    except BaseException:
                        failed.append(1)
                        for e in done_f:
                            e.set()
                        raise

                def inv_thread(w=w, hy=hy, hz=hz, done_f=done_f, done_i=done_i, failed=failed, nb=nb, half=half):
                    try:
                        for s in range(k):
                            done_f[s].wait()
                            if s == 0 and half:
                                time.sleep(half)
                            if not failed:
                                call(w, hy[s % nb], hz, True)
                            done_i[s].set()
                    except BaseException:
                        failed.append(1)
                        for e in done_i:
                            e.set()
                        raise

                futs += [pf.submit(fwd_thread), pi.submit(inv_thread)]
            for f in futs:
                f.result()

        def e2e_chains_run(k):
            # Per item `nchain` chains, each running whole steps (forward, then inverse of its
            # result) on its own buffers: chain c takes steps c, c + nchain, ... Chain c starts c
            # uploads' time later, so that while one chain copies a call's input to the device
            # another copies a result back, and they keep that offset (their work is equal).
            futs = []
            for (w, hx, hy, hz), pc in zip(host, chain_pools):
                up_s = 8.0 * (1 << w["log2n"]) * w["batch"] / 50e9  # one input at ~50 GB/s

                def chain(c, w=w, hx=hx, hy=hy, hz=hz, up_s=up_s):
                    time.sleep(c * up_s * 2.0 / nchain)
                    for s in range(c, k, nchain):
                        call(w, hx, hy[c], False)
                        call(w, hy[c], hz[c], True)

                futs += [pc[c].submit(chain, c) for c in range(nchain)]
            for f in futs:
                f.result()

        if offset:  # three intermediates: forward s waits only for inverse s - 3
            for i, (w, hx, hy, hz) in enumerate(host):
                host[i] = (w, hx, hy + [torch.empty_like(hx, pin_memory=True)], hz)
        if args.e2e_schedule == "chains":
            for i, (w, hx, hy, hz) in enumerate(host):  # per chain its own intermediate and result
                hy = hy + [torch.empty_like(hx, pin_memory=True) for _ in range(nchain - len(hy))]
                host[i] = (w, hx, hy, [hz] + [torch.empty_like(hz, pin_memory=True) for _ in range(nchain - 1)])
            e2e_steps_run = e2e_chains_run  # noqa: F811
        e2e_steps_run(2)  # per-thread streams and staging buffers are set up here
        e2e_steps = max(2, min(args.steps, 12))
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        e2e_steps_run(e2e_steps)
        t_e2e = (time.perf_counter() - t0) / e2e_steps
        t_e2e = max_over_ranks(t_e2e, device="cuda")
        same = all(torch.equal(hy[0][:4096].cuda(), w["y"][:4096]) and
                   torch.equal((hz[0] if isinstance(hz, list) else hz)[:4096].cuda(), w["z"][:4096])
                   for w, hx, hy, hz in host)
        nbytes = sum(2 * 8 * (1 << w["log2n"]) * w["batch"] for w in work)
        link = pcie_ceiling(torch)
        e2e = {"value": world * STEP_FLOPS / t_e2e / 1e9, "unit": "GFLOP/s", "h2d_bytes_per_step": nbytes,
               "link": link, "ms_per_step_at_link_ceiling": 1e3 * 2 * nbytes / (link["both_ways_gbs"] * 1e9),
               "d2h_bytes_per_step": nbytes, "ms_per_step": 1e3 * t_e2e, "steps": e2e_steps,
               "matches_device_path": bool(same),
               "calls": "onefft_plan_forward/_inverse (single) and onefft_plan_forward/_inverse_batched (batch), "
                        "pinned host buffers",
               "schedule": {"pairs": "per item one forward and one inverse host thread; step s+1's forward "
                                     "overlaps step s's inverse (intermediates double-buffered); time of all "
                                     "steps / steps",
                            "offset": "per item one forward and one inverse host thread, the inverse thread "
                                      "half a call behind (its uploads meet the forward thread's downloads); "
                                      "three intermediates; time of all steps / steps",
                            "chains": "per item two host threads, each running whole steps (forward, then "
                                      "inverse) on its own buffers, the second started one upload later so one "
                                      "uploads while the other downloads; time of all steps / steps"}[args.e2e_schedule]}
        for pf, pi in pools:
            pf.shutdown()
            pi.shutdown()
        for pc in chain_pools:
            for p in pc:
                p.shutdown()
        del host

    # ---- the other configurations, measured beside the headline (rank 0, N = 1) ----
    configs = None
    if rank == 0 and world == 1 and not args.no_configs:
        for w in work:  # free the headline buffers first
            w["x"] = w["y"] = w["z"] = None
        torch.cuda.empty_cache()
        configs = other_configs(torch, ofb, L, stream, peak)

    # ---- CPU baseline: the reference library on this host (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            times, cores, kind, impl = cpu_step_times(3, 1)
            tc = min(times)
            cpu = {"value": STEP_FLOPS / tc / 1e9, "unit": "GFLOP/s", "cores": cores, "kind": kind,
                   "ms_per_step": 1e3 * tc,
                   "sample": f"the whole step (all items, both directions), min of 3 runs after 1 warm-up; "
                             f"{impl} kernels, {cores} threads, largest transforms first"}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "GFLOP/s", "cores": None, "kind": None, "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": 1e3 * per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(WORKLOAD, parallelism=f"dp{world} (independent work per GPU, no collective)"),
                "impl": "ours", "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": launches, "detail": detail, "configs": configs}
        print(json.dumps(line), flush=True)
    for w in work:
        w["plan"].destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
