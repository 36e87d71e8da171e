"""Benchmark of the B200 FFT path: batched FP32 complex FFT, 16384 transforms of n = 4096.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one forward transform of the whole batch (16384 x 4096 complex64, 512 MiB in and
512 MiB out, larger than the 126 MB L2, so no flush is needed between steps), launched through
the C ABI's device-pointer batched entry point on the current torch stream and timed with CUDA
events over exactly K steps, barrier + synchronize on both sides, max over ranks.

Printed (rank 0, one JSON line):
  value       5 n log2(n) batch / t summed over ranks, GFLOP/s (the reference's unit)
  e2e         the same metric through the drop-in host-pointer call onefft_plan_forward_batched
              with pinned host buffers: the host->device copy of the inputs and the
              device->host copy of all outputs are inside the timed region of every step
  roofline    the transform kernel against the measured HBM copy bandwidth: algorithmic bytes
              16 n per transform (read 8n + write 8n) / average kernel time
  cpu_baseline  the reference library (compiled from its own sources) on this host's cores,
              one shared plan and all cores pulling transforms from an atomic counter
  detail      single large transforms n = 2^20, 2^24, 2^27 (time, GFLOP/s, GB/s of 16 n)

With --impl reference only rank 0 runs: it times the reference CPU library on the same workload
with all host threads and prints the same metric with "impl": "reference".
Multi-GPU (torchrun, one process per GPU): each rank transforms its own 16384 x 4096 batch
(weak scaling, no collective on the data path).
"""
from __future__ import annotations

import argparse
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

N_LOG2 = 12
N = 1 << N_LOG2
BATCH = 16384
FLOP_PER_TRANSFORM = 5 * N * N_LOG2
BYTES_PER_TRANSFORM = 16 * N
METRIC = "5n*log2(n)/t GFLOP/s, batched FP32 c2c FFT"
WORKLOAD = {"workload": "batched FP32 complex FFT, 16384 x n=4096, forward, interleaved complex64",
            "n": N, "batch": BATCH, "direction": "forward", "input": "standard normal re/im (seeded)",
            "l2": "inputs larger than L2 (512 MiB per buffer), no flush needed"}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-detail", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    return ap.parse_args()


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "of measured"
    except Exception:
        return 6650.0, "of fallback"


def ncu_traffic():
    """DRAM bytes per launch of the transform kernel from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", "ncu_dram_bytes.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d.get("k_batched_4096", {}).get("dram_bytes_per_launch")
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
        self.t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
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
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_time(x_host: np.ndarray, threads: int, samples: int, kind: str, batch: int = BATCH) -> float:
    """Seconds for `batch` forward transforms of n=4096 with the CPU library (minimum of samples)."""
    import oracle
    oracle.build()
    out = np.empty_like(x_host[:2 * N * batch])
    t = oracle.cpu_bench_batched(N, batch, threads, False, x_host, out, samples, kind=kind)
    if t <= 0:
        raise RuntimeError("CPU reference run failed")
    return t


def run_reference(args, rank: int):
    """--impl reference: the reference CPU library on this host, rank 0 only."""
    if rank != 0:
        return
    import oracle
    oracle.build()
    kind = "reference" if oracle.have_reference() else "port"
    cores = oracle.cpu_cores(kind)
    rng = np.random.default_rng(12345)
    x = rng.standard_normal(2 * N * BATCH, dtype=np.float32)
    out = np.empty_like(x)
    for _ in range(max(1, args.warmup)):
        oracle.cpu_bench_batched(N, BATCH, cores, False, x, out, 1, kind=kind)
    times = []
    for _ in range(args.steps if args.steps <= 20 else 20):
        times.append(oracle.cpu_bench_batched(N, BATCH, cores, False, x, out, 1, kind=kind))
    t = sum(times) / len(times)
    value = FLOP_PER_TRANSFORM * BATCH / t / 1e9
    line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": args.gpus, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "impl": "reference",
            "config": dict(WORKLOAD, parallelism="host threads"),
            "cpu_baseline": {"value": value, "unit": "GFLOP/s", "cores": cores, "kind": kind,
                             "sample": f"the full 16384 x 4096 forward batch per step ({oracle.cpu_impl(kind)} kernels)"},
            "e2e": {"value": value, "unit": "GFLOP/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import onefft_b200 as ofb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))

    L = ofb.lib()
    plan = ofb.Plan(N)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(1234 + rank)
    d_in = torch.randn(2 * N * BATCH, device="cuda", generator=gen, dtype=torch.float32)
    d_out = torch.empty_like(d_in)
    stream = torch.cuda.current_stream()
    sptr = stream.cuda_stream

    def step():
        rc = L.onefft_dev_forward_batched(plan.handle, d_in.data_ptr(), d_out.data_ptr(), BATCH, sptr)
        if rc != 0:
            raise RuntimeError(ofb.last_error())

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    launches0 = L.onefft_debug_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    launches = int(L.onefft_debug_launch_count() - launches0)
    clk = clocks.stop()
    t = ev0.elapsed_time(ev1) / 1e3
    if dist:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t = tt.item()
    per_step = t / args.steps
    value = world * FLOP_PER_TRANSFORM * BATCH / per_step / 1e9
    peak, peak_kind = measured_peaks()
    achieved = BYTES_PER_TRANSFORM * BATCH / per_step / 1e9  # one kernel launch per step
    traffic = ncu_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": peak_kind, "traffic": traffic, "traffic_unit": "bytes per launch",
                "algorithmic_bytes_per_launch": BYTES_PER_TRANSFORM * BATCH,
                "frac_of_8TBs_nominal": achieved / 8000.0}

    # ---- end to end through the drop-in host-pointer call (pinned host buffers) ----
    h_in = torch.empty(2 * N * BATCH, dtype=torch.float32, pin_memory=True)
    h_out = torch.empty_like(h_in, pin_memory=True)
    h_in.copy_(d_in.cpu())
    e2e_steps = max(1, min(args.steps, 10))
    rc = L.onefft_plan_forward_batched(plan.handle, h_in.data_ptr(), h_out.data_ptr(), BATCH)  # warm-up
    if rc != 0:
        raise RuntimeError(ofb.last_error())
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        L.onefft_plan_forward_batched(plan.handle, h_in.data_ptr(), h_out.data_ptr(), BATCH)
    t_e2e = (time.perf_counter() - t0) / e2e_steps
    if dist:
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = tt.item()
    torch.cuda.synchronize()
    ok_e2e = torch.equal(h_out[:2 * N].cuda(), d_out[:2 * N])
    e2e = {"value": world * FLOP_PER_TRANSFORM * BATCH / t_e2e / 1e9, "unit": "GFLOP/s",
           "h2d_bytes_per_step": 8 * N * BATCH, "d2h_bytes_per_step": 8 * N * BATCH,
           "ms_per_step": 1e3 * t_e2e, "steps": e2e_steps, "matches_device_path": bool(ok_e2e),
           "call": "onefft_plan_forward_batched (pinned host in/out)"}
    del h_in, h_out

    # ---- single large transforms (same run, reported beside the headline) ----
    detail = {}
    if not args.no_detail:
        for lg in (20, 24, 27):
            n = 1 << lg
            p = ofb.Plan(n)
            a = torch.randn(2 * n, device="cuda", generator=gen)
            b = torch.empty_like(a)
            flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")  # 256 MiB > L2
            reps = 20 if lg < 27 else 5
            tot = 0.0
            for r in range(reps + 3):
                flush.zero_()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                L.onefft_dev_forward_batched(p.handle, a.data_ptr(), b.data_ptr(), 1, sptr)
                e1.record(stream)
                torch.cuda.synchronize()
                if r >= 3:
                    tot += e0.elapsed_time(e1) / 1e3
            ts = tot / reps
            detail[f"n=2^{lg}"] = {"us": 1e6 * ts, "gflops": 5 * n * lg / ts / 1e9, "gbs_16n": 16 * n / ts / 1e9,
                                   "frac_hbm": 16 * n / ts / 1e9 / peak, "passes": list(p.passes()),
                                   "l2": "flushed (256 MiB write) before each rep"}
            p.destroy()
            del a, b, flush

    # ---- CPU baseline: the reference library on this host (rank 0, N = 1) ----
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            import oracle
            oracle.build()
            kind = "reference" if oracle.have_reference() else "port"
            cores = oracle.cpu_cores(kind)
            xh = d_in.cpu().numpy()
            tc = cpu_reference_time(xh, cores, 5, kind)
            cpu = {"value": FLOP_PER_TRANSFORM * BATCH / tc / 1e9, "unit": "GFLOP/s", "cores": cores, "kind": kind,
                   "sample": f"full 16384 x 4096 forward batch, min of 5 passes, {oracle.cpu_impl(kind)} kernels",
                   "ms_per_step": 1e3 * tc}
        except Exception as e:  # reported, not fatal
            cpu = {"value": None, "unit": "GFLOP/s", "cores": None, "kind": None, "sample": f"failed: {e}"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "GFLOP/s", "n_gpus": world, "steps": args.steps,
                "warmup": max(3, args.warmup), "ms_per_step": 1e3 * per_step, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": dict(WORKLOAD, parallelism=f"dp{world} (independent batches per GPU)"),
                "impl": "ours", "e2e": e2e, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
                "gpu_launches": launches, "detail": detail}
        print(json.dumps(line), flush=True)
    plan.destroy()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
