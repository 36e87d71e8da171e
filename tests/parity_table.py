"""Writes the per-size error table of the GPU path against the FP64 oracle, beside the reference
library's own errors on the same inputs (run on a machine with a GPU):

    python tests/parity_table.py OUT.md

Rows, each forward and inverse:
  - uniform [-1,1) inputs of the reference test's sequence (tests/test_onefft.c:57-61, 122), n =
    2^0 .. 2^20, through the drop-in host call onefft_plan_forward / _inverse;
  - standard normal inputs at 2^10, 2^12, 2^13, 2^16, 2^20, 2^22, 2^24 .. 2^27 (the batched
    configuration's single sizes), through the device-pointer calls;
  - the 16384 x 4096 batch (standard normal): the worst of 64 sampled transforms;
  - the distributed four-step (onefft_b200/distributed.py) on the standard normal inputs of 2^22,
    2^24, 2^25 and 2^27, its P ranks' column transforms run one after another on this GPU with
    the all-to-all done by indexing (the same exchange the multi-rank tests run through gloo).
Columns: relative RMS against FP64 (tests/test_onefft.c:64-71) of this library and of the
reference (tests/golden/ref_errors.json, the reference library run on the same inputs), their
ratio (the parity rule asks <= 2), and the max-abs error of each.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402


def main(out_path: str) -> None:
    import torch

    import onefft_b200 as ofb
    O.build()
    with open(os.path.join(HERE, "golden", "ref_errors.json")) as f:
        ref = json.load(f)
    L = ofb.lib()
    rows = []

    def add(label, log2n, d, got, want, r):
        err, mab = O.rel_rms(got, want), O.max_abs(got, want)
        # n = 1 is exact in both (ratio 1 by definition); otherwise ours over the reference's
        ratio = err / r["rel_rms"] if r["rel_rms"] else (1.0 if err == 0 else float("inf"))
        rows.append((label, log2n, d, err, r["rel_rms"], ratio, mab, r["max_abs"]))

    st = O.SEED_TESTS
    for l in range(21):
        n = 1 << l
        x, st = O.gen_uniform(2 * n, st)
        plan = ofb.Plan(n)
        for inv in (0, 1):
            d = "inverse" if inv else "forward"
            out = np.empty_like(x)
            (L.onefft_plan_inverse if inv else L.onefft_plan_forward)(plan.handle, x.ctypes.data, out.ctypes.data)
            want = O.fft64(x, bool(inv)) if l <= 12 else O.fft64_numpy(x, bool(inv))
            add("uniform", l, d, out, want, ref["uniform"][str(l)][d])
        plan.destroy()
    for l in (10, 12, 13, 16, 20, 22, 24, 25, 26, 27):
        n = 1 << l
        x = O.gen_normal(2 * n, ref["seed_normal"] + l)
        plan = ofb.Plan(n)
        d_in = torch.from_numpy(x).cuda()
        d_out = torch.empty_like(d_in)
        for inv in (0, 1):
            d = "inverse" if inv else "forward"
            (plan.dev_inverse if inv else plan.dev_forward)(d_in.data_ptr(), d_out.data_ptr(), 1)
            torch.cuda.synchronize()
            plan.check()
            got = d_out.cpu().numpy()
            add("normal", l, d, got, O.fft64_numpy(x, bool(inv)), ref["normal"][str(l)][d])
            del got
        del d_in, d_out
        plan.destroy()
        print("normal", l, flush=True)
    # the distributed four-step: (log2 n, ranks, log2 n1)
    from test_multigpu_gloo import emulate_ranks

    from onefft_b200.distributed import clear_cache, gpu_columns

    def columns(v, n, cols, blocks, big_n, col0, flags):
        t = torch.from_numpy(np.ascontiguousarray(v, np.complex64)).cuda()
        return gpu_columns(t, n, cols, blocks, big_n, col0, flags).cpu().numpy()

    for l, world, l1 in ((22, 4, 10), (24, 8, 10), (25, 8, 12), (27, 8, 10)):
        n = 1 << l
        x = O.gen_normal(2 * n, ref["seed_normal"] + l)
        n1, n2 = 1 << l1, n >> l1
        for inv in (0, 1):
            d = "inverse" if inv else "forward"
            blocks = emulate_ranks(x.view(np.complex64), n1, n2, world, columns, bool(inv))  # [k1][k2]
            got = np.ascontiguousarray(blocks.T).reshape(-1).view(np.float32)  # natural order
            del blocks
            add(f"normal, distributed over {world} ranks (n1 = 2^{l1})", l, d, got, O.fft64_numpy(x, bool(inv)),
                ref["normal"][str(l)][d])
            del got
        clear_cache()
        print("distributed", l, flush=True)
    # the 16384 x 4096 batch: worst ratio over 64 sampled transforms
    n, batch = 4096, 16384
    x = O.gen_normal(2 * n * batch, 0xC0F2)
    plan = ofb.Plan(n)
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.empty_like(d_in)
    sample = np.sort(np.random.default_rng(5).choice(batch, 64, replace=False))
    for inv in (0, 1):
        d = "inverse" if inv else "forward"
        (plan.dev_inverse if inv else plan.dev_forward)(d_in.data_ptr(), d_out.data_ptr(), batch)
        torch.cuda.synchronize()
        out = d_out.view(batch, 2 * n).cpu().numpy()
        worst = None
        for b in sample:
            xb = x[2 * n * b:2 * n * (b + 1)]
            want = O.fft64(xb, bool(inv))
            got = out[b]
            r = O.ref_fft(xb, bool(inv))
            e, re_ = O.rel_rms(got, want), O.rel_rms(r, want)
            row = ("batch 16384 (worst of 64)", 12, d, e, re_, e / re_, O.max_abs(got, want), O.max_abs(r, want))
            if worst is None or row[5] > worst[5]:
                worst = row
        rows.append(worst)
    plan.destroy()
    with open(out_path, "w") as f:
        f.write("| input | log2 n | direction | rel RMS (this library) | rel RMS (reference) | ratio | "
                "max-abs (this library) | max-abs (reference) |\n|---|---|---|---|---|---|---|---|\n")
        for label, l, d, e, r, q, m1, m2 in rows:
            f.write(f"| {label} | {l} | {d} | {e:.3e} | {r:.3e} | {q:.3f} | {m1:.3e} | {m2:.3e} |\n")
        worst = max(rows, key=lambda r: r[5])
        f.write(f"\nWorst ratio {worst[5]:.3f} ({worst[0]}, 2^{worst[1]} {worst[2]}; n = 1 is exact in both); "
                f"reference library: {ref['reference_impl']} build of OneFFT's src/onefft.c.\n")
    print(f"wrote {out_path}: {len(rows)} rows, worst ratio {worst[5]:.3f}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "parity_table.md")
