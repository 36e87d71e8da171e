"""Generates the golden fixtures of the parity tests by running the reference library.

The reference (OneFFT) ships no golden vector files; its tests compare against an FP64 FFT
(tests/test_onefft.c:31-55). The fixtures here are therefore made by the reference itself: the
oracle Makefile compiles OneFFT's unmodified src/onefft.c (its SIMD build and its
ONEFFT_NO_SIMD portable build) into oracle/_ref/, and this script runs both on the seeded inputs
of the test suite and stores

  ref_small.npz     inputs and the SIMD build's forward/inverse outputs for n = 2^0 .. 2^11,
                    xorshift32 uniform [-1,1) inputs drawn in sequence from seed 0x9e3779b9
                    as tests/test_onefft.c:57-61, 122 does;
  ref_errors.json   the reference's relative RMS (tests/test_onefft.c:64-71) and max-abs error
                    against the FP64 oracle, per size and direction, on the suite's inputs for
                    every size of the configurations (uniform per size up to 2^20; standard
                    normal at 2^10, 2^12, 2^13, 2^16, 2^20, 2^22 and 2^24 .. 2^27).

Usage:  python tests/golden/make_golden.py   (needs the reference tree; run where it exists)
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

SEED_NORMAL = 0x5EED0002


def uniform_inputs(max_log2: int):
    """Per-size xorshift inputs drawn in one sequence, as the reference test walks sizes."""
    st = O.SEED_TESTS
    out = {}
    for l in range(max_log2 + 1):
        x, st = O.gen_uniform(2 * (1 << l), st)
        out[l] = x
    return out


def err_pair(got, want):
    return {"rel_rms": O.rel_rms(got, want), "max_abs": O.max_abs(got, want)}


def main() -> None:
    O.build()
    if not O.have_reference():
        raise SystemExit("reference library not built (reference tree absent?)")
    impl = O.reference_lib().onefft_implementation().decode()
    small = {}
    uni = uniform_inputs(20)
    errors = {"reference_impl": impl, "uniform": {}, "normal": {}}
    for l, x in uni.items():
        rec = {}
        for inv in (0, 1):
            got = O.ref_fft(x, bool(inv))
            gotp = O.ref_fft(x, bool(inv), portable=True)
            want = O.fft64_numpy(x, bool(inv)) if l > 12 else O.fft64(x, bool(inv))
            d = "inverse" if inv else "forward"
            rec[d] = err_pair(got, want)
            rec[d + "_portable"] = err_pair(gotp, want)
            if l <= 11:
                small[f"out_{d}_{l}"] = got
        if l <= 11:
            small[f"in_{l}"] = x
        errors["uniform"][str(l)] = rec
        print(l, rec["forward"]["rel_rms"], rec["inverse"]["rel_rms"], flush=True)
    for l in (10, 12, 13, 16, 20, 22, 24, 25, 26, 27):
        x = O.gen_normal(2 * (1 << l), SEED_NORMAL + l)
        rec = {}
        for inv in (0, 1):
            d = "inverse" if inv else "forward"
            rec[d] = err_pair(O.ref_fft(x, bool(inv)), O.fft64_numpy(x, bool(inv)))
        errors["normal"][str(l)] = rec
        print("normal", l, rec["forward"]["rel_rms"], flush=True)
    errors["seed_normal"] = SEED_NORMAL
    np.savez_compressed(os.path.join(HERE, "ref_small.npz"), **small)
    with open(os.path.join(HERE, "ref_errors.json"), "w") as f:
        json.dump(errors, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
