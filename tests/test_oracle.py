"""CPU tests of the oracle: it must reproduce the reference before it may check the GPU path.

Pins (reference file:line in OneFFT):
  * the restated portable transform equals the reference's own ONEFFT_NO_SIMD build bit for bit
    (src/onefft.c:158-230), and the golden vectors of its SIMD build within the test bound;
  * the twiddle rule's symmetry and exactness claims (src/onefft.c:112-135);
  * the FP64 checks agree with numpy's FP64 FFT;
  * the reference test's known answers: impulse and constant (tests/test_onefft.c:142-164).
"""
from __future__ import annotations

import math

import numpy as np
import pytest


def test_port_matches_reference_portable_build_bitwise(oracle, uniform_inputs):
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    for l in range(0, 15):
        x = uniform_inputs[l]
        for inv in (False, True):
            a = oracle.port_fft(x, inv)
            b = oracle.ref_fft(x, inv, portable=True)
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (l, inv)


def test_golden_vectors_reproduced_by_reference(oracle, ref_small):
    """The committed fixtures are the SIMD reference's outputs; the live build must agree."""
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    for l in range(0, 12):
        x = ref_small[f"in_{l}"]
        for d, inv in (("forward", False), ("inverse", True)):
            got = oracle.ref_fft(x, inv)
            assert np.array_equal(got, ref_small[f"out_{d}_{l}"]), (l, d)


def test_port_vs_golden_within_reference_bound(oracle, ref_small, uniform_inputs):
    for l in range(0, 12):
        x = ref_small[f"in_{l}"]
        assert np.array_equal(x, uniform_inputs[l])
        for d, inv in (("forward", False), ("inverse", True)):
            want = oracle.fft64(x, inv)
            port = oracle.port_fft(x, inv)
            gold = ref_small[f"out_{d}_{l}"]
            assert oracle.rel_rms(port, want) < oracle.tolerance(l)
            assert oracle.rel_rms(gold, want) < oracle.tolerance(l)
            # port and reference differ only by rounding
            assert oracle.rel_rms(port, gold.astype(np.float64)) < 2 * oracle.tolerance(l)


def test_fft64_agrees_with_numpy(oracle, uniform_inputs):
    for l in (0, 1, 5, 10, 14):
        x = uniform_inputs[l]
        for inv in (False, True):
            a = oracle.fft64(x, inv)
            b = oracle.fft64_numpy(x, inv)
            assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(b).max())


def test_dft_bins_agree_with_fft64(oracle, uniform_inputs):
    x = uniform_inputs[9]
    bins = [0, 1, 77, 256, 511]
    for inv in (False, True):
        full = oracle.fft64(x, inv).reshape(-1, 2)
        got = oracle.dft_bins(x, bins, inv).reshape(-1, 2)
        assert np.abs(got - full[bins]).max() < 1e-11


def test_twiddle_rule_symmetry_and_exact_points(oracle):
    # exact at multiples of an eighth turn (src/onefft.c:112-114)
    r = math.sqrt(0.5)
    assert oracle.root_f64(0, 10) == (1.0, -0.0) or oracle.root_f64(0, 10) == (1.0, 0.0)
    assert oracle.root_f64(256, 10) == (0.0, -1.0)
    assert oracle.root_f64(512, 10) == (-1.0, 0.0)
    re, im = oracle.root_f64(128, 10)
    assert abs(re - r) < 2e-16 and abs(im + r) < 2e-16
    # exactly symmetric: w^(n/4 - k) = -i conj(w^k) ... i.e. re/im swap with signs
    for l in (5, 12, 20):
        n = 1 << l
        for k in (1, 3, n // 16 + 1):
            a = oracle.root_f64(k, l)
            b = oracle.root_f64(n // 4 - k, l)
            assert b == (-a[1], -a[0])
    # FP32 table entries are the FP64 values rounded once
    t = oracle.twiddle_table(12, 4096).reshape(-1, 2)
    for k in (0, 1, 1000, 4095):
        re, im = oracle.root_f64(k, 12)
        assert t[k, 0] == np.float32(re) and t[k, 1] == np.float32(im)


def test_known_answers_on_port(oracle):
    """Impulse and constant KATs of tests/test_onefft.c:142-164 on the restated transform."""
    for l in range(0, 13):
        n = 1 << l
        j = 1 + (n // 3) % (n - 1) if n > 1 else 0
        x = np.zeros(2 * n, np.float32)
        x[2 * j] = 1.0
        y = oracle.port_fft(x).reshape(-1, 2).astype(np.float64)
        k = np.arange(n, dtype=np.uint64)
        ang = -2 * math.pi * ((j * k) % n).astype(np.float64) / n
        assert np.hypot(y[:, 0] - np.cos(ang), y[:, 1] - np.sin(ang)).max() < 4e-6
        c = np.tile(np.array([0.5, -0.25], np.float32), n)
        y = oracle.port_fft(c).reshape(-1, 2).astype(np.float64)
        worst = math.hypot(y[0, 0] - 0.5 * n, y[0, 1] + 0.25 * n) / n
        if n > 1:
            worst = max(worst, np.hypot(y[1:, 0], y[1:, 1]).max() / n)
        assert worst < 1e-6


def test_invalid_sizes_on_port(oracle):
    x = np.zeros(8, np.float32)
    for n in (0, 3, 5, 6, 7, 12):
        with pytest.raises(ValueError):
            oracle.port_fft(np.zeros(2 * n, np.float32) if n else x[:0])


def test_generators_are_seeded_and_sliceable(oracle):
    a = oracle.gen_normal(1000, 7)
    b = oracle.gen_normal(400, 7, first=600)
    assert np.array_equal(a[600:], b)
    assert abs(a.mean()) < 0.15 and abs(a.std() - 1) < 0.1
    w = oracle.gen_wide(20000, 9).reshape(-1, 2)
    big = (np.abs(w).max(axis=1) > 50).mean()
    assert 0.005 < big < 0.02
    u, st = oracle.gen_uniform(10, oracle.SEED_TESTS)
    assert (u >= -1).all() and (u < 1).all()


def test_reference_errors_fixture_is_consistent(ref_errors, oracle, uniform_inputs):
    """The stored reference errors are the live reference's on the same inputs."""
    if not oracle.have_reference():
        pytest.skip("reference library not built")
    for l in (3, 10, 12):
        x = uniform_inputs[l]
        want = oracle.fft64(x)
        e = oracle.rel_rms(oracle.ref_fft(x), want)
        assert e == pytest.approx(ref_errors["uniform"][str(l)]["forward"]["rel_rms"], rel=1e-12)
