/*
 * A C caller of the drop-in API, compiled as C99 against include/onefft.h and linked to
 * libonefft_cuda.so (tests/test_c_api.py builds and runs it). It makes the checks a OneFFT
 * caller relies on (the same kinds of checks as OneFFT's tests/test_onefft.c), with its own FP64
 * reference transform:
 *   - forward and inverse of every n = 2^0 .. 2^16 within 4e-7 + 1e-7 log2 n relative RMS of FP64,
 *     through onefft_forward/_inverse and through a plan, with the input misaligned by one float
 *     and the output by three, guard bands untouched and the input unmodified;
 *   - the round trip inverse(forward(x)) = n x;
 *   - an impulse's spectrum;
 *   - invalid sizes return -1 / NULL and leave the output untouched;
 *   - cache and plan results equal bit for bit.
 * Prints one line per failed check and "c api: all checks passed" at the end; exit status 0 only
 * when every check passed.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "onefft.h"

#define GUARD 64
#define SENTINEL 12345.0f

static int failures = 0;

#define CHECK(cond, ...)                       \
    do {                                       \
        if (!(cond)) {                         \
            ++failures;                        \
            fprintf(stderr, "FAILED: " __VA_ARGS__); \
            fprintf(stderr, "\n");             \
        }                                      \
    } while (0)

/* xorshift64 with a fixed seed: inputs uniform in [-1, 1) */
static uint64_t rng_state = 0x243F6A8885A308D3ull;
static float next_uniform(void) {
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return (float)((double)(rng_state >> 11) * (2.0 / 9007199254740992.0) - 1.0);
}

/* FP64 radix-2 decimation-in-time FFT, in place on interleaved re,im; sign -1 forward, +1
 * inverse (unnormalised). Angles from the integer exponent reduced modulo n. */
static void fft64(double *a, size_t n, int sign) {
    for (size_t i = 1, j = 0; i < n; ++i) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double t0 = a[2 * i], t1 = a[2 * i + 1];
            a[2 * i] = a[2 * j];
            a[2 * i + 1] = a[2 * j + 1];
            a[2 * j] = t0;
            a[2 * j + 1] = t1;
        }
    }
    const double two_pi = 6.283185307179586476925286766559;
    for (size_t len = 2; len <= n; len <<= 1) {
        const size_t half = len >> 1, step = n / len;
        for (size_t k = 0; k < half; ++k) {
            const size_t e = (k * step) % n;
            const double ang = sign * two_pi * (double)e / (double)n;
            const double wr = cos(ang), wi = sin(ang);
            for (size_t s = 0; s < n; s += len) {
                double *u = a + 2 * (s + k), *v = a + 2 * (s + k + half);
                const double vr = v[0] * wr - v[1] * wi, vi = v[0] * wi + v[1] * wr;
                v[0] = u[0] - vr;
                v[1] = u[1] - vi;
                u[0] += vr;
                u[1] += vi;
            }
        }
    }
}

static double rel_rms(const float *got, const double *want, size_t count) {
    double num = 0.0, den = 0.0;
    for (size_t i = 0; i < count; ++i) {
        const double d = (double)got[i] - want[i];
        num += d * d;
        den += want[i] * want[i];
    }
    return den > 0.0 ? sqrt(num / den) : sqrt(num);
}

/* a buffer of `count` floats at `misalign` floats past a band of sentinels, with a band after */
typedef struct {
    float *base;
    float *data;
    size_t count;
} Guarded;

static Guarded guarded_new(size_t count, size_t misalign) {
    Guarded g;
    g.count = count;
    g.base = (float *)malloc(sizeof(float) * (count + 2 * GUARD + 16));
    for (size_t i = 0; i < count + 2 * GUARD + 16; ++i) g.base[i] = SENTINEL;
    g.data = g.base + GUARD + misalign;
    return g;
}

static int guarded_intact(const Guarded *g) {
    for (float *p = g->base; p < g->data; ++p)
        if (*p != SENTINEL) return 0;
    for (size_t i = 0; i < GUARD; ++i)
        if (g->data[g->count + i] != SENTINEL) return 0;
    return 1;
}

static void check_size(unsigned log2n) {
    const size_t n = (size_t)1 << log2n;
    const double tol = 4e-7 + 1e-7 * log2n;
    Guarded in = guarded_new(2 * n, 1), out = guarded_new(2 * n, 3), back = guarded_new(2 * n, 0);
    float *copy = (float *)malloc(sizeof(float) * 2 * n);
    double *want = (double *)malloc(sizeof(double) * 2 * n);
    for (size_t i = 0; i < 2 * n; ++i) copy[i] = in.data[i] = next_uniform();
    onefft_plan *plan = onefft_plan_create(n);
    CHECK(plan != NULL, "plan_create(2^%u)", log2n);
    if (plan) CHECK(onefft_plan_size(plan) == n, "plan_size(2^%u)", log2n);
    for (int inverse = 0; inverse <= 1; ++inverse) {
        for (size_t i = 0; i < 2 * n; ++i) want[i] = copy[i];
        fft64(want, n, inverse ? 1 : -1);
        /* cache path */
        const int rc = inverse ? onefft_inverse(in.data, out.data, n) : onefft_forward(in.data, out.data, n);
        CHECK(rc == 0, "%s(2^%u) returned %d", inverse ? "onefft_inverse" : "onefft_forward", log2n, rc);
        const double err = rel_rms(out.data, want, 2 * n);
        CHECK(err < tol, "2^%u %s: relative RMS %.3g above %.3g", log2n, inverse ? "inverse" : "forward", err, tol);
        CHECK(guarded_intact(&out), "2^%u: wrote outside the output", log2n);
        CHECK(guarded_intact(&in) && memcmp(in.data, copy, sizeof(float) * 2 * n) == 0, "2^%u: input modified",
              log2n);
        /* plan path: bit for bit the cache path's result */
        if (plan) {
            float *again = (float *)malloc(sizeof(float) * 2 * n);
            if (inverse) onefft_plan_inverse(plan, in.data, again);
            else onefft_plan_forward(plan, in.data, again);
            CHECK(memcmp(again, out.data, sizeof(float) * 2 * n) == 0, "2^%u: plan and cache results differ", log2n);
            free(again);
        }
    }
    /* round trip */
    onefft_forward(in.data, out.data, n);
    onefft_inverse(out.data, back.data, n);
    for (size_t i = 0; i < 2 * n; ++i) want[i] = (double)copy[i] * (double)n;
    CHECK(rel_rms(back.data, want, 2 * n) < 2 * tol, "2^%u: round trip", log2n);
    CHECK(guarded_intact(&back), "2^%u: round trip wrote outside its output", log2n);
    /* impulse at j: X[k] = exp(-2 pi i j k / n) */
    if (n > 1) {
        const size_t j = 1 + (n / 3) % (n - 1);
        memset(in.data, 0, sizeof(float) * 2 * n);
        in.data[2 * j] = 1.0f;
        onefft_forward(in.data, out.data, n);
        double worst = 0.0;
        for (size_t k = 0; k < n; ++k) {
            const double ang = -6.283185307179586476925286766559 * (double)((j * k) % n) / (double)n;
            const double dr = out.data[2 * k] - cos(ang), di = out.data[2 * k + 1] - sin(ang);
            const double d = sqrt(dr * dr + di * di);
            if (d > worst) worst = d;
        }
        CHECK(worst < 4e-6, "2^%u: impulse off by %.3g", log2n, worst);
    }
    onefft_plan_destroy(plan);
    free(in.base);
    free(out.base);
    free(back.base);
    free(copy);
    free(want);
}

int main(void) {
    printf("implementation: %s, version %d.%d.%d\n", onefft_implementation(), ONEFFT_VERSION_MAJOR,
           ONEFFT_VERSION_MINOR, ONEFFT_VERSION_PATCH);
    for (unsigned m = 0; m <= 16; ++m) check_size(m);
    /* invalid sizes: -1 / NULL, output untouched */
    const size_t bad[] = {0, 3, 5, 6, 12, 1000, 1023, 1025, (size_t)1 << 31};
    float x[6] = {0}, out[6];
    for (size_t i = 0; i < sizeof bad / sizeof bad[0]; ++i) {
        for (int k = 0; k < 6; ++k) out[k] = 7.0f;
        CHECK(onefft_plan_create(bad[i]) == NULL, "plan_create(%zu) accepted", bad[i]);
        CHECK(onefft_forward(x, out, bad[i]) == -1 && out[0] == 7.0f && out[5] == 7.0f, "forward(%zu) accepted",
              bad[i]);
        CHECK(onefft_cache_prepare(bad[i]) == -1, "cache_prepare(%zu) accepted", bad[i]);
    }
    onefft_plan_destroy(NULL);
    CHECK(onefft_cache_prepare(4096) == 0, "cache_prepare(4096)");
    onefft_cache_clear();
    if (failures) {
        printf("c api: %d checks failed\n", failures);
        return 1;
    }
    printf("c api: all checks passed\n");
    return 0;
}
