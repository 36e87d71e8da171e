/*
 * CPU oracle for the onefft_b200 test suite — TEST INFRASTRUCTURE, NOT PART OF THE PRODUCT.
 *
 * Only the tests, the smoke check and the benchmark's CPU-baseline leg load this file (built as
 * oracle/liboracle.so). The CUDA library never links it and never falls back to it.
 *
 * It restates, in plain C, what OneFFT computes for its one hot path (power-of-two, single
 * precision, complex-to-complex, out-of-place, unnormalised FFT on interleaved re,im floats):
 *
 *   - the twiddle rule: FP64 root of unity with the angle folded into the first octant through a
 *     0.64 fixed-point phase, rounded to FP32 (OneFFT src/onefft.c:115-141);
 *   - the portable FP32 transform: sizes 1, 2, 4 written out, otherwise a bit-reversed copy and
 *     an iterative radix-2 over a per-size FP32 twiddle table, inverse = exchange re/im on the
 *     way in and out (src/onefft.c:158-230, docs/design.md "The inverse transform");
 *   - the FP64 checks of the reference's own tests: an in-place radix-2 FP64 FFT
 *     (tests/test_onefft.c:31-55), a direct DFT with the angle reduced in integers
 *     (tests/test_onefft.c:149-150), the relative RMS metric (tests/test_onefft.c:64-71) and the
 *     error bound 4e-7 + 1e-7*log2n (tests/test_onefft.c:101);
 *   - the seeded input generators shared by every harness: xorshift32 uniform in [-1,1)
 *     (tests/test_onefft.c:57-61), a splitmix64 + Box-Muller standard normal, and the
 *     "1% of entries x1e3" wide-range variant.
 *
 * Parity of this restatement is pinned against the reference library compiled from its own
 * sources (oracle/Makefile -> oracle/_ref/) and against golden vectors produced by it
 * (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_EXPORT __attribute__((visibility("default")))

static const double kTwoPi = 6.283185307179586476925286766559;

/* exp(-2 pi i k / 2^log2size) in FP64. The phase k/2^log2size is a 0.64 fixed-point fraction of
 * a turn; its top two bits select the quadrant and the rest is folded into [0, 1/8] turn, so the
 * values are exactly symmetric and exact at multiples of pi/4 (src/onefft.c:112-135). */
ORACLE_EXPORT void oracle_root_f64(uint64_t k, unsigned log2size, double *re, double *im) {
    uint64_t phase = log2size ? k << (64 - log2size) : 0;
    unsigned quadrant = (unsigned)(phase >> 62);
    uint64_t rest = phase & ((UINT64_C(1) << 62) - 1);
    const double turn_per_unit = kTwoPi / 18446744073709551616.0;
    double c, s;
    if (rest > (UINT64_C(1) << 61)) { /* second octant of the quadrant: mirror */
        double a = (double)((UINT64_C(1) << 62) - rest) * turn_per_unit;
        c = sin(a);
        s = cos(a);
    } else {
        double a = (double)rest * turn_per_unit;
        c = cos(a);
        s = sin(a);
    }
    /* (c - i s) rotated by (-i)^quadrant */
    switch (quadrant) {
    case 0: *re = c; *im = -s; break;
    case 1: *re = -s; *im = -c; break;
    case 2: *re = -c; *im = s; break;
    default: *re = s; *im = c; break;
    }
}

/* The FP32 twiddle: the FP64 value rounded once (src/onefft.c:137-141). */
ORACLE_EXPORT void oracle_root_f32(uint64_t k, unsigned log2size, float *re, float *im) {
    double c, s;
    oracle_root_f64(k, log2size, &c, &s);
    *re = (float)c;
    *im = (float)s;
}

/* table[2k], table[2k+1] = FP32 twiddle k of size 2^log2n, for k in [0, count). */
ORACLE_EXPORT void oracle_twiddle_table(unsigned log2n, size_t count, float *table) {
    for (size_t k = 0; k < count; k++) oracle_root_f32(k, log2n, &table[2 * k], &table[2 * k + 1]);
}

static size_t bit_reverse(size_t v, unsigned bits) {
    size_t r = 0;
    for (unsigned i = 0; i < bits; i++) {
        r = (r << 1) | (v & 1);
        v >>= 1;
    }
    return r;
}

static int log2_exact(size_t n, unsigned *log2n) {
    if (n == 0 || (n & (n - 1)) != 0) return -1;
    unsigned l = 0;
    while (((size_t)1 << l) < n) l++;
    if (l > 30) return -1;
    *log2n = l;
    return 0;
}

/* ---- portable FP32 transform (restates src/onefft.c:158-230) --------------------------------
 *
 * A "port plan" holds n and the FP32 table of the n/2 roots the radix-2 stages use. */
typedef struct {
    size_t n;
    unsigned log2n;
    float *tw; /* n/2 interleaved twiddles, NULL for n <= 4 */
} oracle_plan;

ORACLE_EXPORT oracle_plan *oracle_plan_create(size_t n) {
    unsigned log2n;
    if (log2_exact(n, &log2n)) return NULL;
    oracle_plan *p = (oracle_plan *)calloc(1, sizeof(oracle_plan));
    if (!p) return NULL;
    p->n = n;
    p->log2n = log2n;
    if (log2n > 2) {
        p->tw = (float *)malloc(n * sizeof(float)); /* n/2 complex */
        if (!p->tw) {
            free(p);
            return NULL;
        }
        oracle_twiddle_table(log2n, n / 2, p->tw);
    }
    return p;
}

ORACLE_EXPORT void oracle_plan_destroy(oracle_plan *p) {
    if (!p) return;
    free(p->tw);
    free(p);
}

ORACLE_EXPORT size_t oracle_plan_size(const oracle_plan *p) { return p->n; }

static void port_execute(const oracle_plan *p, const float *in, float *out, int inv) {
    size_t n = p->n;
    if (n == 1) { /* src/onefft.c:158-161 */
        out[0] = in[0];
        out[1] = in[1];
        return;
    }
    if (n == 2) { /* src/onefft.c:163-168: the same for both directions */
        float ar = in[0], ai = in[1], br = in[2], bi = in[3];
        out[0] = ar + br;
        out[1] = ai + bi;
        out[2] = ar - br;
        out[3] = ai - bi;
        return;
    }
    if (n == 4) { /* src/onefft.c:170-181: the inverse negates x1 - x3 */
        float s02r = in[0] + in[4], s02i = in[1] + in[5];
        float d02r = in[0] - in[4], d02i = in[1] - in[5];
        float s13r = in[2] + in[6], s13i = in[3] + in[7];
        float d13r = in[2] - in[6], d13i = in[3] - in[7];
        if (inv) {
            d13r = -d13r;
            d13i = -d13i;
        }
        out[0] = s02r + s13r;
        out[1] = s02i + s13i;
        out[2] = d02r + d13i;
        out[3] = d02i - d13r;
        out[4] = s02r - s13r;
        out[5] = s02i - s13i;
        out[6] = d02r - d13i;
        out[7] = d02i + d13r;
        return;
    }
    /* bit-reversed copy; the inverse exchanges re and im (src/onefft.c:186-191) */
    for (size_t i = 0; i < n; i++) {
        size_t j = bit_reverse(i, p->log2n);
        out[2 * j + inv] = in[2 * i];
        out[2 * j + 1 - inv] = in[2 * i + 1];
    }
    /* radix-2 stages, twiddle k*step of the size-n table (src/onefft.c:192-205) */
    for (size_t half = 1; half < n; half *= 2) {
        size_t step = n / (2 * half);
        for (size_t start = 0; start < n; start += 2 * half) {
            for (size_t k = 0; k < half; k++) {
                float wr = p->tw[2 * k * step], wi = p->tw[2 * k * step + 1];
                float *a = out + 2 * (start + k), *b = a + 2 * half;
                float tr = b[0] * wr - b[1] * wi;
                float ti = b[0] * wi + b[1] * wr;
                b[0] = a[0] - tr;
                b[1] = a[1] - ti;
                a[0] += tr;
                a[1] += ti;
            }
        }
    }
    if (inv) { /* src/onefft.c:206-211 */
        for (size_t i = 0; i < n; i++) {
            float t = out[2 * i];
            out[2 * i] = out[2 * i + 1];
            out[2 * i + 1] = t;
        }
    }
}

ORACLE_EXPORT void oracle_plan_forward(const oracle_plan *p, const float *in, float *out) { port_execute(p, in, out, 0); }
ORACLE_EXPORT void oracle_plan_inverse(const oracle_plan *p, const float *in, float *out) { port_execute(p, in, out, 1); }

/* One-shot FP32 transform; -1 (out untouched) for an invalid n, as onefft_forward does. */
ORACLE_EXPORT int oracle_fft_f32(const float *in, float *out, size_t n, int inverse) {
    oracle_plan *p = oracle_plan_create(n);
    if (!p) return -1;
    port_execute(p, in, out, inverse ? 1 : 0);
    oracle_plan_destroy(p);
    return 0;
}

/* ---- FP64 checks ---------------------------------------------------------------------------- */

/* In-place iterative radix-2 in FP64 on interleaved doubles, sign -1 forward and +1 inverse, with
 * cos/sin of the exact angle per stage (tests/test_onefft.c:31-55). */
ORACLE_EXPORT void oracle_fft_f64(double *x, size_t n, int inverse) {
    for (size_t i = 1, j = 0; i < n; i++) {
        size_t bit = n >> 1;
        for (; j & bit; bit >>= 1) j ^= bit;
        j ^= bit;
        if (i < j) {
            double tr = x[2 * i], ti = x[2 * i + 1];
            x[2 * i] = x[2 * j];
            x[2 * i + 1] = x[2 * j + 1];
            x[2 * j] = tr;
            x[2 * j + 1] = ti;
        }
    }
    for (size_t len = 2; len <= n; len <<= 1) {
        for (size_t k = 0; k < len / 2; k++) {
            double angle = (inverse ? kTwoPi : -kTwoPi) * (double)k / (double)len;
            double wr = cos(angle), wi = sin(angle);
            for (size_t i = k; i < n; i += len) {
                size_t j = i + len / 2;
                double tr = x[2 * j] * wr - x[2 * j + 1] * wi;
                double ti = x[2 * j] * wi + x[2 * j + 1] * wr;
                x[2 * j] = x[2 * i] - tr;
                x[2 * j + 1] = x[2 * i + 1] - ti;
                x[2 * i] += tr;
                x[2 * i + 1] += ti;
            }
        }
    }
}

/* FP64 FFT of FP32 input (converted first), written to `out` (2n doubles). */
ORACLE_EXPORT void oracle_fft_f64_from_f32(const float *in, double *out, size_t n, int inverse) {
    for (size_t i = 0; i < 2 * n; i++) out[i] = (double)in[i];
    oracle_fft_f64(out, n, inverse);
}

/* Direct DFT of the selected output bins in FP64; the angle of j*k is reduced modulo n in
 * integers before it becomes a double (tests/test_onefft.c:148-150). */
ORACLE_EXPORT void oracle_dft_bins(const float *in, size_t n, int inverse, const uint64_t *bins, size_t nbins,
                                   double *out) {
    double sign = inverse ? kTwoPi : -kTwoPi;
    for (size_t b = 0; b < nbins; b++) {
        uint64_t k = bins[b];
        double sr = 0, si = 0;
        for (size_t j = 0; j < n; j++) {
            double angle = sign * (double)(((uint64_t)j * k) % n) / (double)n;
            double c = cos(angle), s = sin(angle);
            double xr = in[2 * j], xi = in[2 * j + 1];
            sr += xr * c - xi * s;
            si += xr * s + xi * c;
        }
        out[2 * b] = sr;
        out[2 * b + 1] = si;
    }
}

/* sqrt(sum (got-want)^2 / sum want^2) over `count` floats (tests/test_onefft.c:63-71). */
ORACLE_EXPORT double oracle_rel_rms(const float *got, const double *want, size_t count) {
    double err = 0, norm = 0;
    for (size_t i = 0; i < count; i++) {
        double d = (double)got[i] - want[i];
        err += d * d;
        norm += want[i] * want[i];
    }
    return norm > 0 ? sqrt(err / norm) : sqrt(err);
}

/* Largest |got - want| over complex values (the modulus, as tests/test_onefft.c:151 uses). */
ORACLE_EXPORT double oracle_max_abs(const float *got, const double *want, size_t n_complex) {
    double worst = 0;
    for (size_t i = 0; i < n_complex; i++) {
        double d = hypot((double)got[2 * i] - want[2 * i], (double)got[2 * i + 1] - want[2 * i + 1]);
        if (d > worst) worst = d;
    }
    return worst;
}

/* Error bound of the reference's tests for 2^log2n points (tests/test_onefft.c:99-101). */
ORACLE_EXPORT double oracle_tolerance(unsigned log2n) { return 4e-7 + 1e-7 * (double)log2n; }

/* ---- seeded generators ---------------------------------------------------------------------- */

/* xorshift32 uniform in [-1,1): *state evolves as in tests/test_onefft.c:57-61 and
 * bench/bench.c:94-98. */
ORACLE_EXPORT void oracle_gen_uniform(uint32_t *state, float *out, size_t count) {
    uint32_t s = *state;
    for (size_t i = 0; i < count; i++) {
        s ^= s << 13;
        s ^= s >> 17;
        s ^= s << 5;
        out[i] = (float)(int32_t)s * (1.0f / 2147483648.0f);
    }
    *state = s;
}

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += UINT64_C(0x9E3779B97F4A7C15));
    z = (z ^ (z >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
    z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
    return z ^ (z >> 31);
}

/* (0,1] double from the top 53 bits */
static double unit_open(uint64_t *x) { return ((double)(splitmix64(x) >> 11) + 1.0) * (1.0 / 9007199254740992.0); }

/* Standard normal floats: Box-Muller in FP64 over splitmix64 uniforms, rounded to float. Values
 * come in pairs; element i depends only on (seed, i / 2), so any slice can be regenerated. */
ORACLE_EXPORT void oracle_gen_normal(uint64_t seed, uint64_t first, float *out, size_t count) {
    for (size_t i = 0; i < count; i++) {
        uint64_t e = first + i;
        uint64_t x = seed ^ (UINT64_C(0xD1B54A32D192ED03) * ((e >> 1) + 1));
        double u1 = unit_open(&x), u2 = unit_open(&x);
        double r = sqrt(-2.0 * log(u1));
        double a = kTwoPi * u2;
        out[i] = (float)((e & 1) ? r * sin(a) : r * cos(a));
    }
}

/* Normal values with 1% of the complex entries (chosen by a seeded hash) scaled by 1e3. */
ORACLE_EXPORT void oracle_gen_wide(uint64_t seed, uint64_t first_complex, float *out, size_t n_complex) {
    oracle_gen_normal(seed, 2 * first_complex, out, 2 * n_complex);
    for (size_t i = 0; i < n_complex; i++) {
        uint64_t x = (seed + UINT64_C(0x632BE59BD9B4E019)) ^ (first_complex + i) * UINT64_C(0x9E3779B97F4A7C15);
        if (splitmix64(&x) % 100 == 0) {
            out[2 * i] *= 1e3f;
            out[2 * i + 1] *= 1e3f;
        }
    }
}
