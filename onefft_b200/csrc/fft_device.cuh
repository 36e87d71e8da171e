// Device building blocks of the B200 transform: complex arithmetic, register DFTs of radix
// 2/4/8/16, the FP64 twiddle rule, and the Stockham tile engine that every kernel runs.
//
// Conventions (OneFFT include/onefft.h:26-35): complex values are float2 {re, im}; forward uses
// w_N = exp(-2 pi i / N); neither direction normalises. The inverse transform is the forward one
// with re and im exchanged on load and on store (OneFFT docs/design.md "The inverse transform",
// src/onefft.c:186-191), so every kernel body computes forward arithmetic only and inverse
// results are bit-for-bit mirror images of forward ones.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ofb {

// ---- complex helpers ---------------------------------------------------------------------------

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 w) {
    return make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}
// a * (-i)
__device__ __forceinline__ float2 mul_mi(float2 a) { return make_float2(a.y, -a.x); }
__device__ __forceinline__ float2 swap_ri(float2 a) { return make_float2(a.y, a.x); }

// w_16^1 = cos(pi/8) - i sin(pi/8), w_8^1 = sqrt(1/2) (1 - i): exact decimal expansions rounded
// to float by the compiler.
constexpr float kC8 = 0.92387953251128675613f;   // cos(pi/8)
constexpr float kS8 = 0.38268343236508977173f;   // sin(pi/8)
constexpr float kR2 = 0.70710678118654752440f;   // sqrt(1/2)

// a * w_8^1 = sqrt(1/2) ((x + y) + i (y - x))
__device__ __forceinline__ float2 mul_w8_1(float2 a) { return make_float2(kR2 * (a.x + a.y), kR2 * (a.y - a.x)); }
// a * w_8^3 = sqrt(1/2) ((y - x) - i (x + y))
__device__ __forceinline__ float2 mul_w8_3(float2 a) { return make_float2(kR2 * (a.y - a.x), -kR2 * (a.x + a.y)); }
// a * w_16^1, a * w_16^3, a * w_16^9 = -(a * w_16^1)
__device__ __forceinline__ float2 mul_w16_1(float2 a) { return cmul(a, make_float2(kC8, -kS8)); }
__device__ __forceinline__ float2 mul_w16_3(float2 a) { return cmul(a, make_float2(kS8, -kC8)); }
__device__ __forceinline__ float2 mul_w16_9(float2 a) { return cmul(a, make_float2(-kC8, kS8)); }

// ---- register DFTs (forward, natural order in and out) ------------------------------------------

template <int S>
__device__ __forceinline__ void dft2(float2* v) {
    float2 a = v[0], b = v[S];
    v[0] = cadd(a, b);
    v[S] = csub(a, b);
}

// v[0], v[S], v[2S], v[3S]
template <int S>
__device__ __forceinline__ void dft4(float2* v) {
    float2 s02 = cadd(v[0], v[2 * S]), d02 = csub(v[0], v[2 * S]);
    float2 s13 = cadd(v[S], v[3 * S]), d13 = mul_mi(csub(v[S], v[3 * S]));
    v[0] = cadd(s02, s13);
    v[2 * S] = csub(s02, s13);
    v[S] = cadd(d02, d13);
    v[3 * S] = csub(d02, d13);
}

// 8 = 2 x 4: four-point DFTs over q1 for q0 = 0, 1, twiddle w_8^(q0 p_lo), two-point DFTs over q0.
__device__ __forceinline__ void dft8(float2 (&v)[8]) {
    dft4<2>(&v[0]);
    dft4<2>(&v[1]);
    v[3] = mul_w8_1(v[3]);
    v[5] = mul_mi(v[5]);
    v[7] = mul_w8_3(v[7]);
    // y[p_lo + 4 p_hi] = v[2 p_lo + p_hi] after the two-point DFTs
    float2 t[8];
#pragma unroll
    for (int pl = 0; pl < 4; ++pl) {
        t[pl] = cadd(v[2 * pl], v[2 * pl + 1]);
        t[pl + 4] = csub(v[2 * pl], v[2 * pl + 1]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = t[i];
}

// 16 = 4 x 4: four-point DFTs over q1 (stride 4), twiddles w_16^(q0 p_lo), four-point DFTs over
// q0, then the 4x4 index transpose (a renaming once unrolled).
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
#pragma unroll
    for (int q0 = 0; q0 < 4; ++q0) dft4<4>(&v[q0]);
    // v[q0 + 4 p_lo] *= w_16^(q0 p_lo)
    v[5] = mul_w16_1(v[5]);
    v[6] = mul_w8_1(v[6]);
    v[7] = mul_w16_3(v[7]);
    v[9] = mul_w8_1(v[9]);
    v[10] = mul_mi(v[10]);
    v[11] = mul_w8_3(v[11]);
    v[13] = mul_w16_3(v[13]);
    v[14] = mul_w8_3(v[14]);
    v[15] = mul_w16_9(v[15]);
#pragma unroll
    for (int pl = 0; pl < 4; ++pl) dft4<1>(&v[4 * pl]);
    float2 t[16];
#pragma unroll
    for (int pl = 0; pl < 4; ++pl)
#pragma unroll
        for (int ph = 0; ph < 4; ++ph) t[pl + 4 * ph] = v[4 * pl + ph];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

template <int R>
__device__ __forceinline__ void dft(float2 (&a)[R]);
template <>
__device__ __forceinline__ void dft<1>(float2 (&)[1]) {}
template <>
__device__ __forceinline__ void dft<2>(float2 (&a)[2]) { dft2<1>(a); }
template <>
__device__ __forceinline__ void dft<4>(float2 (&a)[4]) { dft4<1>(a); }
template <>
__device__ __forceinline__ void dft<8>(float2 (&a)[8]) { dft8(a); }
template <>
__device__ __forceinline__ void dft<16>(float2 (&a)[16]) { dft16(a); }

// ---- twiddle rule (FP64, OneFFT src/onefft.c:112-141) ----------------------------------------------
//
// exp(-2 pi i k / 2^log2size): the phase is a 0.64 fixed-point fraction of a turn; the top two
// bits pick the quadrant and the rest is folded into the first octant before sin/cos, which
// makes tables exactly symmetric and exact at multiples of pi/4.
__device__ __forceinline__ double2 root_f64(unsigned long long k, unsigned log2size) {
    unsigned long long phase = log2size ? (k << (64 - log2size)) : 0ull;
    unsigned quadrant = (unsigned)(phase >> 62);
    unsigned long long rest = phase & ((1ull << 62) - 1);
    const double unit = 6.283185307179586476925286766559 / 18446744073709551616.0;
    double c, s;
    if (rest > (1ull << 61)) {
        double a = (double)((1ull << 62) - rest) * unit;
        sincos(a, &s, &c);
        double t = c;
        c = s;
        s = t;
    } else {
        double a = (double)rest * unit;
        sincos(a, &s, &c);
    }
    switch (quadrant) {
    case 0: return make_double2(c, -s);
    case 1: return make_double2(-s, -c);
    case 2: return make_double2(-c, s);
    default: return make_double2(s, c);
    }
}

// ---- Stockham stage schedule of a tile of length L = 2^LOG_L (LOG_L >= 4) --------------------------
//
// Radix-16 stages first, then one stage of radix 2^(LOG_L mod 4) if needed. Every thread owns 16
// values of one column: before each stage v[k] = X[j + T k] with T = L / 16. Stage s has stride
// Ns = 16^s; butterfly b reads X[b + q L/R], multiplies input q by w_{R Ns}^((b mod Ns) q),
// runs the R-point DFT and writes output p to Y[(b / Ns) R Ns + (b mod Ns) + p Ns]. After the
// last stage v[k] = output[j + T k] in natural order (auto-sort, no bit reversal).
template <int LOG_L>
struct Stages {
    static_assert(LOG_L >= 4 && LOG_L <= 16, "tile length");
    static constexpr int L = 1 << LOG_L;
    static constexpr int T = L / 16;
    static constexpr int N16 = LOG_L / 4;
    static constexpr int REM = LOG_L % 4;
    static constexpr int COUNT = N16 + (REM ? 1 : 0);
    __host__ __device__ static constexpr int log2_radix(int s) { return s < N16 ? 4 : REM; }
    __host__ __device__ static constexpr int log2_ns(int s) { return 4 * s; }
    // Twiddle table: for each stage s >= 1, (R-1) rows of Ns entries; row q-1, column r holds
    // w_{R Ns}^(r q). Offsets of each stage's rows in one array per tile length.
    __host__ __device__ static constexpr int tw_offset(int s) {
        int o = 0;
        for (int i = 1; i < s; ++i) o += ((1 << log2_radix(i)) - 1) << log2_ns(i);
        return o;
    }
    static constexpr int TW_TOTAL = tw_offset(COUNT);
};

// Stage table length for a runtime tile length (host side sizing).
__host__ __device__ constexpr int stage_table_entries(int log_l) {
    if (log_l < 4) return 0;
    int n16 = log_l / 4, rem = log_l % 4, count = n16 + (rem ? 1 : 0), o = 0;
    for (int s = 1; s < count; ++s) o += ((1 << (s < n16 ? 4 : rem)) - 1) << (4 * s);
    return o;
}

// Compute stage s in registers: twiddle the inputs (s > 0), run 16/R butterflies of radix R.
// Butterfly i of this thread has b = j + T i and inputs v[i + (16/R) q]; its output p is left in
// v[i + (16/R) p].
template <int LOG_L, int S>
__device__ __forceinline__ void stage_compute(float2 (&v)[16], int j, const float2* __restrict__ stw) {
    using St = Stages<LOG_L>;
    constexpr int LR = St::log2_radix(S);
    constexpr int R = 1 << LR;
    constexpr int NS = 1 << St::log2_ns(S);
    constexpr int BPT = 16 / R;
#pragma unroll
    for (int i = 0; i < BPT; ++i) {
        float2 a[R];
#pragma unroll
        for (int q = 0; q < R; ++q) a[q] = v[i + BPT * q];
        if (S > 0) {
            const int r = (j + St::T * i) & (NS - 1);
            const float2* tw = stw + St::tw_offset(S) + r;
#pragma unroll
            for (int q = 1; q < R; ++q) a[q] = cmul(a[q], __ldg(tw + (q - 1) * NS));
        }
        dft<R>(a);
#pragma unroll
        for (int p = 0; p < R; ++p) v[i + BPT * p] = a[p];
    }
}

// Index in the stage's output Y of output p of butterfly b.
template <int LOG_L, int S>
__device__ __forceinline__ int stage_out_index(int b, int p) {
    using St = Stages<LOG_L>;
    constexpr int LR = St::log2_radix(S);
    constexpr int LNS = St::log2_ns(S);
    return ((b >> LNS) << (LR + LNS)) + (b & ((1 << LNS) - 1)) + (p << LNS);
}

// Shared-memory slot of linear tile index x: one pad slot every 16 entries keeps the stride-16
// writes of the first stage and the column-interleaved layouts free of bank conflicts for 8-byte
// accesses.
__device__ __forceinline__ int spad(int x) { return x + (x >> 4); }
// Padded size of a compile-time displacement D. Every access below is spad(x0) + padc(D) with a
// per-thread base x0 and a compile-time D such that (x0 mod 16) + (D mod 16) < 16, which makes
// spad(x0 + D) == spad(x0) + padc(D): the address is one register plus an immediate.
__host__ __device__ constexpr int padc(int d) { return d + (d >> 4); }

// Runs every stage of one column's FFT. On entry v[k] = X[j + T k]; on exit v[k] = Y[j + T k].
// The column's element e lives at linear tile index e * LM + cofs: LM = C, cofs = c for the
// column-interleaved layout ([e][c], C columns), LM = 1, cofs = c L for whole columns ([c][e]).
// All threads of the block must call this (it synchronises).
template <int LOG_L, int LM, int S = 0>
__device__ __forceinline__ void tile_fft(float2 (&v)[16], int j, const float2* __restrict__ stw, float2* smem,
                                         int cofs) {
    using St = Stages<LOG_L>;
    stage_compute<LOG_L, S>(v, j, stw);
    if constexpr (S + 1 < St::COUNT) {
        // intermediate stages are radix 16: one butterfly per thread, b = j, output p at
        // E0 + p Ns with E0 = (j / Ns) 16 Ns + (j mod Ns)
        constexpr int LNS = St::log2_ns(S);
        constexpr int NS = 1 << LNS;
        float2* w = smem + spad((((j >> LNS) << (4 + LNS)) + (j & (NS - 1))) * LM + cofs);
#pragma unroll
        for (int p = 0; p < 16; ++p) w[padc(p * NS * LM)] = v[p];
        __syncthreads();
        const float2* r = smem + spad(j * LM + cofs);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = r[padc(k * St::T * LM)];
        __syncthreads();
        tile_fft<LOG_L, LM, S + 1>(v, j, stw, smem, cofs);
    }
}

}  // namespace ofb
