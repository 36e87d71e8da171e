// Tile bodies shared by the stand-alone kernels (fft_kernels.cu) and the persistent uneven-batch
// kernel (uneven.cu): the same arithmetic in both, so an uneven batch reproduces the plain
// per-size path.
#pragma once

#include "fft_device.cuh"
#include "fft_launch.h"
#include "fft_tc.cuh"

namespace ofb {

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// w_n^t for t < n from the two-level tables, in FP64.
__device__ __forceinline__ double2 big_twiddle_f64(const double2* __restrict__ lo, const double2* __restrict__ hi,
                                                   int lo_bits, unsigned t) {
    return zmul(__ldg(lo + (t & ((1u << lo_bits) - 1))), __ldg(hi + (t >> lo_bits)));
}

// w^e for e < 2^BITS by square-and-multiply in FP64. With w from the two-level tables (error
// ~1e-16), the result is within ~BITS * 2^(BITS+1) * 1e-16 of exact, far below FP32 rounding.
template <int BITS>
__device__ __forceinline__ double2 zpow(double2 w, unsigned e) {
    double2 r = make_double2(1.0, 0.0);
#pragma unroll
    for (int b = 0; b < BITS; ++b) {
        if ((e >> b) & 1u) r = zmul(r, w);
        if (b + 1 < BITS) w = zmul(w, w);
    }
    return r;
}

// Inter-pass twiddles of a pass tile: output j + T kk of a column with factor F (first pass:
// the column index; middle pass: S h) is multiplied by w_n^(F j) * w_n^(F T kk), each factor
// rounded once to FP32. Both factors are powers of ONE table product per column (w_n^F and
// w_n^(F T)), so a tile reads the FP64 tables at C addresses instead of once per factor.
// The 16 factors w_n^(F T kk) of each column go to shared memory (rows of 17).
template <int LOG_L, int LOG_C, int MODE>
__device__ __forceinline__ void pass_twiddle_rows(const PassArgs& a, unsigned col0, float2* tws, int tid, int nthreads) {
    constexpr unsigned T = 1u << (LOG_L - 4);
    constexpr int C = 1 << LOG_C;
    const unsigned hs = (col0 >> a.log_s) << a.log_s;
    for (int i = tid; i < (MODE == 0 ? C : 1) * 16; i += nthreads) {
        const int cc = i >> 4, kk = i & 15;
        const unsigned f = MODE == 0 ? col0 + cc : hs;
        const double2 w = zpow<4>(big_twiddle_f64(a.tw_lo, a.tw_hi, a.lo_bits, f * T), (unsigned)kk);
        tws[cc * 17 + kk] = make_float2((float)w.x, (float)w.y);
    }
}
// ... and the thread's own factor w_n^(F j).
template <int LOG_L>
__device__ __forceinline__ float2 pass_twiddle_lane(const PassArgs& a, unsigned f, int j) {
    const double2 w = zpow<LOG_L - 4>(big_twiddle_f64(a.tw_lo, a.tw_hi, a.lo_bits, f), (unsigned)j);
    return make_float2((float)w.x, (float)w.y);
}

// Column transforms (PassArgs' column fields): w_N^t, N = 2^a.xlog2n <= 2^40, for any 64-bit t
// (reduced mod N; unsigned products wrap mod 2^64, a multiple of N).
__device__ __forceinline__ double2 wide_twiddle_f64(const PassArgs& a, unsigned long long t) {
    t &= (1ull << a.xlog2n) - 1;
    return zmul(__ldg(a.tw_lo + (t & ((1ull << a.lo_bits) - 1))), __ldg(a.tw_hi + (t >> a.lo_bits)));
}
// The factors of a column-transform tile, split like the inter-pass twiddles above (one FP32
// rounding per factor). First pass: output j + T kk of column col gets w_N^(F (j + T kk)),
// F = xcol0 + (col >> tw_shift): rows w_N^(F T kk) per column, lane w_N^(F j). Last pass: output
// k = q + 2^log_s (j + T kk) of transform h = col >> log_s (q = col mod 2^log_s) gets
// w_N^((xcol0 + h) k): rows w_N^((xcol0 + h) 2^log_s T kk), one per tile (a tile's columns share
// h), lane w_N^((xcol0 + h)(q + 2^log_s j)).
template <int LOG_L, int LOG_C, int MODE>
__device__ __forceinline__ void column_twiddle_rows(const PassArgs& a, unsigned col0, float2* tws, int tid, int nthreads) {
    constexpr unsigned long long T = 1ull << (LOG_L - 4);
    constexpr int C = 1 << LOG_C;
    for (int i = tid; i < (MODE == 0 ? C : 1) * 16; i += nthreads) {
        const int cc = i >> 4, kk = i & 15;
        const unsigned long long step = MODE == 0 ? (a.xcol0 + ((col0 + cc) >> a.tw_shift)) * T
                                                  : ((a.xcol0 + (col0 >> a.log_s)) << a.log_s) * T;
        const double2 w = zpow<4>(wide_twiddle_f64(a, step), (unsigned)kk);
        tws[cc * 17 + kk] = make_float2((float)w.x, (float)w.y);
    }
}
template <int LOG_L, int MODE>
__device__ __forceinline__ float2 column_twiddle_lane(const PassArgs& a, unsigned col0, int c, int j) {
    double2 w;
    if (MODE == 0) {
        w = zpow<LOG_L - 4>(wide_twiddle_f64(a, a.xcol0 + ((col0 + c) >> a.tw_shift)), (unsigned)j);
    } else {
        const unsigned long long f = a.xcol0 + (col0 >> a.log_s);
        const unsigned long long q = (col0 & ((1u << a.log_s) - 1)) + c;
        w = wide_twiddle_f64(a, f * (q + ((unsigned long long)j << a.log_s)));
    }
    return make_float2((float)w.x, (float)w.y);
}
// Destination of output k of transform b in the column layout (PassArgs::colstore).
__device__ __forceinline__ long long column_dst(const PassArgs& a, unsigned long long b, unsigned long long k) {
    return (long long)(((((k >> a.xlog_blk) << a.xlog_cols) + b) << a.xlog_blk) + (k & ((1ull << a.xlog_blk) - 1)));
}

// Loads of data the kernel never writes go through the read-only path; the intermediate array
// between passes may be kept in L2 for the next pass (evict last).
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldg(p); }
__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void st_policy(float2* p, float2 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
}

// Bounded wait until *p >= target (acquire at GPU scope), for counters that other blocks of the
// same launch advance: ~1 us per poll, about a second in all.
constexpr unsigned kCountWaitLimit = 1u << 20;
__device__ __forceinline__ bool wait_count(const unsigned* p, unsigned target) {
    for (unsigned i = 0; i < kCountWaitLimit; ++i) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) return true;
        __nanosleep(128);
    }
    return false;
}

// As wait_count, also giving up as soon as *abort is non-zero (another block's wait ran out).
__device__ __forceinline__ bool wait_count_or_abort(const unsigned* p, unsigned target, const unsigned* abort) {
    for (unsigned i = 0; i < kCountWaitLimit; ++i) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
        if (v >= target) return true;
        if (*(const volatile unsigned*)abort) return false;
        __nanosleep(128);
    }
    return false;
}

// Shared memory (bytes) of a tile of 2^log_c columns of length 2^log_l, with padding.
__host__ __device__ constexpr int smem_bytes(int log_l, int log_c) {
    return (int)sizeof(float2) * ((1 << (log_l + log_c)) + (1 << (log_l + log_c - 4)));
}
// ... plus the inter-pass twiddle factors of a pass tile (17 per column).
__host__ __device__ constexpr int pass_smem_bytes(int log_l, int log_c, int mode) {
    return smem_bytes(log_l, log_c) + (mode == 2 ? 0 : (int)sizeof(float2) * 17 * (1 << log_c));
}

// ---- n <= 8: one transform per thread -------------------------------------------------------------

// W: pointwise weights of the input and output (either pointer NULL), out = post * T(pre * in);
// without W the weights are not compiled in at all.
template <int LOG_N, bool W = false>
__device__ __forceinline__ void tiny_transform(const float2* __restrict__ src, float2* __restrict__ dst, int inverse,
                                               const float2* __restrict__ pre = nullptr,
                                               const float2* __restrict__ post = nullptr) {
    constexpr int N = 1 << LOG_N;
    float2 a[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        a[i] = __ldg(src + i);
        if constexpr (W) {
            if (pre) a[i] = cmul(a[i], __ldg(pre + i));
        }
        if (inverse) a[i] = swap_ri(a[i]);
    }
    dft<N>(a);
#pragma unroll
    for (int i = 0; i < N; ++i) {
        float2 y = inverse ? swap_ri(a[i]) : a[i];
        if constexpr (W) {
            if (post) y = cmul(y, __ldg(post + i));
        }
        dst[i] = y;
    }
}

// ---- one block of whole transforms, n = 16 .. 2^14 --------------------------------------------------
//
// 2^LOG_C transforms of length L = 2^LOG_L, 16 values per thread, thread tid owns column
// c = tid / (L/16) and butterfly lane j = tid mod (L/16). src / dst point at this thread's
// transform; inactive columns (past the end of a batch) compute on zeros and store nothing.
// TC: 0 = FP32 stages; 3 or 6 = the split-BF16 tensor-core stages with that many product terms
// (fft_tc.cuh). W, pre, post as tiny_transform.
template <int LOG_L, int LOG_C, int TC = 0, bool W = false>
__device__ __forceinline__ void batched_tile(const float2* __restrict__ src, float2* __restrict__ dst, bool active,
                                             int inverse, const float2* __restrict__ stw, float2* smem, int tid,
                                             const float2* __restrict__ pre = nullptr,
                                             const float2* __restrict__ post = nullptr) {
    constexpr int L = 1 << LOG_L, T = L / 16;
    const int j = tid & (T - 1);
    const int c = tid >> (LOG_L - 4);
    src += j;
    dst += j;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 x = active ? ld_stream(src + T * k) : make_float2(0.f, 0.f);
        if constexpr (W) {
            if (pre) x = cmul(x, __ldg(pre + j + T * k));
        }
        v[k] = inverse ? swap_ri(x) : x;
    }
    if constexpr (TC != 0) tile_fft_tc<LOG_L, LOG_C, 1, TC>(v, j, stw, smem, c << LOG_L, tid);
    else tile_fft<LOG_L, 1>(v, j, stw, smem, c << LOG_L);
    if (active) {
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float2 y = inverse ? swap_ri(v[k]) : v[k];
            if constexpr (W) {
                if (post) y = cmul(y, __ldg(post + j + T * k));
            }
            dst[T * k] = y;
        }
    }
}

// ---- one tile of a pass of the multi-pass decomposition -----------------------------------------
//
// MODE 0: first pass, in -> out with digit-reversed contiguous column runs and w_n^(r k).
// MODE 1: middle pass, in place on out, twiddle w_n^((h k) S).
// MODE 2: last pass, in place on out, no twiddle.
// Tile t covers 2^LOG_C adjacent columns of the transform at element offset `toff`; tid runs
// over the 2^LOG_C L / 16 threads of the tile.
// W: the first pass multiplies its input by a.pre, the last pass its output by a.post (see
// PassArgs); without W they are not compiled in.
// CG: later passes load through L2 only (ld.global.cg), for data that other blocks of the same
// launch wrote: an SM's L1 may still hold an older copy of a line that it read for a neighbouring
// transform.
// X: a pass of a column transform (PassArgs' column fields): MODE 0 takes its inter-pass factor
// from the column fields and, with colstore, writes the column layout (and a.swap_out: it is
// then the only pass); MODE 2 reads a.in, multiplies by the larger transform's factors and
// writes the column layout to a.out. One matrix per launch (toff 0).
template <int LOG_L, int LOG_C, int MODE, int TC = 0, bool W = false, bool CG = false, bool X = false>
__device__ __forceinline__ void pass_tile(const PassArgs& a, unsigned t, long long toff, float2* smem, int tid) {
    constexpr int L = 1 << LOG_L, T = L / 16, C = 1 << LOG_C;
    const int c = tid & (C - 1);
    const int j = tid >> LOG_C;
    const unsigned col0 = a.tli >= 31 ? (t << LOG_C)
                                      : ((a.outer_base + (t >> a.tli)) << a.outer_shift) + a.inner_base +
                                            ((t & ((1u << a.tli) - 1)) << LOG_C);
    unsigned base;  // element e of this thread's column is at base + (e << a.log_s)
    if (MODE == 0) {
        base = col0 + c;
    } else {
        unsigned q = (col0 & ((1u << a.log_s) - 1)) + c;
        unsigned h = col0 >> a.log_s;
        base = q + (h << (a.log_s + LOG_L));
    }
    // Inter-pass twiddles w_n^(F (j + T kk)) for this thread's outputs, F = r (first pass,
    // per column) or S h (middle pass, per tile), split as w^(F j) * w^(F T kk): the factors
    // w^(F T kk) of each column in shared memory (rows padded to 17 so the columns of a warp hit
    // distinct banks), w^(F j) per thread; each rounded once to FP32, their product applied in
    // FP32 (pass_twiddle_rows / pass_twiddle_lane).
    float2* tws = smem + spad(C * L - 1) + 1;
    float2 wjf = make_float2(1.f, 0.f);
    bool twiddled = MODE != 2;
    if constexpr (X) {
        twiddled = MODE != 1 && a.tw_lo != nullptr;  // the same for the whole block
        if (twiddled) {
            column_twiddle_rows<LOG_L, LOG_C, MODE>(a, col0, tws, tid, C * T);
            wjf = column_twiddle_lane<LOG_L, MODE>(a, col0, c, j);
        }
    } else if (MODE != 2) {
        pass_twiddle_rows<LOG_L, LOG_C, MODE>(a, col0, tws, tid, C * T);
        wjf = pass_twiddle_lane<LOG_L>(a, MODE == 0 ? col0 + c : (col0 >> a.log_s) << a.log_s, j);
    }
    // element j + T k of the column: p0 + k * estep
    const long long estep = (long long)T << a.log_s;
    const long long off0 = toff + base + ((long long)j << a.log_s);
    float2 v[16];
    {
        const float2* p0 = a.in + off0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            // The first pass streams the input, which is never read again. Later passes read
            // and write `out` in place, so they avoid the read-only cache path.
            float2 x = MODE == 0 ? ld_stream(p0 + k * estep) : CG ? __ldcg(p0 + k * estep) : p0[k * estep];
            if constexpr (W && MODE == 0) {
                if (a.pre) x = cmul(x, __ldg(a.pre + (off0 - toff) + k * estep));
            }
            v[k] = a.swap_in ? swap_ri(x) : x;
        }
    }
    if constexpr (TC != 0) tile_fft_tc<LOG_L, LOG_C, C, TC>(v, j, a.stw, smem, c, tid);
    else tile_fft<LOG_L, C>(v, j, a.stw, smem, c);
    if (twiddled) {
        if (Stages<LOG_L>::COUNT == 1) __syncthreads();  // tile_fft had no barrier to publish tws
        const float2* tw = tws + (MODE == 0 ? c * 17 : 0);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = cmul(v[k], cmul(wjf, tw[k]));
    }
    const unsigned long long keep = a.l2_keep ? policy_evict_last() : 0ull;
    if (MODE == 0) {
        // Transpose through shared memory so that each column's L results leave as one
        // contiguous, coalesced run: thread tid then stores values kk0 + T i (i = 0..15) of
        // column cc = tid / T, at its digit-reversed place.
        {
            float2* w = smem + spad(j * C + c);
#pragma unroll
            for (int k = 0; k < 16; ++k) w[padc(k * T * C)] = v[k];
        }
        __syncthreads();
        const int cc = tid >> (LOG_L - 4), kk0 = tid & (T - 1);
        const unsigned rr = col0 + cc;
        if (X && a.colstore) {
            const float2* r = smem + spad(kk0 * C + cc);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float2 x = r[padc(i * T * C)];
                a.out[column_dst(a, rr, (unsigned)(kk0 + i * T))] = a.swap_out ? swap_ri(x) : x;
            }
            return;
        }
        const unsigned j2 = rr & ((1u << a.rev_b2) - 1), j1 = rr >> a.rev_b2;
        float2* q = a.out + toff + (((j1 + (j2 << a.rev_b1)) << LOG_L) + kk0);
        const float2* r = smem + spad(kk0 * C + cc);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float2 x = r[padc(i * T * C)];
            if (a.l2_keep) st_policy(q + i * T, x, keep);
            else q[i * T] = x;
        }
    } else if (X && MODE == 2) {
        const unsigned long long h = col0 >> a.log_s, q = (col0 & ((1u << a.log_s) - 1)) + c;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float2 x = a.swap_out ? swap_ri(v[k]) : v[k];
            a.out[column_dst(a, h, q + ((unsigned long long)(j + T * k) << a.log_s))] = x;
        }
    } else {
        float2* p0 = a.out + off0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float2 x = a.swap_out ? swap_ri(v[k]) : v[k];
            if constexpr (W && MODE == 2) {
                if (a.post) x = cmul(x, __ldg(a.post + (off0 - toff) + k * estep));
            }
            if (MODE == 1 && a.l2_keep) st_policy(p0 + k * estep, x, keep);
            else p0[k * estep] = x;
        }
    }
}

}  // namespace ofb
