// The transform kernels for sm_100a and their launchers.
//
//   k_tiny     n = 1, 2, 4, 8: one thread per transform, all in registers.
//   k_batched  n = 16 .. 2^14 in one kernel: each block holds C = max(1, 4096 / n) whole
//              transforms (C n / 16 threads, 16 values per thread), Stockham radix-16 stages in
//              registers with exchanges through padded shared memory. Loads and stores are
//              coalesced 8-byte accesses straight between HBM and registers.
//   k_pass     n > 2^14: one pass of a two- or three-pass four-step decomposition
//              n = L0 L1 (L2). A block transforms a tile of C adjacent columns of length Lp.
//              Pass 0 reads the input in natural order (columns are adjacent addresses),
//              multiplies by w_n^(r k) and writes each column's result as one contiguous run
//              into `out`, at a digit-reversed column position; passes 1.. work in place on
//              `out` with the stride of the digits already done, so the final pass leaves the
//              result in natural order and no workspace beyond `out` is needed.
//
// Replaces the generated SIMD pass chain of OneFFT (src/onefft_*.inc driven by
// onefft_execute_passes, src/onefft.c:274-297): the mathematics (a radix split of the DFT with
// twiddles between stages, inverse by exchanging re/im) is the same; the data movement is the
// GPU's own.
#include "fft_device.cuh"
#include "fft_launch.h"

namespace ofb {

// ---- twiddle tables, built on the device in FP64 and rounded once -----------------------------------

// Stage table of a tile of length 2^log_l: entry (s, q, r) = w_{R Ns}^(r q), FP32.
__global__ void k_stage_table(float2* __restrict__ dst, int log_l, int total) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    int n16 = log_l / 4, rem = log_l % 4, off = 0, s = 1;
    for (;;) {
        int lr = s < n16 ? 4 : rem;
        int cnt = ((1 << lr) - 1) << (4 * s);
        if (idx < off + cnt) {
            int local = idx - off;
            int q = (local >> (4 * s)) + 1;
            int r = local & ((1 << (4 * s)) - 1);
            double2 w = root_f64((unsigned long long)r * (unsigned long long)q, (unsigned)(lr + 4 * s));
            dst[idx] = make_float2((float)w.x, (float)w.y);
            return;
        }
        off += cnt;
        ++s;
    }
}

// Two-level FP64 tables of w_n: lo[t] = w_n^t (t < 2^lo_bits), hi[t] = w_n^(t 2^lo_bits).
__global__ void k_big_table(double2* __restrict__ lo, double2* __restrict__ hi, int log2n, int lo_bits) {
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    int nlo = 1 << lo_bits, nhi = 1 << (log2n - lo_bits);
    if (idx < nlo) lo[idx] = root_f64((unsigned long long)idx, (unsigned)log2n);
    else if (idx < nlo + nhi)
        hi[idx - nlo] = root_f64((unsigned long long)(idx - nlo) << lo_bits, (unsigned)log2n);
}

__device__ __forceinline__ double2 zmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// w_n^t for t < n from the two-level tables, in FP64.
__device__ __forceinline__ double2 big_twiddle_f64(const double2* __restrict__ lo, const double2* __restrict__ hi,
                                                   int lo_bits, unsigned t) {
    return zmul(__ldg(lo + (t & ((1u << lo_bits) - 1))), __ldg(hi + (t >> lo_bits)));
}

// L2 cache hints: the input of a transform is read exactly once (evict first); the intermediate
// array between passes should stay in L2 for the next pass (evict last).
__device__ __forceinline__ float2 ld_stream(const float2* p) { return __ldcs(p); }
__device__ __forceinline__ unsigned long long policy_evict_last() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}
__device__ __forceinline__ void st_policy(float2* p, float2 v, unsigned long long pol) {
    asm volatile("st.global.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(v.x), "f"(v.y), "l"(pol)
                 : "memory");
}

// ---- n <= 8 --------------------------------------------------------------------------------------

template <int LOG_N>
__global__ void __launch_bounds__(256) k_tiny(const float2* __restrict__ in, float2* __restrict__ out,
                                              long long batch, int inverse) {
    constexpr int N = 1 << LOG_N;
    long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= batch) return;
    float2 a[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        a[i] = __ldg(in + g * N + i);
        if (inverse) a[i] = swap_ri(a[i]);
    }
    dft<N>(a);
#pragma unroll
    for (int i = 0; i < N; ++i) out[g * N + i] = inverse ? swap_ri(a[i]) : a[i];
}

// ---- single-kernel batched transforms, n = 16 .. 2^14 -------------------------------------------------

template <int LOG_L, int LOG_C>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4))
    k_batched(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
              const float2* __restrict__ stw, int inverse) {
    constexpr int L = 1 << LOG_L, T = L / 16, C = 1 << LOG_C;
    extern __shared__ float2 smem[];
    const int tid = threadIdx.x;
    const int j = tid & (T - 1);
    const int c = tid >> (LOG_L - 4);
    const long long g = (long long)blockIdx.x * C + c;
    const bool active = g < batch;
    const float2* src = in + g * L + j;
    float2* dst = out + g * L + j;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 x = active ? ld_stream(src + T * k) : make_float2(0.f, 0.f);
        v[k] = inverse ? swap_ri(x) : x;
    }
    tile_fft<LOG_L, 1>(v, j, stw, smem, c << LOG_L);
    if (active) {
#pragma unroll
        for (int k = 0; k < 16; ++k) dst[T * k] = inverse ? swap_ri(v[k]) : v[k];
    }
}

// ---- one pass of the multi-pass decomposition -----------------------------------------------------

// MODE 0: first pass, in -> out with digit-reversed contiguous column runs and w_n^(r k).
// MODE 1: middle pass, in place on out, twiddle w_n^((h k) S).
// MODE 2: last pass, in place on out, no twiddle.
template <int LOG_L, int LOG_C, int MODE>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4)) k_pass(PassArgs a) {
    constexpr int L = 1 << LOG_L, T = L / 16, C = 1 << LOG_C;
    extern __shared__ float2 smem[];
    const int tid = threadIdx.x;
    const int c = tid & (C - 1);
    const int j = tid >> LOG_C;
    const long long tstride = 1ll << a.log2n;  // batch stride between transforms
    const unsigned t = blockIdx.x;
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
    // per column) or S h (middle pass, per block), split as w^(F j) * w^(F T kk): the 16 factors
    // w^(F T kk) of each column are evaluated once per block from the FP64 tables into shared
    // memory (rows padded to 17 so the columns of a warp hit distinct banks), w^(F j) once per
    // thread; each is rounded once to FP32 and their product applied in FP32.
    float2* tws = smem + spad(C * L - 1) + 1;
    if (MODE != 2) {
        const unsigned hs = (col0 >> a.log_s) << a.log_s;
        for (int i = tid; i < (MODE == 0 ? C : 1) * 16; i += C * T) {
            const int cc = i >> 4, kk = i & 15;
            const unsigned f = MODE == 0 ? col0 + cc : hs;
            double2 w = big_twiddle_f64(a.tw_lo, a.tw_hi, a.lo_bits, f * (unsigned)T * (unsigned)kk);
            tws[cc * 17 + kk] = make_float2((float)w.x, (float)w.y);
        }
    }
    // element j + T k of the column: p0 + k * estep
    const long long estep = (long long)T << a.log_s;
    const long long off0 = (long long)blockIdx.y * tstride + base + ((long long)j << a.log_s);
    float2 v[16];
    {
        const float2* p0 = a.in + off0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            // The first pass streams the input, which is never read again. Later passes read
            // and write `out` in place, so they avoid the read-only cache path.
            float2 x = MODE == 0 ? ld_stream(p0 + k * estep) : p0[k * estep];
            v[k] = a.swap_in ? swap_ri(x) : x;
        }
    }
    tile_fft<LOG_L, C>(v, j, a.stw, smem, c);
    if (MODE != 2) {
        if (Stages<LOG_L>::COUNT == 1) __syncthreads();  // tile_fft had no barrier to publish tws
        const unsigned f = MODE == 0 ? col0 + c : (col0 >> a.log_s) << a.log_s;
        const double2 wj = big_twiddle_f64(a.tw_lo, a.tw_hi, a.lo_bits, f * (unsigned)j);
        const float2 wjf = make_float2((float)wj.x, (float)wj.y);
        const float2* tw = tws + (MODE == 0 ? c * 17 : 0);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = cmul(v[k], cmul(wjf, tw[k]));
    }
    const unsigned long long keep = a.l2_keep ? policy_evict_last() : 0ull;
    if (MODE == 0) {
        // Transpose through shared memory so that each column's L results leave as one
        // contiguous, coalesced run: thread t then stores values kk0 + T i (i = 0..15) of
        // column cc = t / T, at its digit-reversed place.
        {
            float2* w = smem + spad(j * C + c);
#pragma unroll
            for (int k = 0; k < 16; ++k) w[padc(k * T * C)] = v[k];
        }
        __syncthreads();
        const int cc = tid >> (LOG_L - 4), kk0 = tid & (T - 1);
        const unsigned rr = col0 + cc;
        const unsigned j2 = rr & ((1u << a.rev_b2) - 1), j1 = rr >> a.rev_b2;
        float2* q = a.out + (long long)blockIdx.y * tstride + (((j1 + (j2 << a.rev_b1)) << LOG_L) + kk0);
        const float2* r = smem + spad(kk0 * C + cc);
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float2 x = r[padc(i * T * C)];
            if (a.l2_keep) st_policy(q + i * T, x, keep);
            else q[i * T] = x;
        }
    } else {
        float2* p0 = a.out + off0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float2 x = a.swap_out ? swap_ri(v[k]) : v[k];
            if (MODE == 1 && a.l2_keep) st_policy(p0 + k * estep, x, keep);
            else p0[k * estep] = x;
        }
    }
}

// ---- launchers -------------------------------------------------------------------------------------

template <class K>
static cudaError_t set_smem(K kernel, int bytes) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
}

static constexpr int smem_bytes(int log_l, int log_c) {
    return (int)sizeof(float2) * ((1 << (log_l + log_c)) + (1 << (log_l + log_c - 4)));
}

int batched_log_c(int log_l) { return log_l >= 12 ? 0 : 12 - log_l; }

template <int LOG_L>
static cudaError_t launch_batched_t(const float2* in, float2* out, long long batch, const float2* stw, int inverse,
                                    cudaStream_t stream) {
    constexpr int LOG_C = LOG_L >= 12 ? 0 : 12 - LOG_L;
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = smem_bytes(LOG_L, LOG_C);
    auto kernel = k_batched<LOG_L, LOG_C>;
    static cudaError_t attr = set_smem(kernel, SMEM);
    if (attr != cudaSuccess) return attr;
    const long long per_block = 1ll << LOG_C;
    long long blocks = (batch + per_block - 1) / per_block;
    while (blocks > 0) {  // gridDim.x limit 2^31-1
        long long now = blocks < 0x7fffffffll ? blocks : 0x7fffffffll;
        kernel<<<(unsigned)now, THREADS, SMEM, stream>>>(in, out, batch, stw, inverse);
        long long done = now * per_block;
        in += done << LOG_L;
        out += done << LOG_L;
        batch -= done;
        blocks -= now;
    }
    return cudaGetLastError();
}

template <int LOG_N>
static cudaError_t launch_tiny_t(const float2* in, float2* out, long long batch, int inverse, cudaStream_t stream) {
    long long blocks = (batch + 255) / 256;
    while (blocks > 0) {
        long long now = blocks < 0x7fffffffll ? blocks : 0x7fffffffll;
        k_tiny<LOG_N><<<(unsigned)now, 256, 0, stream>>>(in, out, batch, inverse);
        long long done = now * 256;
        in += done << LOG_N;
        out += done << LOG_N;
        batch -= done;
        blocks -= now;
    }
    return cudaGetLastError();
}

cudaError_t launch_single_kernel(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                 int inverse, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    switch (log2n) {
    case 0: return launch_tiny_t<0>(in, out, batch, inverse, stream);
    case 1: return launch_tiny_t<1>(in, out, batch, inverse, stream);
    case 2: return launch_tiny_t<2>(in, out, batch, inverse, stream);
    case 3: return launch_tiny_t<3>(in, out, batch, inverse, stream);
    case 4: return launch_batched_t<4>(in, out, batch, stw, inverse, stream);
    case 5: return launch_batched_t<5>(in, out, batch, stw, inverse, stream);
    case 6: return launch_batched_t<6>(in, out, batch, stw, inverse, stream);
    case 7: return launch_batched_t<7>(in, out, batch, stw, inverse, stream);
    case 8: return launch_batched_t<8>(in, out, batch, stw, inverse, stream);
    case 9: return launch_batched_t<9>(in, out, batch, stw, inverse, stream);
    case 10: return launch_batched_t<10>(in, out, batch, stw, inverse, stream);
    case 11: return launch_batched_t<11>(in, out, batch, stw, inverse, stream);
    case 12: return launch_batched_t<12>(in, out, batch, stw, inverse, stream);
    case 13: return launch_batched_t<13>(in, out, batch, stw, inverse, stream);
    case 14: return launch_batched_t<14>(in, out, batch, stw, inverse, stream);
    default: return cudaErrorInvalidValue;
    }
}

// Default tile width (columns per block) of a pass of length 2^log_l: 16 columns (one 128-byte
// line per row) up to 512 points, then 8 at 1024 and 4 beyond, so a tile holds at most 16384
// values (136 KiB of shared memory with padding at 4 x 4096).
int pass_log_c(int log_l) { return log_l <= 9 ? 4 : log_l == 10 ? 3 : 2; }

// Tile widths compiled for each pass length: 2^2 .. 2^4 columns with at most 16384 values, and
// 2 columns for lengths 2^10 .. 2^12 (two tiles of adjacent blocks then share each 32-byte
// sector of a row).
bool pass_tile_supported(int log_l, int log_c) {
    return log_l >= 4 && log_l <= 12 && log_c <= 4 && log_l + log_c <= 14 && (log_c >= 2 || (log_c == 1 && log_l >= 10));
}

template <int LOG_L, int LOG_C, int MODE>
static cudaError_t launch_pass_t(const PassArgs& a, int batch, cudaStream_t stream) {
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    // the tile, then the inter-pass twiddle factors (17 per column)
    constexpr int SMEM = smem_bytes(LOG_L, LOG_C) + (MODE == 2 ? 0 : (int)sizeof(float2) * 17 * (1 << LOG_C));
    auto kernel = k_pass<LOG_L, LOG_C, MODE>;
    static cudaError_t attr = set_smem(kernel, SMEM);
    if (attr != cudaSuccess) return attr;
    unsigned cols = 1u << (a.log2n - LOG_L);
    dim3 grid(a.ntiles ? a.ntiles : cols >> LOG_C, 1, 1);
    PassArgs b = a;
    if (!a.ntiles) b.tli = 31;
    while (batch > 0) {
        int now = batch < 65535 ? batch : 65535;
        grid.y = (unsigned)now;
        kernel<<<grid, THREADS, SMEM, stream>>>(b);
        b.in += (long long)now << a.log2n;
        b.out += (long long)now << a.log2n;
        batch -= now;
    }
    return cudaGetLastError();
}

template <int LOG_L, int MODE>
static cudaError_t launch_pass_c(int log_c, const PassArgs& a, int batch, cudaStream_t stream) {
    if constexpr (LOG_L >= 10) {
        if (log_c == 1) return launch_pass_t<LOG_L, 1, MODE>(a, batch, stream);
    }
    if (log_c == 2) return launch_pass_t<LOG_L, 2, MODE>(a, batch, stream);
    if constexpr (LOG_L + 3 <= 14) {
        if (log_c == 3) return launch_pass_t<LOG_L, 3, MODE>(a, batch, stream);
    }
    if constexpr (LOG_L + 4 <= 14) {
        if (log_c == 4) return launch_pass_t<LOG_L, 4, MODE>(a, batch, stream);
    }
    return cudaErrorInvalidValue;
}

template <int MODE>
static cudaError_t launch_pass_mode(int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t stream) {
    switch (log_l) {
    case 4: return launch_pass_c<4, MODE>(log_c, a, batch, stream);
    case 5: return launch_pass_c<5, MODE>(log_c, a, batch, stream);
    case 6: return launch_pass_c<6, MODE>(log_c, a, batch, stream);
    case 7: return launch_pass_c<7, MODE>(log_c, a, batch, stream);
    case 8: return launch_pass_c<8, MODE>(log_c, a, batch, stream);
    case 9: return launch_pass_c<9, MODE>(log_c, a, batch, stream);
    case 10: return launch_pass_c<10, MODE>(log_c, a, batch, stream);
    case 11: return launch_pass_c<11, MODE>(log_c, a, batch, stream);
    case 12: return launch_pass_c<12, MODE>(log_c, a, batch, stream);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_pass(int mode, int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t stream) {
    if (!pass_tile_supported(log_l, log_c)) return cudaErrorInvalidValue;
    switch (mode) {
    case 0: return launch_pass_mode<0>(log_l, log_c, a, batch, stream);
    case 1: return launch_pass_mode<1>(log_l, log_c, a, batch, stream);
    default: return launch_pass_mode<2>(log_l, log_c, a, batch, stream);
    }
}

int stage_table_entries_host(int log_l) { return stage_table_entries(log_l); }

cudaError_t launch_stage_table(float2* dst, int log_l, cudaStream_t stream) {
    int total = stage_table_entries(log_l);
    if (total == 0) return cudaSuccess;
    k_stage_table<<<(total + 255) / 256, 256, 0, stream>>>(dst, log_l, total);
    return cudaGetLastError();
}

cudaError_t launch_big_table(double2* lo, double2* hi, int log2n, int lo_bits, cudaStream_t stream) {
    int total = (1 << lo_bits) + (1 << (log2n - lo_bits));
    k_big_table<<<(total + 255) / 256, 256, 0, stream>>>(lo, hi, log2n, lo_bits);
    return cudaGetLastError();
}

}  // namespace ofb

namespace ofb {

__global__ void k_twiddle_probe(float2* __restrict__ dst, unsigned log2n, unsigned long long count) {
    unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double2 w = root_f64(k, log2n);
    dst[k] = make_float2((float)w.x, (float)w.y);
}

cudaError_t launch_twiddle_probe(float2* dst, unsigned log2n, unsigned long long count, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    k_twiddle_probe<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(dst, log2n, count);
    return cudaGetLastError();
}

}  // namespace ofb
