// The transform kernels for sm_100a and their launchers.
//
//   k_tiny     n = 1, 2, 4, 8: 8 / n transforms per thread in registers, 2048 values per block
//              loaded and stored coalesced through shared memory.
//   k_batched  n = 16 .. 2^14 in one kernel: each block holds C whole transforms (by default
//              max(1, 4096 / n), or half or twice that as the plan's tuned width says; C n / 16
//              threads, 16 values per thread), Stockham radix-16 stages in registers with
//              exchanges through padded shared memory. Loads and stores are 8-byte accesses
//              straight between HBM and registers, or for n <= 64 coalesced through shared memory.
//   k_pass     n > 2^14: one pass of a two- or three-pass four-step decomposition
//              n = L0 L1 (L2). A block transforms a tile of C adjacent columns of length Lp.
//              Pass 0 reads the input in natural order (columns are adjacent addresses),
//              multiplies by w_n^(r k) and writes each column's result as one contiguous run
//              into `out`, at a digit-reversed column position; passes 1.. work in place on
//              `out` with the stride of the digits already done, so the final pass leaves the
//              result in natural order and no workspace beyond `out` is needed.
// The tile bodies live in fft_tiles.cuh, shared with the persistent uneven-batch kernel.
//
// Replaces the generated SIMD pass chain of OneFFT (src/onefft_*.inc driven by
// onefft_execute_passes, src/onefft.c:274-297): the mathematics (a radix split of the DFT with
// twiddles between stages, inverse by exchanging re/im) is the same; the data movement is the
// GPU's own.
#include "fft_tiles.cuh"

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

// FP32-rounded twiddles w_(2^log2n)^k, k < count: the device evaluation of the twiddle rule.
__global__ void k_twiddle_probe(float2* __restrict__ dst, unsigned log2n, unsigned long long count) {
    unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
    double2 w = root_f64(k, log2n);
    dst[k] = make_float2((float)w.x, (float)w.y);
}

// ---- kernels --------------------------------------------------------------------------------------

// W: the pointwise weights pre / post are applied (instantiated only for weighted calls).
// Each thread transforms the 8 / n consecutive transforms of 8 consecutive values, so a block
// covers 2048 values. The block's transforms are one contiguous run, loaded and stored with
// consecutive threads on consecutive values through shared memory (padded one slot per 16, so
// each thread's 8 values, 64 bytes from its neighbour's, sit in distinct banks). Loading each
// thread's own values directly touched 32 lines per warp instruction: an n = 8 batch of 2^26
// values took 324 us (ncu, 39 % of DRAM bandwidth, load/store throttled). Same arithmetic as
// tiny_transform, so the same bits.
constexpr int kTinyValues = 2048;  // values per block
template <int LOG_N, bool W>
__global__ void __launch_bounds__(256) k_tiny(const float2* __restrict__ in, float2* __restrict__ out,
                                              long long batch, int inverse, const float2* __restrict__ pre,
                                              const float2* __restrict__ post) {
    constexpr int N = 1 << LOG_N, PER = 8 >> LOG_N, PB = kTinyValues >> LOG_N;  // per thread, per block
    __shared__ float2 s[kTinyValues + (kTinyValues >> 4)];
    const long long first = (long long)blockIdx.x * PB;
    const int count = batch - first < PB ? (int)(batch - first) : PB;
    const int total = count << LOG_N;
    const float2* src = in + (first << LOG_N);
    float2* dst = out + (first << LOG_N);
    for (int i = threadIdx.x; i < total; i += 256) s[spad(i)] = __ldg(src + i);
    __syncthreads();
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int t = threadIdx.x * PER + p;
        if (t >= count) break;
        float2 a[N];
#pragma unroll
        for (int i = 0; i < N; ++i) {
            a[i] = s[spad(t * N + i)];
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
            s[spad(t * N + i)] = y;
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < total; i += 256) dst[i] = s[spad(i)];
}

// The block's 2^LOG_C transforms of n = 16 .. 64 through shared memory. Each thread's 16
// values of one transform lie T = n / 16 apart, so direct loads touch 32 / T different lines per
// warp instruction (for n = 16 one value of each); the block's transforms are one contiguous run,
// so it is loaded and stored with consecutive threads on consecutive values instead, in the
// padded layout the exchanges use (transform c's value e at spad(c n + e)). Measured on a B200
// with 2^25 values per batch and 4096-value tiles, forward: n = 16 303 -> 90 us, n = 32 162 -> 94,
// n = 64 104 -> 96 (82 us is the copy bound of the 537 MB moved); 2048-value tiles 86-87 us.
template <int LOG_L, int LOG_C, int INV>
__device__ __forceinline__ void batched_tile_staged(const float2* __restrict__ in, float2* __restrict__ out,
                                                    long long batch, const float2* __restrict__ stw, float2* smem,
                                                    int tid) {
    constexpr int L = 1 << LOG_L, T = L / 16, THREADS = 1 << (LOG_L + LOG_C - 4);
    const long long g0 = (long long)blockIdx.x << LOG_C;
    const long long left = batch - g0;
    const int valid = (left < (1 << LOG_C) ? (int)left : (1 << LOG_C)) << LOG_L;  // values of this block
    const float2* src = in + (g0 << LOG_L);
    float2* dst = out + (g0 << LOG_L);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int x = tid + THREADS * i;
        smem[spad(x)] = x < valid ? ld_stream(src + x) : make_float2(0.f, 0.f);
    }
    __syncthreads();
    const int c = tid >> (LOG_L - 4), j = tid & (T - 1);
    float2 v[16];
    {
        const float2* r = smem + spad(c * L + j);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = INV ? swap_ri(r[padc(k * T)]) : r[padc(k * T)];
    }
    __syncthreads();  // every input is in registers before the exchanges reuse the memory
    tile_fft<LOG_L, 1>(v, j, stw, smem, c << LOG_L);
    __syncthreads();  // n = 16 has no exchange: other threads may still be reading inputs
    {
        float2* w = smem + spad(c * L + j);
#pragma unroll
        for (int k = 0; k < 16; ++k) w[padc(k * T)] = INV ? swap_ri(v[k]) : v[k];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int x = tid + THREADS * i;
        if (x < valid) dst[x] = smem[spad(x)];
    }
}

// INV: the direction as a compile-time constant (the re/im exchanges on load and store then
// cost nothing in the forward kernel and no selects in the inverse one).
template <int LOG_L, int LOG_C, bool W, int INV>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4))
    k_batched(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
              const float2* __restrict__ stw, const float2* __restrict__ pre, const float2* __restrict__ post) {
    extern __shared__ float2 smem[];
    const int tid = threadIdx.x;
    if constexpr (LOG_L <= 6 && !W) {
        batched_tile_staged<LOG_L, LOG_C, INV>(in, out, batch, stw, smem, tid);
    } else {
        const long long g = ((long long)blockIdx.x << LOG_C) + (tid >> (LOG_L - 4));
        batched_tile<LOG_L, LOG_C, false, W>(in + (g << LOG_L), out + (g << LOG_L), g < batch, INV, stw, smem, tid,
                                             pre, post);
    }
}

template <int LOG_L, int LOG_C, int MODE, bool W, bool X = false>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4)) k_pass(PassArgs a) {
    extern __shared__ float2 smem[];
    pass_tile<LOG_L, LOG_C, MODE, 0, W, false, X>(a, blockIdx.x, X ? 0ll : (long long)blockIdx.y << a.log2n, smem,
                                                  threadIdx.x);
}

// ---- launchers -------------------------------------------------------------------------------------

constexpr int default_batched_log_c(int log_l) { return log_l >= 12 ? 0 : 12 - log_l; }

int batched_log_c(int log_l) { return default_batched_log_c(log_l); }

bool batched_log_c_supported(int log_l, int log_c) {
    if (log_l < 4 || log_l > kMaxSingleLog2) return false;
    const int b = default_batched_log_c(log_l);
    return log_c == b || (log_c >= 0 && log_c >= b - 1 && log_c <= b + 1 && log_l + log_c <= 13);
}

template <int LOG_L, bool W, int LOG_C>
static cudaError_t launch_batched_w(const float2* in, float2* out, long long batch, const float2* stw, int inverse,
                                    cudaStream_t stream, const float2* pre, const float2* post) {
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = smem_bytes(LOG_L, LOG_C);
    auto kernel = inverse ? k_batched<LOG_L, LOG_C, W, 1> : k_batched<LOG_L, LOG_C, W, 0>;
    static std::atomic<unsigned long long> done_fwd{0}, done_inv{0};
    cudaError_t attr = inverse ? smem_limit((const void*)k_batched<LOG_L, LOG_C, W, 1>, SMEM, done_inv)
                               : smem_limit((const void*)k_batched<LOG_L, LOG_C, W, 0>, SMEM, done_fwd);
    if (attr != cudaSuccess) return attr;
    const long long per_block = 1ll << LOG_C;
    long long blocks = (batch + per_block - 1) / per_block;
    while (blocks > 0) {  // gridDim.x limit 2^31-1
        long long now = blocks < 0x7fffffffll ? blocks : 0x7fffffffll;
        kernel<<<(unsigned)now, THREADS, SMEM, stream>>>(in, out, batch, stw, pre, post);
        long long done = now * per_block;
        in += done << LOG_L;
        out += done << LOG_L;
        batch -= done;
        blocks -= now;
    }
    return cudaGetLastError();
}

template <int LOG_L>
static cudaError_t launch_batched_t(const float2* in, float2* out, long long batch, const float2* stw, int inverse,
                                    cudaStream_t stream, const float2* pre, const float2* post, int log_c) {
    constexpr int B = default_batched_log_c(LOG_L);
    if (pre || post) return launch_batched_w<LOG_L, true, B>(in, out, batch, stw, inverse, stream, pre, post);
    if constexpr (B >= 1)
        if (log_c == B - 1)
            return launch_batched_w<LOG_L, false, B - 1>(in, out, batch, stw, inverse, stream, nullptr, nullptr);
    if constexpr (LOG_L + B + 1 <= 13)
        if (log_c == B + 1)
            return launch_batched_w<LOG_L, false, B + 1>(in, out, batch, stw, inverse, stream, nullptr, nullptr);
    return launch_batched_w<LOG_L, false, B>(in, out, batch, stw, inverse, stream, nullptr, nullptr);
}

template <int LOG_N>
static cudaError_t launch_tiny_t(const float2* in, float2* out, long long batch, int inverse, cudaStream_t stream,
                                 const float2* pre, const float2* post) {
    const bool w = pre || post;
    constexpr long long PB = kTinyValues >> LOG_N;  // transforms per block
    long long blocks = (batch + PB - 1) / PB;
    while (blocks > 0) {
        long long now = blocks < 0x7fffffffll ? blocks : 0x7fffffffll;
        if (w) k_tiny<LOG_N, true><<<(unsigned)now, 256, 0, stream>>>(in, out, batch, inverse, pre, post);
        else k_tiny<LOG_N, false><<<(unsigned)now, 256, 0, stream>>>(in, out, batch, inverse, nullptr, nullptr);
        long long done = now * PB;
        in += done << LOG_N;
        out += done << LOG_N;
        batch -= done;
        blocks -= now;
    }
    return cudaGetLastError();
}

cudaError_t launch_single_kernel(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                 int inverse, cudaStream_t stream, const float2* pre, const float2* post,
                                 int log_c) {
    if (batch <= 0) return cudaSuccess;
    switch (log2n) {
    case 0: return launch_tiny_t<0>(in, out, batch, inverse, stream, pre, post);
    case 1: return launch_tiny_t<1>(in, out, batch, inverse, stream, pre, post);
    case 2: return launch_tiny_t<2>(in, out, batch, inverse, stream, pre, post);
    case 3: return launch_tiny_t<3>(in, out, batch, inverse, stream, pre, post);
    case 4: return launch_batched_t<4>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 5: return launch_batched_t<5>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 6: return launch_batched_t<6>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 7: return launch_batched_t<7>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 8: return launch_batched_t<8>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 9: return launch_batched_t<9>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 10: return launch_batched_t<10>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 11: return launch_batched_t<11>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 12: return launch_batched_t<12>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 13: return launch_batched_t<13>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    case 14: return launch_batched_t<14>(in, out, batch, stw, inverse, stream, pre, post, log_c);
    default: return cudaErrorInvalidValue;
    }
}

// Default tile width (columns per block) of a pass of length 2^log_l: 16 columns (one 128-byte
// line per row) up to 512 points, then 8 at 1024 and 4 beyond, so a tile holds at most 16384
// values (136 KiB of shared memory with padding at 4 x 4096).
constexpr int default_pass_log_c(int log_l) { return log_l <= 9 ? 4 : log_l == 10 ? 3 : 2; }

int pass_log_c(int log_l) { return default_pass_log_c(log_l); }

// Tile widths compiled for each pass length: 2^2 .. 2^4 columns with at most 16384 values, and
// 2 columns for lengths 2^10 .. 2^12 (two tiles of adjacent blocks then share each 32-byte
// sector of a row).
bool pass_tile_supported(int log_l, int log_c) {
    return log_l >= 4 && log_l <= 12 && log_c <= 4 && log_l + log_c <= 14 &&
           (log_c >= 2 || (log_c == 1 && log_l >= 10));
}

template <int LOG_L, int LOG_C, int MODE, bool W>
static cudaError_t launch_pass_w(const PassArgs& a, int batch, cudaStream_t stream) {
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = pass_smem_bytes(LOG_L, LOG_C, MODE);
    auto kernel = k_pass<LOG_L, LOG_C, MODE, W>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
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

// The weighted kernel only where a weight applies: the first pass's input, the last pass's output.
template <int LOG_L, int LOG_C, int MODE>
static cudaError_t launch_pass_t(const PassArgs& a, int batch, cudaStream_t stream) {
    if constexpr (MODE != 1) {
        if (MODE == 0 ? a.pre != nullptr : a.post != nullptr) return launch_pass_w<LOG_L, LOG_C, MODE, true>(a, batch, stream);
    }
    return launch_pass_w<LOG_L, LOG_C, MODE, false>(a, batch, stream);
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

// Column transforms: one launch over the whole matrix, default tile width, twiddle rows in
// shared memory in both modes.
template <int LOG_L, int MODE>
static cudaError_t launch_columns_t(const PassArgs& a, cudaStream_t stream) {
    constexpr int LOG_C = default_pass_log_c(LOG_L);
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = pass_smem_bytes(LOG_L, LOG_C, 1);
    auto kernel = k_pass<LOG_L, LOG_C, MODE, false, true>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    if (a.log2n > 31 || a.log2n < LOG_L + LOG_C) return cudaErrorInvalidValue;
    PassArgs b = a;
    b.tli = 31;
    kernel<<<1u << (a.log2n - LOG_L - LOG_C), THREADS, SMEM, stream>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_pass_columns(int mode, int log_l, const PassArgs& a, cudaStream_t stream) {
    if (mode != 0 && mode != 2) return cudaErrorInvalidValue;
#define OFB_COLUMNS_CASE(LL) \
    case LL: return mode == 0 ? launch_columns_t<LL, 0>(a, stream) : launch_columns_t<LL, 2>(a, stream);
    switch (log_l) {
        OFB_COLUMNS_CASE(4)
        OFB_COLUMNS_CASE(5)
        OFB_COLUMNS_CASE(6)
        OFB_COLUMNS_CASE(7)
        OFB_COLUMNS_CASE(8)
        OFB_COLUMNS_CASE(9)
        OFB_COLUMNS_CASE(10)
        OFB_COLUMNS_CASE(11)
        OFB_COLUMNS_CASE(12)
    default: return cudaErrorInvalidValue;
    }
#undef OFB_COLUMNS_CASE
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

cudaError_t launch_twiddle_probe(float2* dst, unsigned log2n, unsigned long long count, cudaStream_t stream) {
    if (count == 0) return cudaSuccess;
    k_twiddle_probe<<<(unsigned)((count + 255) / 256), 256, 0, stream>>>(dst, log2n, count);
    return cudaGetLastError();
}

}  // namespace ofb
