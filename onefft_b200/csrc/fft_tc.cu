// Kernels and launchers of the split-BF16 tensor-core variants (engine in fft_tc.cuh): the same
// tiles, passes and tables as the FP32 kernels in fft_kernels.cu, with the radix-16 stages
// computed by mma.sync bf16 split products of TERMS = 3 (hi/lo) or 6 (hi/mid/lo) terms.
#include "fft_tiles.cuh"

namespace ofb {

template <int LOG_L, int LOG_C, int TERMS>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4))
    k_batched_tc(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                 const float2* __restrict__ stw, int inverse) {
    extern __shared__ float2 smem[];
    const int tid = threadIdx.x;
    const long long g = ((long long)blockIdx.x << LOG_C) + (tid >> (LOG_L - 4));
    batched_tile<LOG_L, LOG_C, TERMS>(in + (g << LOG_L), out + (g << LOG_L), g < batch, inverse, stw, smem, tid);
}

template <int LOG_L, int LOG_C, int MODE, int TERMS>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4)) k_pass_tc(PassArgs a) {
    extern __shared__ float2 smem[];
    pass_tile<LOG_L, LOG_C, MODE, TERMS>(a, blockIdx.x, (long long)blockIdx.y << a.log2n, smem, threadIdx.x);
}

template <int LOG_L, int TERMS>
static cudaError_t launch_batched_tc_t(const float2* in, float2* out, long long batch, const float2* stw, int inverse,
                                       cudaStream_t stream) {
    constexpr int LOG_C = LOG_L >= 12 ? 0 : 12 - LOG_L;
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = smem_bytes(LOG_L, LOG_C);
    auto kernel = k_batched_tc<LOG_L, LOG_C, TERMS>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    const long long per_block = 1ll << LOG_C;
    long long blocks = (batch + per_block - 1) / per_block;
    while (blocks > 0) {
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

template <int TERMS>
static cudaError_t launch_single_tc_terms(int log2n, const float2* in, float2* out, long long batch,
                                          const float2* stw, int inverse, cudaStream_t stream) {
    switch (log2n) {
    case 4: return launch_batched_tc_t<4, TERMS>(in, out, batch, stw, inverse, stream);
    case 5: return launch_batched_tc_t<5, TERMS>(in, out, batch, stw, inverse, stream);
    case 6: return launch_batched_tc_t<6, TERMS>(in, out, batch, stw, inverse, stream);
    case 7: return launch_batched_tc_t<7, TERMS>(in, out, batch, stw, inverse, stream);
    case 8: return launch_batched_tc_t<8, TERMS>(in, out, batch, stw, inverse, stream);
    case 9: return launch_batched_tc_t<9, TERMS>(in, out, batch, stw, inverse, stream);
    case 10: return launch_batched_tc_t<10, TERMS>(in, out, batch, stw, inverse, stream);
    case 11: return launch_batched_tc_t<11, TERMS>(in, out, batch, stw, inverse, stream);
    case 12: return launch_batched_tc_t<12, TERMS>(in, out, batch, stw, inverse, stream);
    case 13: return launch_batched_tc_t<13, TERMS>(in, out, batch, stw, inverse, stream);
    case 14: return launch_batched_tc_t<14, TERMS>(in, out, batch, stw, inverse, stream);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_single_kernel_tc(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                    int inverse, int terms, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    return terms == 6 ? launch_single_tc_terms<6>(log2n, in, out, batch, stw, inverse, stream)
                      : launch_single_tc_terms<3>(log2n, in, out, batch, stw, inverse, stream);
}

// Tensor-core passes use the default tile width of each length (pass_log_c) and need whole
// warps: lengths 2^5 .. 2^12.
template <int LOG_L, int MODE, int TERMS>
static cudaError_t launch_pass_tc_t(const PassArgs& a, int batch, cudaStream_t stream) {
    constexpr int LOG_C = LOG_L <= 9 ? 4 : LOG_L == 10 ? 3 : 2;
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = pass_smem_bytes(LOG_L, LOG_C, MODE);
    auto kernel = k_pass_tc<LOG_L, LOG_C, MODE, TERMS>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    dim3 grid(1u << (a.log2n - LOG_L - LOG_C), 1, 1);
    PassArgs b = a;
    b.tli = 31;
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

template <int MODE, int TERMS>
static cudaError_t launch_pass_tc_mode(int log_l, const PassArgs& a, int batch, cudaStream_t stream) {
    switch (log_l) {
    case 5: return launch_pass_tc_t<5, MODE, TERMS>(a, batch, stream);
    case 6: return launch_pass_tc_t<6, MODE, TERMS>(a, batch, stream);
    case 7: return launch_pass_tc_t<7, MODE, TERMS>(a, batch, stream);
    case 8: return launch_pass_tc_t<8, MODE, TERMS>(a, batch, stream);
    case 9: return launch_pass_tc_t<9, MODE, TERMS>(a, batch, stream);
    case 10: return launch_pass_tc_t<10, MODE, TERMS>(a, batch, stream);
    case 11: return launch_pass_tc_t<11, MODE, TERMS>(a, batch, stream);
    case 12: return launch_pass_tc_t<12, MODE, TERMS>(a, batch, stream);
    default: return cudaErrorInvalidValue;
    }
}

template <int TERMS>
static cudaError_t launch_pass_tc_terms(int mode, int log_l, const PassArgs& a, int batch, cudaStream_t stream) {
    switch (mode) {
    case 0: return launch_pass_tc_mode<0, TERMS>(log_l, a, batch, stream);
    case 1: return launch_pass_tc_mode<1, TERMS>(log_l, a, batch, stream);
    default: return launch_pass_tc_mode<2, TERMS>(log_l, a, batch, stream);
    }
}

cudaError_t launch_pass_tc(int mode, int log_l, const PassArgs& a, int batch, int terms, cudaStream_t stream) {
    return terms == 6 ? launch_pass_tc_terms<6>(mode, log_l, a, batch, stream)
                      : launch_pass_tc_terms<3>(mode, log_l, a, batch, stream);
}

}  // namespace ofb
