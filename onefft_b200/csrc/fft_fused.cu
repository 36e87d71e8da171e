// Fused weighted power loss and its gradient, one kernel per batch.
//
// For the differentiable-layer workload, loss = sum over transforms and k of w_k^2 |(F x)_k|^2
// and its gradient (torch's conjugate-Wirtinger convention) grad = F^H (2 w^2 * F x). Unfused this
// is a forward kernel, elementwise work on y in HBM and an adjoint kernel: about four round trips
// of the data. Here one block keeps each transform on chip: load x, forward Stockham stages,
// accumulate w^2 |y|^2, scale y by 2 w^2, adjoint stages (the forward engine with re/im exchanged
// on the way in and out), store the gradient — one read and one write of n values per transform.
// The arithmetic equals the unfused path's (the same tile engine, 2 w^2 y with exact scalings), so
// the gradient matches it bit for bit; the loss is a sum in another order.
#include "fft_tiles.cuh"

namespace ofb {

// Tiles of 2^11 .. 2^14 values are sized for 64 registers per thread (4 blocks of 256 threads or
// 2 of 512 per SM, without spills): left to itself the compiler took up to 80, which held the
// 8192-point tile to ONE block per SM (ncu: 24 % DRAM throughput, latency-bound); measured on a
// B200, 4096 x 8192 went from 256 to 220 us and 512 x 8192 from 43.7 to 41.2 us. Smaller tiles
// keep the compiler's choice (at 64 registers some spill and run slower).
template <int LOG_L, int LOG_C>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4), LOG_L >= 11 ? 65536 / (64 << (LOG_L + LOG_C - 4)) : 0)
    k_power_loss_grad(const float2* __restrict__ x, const float* __restrict__ w, float2* __restrict__ grad,
                      double* __restrict__ loss, long long batch, const float2* __restrict__ stw) {
    constexpr int L = 1 << LOG_L, T = L / 16, THREADS = 1 << (LOG_L + LOG_C - 4);
    extern __shared__ float2 smem[];
    __shared__ double warp_sum[THREADS / 32 > 0 ? THREADS / 32 : 1];
    const int tid = threadIdx.x;
    const int j = tid & (T - 1);
    const int c = tid >> (LOG_L - 4);
    const long long g = ((long long)blockIdx.x << LOG_C) + c;
    const bool active = g < batch;
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = active ? ld_stream(x + (g << LOG_L) + j + T * k) : make_float2(0.f, 0.f);
    tile_fft<LOG_L, 1>(v, j, stw, smem, c << LOG_L);
    // v[k] = y[j + T k]: loss terms and the scaled spectrum 2 w^2 y
    float part = 0.f;
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        const float wk = __ldg(w + j + T * k);
        const float w2 = wk * wk;
        part += (v[k].x * v[k].x + v[k].y * v[k].y) * w2;
        v[k] = make_float2(2.f * v[k].x * w2, 2.f * v[k].y * w2);
    }
    if (!active) part = 0.f;
    // block sum -> one double atomic per block
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
    if (THREADS >= 32) {
        if ((tid & 31) == 0) warp_sum[tid >> 5] = part;
    }
    // adjoint: F^H u = swap(F(swap(u)))
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = swap_ri(v[k]);
    tile_fft<LOG_L, 1>(v, j, stw, smem, c << LOG_L);  // its barriers also publish warp_sum
    if (Stages<LOG_L>::COUNT == 1) __syncthreads();
    if (tid == 0) {
        double s = 0;
        for (int i = 0; i < (THREADS >= 32 ? THREADS / 32 : 1); ++i) s += warp_sum[i];
        atomicAdd(loss, s);
    }
    if (active && grad) {
#pragma unroll
        for (int k = 0; k < 16; ++k) grad[(g << LOG_L) + j + T * k] = swap_ri(v[k]);
    }
}

template <int LOG_L>
static cudaError_t launch_loss_t(const float2* x, const float* w, float2* grad, double* loss, long long batch,
                                 const float2* stw, cudaStream_t stream) {
    constexpr int LOG_C = LOG_L >= 12 ? 0 : 12 - LOG_L;
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = smem_bytes(LOG_L, LOG_C);
    auto kernel = k_power_loss_grad<LOG_L, LOG_C>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    const long long per_block = 1ll << LOG_C;
    long long blocks = (batch + per_block - 1) / per_block;
    while (blocks > 0) {
        long long now = blocks < 0x7fffffffll ? blocks : 0x7fffffffll;
        kernel<<<(unsigned)now, THREADS, SMEM, stream>>>(x, w, grad, loss, batch, stw);
        long long done = now * per_block;
        x += done << LOG_L;
        if (grad) grad += done << LOG_L;
        batch -= done;
        blocks -= now;
    }
    return cudaGetLastError();
}

cudaError_t launch_power_loss_grad(int log2n, const float2* x, const float* w, float2* grad, double* loss,
                                   long long batch, const float2* stw, cudaStream_t stream) {
    switch (log2n) {
    case 4: return launch_loss_t<4>(x, w, grad, loss, batch, stw, stream);
    case 5: return launch_loss_t<5>(x, w, grad, loss, batch, stw, stream);
    case 6: return launch_loss_t<6>(x, w, grad, loss, batch, stw, stream);
    case 7: return launch_loss_t<7>(x, w, grad, loss, batch, stw, stream);
    case 8: return launch_loss_t<8>(x, w, grad, loss, batch, stw, stream);
    case 9: return launch_loss_t<9>(x, w, grad, loss, batch, stw, stream);
    case 10: return launch_loss_t<10>(x, w, grad, loss, batch, stw, stream);
    case 11: return launch_loss_t<11>(x, w, grad, loss, batch, stw, stream);
    case 12: return launch_loss_t<12>(x, w, grad, loss, batch, stw, stream);
    case 13: return launch_loss_t<13>(x, w, grad, loss, batch, stw, stream);
    case 14: return launch_loss_t<14>(x, w, grad, loss, batch, stw, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace ofb
