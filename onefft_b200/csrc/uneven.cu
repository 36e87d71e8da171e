// Uneven batches: many transforms of different power-of-two sizes in ONE persistent launch.
//
// OneFFT has no batch interface: its callers loop over transforms, one onefft_plan_forward /
// _inverse call each, possibly from several threads (OneFFT include/onefft.h:102-106). Here the
// whole list runs as one kernel:
//   - onefft_uneven_create() validates the (log2 n, offset, direction) descriptors on the host,
//     sorts them largest first (longest-processing-time order) and groups equal sizes into work
//     items: up to 256 transforms of n <= 8 (one thread each), 4096 / n transforms of
//     16 <= n <= 4096 (one block tile, the plain path's batched tile), or one transform of
//     2^13 .. 2^16 (both passes of a two-pass split run by the same block, tile after tile, with
//     the intermediate values in `out`, i.e. in L2);
//   - k_uneven: every block loops, taking the next work item from a device counter, until the
//     queue is empty. No block ever waits for another.
//   - the memset of the counter plus the launch form a CUDA graph built at creation; execute
//     patches the buffer pointers into the kernel node and replays it.
// Per work item the arithmetic is the plain path's tile body (fft_tiles.cuh) with the plain
// path's tables, so results equal onefft_dev_*_batched of each transform bit for bit wherever
// the split is the same (every size except 2^13 and 2^14, which the plain path runs as one
// kernel of 512 / 1024 threads and the uneven kernel as two passes of 256-thread tiles).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <new>
#include <vector>

#include "onefft_cuda.h"
#include "fft_tiles.cuh"
#include "uneven.h"

namespace ofb {

// Two-pass split of the sizes handled by one block: (L0, L1) per log2 n.
template <int M>
struct BigSplit;
template <>
struct BigSplit<13> {
    static constexpr int L0 = 7, L1 = 6;
};
template <>
struct BigSplit<14> {
    static constexpr int L0 = 7, L1 = 7;
};
template <>
struct BigSplit<15> {
    static constexpr int L0 = 8, L1 = 7;
};
template <>
struct BigSplit<16> {
    static constexpr int L0 = 8, L1 = 8;
};

int uneven_split(int m, int pass) {
    switch (m) {
    case 13: return pass ? BigSplit<13>::L1 : BigSplit<13>::L0;
    case 14: return pass ? BigSplit<14>::L1 : BigSplit<14>::L0;
    case 15: return pass ? BigSplit<15>::L1 : BigSplit<15>::L0;
    case 16: return pass ? BigSplit<16>::L1 : BigSplit<16>::L0;
    default: return 0;
    }
}

// Tile width of an in-block pass of length 2^L: 16 columns, fewer when the tile would exceed
// 4096 values; such tiles have 16 L / 16 <= 256 threads and 256 / threads of them run side by
// side in one block.
__host__ __device__ constexpr int inblock_log_c(int l) { return l <= 8 ? 4 : 12 - l; }

constexpr int kUnevenThreads = 256;

__host__ __device__ constexpr int inblock_pass_smem(int l, int mode) {
    return (kUnevenThreads >> (l + inblock_log_c(l) - 4)) * pass_smem_bytes(l, inblock_log_c(l), mode);
}

// Both passes of one 2^M transform by one block.
template <int M>
__device__ __forceinline__ void big_item(const UnevenArgs& a, const onefft_desc& d, float2* smem, int tid) {
    constexpr int L0 = BigSplit<M>::L0, L1 = BigSplit<M>::L1;
    PassArgs p{};
    p.in = a.in + d.offset;
    p.out = a.out + d.offset;
    p.log2n = M;
    p.tw_lo = a.tw_lo[M];
    p.tw_hi = a.tw_hi[M];
    p.lo_bits = a.lo_bits[M];
    p.tli = 31;
    {
        constexpr int LC = inblock_log_c(L0), TT = 1 << (L0 + LC - 4), G = kUnevenThreads / TT;
        constexpr int NT = 1 << (M - L0 - LC);
        p.log_s = M - L0;
        p.rev_b1 = L1;
        p.rev_b2 = 0;
        p.swap_in = d.inverse;
        p.swap_out = 0;
        p.stw = a.stw[M][0];
        float2* sm = smem + (tid / TT) * (pass_smem_bytes(L0, LC, 0) / (int)sizeof(float2));
        // A first-pass tile ends by reading its transposed results back from shared memory;
        // the barrier keeps the next tile's exchanges from overwriting them while slower warps
        // still read.
#pragma unroll 1
        for (int t = 0; t < NT; t += G) {
            pass_tile<L0, LC, 0>(p, (unsigned)(t + tid / TT), 0, sm, tid % TT);
            __syncthreads();
        }
    }
    // (the last barrier of the loop makes pass 0's global writes visible to the whole block)
    {
        constexpr int LC = inblock_log_c(L1), TT = 1 << (L1 + LC - 4), G = kUnevenThreads / TT;
        constexpr int NT = 1 << (M - L1 - LC);
        p.in = p.out;
        p.log_s = L0;
        p.swap_in = 0;
        p.swap_out = d.inverse;
        p.stw = a.stw[M][1];
        float2* sm = smem + (tid / TT) * (pass_smem_bytes(L1, LC, 2) / (int)sizeof(float2));
#pragma unroll 1
        for (int t = 0; t < NT; t += G) {
            pass_tile<L1, LC, 2>(p, (unsigned)(t + tid / TT), 0, sm, tid % TT);
            __syncthreads();  // as above (this pass's tiles end in registers; kept for symmetry)
        }
    }
}

template <int M>
__device__ __forceinline__ void batch_item(const UnevenArgs& a, const UnevenItem& w, float2* smem, int tid) {
    constexpr int LOG_C = 12 - M;
    const int c = tid >> (M - 4);
    const bool active = c < w.count;
    const onefft_desc d = a.desc[w.first + (active ? c : 0)];
    batched_tile<M, LOG_C>(a.in + d.offset, a.out + d.offset, active, d.inverse, a.stw[M][0], smem, tid);
}

template <int M>
__device__ __forceinline__ void tiny_item(const UnevenArgs& a, const UnevenItem& w, int tid) {
    if (tid < w.count) {
        const onefft_desc d = a.desc[w.first + tid];
        tiny_transform<M>(a.in + d.offset, a.out + d.offset, d.inverse);
    }
}

// Four resident blocks per SM (64 registers, a few spilled values): measured on a B200 with
// 20000 transforms of 2^4 .. 2^16, 1.21 ms at 2 blocks per SM (128 registers), 1.14 ms at 3
// (80 registers), 1.12 ms at 4; items are latency-bound tile sequences, so more resident blocks
// hide more of each block's waits.
__global__ void __launch_bounds__(kUnevenThreads, 4) k_uneven(UnevenArgs a) {
    extern __shared__ float2 smem[];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int it = s_item;
        __syncthreads();  // every thread has read s_item before it is overwritten
        if (it >= a.nitems) break;
        const UnevenItem w = a.items[it];
        switch (w.log2n) {
        case 0: tiny_item<0>(a, w, tid); break;
        case 1: tiny_item<1>(a, w, tid); break;
        case 2: tiny_item<2>(a, w, tid); break;
        case 3: tiny_item<3>(a, w, tid); break;
        case 4: batch_item<4>(a, w, smem, tid); break;
        case 5: batch_item<5>(a, w, smem, tid); break;
        case 6: batch_item<6>(a, w, smem, tid); break;
        case 7: batch_item<7>(a, w, smem, tid); break;
        case 8: batch_item<8>(a, w, smem, tid); break;
        case 9: batch_item<9>(a, w, smem, tid); break;
        case 10: batch_item<10>(a, w, smem, tid); break;
        case 11: batch_item<11>(a, w, smem, tid); break;
        case 12: batch_item<12>(a, w, smem, tid); break;
        case 13: big_item<13>(a, a.desc[w.first], smem, tid); break;
        case 14: big_item<14>(a, a.desc[w.first], smem, tid); break;
        case 15: big_item<15>(a, a.desc[w.first], smem, tid); break;
        case 16: big_item<16>(a, a.desc[w.first], smem, tid); break;
        default: break;
        }
        __syncthreads();  // the next item may reuse shared memory
    }
}

int uneven_smem_bytes() {
    int s = smem_bytes(12, 0);
    for (int m = 13; m <= 16; ++m) {
        s = std::max(s, inblock_pass_smem(uneven_split(m, 0), 0));
        s = std::max(s, inblock_pass_smem(uneven_split(m, 1), 2));
    }
    return s;
}

const void *uneven_kernel() { return (const void *)k_uneven; }

}  // namespace ofb
