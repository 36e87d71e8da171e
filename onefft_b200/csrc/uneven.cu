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
//   - k_uneven: every block loops, taking the next unit of work from a device counter, until the
//     queue is empty. A transform of 2^13 .. 2^16 is split into steps of 4096 values (its pass-0
//     tiles, then its pass-1 tiles) that any block may take; a pass-1 step waits (bounded) on a
//     per-transform counter of finished pass-0 steps, and the queue places it at least
//     kUnevenLagUnits units after them, so it rarely waits. Many blocks then share the few
//     transforms in flight, and the values between their passes stay in L2, where one block per
//     transform kept hundreds of megabytes of them in flight. (With no unit queue, as in
//     onefft_uneven_execute_noalloc, every block runs whole transforms; the same bits either way.)
//   - the memset of the counter plus the launch form a CUDA graph built at creation; execute
//     patches the buffer pointers into the kernel node and replays it.
// Per work item the arithmetic is the plain path's tile body (fft_tiles.cuh) with the plain
// path's tables, so results equal onefft_dev_*_batched of each transform bit for bit wherever
// the split is the same (every size except 2^13 and 2^14, which the plain path runs as one
// kernel of 512 / 1024 threads and the uneven kernel as two passes of 256-thread tiles).
// The two-pass split of 2^13 .. 2^16 is one of three compiled candidates per size, picked by the
// autotuner (kUnevenTunedSplit); the kernel is compiled once per combination it runs.
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

int uneven_split(int m, int choice, int pass) {
    if (m < 13 || m > 16 || choice < 0 || choice >= kUnevenSplitChoices) return 0;
    return kUnevenSplits[m - 13][choice][pass ? 1 : 0];
}

// Tile width of an in-block pass of length 2^L: 16 columns, fewer when the tile would exceed
// 4096 values; such tiles have 16 L / 16 <= 256 threads and 256 / threads of them run side by
// side in one block.
__host__ __device__ constexpr int inblock_log_c(int l) { return l <= 8 ? 4 : 12 - l; }

constexpr int kUnevenThreads = 256;

__host__ __device__ constexpr int inblock_pass_smem(int l, int mode) {
    return (kUnevenThreads >> (l + inblock_log_c(l) - 4)) * pass_smem_bytes(l, inblock_log_c(l), mode);
}

// What the two passes of one 2^M transform take from UnevenArgs (small enough to pass by value).
struct BigItemArgs {
    const float2* in;
    float2* out;
    const double2* tw_lo;
    const double2* tw_hi;
    const float2* stw0;
    const float2* stw1;
    int lo_bits;
    int inverse;
};

// Both passes of one 2^M transform, split 2^L0 x 2^L1, by one block.
template <int M, int L0, int L1>
__device__ __forceinline__ void big_item(const BigItemArgs& b, float2* smem, int tid) {
    PassArgs p{};
    p.in = b.in;
    p.out = b.out;
    p.log2n = M;
    p.tw_lo = b.tw_lo;
    p.tw_hi = b.tw_hi;
    p.lo_bits = b.lo_bits;
    p.tli = 31;
    {
        constexpr int LC = inblock_log_c(L0), TT = 1 << (L0 + LC - 4), G = kUnevenThreads / TT;
        constexpr int NT = 1 << (M - L0 - LC);
        p.log_s = M - L0;
        p.rev_b1 = L1;
        p.rev_b2 = 0;
        p.swap_in = b.inverse;
        p.swap_out = 0;
        p.stw = b.stw0;
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
        p.swap_out = b.inverse;
        p.stw = b.stw1;
        float2* sm = smem + (tid / TT) * (pass_smem_bytes(L1, LC, 2) / (int)sizeof(float2));
#pragma unroll 1
        for (int t = 0; t < NT; t += G) {
            pass_tile<L1, LC, 2>(p, (unsigned)(t + tid / TT), 0, sm, tid % TT);
            __syncthreads();  // as above (this pass's tiles end in registers; kept for symmetry)
        }
    }
}

// One step (4096 values) of a 2^M transform split 2^L0 x 2^L1, for the step-wise queue: steps
// 0 .. S - 1 run tiles of pass 0 and publish them in the item's counter; steps S .. 2S - 1 run
// tiles of pass 1 once every pass-0 step of the item is published (bounded wait). S = 2^(M - 12).
// The tiles are the ones big_item runs, with the same arithmetic, so results are the same bits.
template <int M, int L0, int L1>
__device__ __forceinline__ void big_step(const BigItemArgs& b, unsigned* done, unsigned* abort, unsigned* err, int step,
                                         float2* smem, int tid) {
    constexpr int S = 1 << (M - 12);
    PassArgs p{};
    p.in = b.in;
    p.out = b.out;
    p.log2n = M;
    p.tw_lo = b.tw_lo;
    p.tw_hi = b.tw_hi;
    p.lo_bits = b.lo_bits;
    p.tli = 31;
    if (step < S) {
        constexpr int LC = inblock_log_c(L0), TT = 1 << (L0 + LC - 4), G = kUnevenThreads / TT;
        p.log_s = M - L0;
        p.rev_b1 = L1;
        p.rev_b2 = 0;
        p.swap_in = b.inverse;
        p.swap_out = 0;
        p.stw = b.stw0;
        float2* sm = smem + (tid / TT) * (pass_smem_bytes(L0, LC, 0) / (int)sizeof(float2));
        pass_tile<L0, LC, 0>(p, (unsigned)(step * G + tid / TT), 0, sm, tid % TT);
        __syncthreads();  // every thread's stores of the step are issued
        if (tid == 0) {
            __threadfence();  // ... and visible at GPU scope before the count says so
            atomicAdd(done, 1u);
        }
    } else {
        bool ready = true;
        if (tid == 0) {
            // abort: the word after the last item's counter, set by the first wait that runs
            // out, so that no other block waits its full limit for work that will not come
            ready = wait_count_or_abort(done, (unsigned)S, abort);
            if (!ready) {
                *(volatile unsigned*)abort = 1u;
                *(volatile unsigned*)err = 3u;
            }
        }
        if (__syncthreads_or(!ready)) return;
        constexpr int LC = inblock_log_c(L1), TT = 1 << (L1 + LC - 4), G = kUnevenThreads / TT;
        p.in = p.out;
        p.log_s = L0;
        p.swap_in = 0;
        p.swap_out = b.inverse;
        p.stw = b.stw1;
        float2* sm = smem + (tid / TT) * (pass_smem_bytes(L1, LC, 2) / (int)sizeof(float2));
        // pass 0 of this transform was written by other blocks: load through L2 only
        pass_tile<L1, LC, 2, false, false, true>(p, (unsigned)((step - S) * G + tid / TT), 0, sm, tid % TT);
    }
}

template <int M, int L0, int L1>
__device__ __noinline__ void big_step_call(const BigItemArgs b, unsigned* done, unsigned* abort, unsigned* err, int step,
                                           float2* smem, int tid) {
    big_step<M, L0, L1>(b, done, abort, err, step, smem, tid);
}

// Any compiled split as a call, for the kernel that picks splits at run time. Inlining every
// split into one kernel raised its spills at 64 registers from 164 to 536 bytes, even with three
// identical splits; fixed kernels inline the one split they run.
template <int M, int L0, int L1>
__device__ __noinline__ void big_item_call(const BigItemArgs b, float2* smem, int tid) {
    big_item<M, L0, L1>(b, smem, tid);
}

// One 2^M transform with split CHOICE, or, for CHOICE = kSplitAtRunTime, the split the batch
// was created with (UnevenArgs::split).
constexpr int kSplitAtRunTime = -1;

template <int M, int CHOICE>
__device__ __forceinline__ void big_choice(const UnevenArgs& a, const onefft_desc& d, float2* smem, int tid) {
    constexpr int I = M - 13;
    const BigItemArgs b{a.in + d.offset, a.out + d.offset, a.tw_lo[M], a.tw_hi[M],
                        a.stw[M][0],     a.stw[M][1],      a.lo_bits[M], d.inverse};
    if constexpr (CHOICE != kSplitAtRunTime) {
        big_item<M, kUnevenSplits[I][CHOICE][0], kUnevenSplits[I][CHOICE][1]>(b, smem, tid);
    } else {
        static_assert(kUnevenSplitChoices == 3, "one branch per compiled split");
        switch (a.split[M]) {
        case 1: big_item_call<M, kUnevenSplits[I][1][0], kUnevenSplits[I][1][1]>(b, smem, tid); break;
        case 2: big_item_call<M, kUnevenSplits[I][2][0], kUnevenSplits[I][2][1]>(b, smem, tid); break;
        default: big_item_call<M, kUnevenSplits[I][0][0], kUnevenSplits[I][0][1]>(b, smem, tid); break;
        }
    }
}

// One step of a 2^M transform (item `it`) with split CHOICE (or the batch's split, see big_choice).
template <int M, int CHOICE>
__device__ __forceinline__ void step_choice(const UnevenArgs& a, int it, const onefft_desc& d, int step, float2* smem,
                                            int tid) {
    constexpr int I = M - 13;
    const BigItemArgs b{a.in + d.offset, a.out + d.offset, a.tw_lo[M], a.tw_hi[M],
                        a.stw[M][0],     a.stw[M][1],      a.lo_bits[M], d.inverse};
    unsigned* abort = a.done + a.nitems;
    if constexpr (CHOICE != kSplitAtRunTime) {
        big_step<M, kUnevenSplits[I][CHOICE][0], kUnevenSplits[I][CHOICE][1]>(b, a.done + it, abort, a.err, step, smem,
                                                                             tid);
    } else {
        switch (a.split[M]) {
        case 1:
            big_step_call<M, kUnevenSplits[I][1][0], kUnevenSplits[I][1][1]>(b, a.done + it, abort, a.err, step, smem,
                                                                           tid);
            break;
        case 2:
            big_step_call<M, kUnevenSplits[I][2][0], kUnevenSplits[I][2][1]>(b, a.done + it, abort, a.err, step, smem,
                                                                           tid);
            break;
        default:
            big_step_call<M, kUnevenSplits[I][0][0], kUnevenSplits[I][0][1]>(b, a.done + it, abort, a.err, step, smem,
                                                                           tid);
            break;
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
// C13 .. C16: the split of each size 2^13 .. 2^16 (an index into kUnevenSplits, or kSplitAtRunTime).
template <int C13, int C14, int C15, int C16>
__global__ void __launch_bounds__(kUnevenThreads, 4) k_uneven(UnevenArgs a) {
    extern __shared__ float2 smem[];
    __shared__ int s_item;
    const int tid = threadIdx.x;
    const int count = a.units ? a.nunits : a.nitems;
    if (tid == 0) s_item = atomicAdd(a.counter, 1);
    __syncthreads();
    int s = s_item;
    for (;; s = s_item) {
        __syncthreads();  // every thread has read s_item before it is overwritten
        if (s >= count) break;
        // the next unit's index, fetched while this one runs (its round trip to L2 would
        // otherwise hold the whole block between units)
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        int it = s, step = -1;
        if (a.units) {
            const UnevenUnit u = a.units[s];
            it = u.item;
            step = u.step;
        }
        const UnevenItem w = a.items[it];
        if (step >= 0) {
            const onefft_desc d = a.desc[w.first];
            switch (w.log2n) {
            case 13: step_choice<13, C13>(a, it, d, step, smem, tid); break;
            case 14: step_choice<14, C14>(a, it, d, step, smem, tid); break;
            case 15: step_choice<15, C15>(a, it, d, step, smem, tid); break;
            case 16: step_choice<16, C16>(a, it, d, step, smem, tid); break;
            default: break;
            }
            __syncthreads();  // the next unit may reuse shared memory
            continue;
        }
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
        case 13: big_choice<13, C13>(a, a.desc[w.first], smem, tid); break;
        case 14: big_choice<14, C14>(a, a.desc[w.first], smem, tid); break;
        case 15: big_choice<15, C15>(a, a.desc[w.first], smem, tid); break;
        case 16: big_choice<16, C16>(a, a.desc[w.first], smem, tid); break;
        default: break;
        }
        __syncthreads();  // the next item may reuse shared memory
    }
}

int uneven_smem_bytes() {
    int s = smem_bytes(12, 0);
    for (int m = 13; m <= 16; ++m)
        for (int c = 0; c < kUnevenSplitChoices; ++c) {
            s = std::max(s, inblock_pass_smem(uneven_split(m, c, 0), 0));
            s = std::max(s, inblock_pass_smem(uneven_split(m, c, 1), 2));
        }
    return s;
}

// The compiled kernels: every split inlined for the plain path's splits (choice 0 everywhere)
// and for the tuned choices, and one that reads the choices from its arguments (any other
// combination; the autotuner times candidates with it).
int uneven_tuned_split(int m) { return m >= 13 && m <= 16 ? kUnevenTunedSplit[m - 13] : 0; }

const void *uneven_kernel(const int *split) {
    bool plain = true, tuned = true;
    for (int m = 13; m <= kUnevenMaxLog2; ++m) {
        const int c = split ? split[m] : 0;
        plain = plain && c == 0;
        tuned = tuned && c == kUnevenTunedSplit[m - 13];
    }
    if (plain) return (const void *)k_uneven<0, 0, 0, 0>;
    if (tuned)
        return (const void *)k_uneven<kUnevenTunedSplit[0], kUnevenTunedSplit[1], kUnevenTunedSplit[2],
                                      kUnevenTunedSplit[3]>;
    return (const void *)k_uneven<kSplitAtRunTime, kSplitAtRunTime, kSplitAtRunTime, kSplitAtRunTime>;
}

}  // namespace ofb
