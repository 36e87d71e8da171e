// TMA-staged pass kernels (sm_100a): the tile of a pass — C adjacent columns of L values at a
// stride of S complex values — arrives in shared memory through ONE cp.async.bulk.tensor copy
// (a 4-D/5-D box over the strided array) instead of C*L/2 narrow strided loads, and the strided
// in-place passes write their tile back with one bulk tensor store. The arithmetic is the FP32
// tile engine of k_pass (fft_tiles.cuh), so results equal k_pass bit for bit.
//
// Why: with narrow tiles (C = 2 .. 8) every warp load touches many 8..64-byte row segments; the
// load/store unit and MIO queues saturate long before HBM does (ncu: lg/mio throttle stalls,
// 22-32 % issue active on the 2^12-point passes). The copy engine moves the same box with no
// per-thread address work.
//
// Waits on the mbarrier are bounded: if a copy does not complete within the limit, the kernel
// records the failure in the plan's error word, waits once more (bounded) and returns without
// touching global memory; host calls that synchronise report it.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "fft_tiles.cuh"

namespace ofb {

constexpr unsigned kWaitLimit = 1u << 22;  // try_wait polls (each may suspend briefly): ~0.1-1 s

// Test hook of the failure path (onefft_debug_expire_waits): when non-zero, the first wait of
// every tile counts as expired without polling. The tile then takes the same path as after a
// real expiry: it records the failure in the plan's error word, lets its copy land (the normal
// bounded wait) and returns without writing.
__device__ int g_expire_waits = 0;

cudaError_t set_expire_waits(int on) {
    const int v = on ? 1 : 0;
    return cudaMemcpyToSymbol(g_expire_waits, &v, sizeof v);
}

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned phase) {
    const unsigned a = smem_u32(bar);
    for (unsigned i = 0; i < kWaitLimit; ++i) {
        unsigned ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5, %6}], [%7];" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void tma_store_5d(const CUtensorMap* map, const void* src, int c0, int c1, int c2, int c3,
                                             int c4) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];" ::"l"(
            (unsigned long long)map),
        "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4)
        : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

// The same copies with an L2 eviction-priority hint (a createpolicy value).
__device__ __forceinline__ void tma_load_4d_hint(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                                 uint64_t* bar, unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, "
        "{%2, %3, %4, %5}], [%6], %7;" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ void tma_load_5d_hint(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                                 int c4, uint64_t* bar, unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1, "
        "{%2, %3, %4, %5, %6}], [%7], %8;" ::"r"(smem_u32(dst)),
        "l"((unsigned long long)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

__device__ __forceinline__ void tma_store_5d_hint(const CUtensorMap* map, const void* src, int c0, int c1, int c2,
                                                  int c3, int c4, unsigned long long policy) {
    asm volatile(
        "cp.async.bulk.tensor.5d.global.shared::cta.tile.bulk_group.L2::cache_hint [%0, {%2, %3, %4, %5, %6}], [%1], "
        "%7;" ::"l"((unsigned long long)map),
        "r"(smem_u32(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "l"(policy)
        : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
}

__device__ __forceinline__ unsigned long long policy_evict_first() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// Blocks per SM that the register allocation must allow (0: the compiler chooses freely). Measured
// on a B200: the last pass with 1024-value tiles of 8 columns (512 threads, 70 KB of shared
// memory) fits 3 blocks per SM at 40 registers instead of 2 at 41, which hides more of the tile
// copy's latency (2^27: 1.18 -> 1.13 ms); the first pass with 256-value tiles of 16 columns and
// the middle pass with 512-value tiles of 8 columns fit 5 at 48 registers instead of 4 at 51 / 55
// (2^27: 1.080 -> 1.073 -> 1.060 ms). Caps on the other shapes were slower (spills, or more
// blocks than the copy bandwidth needs).
template <int LOG_L, int LOG_C, int MODE>
constexpr int tma_min_blocks() {
    return LOG_L == 10 && LOG_C == 3 && MODE == 2 ? 3
           : LOG_L == 8 && LOG_C == 4 && MODE == 0 ? 5
           : LOG_L == 9 && LOG_C == 3 && MODE == 1 ? 5
                                                   : 0;
}

// Shared memory of a TMA-staged tile, in float2 units: the tile (dense as the copy lands, then
// reused padded by the exchanges), the inter-pass twiddle factors (17 per column); the block's
// mbarrier follows at this offset.
__host__ __device__ constexpr int tma_bar_offset(int log_l, int log_c) {
    return (1 << (log_l + log_c)) + (1 << (log_l + log_c - 4)) + 17 * (1 << log_c);
}
__host__ __device__ constexpr int tma_smem_bytes(int log_l, int log_c) {
    return (int)sizeof(float2) * (tma_bar_offset(log_l, log_c) + 2) + 16;
}

// One tile of a pass, MODE as k_pass, run by all threads of the block: the tile arrives through
// one bulk tensor copy completing on the block's mbarrier `bar` (phase parity `parity`); `fresh`:
// the barrier is initialised here (the block's first tile), else the generic accesses of the
// block's previous tile to the landing buffer are ordered before this copy overwrites it. `tin`
// maps the pass's input, `tout` its output (MODE 1/2: the same array, in place). Returns false,
// the same in every thread, if the copy's bounded wait expired: the tile then recorded the
// failure in the plan's error word, let the copy land and wrote nothing.
// W: the first pass multiplies its input by a.pre, the last pass its output by a.post
// (instantiated only for weighted calls).
// Hooks, for the persistent fused kernel: thread 0 calls ready() before issuing the copy (false:
// the tile is not run and tma_tile returns false), and issued() right after issuing it, so that
// work which waits on memory overlaps the copy; every thread calls landed() once the copy has
// landed, before the tile's arithmetic.
// X: a pass of a column transform (PassArgs' column fields, as pass_tile): the first pass takes
// its factor from the column fields and, with colstore, writes the column layout with plain
// stores; the last pass reads its tile from `tin` (a.in, the work array) and writes the column
// layout of a.out with plain stores instead of the bulk tensor store.
struct NoHook {
    __device__ void operator()() const {}
};
struct AlwaysReady {
    __device__ bool operator()() const { return true; }
};

template <int LOG_L, int LOG_C, int MODE, bool W, class Ready = AlwaysReady, class Issued = NoHook,
          class Landed = NoHook, bool X = false>
__device__ __forceinline__ bool tma_tile(const PassArgs& a, const CUtensorMap* tin, const CUtensorMap* tout,
                                         unsigned t, int b, float2* smem, uint64_t* bar, unsigned parity, bool fresh,
                                         int tid, Ready ready = Ready(), Issued issued = Issued(),
                                         Landed landed = Landed()) {
    constexpr int L = 1 << LOG_L, T = L / 16, C = 1 << LOG_C;
    const int c = tid & (C - 1);
    const int j = tid >> LOG_C;
    const unsigned col0 = a.tli >= 31 ? (t << LOG_C)
                                      : ((a.outer_base + (t >> a.tli)) << a.outer_shift) + a.inner_base +
                                            ((t & ((1u << a.tli) - 1)) << LOG_C);
    const int q0 = (int)(col0 & ((1u << a.log_s) - 1)), h = (int)(col0 >> a.log_s);
    bool go = true;
    if (tid == 0) {
        if (fresh) mbar_init(bar, 1);
        else asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        go = ready();
        if (go) {
            mbar_expect_tx(bar, (unsigned)(C * L * sizeof(float2)));
            // With l2_keep the array between passes should stay in L2: the input (read once)
            // and the last pass's tile (read for the last time) are loaded evict-first.
            if (a.l2_keep && MODE != 1) {
                const unsigned long long first = policy_evict_first();
                if (MODE == 0) tma_load_4d_hint(smem, tin, (int)col0, 0, 0, b, bar, first);
                else tma_load_5d_hint(smem, tin, q0, 0, 0, h, b, bar, first);
            } else if (MODE == 0) {
                tma_load_4d(smem, tin, (int)col0, 0, 0, b, bar);
            } else {
                tma_load_5d(smem, tin, q0, 0, 0, h, b, bar);
            }
            issued();
        }
    }
    // inter-pass twiddle factors (as pass_tile) while the copy is in flight
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
    // the barrier is initialised (and armed) before anyone waits on it
    if (__syncthreads_or(!go)) return false;  // nothing was issued: nothing to wait for
    const bool ok = !g_expire_waits && mbar_wait(bar, parity);
    if (__syncthreads_or(!ok)) {
        if (tid == 0) {
            *(volatile unsigned*)a.err = 1u;
            mbar_wait(bar, parity);  // let a late copy land before the memory is reused or released
        }
        return false;
    }
    landed();
    float2 v[16];
#pragma unroll
    for (int k = 0; k < 16; ++k) {
        float2 x = smem[(j + T * k) * C + c];
        // input element col0 + c + (j + T k) S of the transform (first pass only)
        if constexpr (W && MODE == 0) {
            if (a.pre) x = cmul(x, __ldg(a.pre + col0 + c + ((unsigned)(j + T * k) << a.log_s)));
        }
        v[k] = a.swap_in ? swap_ri(x) : x;
    }
    __syncthreads();  // the dense tile is consumed; the exchanges reuse its memory
    tile_fft<LOG_L, C>(v, j, a.stw, smem, c);
    if (twiddled) {
        if (Stages<LOG_L>::COUNT == 1) __syncthreads();
        const float2* tw = tws + (MODE == 0 ? c * 17 : 0);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = cmul(v[k], cmul(wjf, tw[k]));
    }
    if (MODE == 0) {
        // contiguous column runs at their digit-reversed place, as k_pass
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
            return true;
        }
        const unsigned j2 = rr & ((1u << a.rev_b2) - 1), j1 = rr >> a.rev_b2;
        float2* q = a.out + ((long long)b << a.log2n) + (((j1 + (j2 << a.rev_b1)) << LOG_L) + kk0);
        const float2* r = smem + spad(kk0 * C + cc);
        if (a.l2_keep) {
            const unsigned long long keep = policy_evict_last();  // the next pass reads these
#pragma unroll
            for (int i = 0; i < 16; ++i) st_policy(q + i * T, r[padc(i * T * C)], keep);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) q[i * T] = r[padc(i * T * C)];
        }
    } else if (X && MODE == 2) {
        const unsigned long long hh = (unsigned)h, q = (unsigned)(q0 + c);
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const float2 x = a.swap_out ? swap_ri(v[k]) : v[k];
            a.out[column_dst(a, hh, q + ((unsigned long long)(j + T * k) << a.log_s))] = x;
        }
    } else {
        // dense tile back in shared memory, then one bulk tensor store
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            float2 x = a.swap_out ? swap_ri(v[k]) : v[k];
            // output element q0 + c + (j + T k) S + h L S of the transform, natural order (last pass)
            if constexpr (W && MODE == 2) {
                if (a.post)
                    x = cmul(x, __ldg(a.post + (unsigned)(q0 + c) + ((unsigned)(j + T * k) << a.log_s) +
                                     ((unsigned)h << (a.log_s + LOG_L))));
            }
            smem[(j + T * k) * C + c] = x;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            if (MODE == 1 && a.l2_keep) tma_store_5d_hint(tout, smem, q0, 0, 0, h, b, policy_evict_last());
            else tma_store_5d(tout, smem, q0, 0, 0, h, b);
        }
    }
    return true;
}

// One tile per block (blockIdx.x the tile, blockIdx.y the transform of the batch).
template <int LOG_L, int LOG_C, int MODE, bool W, bool X = false>
__global__ void __launch_bounds__(1 << (LOG_L + LOG_C - 4), (X ? 0 : tma_min_blocks<LOG_L, LOG_C, MODE>()))
    k_pass_tma(PassArgs a, const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tout) {
    extern __shared__ __align__(1024) float2 smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + tma_bar_offset(LOG_L, LOG_C));
    if (smem_u32(smem) & 127) {  // bulk tensor copies need a 128-byte aligned destination
        if (threadIdx.x == 0) *(volatile unsigned*)a.err = 2u;
        return;
    }
    tma_tile<LOG_L, LOG_C, MODE, W, AlwaysReady, NoHook, NoHook, X>(a, &tin, &tout, blockIdx.x, (int)blockIdx.y, smem,
                                                                    bar, 0u, true,
                                    (int)threadIdx.x);
}

// ---- passes 0 and 1 of a three-pass transform in one persistent launch -----------------------
//
// n = A B C (pass lengths 2^len[0..2]). Pass 1 on the columns of last digit j_c needs only pass
// 0's outputs for the same j_c, and those form one contiguous region of A B 2^g values per
// chunk of 2^g digits (see plan_enqueue's chunked launches). Here one launch runs both passes,
// chunk by chunk: blocks take tiles in order from a device counter, a sequence that issues
// pass 0 of chunk k + lag before pass 1 of chunk k; a pass-1 tile first waits (bounded) until
// every pass-0 tile of its chunk has published its stores. A chunk's intermediate values are then
// re-read from L2 a few microseconds after they were written, instead of from HBM after the whole
// array went through pass 0, so passes 0 and 1 together move the array through HBM once (read
// the input, write the result) instead of twice. The tile arithmetic is tma_tile's, so results
// equal the separate passes bit for bit.
//
// Counters (one slot per launch, zero at entry; the last block to leave zeroes them again):
// [0] the next tile of the sequence, [1] blocks that have left, [2 + k] pass-0 tiles of chunk k
// published.
struct FusedArgs {
    PassArgs p0;      // pass 0 (inner_base: the chunk's first last-digit column, set per tile)
    PassArgs p1;      // pass 1 (outer_base: the same, set per tile)
    int g;            // log2 last-digit columns per chunk
    unsigned chunks;  // 2^(len[2] - g)
    unsigned lag;     // chunks by which pass 1 trails pass 0 (1 <= lag <= chunks)
    unsigned t0, t1;  // tiles per chunk of pass 0 and of pass 1
    unsigned total;   // chunks (t0 + t1)
    unsigned* ctr;
};

// Tile s of the sequence: `lag` chunks of pass 0, then per chunk k pass 0 of chunk k + lag
// followed by pass 1 of chunk k, then the last `lag` chunks of pass 1.
__device__ __forceinline__ void fused_decode(const FusedArgs& f, unsigned s, int& pass, unsigned& chunk,
                                             unsigned& tile) {
    const unsigned pre = f.lag * f.t0;
    if (s < pre) {
        pass = 0, chunk = s / f.t0, tile = s % f.t0;
        return;
    }
    s -= pre;
    const unsigned step = f.t0 + f.t1, mid = (f.chunks - f.lag) * step;
    if (s < mid) {
        const unsigned k = s / step, r = s % step;
        if (r < f.t0) pass = 0, chunk = k + f.lag, tile = r;
        else pass = 1, chunk = k, tile = r - f.t0;
        return;
    }
    s -= mid;
    pass = 1, chunk = f.chunks - f.lag + s / f.t1, tile = s % f.t1;
}

// Both tile shapes run with the same number of threads: 2^(L0 + C0 - 4) = 2^(L1 + C1 - 4).
// Blocks per SM the register allocation must allow: as many as the separate pass kernels of the
// same tiles get (the fused kernels are latency-bound tile machines, so residency matters).
template <int L0, int C0, int L1, int C1>
constexpr int fused_min_blocks() {
    return L0 + C0 == 11 ? 8 : L0 + C0 == 12 ? 5 : L0 + C0 == 13 ? 2 : 0;
}

template <int L0, int C0, int L1, int C1>
__global__ void __launch_bounds__(1 << (L0 + C0 - 4), (fused_min_blocks<L0, C0, L1, C1>()))
    k_pass01_fused(FusedArgs f, const __grid_constant__ CUtensorMap tin, const __grid_constant__ CUtensorMap tmid) {
    static_assert(L0 + C0 == L1 + C1, "both passes' tiles need the same threads");
    constexpr int BAR = tma_bar_offset(L0, C0) > tma_bar_offset(L1, C1) ? tma_bar_offset(L0, C0)
                                                                        : tma_bar_offset(L1, C1);
    extern __shared__ __align__(1024) float2 smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + BAR);
    // two words after the mbarrier: the next tile's index, alternating by iteration (written by
    // thread 0 while the current tile's copy is in flight, read by all after the tile), then the
    // "last block" flag
    unsigned* shared_word = reinterpret_cast<unsigned*>(smem + BAR + 1);
    const int tid = threadIdx.x;
    if (smem_u32(smem) & 127) {  // bulk tensor copies need a 128-byte aligned destination
        if (tid == 0) *(volatile unsigned*)f.p0.err = 2u;
    } else {
        if (tid == 0) shared_word[0] = atomicAdd(f.ctr, 1u);
        __syncthreads();
        unsigned s = shared_word[0], parity = 0, iter = 0;
        bool fresh = true;
        // A pass-0 tile is counted as done (fence, then the chunk's counter) only once the block's
        // next tile copy has landed: by then its stores have long reached L2 and the fence costs
        // little, where fencing right after the stores held the block for their whole round
        // trip. `pending` is that tile's chunk (-1: none); it is published before any wait on a
        // counter, so no block ever waits for a count that it holds itself.
        int pending = -1;
        auto publish = [&]() {
            if (pending >= 0 && tid == 0) {
                __threadfence();  // the tile's stores (all threads, ordered by the barriers since)
                atomicAdd(f.ctr + 2 + pending, 1u);
            }
            pending = -1;
        };
        while (s < f.total) {
            int pass;
            unsigned chunk, tile;
            fused_decode(f, s, pass, chunk, tile);
            unsigned* next = shared_word + ((iter + 1) & 1);  // read by all only after this tile
            auto fetch_next = [&]() { *next = atomicAdd(f.ctr, 1u); };  // thread 0, copy in flight
            bool ok;
            if (pass == 0) {
                PassArgs a = f.p0;
                a.inner_base = chunk << f.g;
                ok = tma_tile<L0, C0, 0, false>(a, &tin, &tin, tile, 0, smem, bar, parity, fresh, tid, AlwaysReady(),
                                                fetch_next, publish);
                if (ok) pending = (int)chunk;
            } else {
                publish();
                // thread 0: wait until every pass-0 tile of the chunk is published, then issue
                // the copy; the other threads compute the tile's twiddle factors meanwhile
                auto chunk_ready = [&]() {
                    const bool r = !g_expire_waits && wait_count(f.ctr + 2 + chunk, f.t0);
                    // the chunk's values were written by other blocks through the generic proxy;
                    // this block reads them with a bulk tensor copy (the async proxy)
                    asm volatile("fence.proxy.async.global;" ::: "memory");
                    if (!r) *(volatile unsigned*)f.p1.err = 3u;
                    return r;
                };
                PassArgs a = f.p1;
                a.outer_base = chunk << f.g;
                ok = tma_tile<L1, C1, 1, false>(a, &tmid, &tmid, tile, 0, smem, bar, parity, fresh, tid, chunk_ready,
                                                fetch_next);
            }
            if (!ok) break;  // block-uniform: an expired wait, recorded in the error word
            parity ^= 1u;
            fresh = false;
            __syncthreads();  // the next-tile word is written; the tile's stores are issued
            s = *next;
            ++iter;
        }
        publish();  // the last pass-0 tile (after the barrier above, or after a failed tile)
    }
    // The last block to leave zeroes the counters for the next launch on this slot: every other
    // block has left its loop, so none touches them again.
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        *shared_word = atomicAdd(f.ctr + 1, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (*shared_word) {
        for (unsigned k = tid; k < f.chunks + 2; k += blockDim.x) f.ctr[k] = 0;
        __threadfence();
    }
}

// ---- one-kernel sizes as a persistent, double-buffered pipeline ---------------------------------
//
// A whole transform of 2^LOG_L values per block, as k_batched, but the block stays resident and
// walks the batch (transform blockIdx.x, then every gridDim.x-th): while it computes one
// transform, the next one's 8 * 2^LOG_L bytes arrive in its second buffer through ONE bulk copy
// (cp.async.bulk, completing on that buffer's mbarrier). A transform of 2^13 fills a block of 512
// threads and half its SM's shared memory, so k_batched runs two of them per SM, each waiting for
// its own loads; here the load of the next transform overlaps the arithmetic of this one. The
// values then go from the dense buffer to registers and through the same Stockham stages
// (tile_fft) as k_batched, so results equal it bit for bit. Buffers are padded for the exchanges
// (which reuse them once the values are in registers); the two mbarriers follow them.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

template <int LOG_L>
constexpr int pipe_smem_bytes() {
    return 2 * (int)sizeof(float2) * ((1 << LOG_L) + (1 << (LOG_L - 4))) + 2 * (int)sizeof(uint64_t);
}

template <int LOG_L, int INV>
__global__ void __launch_bounds__(1 << (LOG_L - 4), 1)
    k_batched_pipe(const float2* __restrict__ in, float2* __restrict__ out, long long batch,
                   const float2* __restrict__ stw, unsigned* err) {
    constexpr int L = 1 << LOG_L, T = L / 16, BUF = L + L / 16;
    constexpr unsigned BYTES = (unsigned)(L * sizeof(float2));
    extern __shared__ __align__(1024) float2 smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + 2 * BUF);
    const int tid = threadIdx.x;
    const long long stride = gridDim.x;
    long long b = blockIdx.x;
    if (b >= batch) return;
    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        mbar_expect_tx(&bar[0], BYTES);
        bulk_load(smem, in + (b << LOG_L), BYTES, &bar[0]);
    }
    __syncthreads();  // the barriers are initialised before anyone waits on them
    for (int k = 0; b < batch; ++k, b += stride) {
        float2* buf = smem + (k & 1) * BUF;
        const bool next = b + stride < batch;
        if (tid == 0 && next) {
            // the other buffer was last read and written as iteration k - 1's exchange space
            // (generic accesses, ordered before this by the barrier that ended it)
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            mbar_expect_tx(&bar[(k + 1) & 1], BYTES);
            bulk_load(smem + ((k + 1) & 1) * BUF, in + ((b + stride) << LOG_L), BYTES, &bar[(k + 1) & 1]);
        }
        const bool ok = !g_expire_waits && mbar_wait(&bar[k & 1], (unsigned)(k >> 1) & 1u);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                *(volatile unsigned*)err = 4u;
                // let the copies in flight land before the block's memory is released
                mbar_wait(&bar[k & 1], (unsigned)(k >> 1) & 1u);
                if (next) mbar_wait(&bar[(k + 1) & 1], (unsigned)((k + 1) >> 1) & 1u);
            }
            return;
        }
        float2 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = INV ? swap_ri(buf[tid + T * i]) : buf[tid + T * i];
        __syncthreads();  // every value is in registers before the exchanges reuse the buffer
        tile_fft<LOG_L, 1>(v, tid, stw, buf, 0);
        float2* dst = out + (b << LOG_L) + tid;
#pragma unroll
        for (int i = 0; i < 16; ++i) dst[T * i] = INV ? swap_ri(v[i]) : v[i];
        __syncthreads();  // the buffer is free before it is refilled (iteration k + 1 issues into it)
    }
}

// ---- host side ----------------------------------------------------------------------------------

static PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
    });
    return fn;
}

// Tensor map of the pass tile: MODE 0 {column r, row-in-box, row-box, batch} over `in`;
// MODE 1/2 {q, row-in-box, row-box, h, batch} over `out`. 8-byte elements, no swizzle.
static bool make_map(CUtensorMap* m, const float2* base, int mode, int log2n, int log_l, int log_c, int log_s,
                     int batch) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = encode_fn();
    if (!enc) return false;
    const cuuint64_t n = 1ull << log2n, L = 1ull << log_l, elo = L < 256 ? L : 256, ehi = L / elo;
    cuuint64_t dims[5], strides[4];
    cuuint32_t box[5], estr[5] = {1, 1, 1, 1, 1};
    int rank;
    if (mode == 0) {
        const cuuint64_t cols = n >> log_l;
        dims[0] = cols, dims[1] = elo, dims[2] = ehi, dims[3] = (cuuint64_t)batch;
        strides[0] = cols * 8, strides[1] = elo * cols * 8, strides[2] = n * 8;
        box[0] = 1u << log_c, box[1] = (cuuint32_t)elo, box[2] = (cuuint32_t)ehi, box[3] = 1;
        rank = 4;
    } else {
        const cuuint64_t S = 1ull << log_s, H = n >> (log_s + log_l);
        dims[0] = S, dims[1] = elo, dims[2] = ehi, dims[3] = H, dims[4] = (cuuint64_t)batch;
        strides[0] = S * 8, strides[1] = elo * S * 8, strides[2] = L * S * 8, strides[3] = n * 8;
        box[0] = 1u << log_c, box[1] = (cuuint32_t)elo, box[2] = (cuuint32_t)ehi, box[3] = 1, box[4] = 1;
        rank = 5;
    }
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, (cuuint32_t)rank, (void*)base, dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS;
}

template <int LOG_L, int LOG_C, int MODE, bool W>
static cudaError_t launch_tma_w(const PassArgs& a, int batch, cudaStream_t stream) {
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = tma_smem_bytes(LOG_L, LOG_C);
    auto kernel = k_pass_tma<LOG_L, LOG_C, MODE, W>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    // MODE 0 loads from `in` and stores with plain coalesced stores (tout unused); MODE 1/2
    // load and store the same tile of `out`
    CUtensorMap tin;
    if (!make_map(&tin, MODE == 0 ? a.in : a.out, MODE, a.log2n, LOG_L, LOG_C, a.log_s, batch))
        return cudaErrorInvalidValue;
    const CUtensorMap& tout = tin;
    dim3 grid(a.ntiles ? a.ntiles : 1u << (a.log2n - LOG_L - LOG_C), (unsigned)batch, 1);
    PassArgs b = a;
    if (!a.ntiles) b.tli = 31;
    kernel<<<grid, THREADS, SMEM, stream>>>(b, tin, tout);
    return cudaGetLastError();
}

// Tile shapes with a TMA kernel (the only ones pass_tma_supported accepts): widths 2 .. 16
// columns (16-byte minimum row segment), up to 8192 values per tile, and 4 columns of 4096
// (16384 values, 1024 threads, one block per SM) for two-pass 2^24.
#define OFB_TMA_SHAPES(X) \
    X(12, 2)              \
    X(12, 1)              \
    X(11, 1)              \
    X(11, 2)              \
    X(10, 1)              \
    X(10, 2)              \
    X(10, 3)              \
    X(9, 2)               \
    X(9, 3)               \
    X(9, 4)               \
    X(8, 2)               \
    X(8, 3)               \
    X(8, 4)               \
    X(7, 3)               \
    X(7, 4)               \
    X(6, 4)

bool pass_tma_supported(int log_l, int log_c) {
#define OFB_TMA_MATCH(LL, LC) \
    if (log_l == LL && log_c == LC) return true;
    OFB_TMA_SHAPES(OFB_TMA_MATCH)
#undef OFB_TMA_MATCH
    return false;
}

// The weighted kernel only where a weight applies: the first pass's input, the last pass's output.
template <int LOG_L, int LOG_C, int MODE>
static cudaError_t launch_tma_t(const PassArgs& a, int batch, cudaStream_t stream) {
    if constexpr (MODE != 1) {
        if (MODE == 0 ? a.pre != nullptr : a.post != nullptr) return launch_tma_w<LOG_L, LOG_C, MODE, true>(a, batch, stream);
    }
    return launch_tma_w<LOG_L, LOG_C, MODE, false>(a, batch, stream);
}

template <int MODE>
static cudaError_t launch_tma_mode(int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t s) {
#define OFB_TMA_CASE(LL, LC) \
    if (log_l == LL && log_c == LC) return launch_tma_t<LL, LC, MODE>(a, batch, s);
    OFB_TMA_SHAPES(OFB_TMA_CASE)
#undef OFB_TMA_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_pass_tma(int mode, int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t stream) {
    if (!pass_tma_supported(log_l, log_c) || batch > 65535) return cudaErrorInvalidValue;
    switch (mode) {
    case 0: return launch_tma_mode<0>(log_l, log_c, a, batch, stream);
    case 1: return launch_tma_mode<1>(log_l, log_c, a, batch, stream);
    default: return launch_tma_mode<2>(log_l, log_c, a, batch, stream);
    }
}

// ---- column transforms through the bulk-tensor-copy tiles ----------------------------------------

// Tile width (log2 columns) of a column-transform pass of length 2^log_l, -1: no TMA tile.
// Timed on a B200 over 2^27 values (one and two passes): 1024-value columns in tiles of 4 beat 8
// and 2 (445 against 514 / 558 us for one pass); 512 and 256 values in tiles of 8 beat 16 and 4.
int column_tma_log_c(int log_l) {
    switch (log_l) {
    case 12: return 1;
    case 11: return 2;
    case 10: return 2;
    case 9: return 3;
    case 8: return 3;
    case 7: return 4;
    case 6: return 4;
    default: return -1;
    }
}

// Both modes read their tile from a.in (first pass: the matrix; last pass: the work array in the
// first pass's layout) and write a.out with plain stores.
template <int LOG_L, int LOG_C, int MODE>
static cudaError_t launch_columns_tma_t(const PassArgs& a, cudaStream_t stream) {
    constexpr int THREADS = 1 << (LOG_L + LOG_C - 4);
    constexpr int SMEM = tma_smem_bytes(LOG_L, LOG_C);
    auto kernel = k_pass_tma<LOG_L, LOG_C, MODE, false, true>;
    static std::atomic<unsigned long long> done{0};
    const cudaError_t attr = smem_limit((const void*)kernel, SMEM, done);
    if (attr != cudaSuccess) return attr;
    if (a.log2n > 31 || a.log2n < LOG_L + LOG_C) return cudaErrorInvalidValue;
    CUtensorMap tin;
    if (!make_map(&tin, a.in, MODE, a.log2n, LOG_L, LOG_C, a.log_s, 1)) return cudaErrorInvalidValue;
    PassArgs b = a;
    b.tli = 31;
    kernel<<<1u << (a.log2n - LOG_L - LOG_C), THREADS, SMEM, stream>>>(b, tin, tin);
    return cudaGetLastError();
}

cudaError_t launch_pass_columns_tma(int mode, int log_l, const PassArgs& a, cudaStream_t stream) {
    if (mode != 0 && mode != 2) return cudaErrorInvalidValue;
#define OFB_COLUMNS_TMA_CASE(LL, LC) \
    case LL: return mode == 0 ? launch_columns_tma_t<LL, LC, 0>(a, stream) : launch_columns_tma_t<LL, LC, 2>(a, stream);
    switch (log_l) {
        OFB_COLUMNS_TMA_CASE(12, 1)
        OFB_COLUMNS_TMA_CASE(11, 2)
        OFB_COLUMNS_TMA_CASE(10, 2)
        OFB_COLUMNS_TMA_CASE(9, 3)
        OFB_COLUMNS_TMA_CASE(8, 3)
        OFB_COLUMNS_TMA_CASE(7, 4)
        OFB_COLUMNS_TMA_CASE(6, 4)
    default: return cudaErrorInvalidValue;
    }
#undef OFB_COLUMNS_TMA_CASE
}

}  // namespace ofb

namespace ofb {

// ---- fused passes 0+1: host side ----------------------------------------------------------------

// Shapes (L0, C0, L1, C1) with a fused kernel: both tiles have a TMA kernel and the same threads.
#define OFB_FUSED_SHAPES(X) \
    X(8, 4, 9, 3)           \
    X(8, 3, 8, 3)           \
    X(8, 4, 8, 4)           \
    X(8, 3, 7, 4)           \
    X(9, 3, 9, 3)           \
    X(10, 3, 10, 3)         \
    X(10, 3, 11, 2)

bool pass01_fused_supported(int l0, int c0, int l1, int c1) {
#define OFB_FUSED_MATCH(A0, B0, A1, B1) \
    if (l0 == A0 && c0 == B0 && l1 == A1 && c1 == B1) return true;
    OFB_FUSED_SHAPES(OFB_FUSED_MATCH)
#undef OFB_FUSED_MATCH
    return false;
}

template <int L0, int C0, int L1, int C1>
static cudaError_t launch_fused_t(const FusedArgs& f, int log2n, cudaStream_t stream) {
    constexpr int THREADS = 1 << (L0 + C0 - 4);
    constexpr int SMEM = tma_smem_bytes(L0, C0) > tma_smem_bytes(L1, C1) ? tma_smem_bytes(L0, C0)
                                                                        : tma_smem_bytes(L1, C1);
    auto kernel = k_pass01_fused<L0, C0, L1, C1>;
    static std::atomic<unsigned long long> done{0};
    cudaError_t e = smem_limit((const void*)kernel, SMEM, done);
    if (e != cudaSuccess) return e;
    // persistent grid: as many blocks as fit on the device at once (per device, computed once)
    static std::atomic<int> grid_of[64];
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    int grid = grid_of[dev & 63].load(std::memory_order_relaxed);
    if (grid == 0) {
        int per_sm = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, THREADS, SMEM)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        grid = per_sm * sms > 0 ? per_sm * sms : 1;
        grid_of[dev & 63].store(grid, std::memory_order_relaxed);
    }
    if ((unsigned)grid > f.total) grid = (int)f.total;
    CUtensorMap tin, tmid;
    if (!make_map(&tin, f.p0.in, 0, log2n, L0, C0, f.p0.log_s, 1) ||
        !make_map(&tmid, f.p1.out, 1, log2n, L1, C1, f.p1.log_s, 1))
        return cudaErrorInvalidValue;
    kernel<<<grid, THREADS, SMEM, stream>>>(f, tin, tmid);
    return cudaGetLastError();
}

cudaError_t launch_pass01_fused(int l0, int c0, int l1, int c1, const PassArgs& a0, const PassArgs& a1, int g,
                                int len2, int lag, unsigned* ctr, cudaStream_t stream) {
    if (!pass01_fused_supported(l0, c0, l1, c1) || g < c0 || g > len2) return cudaErrorInvalidValue;
    FusedArgs f{};
    f.p0 = a0;
    f.p1 = a1;
    f.g = g;
    f.chunks = 1u << (len2 - g);
    f.lag = lag < 1 ? 1u : (unsigned)lag > f.chunks ? f.chunks : (unsigned)lag;
    f.t0 = a0.ntiles;
    f.t1 = a1.ntiles;
    f.total = f.chunks * (f.t0 + f.t1);
    f.ctr = ctr;
#define OFB_FUSED_CASE(A0, B0, A1, B1) \
    if (l0 == A0 && c0 == B0 && l1 == A1 && c1 == B1) return launch_fused_t<A0, B0, A1, B1>(f, a0.log2n, stream);
    OFB_FUSED_SHAPES(OFB_FUSED_CASE)
#undef OFB_FUSED_CASE
    return cudaErrorInvalidValue;
}

}  // namespace ofb

namespace ofb {

// ---- the pipelined one-kernel sizes: host side ---------------------------------------------------

bool batched_pipe_supported(int log2n) { return log2n == 12 || log2n == 13; }

template <int LOG_L>
static cudaError_t launch_pipe_t(const float2* in, float2* out, long long batch, const float2* stw, int inverse,
                                 unsigned* err, cudaStream_t stream) {
    constexpr int THREADS = 1 << (LOG_L - 4), SMEM = pipe_smem_bytes<LOG_L>();
    auto kernel = inverse ? k_batched_pipe<LOG_L, 1> : k_batched_pipe<LOG_L, 0>;
    static std::atomic<unsigned long long> done_fwd{0}, done_inv{0};
    cudaError_t e = smem_limit((const void*)kernel, SMEM, inverse ? done_inv : done_fwd);
    if (e != cudaSuccess) return e;
    // persistent grid: the blocks that fit on the device at once (per device and direction)
    static std::atomic<int> grid_of[2][64];
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    int grid = grid_of[inverse ? 1 : 0][dev & 63].load(std::memory_order_relaxed);
    if (grid == 0) {
        int per_sm = 0, sms = 0;
        if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, THREADS, SMEM)) != cudaSuccess) return e;
        if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
        grid = per_sm * sms > 0 ? per_sm * sms : 1;
        grid_of[inverse ? 1 : 0][dev & 63].store(grid, std::memory_order_relaxed);
    }
    if ((long long)grid > batch) grid = (int)batch;
    kernel<<<grid, THREADS, SMEM, stream>>>(in, out, batch, stw, err);
    return cudaGetLastError();
}

cudaError_t launch_batched_pipe(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                int inverse, unsigned* err, cudaStream_t stream) {
    if (batch <= 0) return cudaSuccess;
    if ((uintptr_t)in & 15) return cudaErrorInvalidValue;  // bulk copies start on 16-byte boundaries
    switch (log2n) {
    case 12: return launch_pipe_t<12>(in, out, batch, stw, inverse, err, stream);
    case 13: return launch_pipe_t<13>(in, out, batch, stw, inverse, err, stream);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace ofb
