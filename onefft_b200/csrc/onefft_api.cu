// C-ABI layer of libonefft_cuda.so: plans, the plan cache, the host-pointer drop-in calls and the
// device-pointer batched calls.
//
// OneFFT's runtime (src/onefft.c:1094-1189) is restated for the device:
//   - a plan is immutable after creation and holds every table in one allocation, here one
//     cudaMalloc filled by kernels that evaluate the FP64 twiddle rule on the device;
//   - the cache is one slot per log2 n (and per device), filled lock-free by compare-and-swap;
//     the loser of a race destroys its copy (src/onefft.c:1151-1167);
//   - invalid sizes and allocation failures return -1 / NULL with the output untouched
//     (include/onefft.h:73-75).
// The host-pointer calls stage through per-thread device buffers on a per-thread stream, so
// concurrent callers never share mutable state.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "onefft_cuda.h"
#include "fft_launch.h"
#include "uneven.h"

#include <algorithm>
#include <numeric>
#include <vector>

using namespace ofb;

// ---- errors, test hooks, counters --------------------------------------------------------------

static thread_local std::string t_last_error;
static std::atomic<int> g_fail_alloc_countdown{0};
std::atomic<unsigned long long> ofb::g_launches{0};

static int set_error(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
static int set_error(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
    return code;
}

// Sets the calling thread's onefft_last_error() message (for entry points in other files).
void ofb::record_error(const char *msg) { t_last_error = msg; }

static int cuda_error(cudaError_t e, const char *what) {
    cudaGetLastError();  // clear a non-sticky error so later calls start clean
    return set_error(ONEFFT_ERR_CUDA_BASE - (int)e, "%s: %s", what, cudaGetErrorString(e));
}

// Device allocation with the test hook of onefft_debug_fail_alloc().
static cudaError_t dev_alloc(void **p, size_t bytes) {
    int k = g_fail_alloc_countdown.load();
    while (k > 0) {
        if (g_fail_alloc_countdown.compare_exchange_weak(k, k - 1)) {
            if (k == 1) {
                *p = nullptr;
                return cudaErrorMemoryAllocation;
            }
            break;
        }
    }
    return cudaMalloc(p, bytes);
}

static bool size_log2(size_t n, int *log2n) {
    if (n == 0 || (n & (n - 1)) != 0) return false;
    int l = 0;
    while (((size_t)1 << l) < n) ++l;
    if (l > 30) return false;
    *log2n = l;
    return true;
}

// ---- plans -------------------------------------------------------------------------------------

// Counter slot of the fused pass-0/1 kernel: launches that take the same slot are ordered by
// its event (the slot's previous launch has finished and left the counters zeroed).
struct FusedSlot {
    std::mutex m;
    cudaEvent_t done = nullptr;
    bool used = false;
};
constexpr int kFusedSlots = 4;

struct onefft_plan {
    size_t n;
    int log2n;
    int device;
    int npass;
    int len[3];            // log2 of each pass length
    int cols[3];           // log2 of the tile width (columns per block) of each pass; one kernel:
                           // cols[0] = log2 of the transforms per block (-1 = default)
    int l2_keep;           // intermediate stores with L2 evict-last priority
    int chunk;             // three passes: log2 of the last-digit columns per chunk of passes 0+1 (0 = none)
    int tc;                // radix-16 stages as split-BF16 tensor-core products of this many terms (3: hi/lo,
                           // onefft_plan_create_bf16x3; 6: hi/mid/lo, onefft_plan_create_bf16x6); 0 = FP32
    int tma;               // passes staged through bulk tensor copies where the tile shape has a TMA kernel
    int fuse_lag;          // three passes, chunked: passes 0+1 as one persistent launch with pass 1
                           // trailing by this many chunks (0 = separate launches)
    unsigned *fused_ctr;   // kFusedSlots counter slots of fused_words words each, in `mem`
    size_t fused_words;
    FusedSlot *slots;
    mutable std::atomic<unsigned> next_slot{0};
    unsigned *err;         // error word as kernels address it: set by a kernel whose bounded wait ran out
    unsigned *err_host;    // the same word on the host (mapped pinned memory: read without a copy)
    void *mem;             // the one device allocation
    size_t mem_bytes;
    const float2 *stw[3];  // stage twiddles of each pass's length
    const double2 *tw_lo;  // two-level FP64 tables of w_n (npass >= 2)
    const double2 *tw_hi;
    int lo_bits;
};

// How a size runs: number of passes, their lengths and tile widths. The table below is the
// tuned choice per log2 n (onefft_b200/autotune.py measures the candidates on the device and
// prints this table); sizes up to 2^14 run as one kernel.
struct Shape {
    int npass;
    int len[3];
    int cols[3];
    int l2_keep;
    int chunk;
    int tma;
    int fuse_lag = 0;  // the tuned table leaves it out: no size runs the fused passes by default
};

// Fastest shapes measured on a B200 by onefft_b200/autotune.py (forward transform, L2 flushed
// before each repetition): {npass, {log2 lengths}, {log2 tile widths}, l2_keep, chunk, tma}.
// 2^16 keeps the (8, 8) split (as fast as the best) so the uneven batch's in-block passes,
// which use it, stay bit-identical to this path.
static const Shape kTuned[] = {
    /* 15 */ {2, {8, 7, 0}, {3, 4, 0}, 0, 0, 1},
    /* 16 */ {2, {8, 8, 0}, {3, 3, 0}, 0, 0, 1},
    /* 17 */ {2, {10, 7, 0}, {1, 4, 0}, 0, 0, 0},
    /* 18 */ {2, {10, 8, 0}, {2, 3, 0}, 0, 0, 0},
    /* 19 */ {2, {8, 11, 0}, {4, 1, 0}, 1, 0, 0},
    /* 20 */ {2, {12, 8, 0}, {1, 3, 0}, 1, 0, 1},
    /* 21 */ {2, {11, 10, 0}, {1, 4, 0}, 0, 0, 1},
    /* 22 */ {3, {8, 7, 7}, {3, 4, 4}, 1, 0, 1},
    /* 23 */ {3, {8, 8, 7}, {3, 4, 4}, 1, 0, 1},
    /* 24 */ {3, {8, 8, 8}, {3, 3, 3}, 0, 0, 1},
    /* 25 */ {3, {8, 8, 9}, {3, 3, 3}, 0, 0, 1},
    /* 26 */ {3, {8, 8, 10}, {3, 3, 3}, 0, 0, 1},
    /* 27 */ {3, {8, 9, 10}, {4, 3, 3}, 0, 0, 1},
    // 2^28 .. 2^30 (one 2^30 transform holds 16 GiB of buffers), timed among three-pass splits
    // with default tile widths: 2^28 (10,10,8) 2.57 ms against (10,9,9) 2.62; 2^29 (10,10,9)
    // 5.28 ms, the fastest of six; 2^30 (10,11,9) 11.2 ms against 12.6-16.2 ms for seven others,
    // (10,10,10) 12.9 ms.
    /* 28 */ {3, {10, 10, 8}, {3, 3, 4}, 1, 0, 1},
    /* 29 */ {3, {10, 10, 9}, {3, 3, 4}, 1, 0, 1},
    /* 30 */ {3, {10, 11, 9}, {3, 2, 4}, 1, 0, 1},
};
static_assert(sizeof(kTuned) / sizeof(kTuned[0]) == 30 - 15 + 1, "one shape per size 2^15 .. 2^30");

// Transforms per block (log2) of the one-kernel sizes 2^4 .. 2^14, from
// `python -m onefft_b200.autotune --batched` on a B200 (forward, 2^25 values per batch, median of
// 9): 2048-value tiles up to n = 2^9 and at 2^11 (2^4 87 us against 90 / 96 for 4096 / 8192, 2^5
// 86 against 94 / 131, 2^6 87 against 96 / 133; 2^7 .. 2^9 and 2^11 by one timer tick, ~2 us),
// the default 4096 at 2^10 and 2^12; 2^13 / 2^14 have one width. -1 = the default.
static const int kBatchedTunedLogC[kMaxSingleLog2 + 1] = {-1, -1, -1, -1, 7, 6, 5, 4, 3, 2, 2, 0, 0, 0, 0};

static Shape tuned_shape(int m) {
    Shape s{};
    if (m <= kMaxSingleLog2) {
        s.npass = 1;
        s.len[0] = m;
        s.cols[0] = kBatchedTunedLogC[m];
        return s;
    }
    return kTuned[m - 15];
}

// One kernel, cols[0] = this: the persistent pipelined kernel (launch_batched_pipe) instead of
// k_batched (ONEFFT_COLS_PIPELINED in onefft_cuda.h).
constexpr int kPipelinedCols = 15;

static bool valid_shape(int m, const Shape &s) {
    if (s.npass == 1)
        return s.len[0] == m && m <= kMaxSingleLog2 &&
               (s.cols[0] == -1 || batched_log_c_supported(m, s.cols[0]) ||
                (s.cols[0] == kPipelinedCols && batched_pipe_supported(m)));
    if (s.npass < 2 || s.npass > 3) return false;
    int sum = 0;
    for (int p = 0; p < s.npass; ++p) {
        if (!pass_tile_supported(s.len[p], s.cols[p])) return false;
        sum += s.len[p];
    }
    // the first pass's tile must not straddle a column digit of the last pass (three passes),
    // and a chunk holds whole first-pass tiles
    if (s.npass == 3 && s.cols[0] > s.len[2]) return false;
    if (s.chunk && (s.npass != 3 || s.chunk < s.cols[0] || s.chunk > s.len[2])) return false;
    // the fused passes 0+1 need chunks, bulk tensor copies and a compiled tile pair
    if (s.fuse_lag && (!s.chunk || !s.tma || s.fuse_lag > 15 ||
                       !pass01_fused_supported(s.len[0], s.cols[0], s.len[1], s.cols[1])))
        return false;
    return sum == m;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

static onefft_plan *plan_build(size_t n, int m, const Shape &shape) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        cuda_error(e, "no CUDA device");
        return nullptr;
    }
    onefft_plan *p = new (std::nothrow) onefft_plan();
    if (!p) {
        set_error(ONEFFT_ERR_SIZE, "out of host memory");
        return nullptr;
    }
    p->n = n;
    p->log2n = m;
    p->device = device;
    p->npass = shape.npass;
    p->l2_keep = shape.l2_keep;
    p->chunk = shape.chunk;
    p->tma = shape.tma;
    p->fuse_lag = shape.fuse_lag;
    for (int i = 0; i < shape.npass; ++i) {
        p->len[i] = shape.len[i];
        p->cols[i] = shape.cols[i];
    }
    // layout: stage tables per pass, then the FP64 tables
    size_t off[3], bytes = 0;
    for (int i = 0; i < p->npass; ++i) {
        off[i] = bytes;
        bytes = align256(bytes + sizeof(float2) * (size_t)stage_table_entries_host(p->len[i]));
    }
    size_t lo_off = bytes, hi_off = bytes;
    if (p->npass >= 2) {
        p->lo_bits = m / 2;
        lo_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << p->lo_bits));
        hi_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << (m - p->lo_bits)));
    }
    size_t ctr_off = bytes;
    if (p->fuse_lag) {  // counter slots of the fused passes: next tile, blocks done, one per chunk
        p->fused_words = align256(sizeof(unsigned) * (2 + ((size_t)1 << (p->len[2] - p->chunk)))) / sizeof(unsigned);
        bytes += kFusedSlots * p->fused_words * sizeof(unsigned);
        p->slots = new (std::nothrow) FusedSlot[kFusedSlots];
        if (!p->slots) {
            delete p;
            set_error(ONEFFT_ERR_SIZE, "out of host memory");
            return nullptr;
        }
    }
    e = dev_alloc(&p->mem, bytes);
    if (e != cudaSuccess) {
        delete[] p->slots;
        delete p;
        cuda_error(e, "plan table allocation");
        set_error(ONEFFT_ERR_SIZE, "plan table allocation failed");
        return nullptr;
    }
    p->mem_bytes = bytes;
    char *base = (char *)p->mem;
    // The error word lives in mapped pinned host memory: kernels write it over the bus (only
    // when a wait expires) and a host call reads it with a plain load after its stream
    // synchronises, so checking it needs no copy that could queue behind other threads' large
    // transfers on a copy engine.
    e = cudaHostAlloc((void **)&p->err_host, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e == cudaSuccess) {
        *(volatile unsigned *)p->err_host = 0;
        e = cudaHostGetDevicePointer((void **)&p->err, p->err_host, 0);
    } else {
        p->err_host = nullptr;
    }
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        for (int i = 0; i < p->npass && e == cudaSuccess; ++i) {
            p->stw[i] = (const float2 *)(base + off[i]);
            e = launch_stage_table((float2 *)(base + off[i]), p->len[i], s);
        }
        if (p->npass >= 2 && e == cudaSuccess) {
            p->tw_lo = (const double2 *)(base + lo_off);
            p->tw_hi = (const double2 *)(base + hi_off);
            e = launch_big_table((double2 *)p->tw_lo, (double2 *)p->tw_hi, m, p->lo_bits, s);
        }
        if (p->fuse_lag && e == cudaSuccess) {
            p->fused_ctr = (unsigned *)(base + ctr_off);
            e = cudaMemsetAsync(p->fused_ctr, 0, kFusedSlots * p->fused_words * sizeof(unsigned), s);
            for (int i = 0; i < kFusedSlots && e == cudaSuccess; ++i)
                e = cudaEventCreateWithFlags(&p->slots[i].done, cudaEventDisableTiming);
        }
        cudaError_t e2 = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = e2;
        cudaStreamDestroy(s);
    }
    if (e != cudaSuccess) {
        cudaFree(p->mem);
        if (p->err_host) cudaFreeHost(p->err_host);
        if (p->slots)
            for (int i = 0; i < kFusedSlots; ++i)
                if (p->slots[i].done) cudaEventDestroy(p->slots[i].done);
        delete[] p->slots;
        delete p;
        cuda_error(e, "plan table build");
        return nullptr;
    }
    return p;
}

extern "C" onefft_plan *onefft_plan_create(size_t n) {
    int m;
    if (!size_log2(n, &m)) {
        set_error(ONEFFT_ERR_SIZE, "n=%zu is not a power of two in [1, 2^30]", n);
        return nullptr;
    }
    return plan_build(n, m, tuned_shape(m));
}

extern "C" onefft_plan *onefft_plan_create_tiles(size_t n, int npass, const int *log2_len, const int *log2_cols,
                                                 int options, int log2_chunk) {
    int m;
    if (!size_log2(n, &m)) {
        set_error(ONEFFT_ERR_SIZE, "n=%zu is not a power of two in [1, 2^30]", n);
        return nullptr;
    }
    if (!log2_len || npass < 1 || npass > 3) {
        set_error(ONEFFT_ERR_ARG, "invalid pass split for n=%zu", n);
        return nullptr;
    }
    Shape s{};
    s.npass = npass;
    s.l2_keep = (options & ONEFFT_OPT_L2_KEEP) ? 1 : 0;
    s.tma = (options & ONEFFT_OPT_TMA) ? 1 : 0;
    s.chunk = log2_chunk > 0 ? log2_chunk : 0;
    if (options & ONEFFT_OPT_FUSED) s.fuse_lag = ((options >> 8) & 15) ? ((options >> 8) & 15) : 1;
    for (int i = 0; i < npass; ++i) {
        s.len[i] = log2_len[i];
        s.cols[i] = log2_cols ? log2_cols[i] : pass_log_c(log2_len[i]);
    }
    // one kernel: cols[0] is the transforms per block (log2), the tuned one unless given
    if (npass == 1 && (!log2_cols || log2_cols[0] == -1)) s.cols[0] = m <= kMaxSingleLog2 ? tuned_shape(m).cols[0] : -1;
    if (!valid_shape(m, s)) {
        set_error(ONEFFT_ERR_ARG, "invalid pass split for n=%zu", n);
        return nullptr;
    }
    return plan_build(n, m, s);
}

// Sizes (bit log2 n) at which each split-BF16 tensor-core variant meets the FP32 path's error
// bound (relative RMS against FP64 at most 2x OneFFT's own on the same input), measured on a
// B200 with standard normal inputs with 1 % of the values scaled by 1e3, the worst of three
// transforms per size and both directions. Three terms: 33-64x OneFFT's error at every size
// 2^4 .. 2^26, so none. Six terms: 1.22-1.90x at 2^4 .. 2^23, then 2.00, 1.99, 1.94 at 2^24 ..
// 2^26; accepted where the worst measured ratio is at most 1.9 (a margin for other inputs), and
// not at the sizes beyond, which were at the bound or not measured.
static const unsigned long long kBf16x3Accepted = 0;
static const unsigned long long kBf16x6Accepted = ((1ull << 24) - 1) & ~((1ull << 4) - 1);  // 2^4 .. 2^23

static onefft_plan *create_bf16(size_t n, int terms, unsigned long long accepted, int require_accepted) {
    int m;
    if (!size_log2(n, &m) || m < 4) {
        set_error(ONEFFT_ERR_SIZE, "n=%zu: the tensor-core variant needs a power of two in [16, 2^30]", n);
        return nullptr;
    }
    if (require_accepted && !((accepted >> m) & 1)) {
        set_error(ONEFFT_ERR_SIZE, "n=2^%d: split-BF16 (%d terms) does not meet the FP32 error bound at this size", m,
                  terms);
        return nullptr;
    }
    Shape s = tuned_shape(m);
    s.chunk = 0;
    s.tma = 0;
    s.fuse_lag = 0;
    for (int i = 0; i < s.npass; ++i) {
        s.cols[i] = pass_log_c(s.len[i]);
        if (s.npass > 1 && s.len[i] < 5) {
            set_error(ONEFFT_ERR_SIZE, "n=2^%d: no tensor-core split", m);
            return nullptr;
        }
    }
    onefft_plan *p = plan_build(n, m, s);
    if (p) p->tc = terms;
    return p;
}

extern "C" onefft_plan *onefft_plan_create_bf16x3(size_t n, int require_accepted) {
    return create_bf16(n, 3, kBf16x3Accepted, require_accepted);
}

extern "C" onefft_plan *onefft_plan_create_bf16x6(size_t n, int require_accepted) {
    return create_bf16(n, 6, kBf16x6Accepted, require_accepted);
}

extern "C" onefft_plan *onefft_plan_create_split(size_t n, int npass, const int *log2_len) {
    return onefft_plan_create_tiles(n, npass, log2_len, nullptr, ONEFFT_OPT_L2_KEEP, 0);
}

extern "C" void onefft_plan_destroy(onefft_plan *plan) {
    if (!plan) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != plan->device) cudaSetDevice(plan->device);
    cudaFree(plan->mem);
    if (plan->err_host) cudaFreeHost(plan->err_host);
    if (plan->slots)
        for (int i = 0; i < kFusedSlots; ++i)
            if (plan->slots[i].done) cudaEventDestroy(plan->slots[i].done);
    delete[] plan->slots;
    if (cur >= 0 && cur != plan->device) cudaSetDevice(cur);
    delete plan;
}

extern "C" size_t onefft_plan_size(const onefft_plan *plan) { return plan ? plan->n : 0; }

extern "C" int onefft_plan_passes(const onefft_plan *plan, int *log2_len) {
    if (!plan) return 0;
    for (int i = 0; i < plan->npass && log2_len; ++i) log2_len[i] = plan->len[i];
    return plan->npass;
}

extern "C" const char *onefft_implementation(void) { return "cuda sm_100a"; }

extern "C" const char *onefft_last_error(void) { return t_last_error.c_str(); }

extern "C" void onefft_debug_fail_alloc(int k) { g_fail_alloc_countdown.store(k < 0 ? 0 : k); }

extern "C" unsigned long long onefft_debug_launch_count(void) { return g_launches.load(); }

// ---- execution on device memory ---------------------------------------------------------------

// Enqueues `batch` transforms; d_in / d_out are 8-byte aligned device pointers, not overlapping.
// pre / post: optional pointwise weights (n complex values) applied by the kernel that reads the
// input and by the one that writes the output; split-BF16 plans take none (callers check).
static cudaError_t plan_enqueue(const onefft_plan *p, const float2 *in, float2 *out, long long batch, int inverse,
                                cudaStream_t s, const float2 *pre = nullptr, const float2 *post = nullptr) {
    if (batch <= 0) return cudaSuccess;
    if (p->npass == 1) {
        g_launches.fetch_add(1);
        if (p->tc) return launch_single_kernel_tc(p->log2n, in, out, batch, p->stw[0], inverse, p->tc, s);
        if (p->cols[0] == kPipelinedCols) {
            // bulk copies need 16-byte aligned transforms; weighted calls use k_batched's weights
            if (!pre && !post && !((uintptr_t)in & 15))
                return launch_batched_pipe(p->log2n, in, out, batch, p->stw[0], inverse, p->err, s);
            return launch_single_kernel(p->log2n, in, out, batch, p->stw[0], inverse, s, pre, post, -1);
        }
        return launch_single_kernel(p->log2n, in, out, batch, p->stw[0], inverse, s, pre, post, p->cols[0]);
    }
    PassArgs a{};
    a.log2n = p->log2n;
    a.tw_lo = p->tw_lo;
    a.tw_hi = p->tw_hi;
    a.lo_bits = p->lo_bits;
    a.l2_keep = p->l2_keep;
    a.tli = 31;
    a.err = p->err;
    a.pre = pre;
    a.post = post;
    // pass i through its TMA kernel where the plan asks for it and the shape and buffers allow
    const bool use_tma = p->tma && !p->tc && batch <= 65535 && ((((uintptr_t)in | (uintptr_t)out) & 15) == 0);
    auto run = [&](int mode, int i, const PassArgs &x) {
        if (use_tma && pass_tma_supported(p->len[i], p->cols[i]))
            return launch_pass_tma(mode, p->len[i], p->cols[i], x, (int)batch, s);
        return p->tc ? launch_pass_tc(mode, p->len[i], x, (int)batch, p->tc, s)
                     : launch_pass(mode, p->len[i], p->cols[i], x, (int)batch, s);
    };
    if (p->npass == 3 && p->fuse_lag && use_tma && !pre) {
        // Passes 0 and 1 in one persistent launch per transform (k_pass01_fused), then pass 2
        // over the batch. The launch needs a counter slot that no launch running at the same
        // time uses: slots are taken in turn, and a slot's next launch waits on the GPU for the
        // event recorded after its previous one. Stream capture would record that wait on an
        // event from outside the graph, so captured calls take the separate launches below.
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
            cudaGetLastError();
            cs = cudaStreamCaptureStatusActive;
        }
        if (cs == cudaStreamCaptureStatusNone) {
            const int A = p->len[0], B = p->len[1], Cd = p->len[2], G = p->chunk;
            PassArgs c0 = a, c1 = a;
            c0.stw = p->stw[0];
            c0.swap_in = inverse;
            c0.swap_out = 0;
            c0.log_s = p->log2n - A;
            c0.rev_b1 = B;
            c0.rev_b2 = Cd;
            c0.tli = G - p->cols[0];
            c0.outer_shift = Cd;
            c0.outer_base = 0;
            c0.ntiles = 1u << (B + G - p->cols[0]);
            c1.stw = p->stw[1];
            c1.swap_in = c1.swap_out = 0;
            c1.log_s = A;
            c1.tli = A - p->cols[1];
            c1.outer_shift = A;
            c1.inner_base = 0;
            c1.ntiles = 1u << (G + A - p->cols[1]);
            const unsigned k = p->next_slot.fetch_add(1, std::memory_order_relaxed) % kFusedSlots;
            FusedSlot &slot = p->slots[k];
            std::lock_guard<std::mutex> lock(slot.m);
            cudaError_t e = slot.used ? cudaStreamWaitEvent(s, slot.done, 0) : cudaSuccess;
            for (long long b = 0; b < batch && e == cudaSuccess; ++b) {
                c0.in = in + (b << p->log2n);
                c0.out = c1.out = out + (b << p->log2n);
                c1.in = c1.out;
                g_launches.fetch_add(1);
                e = launch_pass01_fused(A, p->cols[0], B, p->cols[1], c0, c1, G, Cd, p->fuse_lag,
                                        p->fused_ctr + k * p->fused_words, s);
            }
            if (e == cudaSuccess) e = cudaEventRecord(slot.done, s);
            if (e != cudaSuccess) return e;
            slot.used = true;
            a.in = out;
            a.out = out;
            a.stw = p->stw[2];
            a.swap_in = 0;
            a.swap_out = inverse;
            a.log_s = A + B;
            g_launches.fetch_add(1);
            return run(2, 2, a);
        }
    }
    if (p->npass == 3 && p->chunk > 0) {
        // Passes 0 and 1 of a three-pass transform n = A B C run chunk by chunk over the last
        // digit j_c: pass 1 on columns j_c needs only pass 0's outputs for the same j_c, which
        // form one contiguous region of A B 2^chunk values, small enough to stay in L2 between
        // the two launches. Pass 2 then runs over the whole array.
        const int A = p->len[0], B = p->len[1], Cd = p->len[2], G = p->chunk;
        PassArgs c0 = a, c1 = a;
        c0.in = in;
        c0.out = out;
        c0.stw = p->stw[0];
        c0.swap_in = inverse;
        c0.swap_out = 0;
        c0.log_s = p->log2n - A;
        c0.rev_b1 = B;
        c0.rev_b2 = Cd;
        c0.tli = G - p->cols[0];
        c0.outer_shift = Cd;
        c0.outer_base = 0;
        c0.ntiles = 1u << (B + G - p->cols[0]);
        c1.in = out;
        c1.out = out;
        c1.stw = p->stw[1];
        c1.swap_in = c1.swap_out = 0;
        c1.log_s = A;
        c1.tli = A - p->cols[1];
        c1.outer_shift = A;
        c1.inner_base = 0;
        c1.ntiles = 1u << (G + A - p->cols[1]);
        for (unsigned g = 0; g < (1u << Cd); g += 1u << G) {
            c0.inner_base = g;
            c1.outer_base = g;
            g_launches.fetch_add(2);
            cudaError_t e = run(0, 0, c0);
            if (e == cudaSuccess) e = run(1, 1, c1);
            if (e != cudaSuccess) return e;
        }
        a.in = out;
        a.out = out;
        a.stw = p->stw[2];
        a.swap_in = 0;
        a.swap_out = inverse;
        a.log_s = A + B;
        g_launches.fetch_add(1);
        return run(2, 2, a);
    }
    int done = 0;  // log2 of the digits transformed so far
    for (int i = 0; i < p->npass; ++i) {
        const bool first = i == 0, last = i == p->npass - 1;
        a.in = first ? in : out;
        a.out = out;
        a.stw = p->stw[i];
        a.swap_in = first && inverse;
        a.swap_out = last && inverse;
        if (first) {
            a.log_s = p->log2n - p->len[0];
            a.rev_b1 = p->len[1];
            a.rev_b2 = p->npass == 3 ? p->len[2] : 0;
        } else {
            a.log_s = done;
        }
        int mode = first ? 0 : last ? 2 : 1;
        g_launches.fetch_add(1);
        cudaError_t e = run(mode, i, a);
        if (e != cudaSuccess) return e;
        done += p->len[i];
    }
    return cudaSuccess;
}

static bool is_device_pointer(const void *ptr) {
    cudaPointerAttributes attr;
    if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

static bool ranges_overlap(const void *a, const void *b, size_t bytes) {
    uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + bytes && y < x + bytes;
}

static int dev_batched(const onefft_plan *p, const float *d_in, float *d_out, size_t batch, int inverse,
                       void *stream, const float *d_pre = nullptr, const float *d_post = nullptr) {
    t_last_error.clear();
    if (!p) return set_error(ONEFFT_ERR_ARG, "NULL plan");
    if (batch == 0) return 0;
    if (!d_in || !d_out) return set_error(ONEFFT_ERR_ARG, "NULL buffer");
    if (((uintptr_t)d_in | (uintptr_t)d_out) & 7) return set_error(ONEFFT_ERR_ARG, "device buffers must be 8-byte aligned");
    if (batch > ((size_t)1 << 40) / p->n) return set_error(ONEFFT_ERR_ARG, "batch too large");
    size_t bytes = batch * p->n * sizeof(float2);
    if (ranges_overlap(d_in, d_out, bytes)) return set_error(ONEFFT_ERR_ARG, "input and output overlap");
    if (d_pre || d_post) {
        if (p->tc) return set_error(ONEFFT_ERR_ARG, "pointwise weights need an FP32 plan");
        if (((uintptr_t)d_pre | (uintptr_t)d_post) & 7) return set_error(ONEFFT_ERR_ARG, "weights must be 8-byte aligned");
        // the weights are read while the output is written: they may not share bytes with it
        const uintptr_t o = (uintptr_t)d_out, wb = p->n * sizeof(float2);
        for (const float *w : {d_pre, d_post})
            if (w && (uintptr_t)w < o + bytes && o < (uintptr_t)w + wb)
                return set_error(ONEFFT_ERR_ARG, "weights overlap the output");
    }
    cudaError_t e = plan_enqueue(p, (const float2 *)d_in, (float2 *)d_out, (long long)batch, inverse,
                                 (cudaStream_t)stream, (const float2 *)d_pre, (const float2 *)d_post);
    if (e != cudaSuccess) return cuda_error(e, "kernel launch");
    return 0;
}

extern "C" int onefft_dev_forward_batched(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                          void *stream) {
    return dev_batched(plan, d_in, d_out, batch, 0, stream);
}

extern "C" int onefft_dev_inverse_batched(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                          void *stream) {
    return dev_batched(plan, d_in, d_out, batch, 1, stream);
}

extern "C" int onefft_dev_forward_weighted(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                           const float *d_pre, const float *d_post, void *stream) {
    return dev_batched(plan, d_in, d_out, batch, 0, stream, d_pre, d_post);
}

extern "C" int onefft_dev_inverse_weighted(const onefft_plan *plan, const float *d_in, float *d_out, size_t batch,
                                           const float *d_pre, const float *d_post, void *stream) {
    return dev_batched(plan, d_in, d_out, batch, 1, stream, d_pre, d_post);
}

extern "C" int onefft_dev_adjoint_batched(const onefft_plan *plan, const float *d_grad_out, float *d_grad_in,
                                          size_t batch, void *stream) {
    // F^H = conj(F): the unnormalised inverse transform, i.e. the forward kernels with re/im
    // exchanged on load and store.
    return dev_batched(plan, d_grad_out, d_grad_in, batch, 1, stream);
}

extern "C" int onefft_dev_weighted_power_loss(const onefft_plan *plan, const float *d_x, const float *d_w,
                                              float *d_grad, size_t batch, double *d_loss, void *stream) {
    t_last_error.clear();
    if (!plan) return set_error(ONEFFT_ERR_ARG, "NULL plan");
    if (plan->npass != 1 || plan->tc || plan->log2n < 4)
        return set_error(ONEFFT_ERR_ARG, "the fused loss needs an FP32 plan of 16 .. 2^14 points");
    if (!d_x || !d_w || !d_loss || batch == 0) return set_error(ONEFFT_ERR_ARG, "NULL buffer or empty batch");
    if ((((uintptr_t)d_x | (uintptr_t)d_grad | (uintptr_t)d_loss) & 7) || ((uintptr_t)d_w & 3))
        return set_error(ONEFFT_ERR_ARG, "misaligned device buffer");
    if (batch > ((size_t)1 << 40) / plan->n) return set_error(ONEFFT_ERR_ARG, "batch too large");
    if (d_grad && ranges_overlap(d_x, d_grad, batch * plan->n * sizeof(float2)))
        return set_error(ONEFFT_ERR_ARG, "input and gradient overlap");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(d_loss, 0, sizeof(double), s);
    if (e == cudaSuccess) {
        g_launches.fetch_add(1);
        e = launch_power_loss_grad(plan->log2n, (const float2 *)d_x, d_w, (float2 *)d_grad, d_loss, (long long)batch,
                                   plan->stw[0], s);
    }
    return e == cudaSuccess ? 0 : cuda_error(e, "fused loss launch");
}

// ---- per-thread host staging -------------------------------------------------------------------

namespace {

constexpr int kStreams = 3;

struct ThreadCtx {
    int device = -1;
    cudaStream_t stream[kStreams] = {};
    cudaEvent_t done[kStreams] = {};
    void *buf[kStreams] = {};  // device staging, in + out per stream
    size_t cap[kStreams] = {};

    ~ThreadCtx() {
        // may run after the CUDA runtime has shut down at process exit: ignore errors
        for (int i = 0; i < kStreams; ++i) {
            if (buf[i]) cudaFree(buf[i]);
            if (stream[i]) cudaStreamDestroy(stream[i]);
            if (done[i]) cudaEventDestroy(done[i]);
        }
    }

    cudaError_t init(int dev) {
        if (device == dev) return cudaSuccess;
        if (device >= 0) return cudaErrorInvalidDevice;  // one device per thread context
        for (int i = 0; i < kStreams; ++i) {
            cudaError_t e = cudaStreamCreateWithFlags(&stream[i], cudaStreamNonBlocking);
            if (e != cudaSuccess) return e;
            e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
            if (e != cudaSuccess) return e;
        }
        device = dev;
        return cudaSuccess;
    }

    cudaError_t reserve(int i, size_t bytes) {
        if (cap[i] >= bytes) return cudaSuccess;
        if (buf[i]) {
            cudaStreamSynchronize(stream[i]);
            cudaFree(buf[i]);
            buf[i] = nullptr;
            cap[i] = 0;
        }
        cudaError_t e = dev_alloc(&buf[i], bytes);
        if (e != cudaSuccess) {
            buf[i] = nullptr;
            return e;
        }
        cap[i] = bytes;
        return cudaSuccess;
    }
};

// Contexts per device for this thread (a thread may use plans of several devices).
constexpr int kMaxDevices = 64;
thread_local ThreadCtx *t_ctx[kMaxDevices];
struct CtxReaper {
    ~CtxReaper() {
        for (int i = 0; i < kMaxDevices; ++i) delete t_ctx[i];
    }
};
thread_local CtxReaper t_reaper;

ThreadCtx *thread_ctx(int device, cudaError_t *err) {
    (void)&t_reaper;  // odr-use so the reaper is constructed for this thread
    if (device < 0 || device >= kMaxDevices) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    ThreadCtx *&c = t_ctx[device];
    if (!c) c = new (std::nothrow) ThreadCtx();
    if (!c) {
        *err = cudaErrorMemoryAllocation;
        return nullptr;
    }
    *err = c->init(device);
    return *err == cudaSuccess ? c : nullptr;
}

// Switches to a plan's device for the duration of a call.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

}  // namespace

// After a synchronise: 0, or an error if a kernel of the plan recorded an expired bounded wait
// in the plan's error word (which is then cleared).
static int kernel_error(const onefft_plan *p) {
    if (!p->err_host) return 0;
    volatile unsigned *word = p->err_host;
    const unsigned flag = *word;
    if (!flag) return 0;
    *word = 0;
    return set_error(ONEFFT_ERR_CUDA_BASE, "a bulk tensor copy did not complete in time (code %u)", flag);
}

// One transform (or `batch`) through host or device buffers, synchronous. Returns 0 or an error;
// `out` is written only by the final copy, after every kernel succeeded.
static int host_execute(const onefft_plan *p, const float *in, float *out, size_t batch, int inverse) {
    t_last_error.clear();
    if (!p) return set_error(ONEFFT_ERR_ARG, "NULL plan");
    if (batch == 0) return 0;
    if (!in || !out) return set_error(ONEFFT_ERR_ARG, "NULL buffer");
    DeviceGuard guard(p->device);
    cudaError_t e;
    ThreadCtx *ctx = thread_ctx(p->device, &e);
    if (!ctx) return cuda_error(e, "thread context");
    const size_t tbytes = p->n * sizeof(float2);
    const bool in_dev = is_device_pointer(in), out_dev = is_device_pointer(out);
    const bool aligned = (((uintptr_t)in | (uintptr_t)out) & 7) == 0;
    if (in_dev && out_dev && aligned && !ranges_overlap(in, out, tbytes * batch)) {
        // device memory of the caller: transform in place of the caller's buffers
        e = plan_enqueue(p, (const float2 *)in, (float2 *)out, (long long)batch, inverse, ctx->stream[0]);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream[0]);
        if (e != cudaSuccess) return cuda_error(e, "transform");
        return kernel_error(p);
    }
    // Chunks of whole transforms, round-robin over the streams: chunk k's copy-in overlaps the
    // kernels and copy-out of chunks k-1 and k-2.
    size_t per_chunk = batch;
    const size_t target = (size_t)32 << 20;  // ~32 MiB of input per chunk
    if (batch > 1 && tbytes * batch > 2 * target) {
        per_chunk = target / tbytes;
        if (per_chunk == 0) per_chunk = 1;
    }
    const size_t chunks = (batch + per_chunk - 1) / per_chunk;
    const int nstreams = chunks == 1 ? 1 : kStreams;
    for (int i = 0; i < nstreams; ++i) {
        e = ctx->reserve(i, 2 * tbytes * per_chunk);
        if (e != cudaSuccess) return set_error(ONEFFT_ERR_SIZE, "staging allocation failed: %s", cudaGetErrorString(e));
    }
    // Input copies of every chunk may all be issued before any output is written back, so a
    // failure in any kernel can still leave `out` untouched: outputs are copied only after the
    // kernels of all chunks were enqueued without error. For several chunks the copy-out of a
    // chunk is issued right after its kernels (overlap); a device fault then surfaces at the sync.
    for (size_t k = 0; k < chunks; ++k) {
        const int si = (int)(k % nstreams);
        cudaStream_t s = ctx->stream[si];
        const size_t first = k * per_chunk;
        const size_t cnt = (first + per_chunk <= batch) ? per_chunk : batch - first;
        float2 *d_in = (float2 *)ctx->buf[si];
        float2 *d_out = d_in + per_chunk * p->n;
        e = cudaMemcpyAsync(d_in, (const char *)in + first * tbytes, cnt * tbytes, cudaMemcpyDefault, s);
        if (e != cudaSuccess) break;
        e = plan_enqueue(p, d_in, d_out, (long long)cnt, inverse, s);
        if (e != cudaSuccess) break;
        if (chunks == 1) {
            // single chunk: check the kernels before the output is touched
            e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) break;
            if (kernel_error(p)) return ONEFFT_ERR_CUDA_BASE;
        }
        e = cudaMemcpyAsync((char *)out + first * tbytes, d_out, cnt * tbytes, cudaMemcpyDefault, s);
        if (e != cudaSuccess) break;
    }
    cudaError_t e2 = cudaSuccess;
    for (int i = 0; i < nstreams; ++i) {
        cudaError_t es = cudaStreamSynchronize(ctx->stream[i]);
        if (e2 == cudaSuccess) e2 = es;
    }
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_error(e, "transform");
    return kernel_error(p);
}

extern "C" int onefft_plan_status(const onefft_plan *plan) {
    t_last_error.clear();
    if (!plan) return set_error(ONEFFT_ERR_ARG, "NULL plan");
    return kernel_error(plan);
}

extern "C" int onefft_debug_expire_waits(int on) {
    t_last_error.clear();
    const cudaError_t e = set_expire_waits(on);
    return e == cudaSuccess ? 0 : cuda_error(e, "wait-expiry hook");
}

extern "C" void onefft_plan_forward(const onefft_plan *plan, const float *in, float *out) {
    host_execute(plan, in, out, 1, 0);
}

extern "C" void onefft_plan_inverse(const onefft_plan *plan, const float *in, float *out) {
    host_execute(plan, in, out, 1, 1);
}

extern "C" int onefft_plan_forward_batched(const onefft_plan *plan, const float *in, float *out, size_t batch) {
    return host_execute(plan, in, out, batch, 0);
}

extern "C" int onefft_plan_inverse_batched(const onefft_plan *plan, const float *in, float *out, size_t batch) {
    return host_execute(plan, in, out, batch, 1);
}

// ---- the plan cache (src/onefft.c:1151-1189) -----------------------------------------------------

static std::atomic<onefft_plan *> g_cache[kMaxDevices][31];

static const onefft_plan *cache_get(size_t n, int *err) {
    int m;
    if (!size_log2(n, &m)) {
        *err = set_error(ONEFFT_ERR_SIZE, "n=%zu is not a power of two in [1, 2^30]", n);
        return nullptr;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *err = cuda_error(e, "no CUDA device");
        return nullptr;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        *err = set_error(ONEFFT_ERR_ARG, "device %d out of range", dev);
        return nullptr;
    }
    std::atomic<onefft_plan *> &slot = g_cache[dev][m];
    onefft_plan *p = slot.load(std::memory_order_acquire);
    if (p) return p;
    p = onefft_plan_create(n);
    if (!p) {
        *err = ONEFFT_ERR_SIZE;
        return nullptr;
    }
    onefft_plan *expected = nullptr;
    if (!slot.compare_exchange_strong(expected, p, std::memory_order_acq_rel, std::memory_order_acquire)) {
        onefft_plan_destroy(p);
        p = expected;
    }
    return p;
}

extern "C" int onefft_forward(const float *in, float *out, size_t n) {
    int err = 0;
    const onefft_plan *p = cache_get(n, &err);
    if (!p) return -1;
    return host_execute(p, in, out, 1, 0) == 0 ? 0 : -1;
}

extern "C" int onefft_inverse(const float *in, float *out, size_t n) {
    int err = 0;
    const onefft_plan *p = cache_get(n, &err);
    if (!p) return -1;
    return host_execute(p, in, out, 1, 1) == 0 ? 0 : -1;
}

extern "C" int onefft_cache_prepare(size_t n) {
    int err = 0;
    return cache_get(n, &err) ? 0 : -1;
}

extern "C" void onefft_cache_clear(void) {
    for (int d = 0; d < kMaxDevices; ++d)
        for (int m = 0; m < 31; ++m) onefft_plan_destroy(g_cache[d][m].exchange(nullptr, std::memory_order_acq_rel));
}

extern "C" int onefft_debug_twiddles(unsigned log2n, size_t count, float *out) {
    t_last_error.clear();
    if (log2n > 30 || !out || count > ((size_t)1 << 30)) return set_error(ONEFFT_ERR_ARG, "invalid twiddle probe");
    if (count == 0) return 0;
    void *d = nullptr;
    cudaError_t e = dev_alloc(&d, count * sizeof(float2));
    if (e != cudaSuccess) return set_error(ONEFFT_ERR_SIZE, "probe allocation failed");
    e = launch_twiddle_probe((float2 *)d, log2n, count, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d, count * sizeof(float2), cudaMemcpyDeviceToHost);
    cudaFree(d);
    return e == cudaSuccess ? 0 : cuda_error(e, "twiddle probe");
}

// ---- uneven batches (kernel in uneven.cu) --------------------------------------------------------

struct onefft_uneven {
    int device;
    size_t count;
    size_t span;
    onefft_plan *plans[kUnevenMaxLog2 + 1];
    void *mem;  // sorted descriptors, work items, units, queue counter + per-item step counters
    unsigned *err_host;  // error word (mapped pinned host memory), as the plans'
    UnevenArgs args;
    int grid;
    int smem;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    cudaGraphNode_t knode;
};

extern "C" void onefft_uneven_destroy(onefft_uneven *u) {
    if (!u) return;
    if (u->exec) cudaGraphExecDestroy(u->exec);
    if (u->graph) cudaGraphDestroy(u->graph);
    if (u->mem) cudaFree(u->mem);
    if (u->err_host) cudaFreeHost(u->err_host);
    for (int m = 0; m <= kUnevenMaxLog2; ++m) onefft_plan_destroy(u->plans[m]);
    delete u;
}

extern "C" size_t onefft_uneven_span(const onefft_uneven *u) { return u ? u->span : 0; }

extern "C" int onefft_uneven_status(onefft_uneven *u) {
    t_last_error.clear();
    if (!u) return set_error(ONEFFT_ERR_ARG, "NULL batch");
    volatile unsigned *word = u->err_host;
    const unsigned flag = *word;
    if (!flag) return 0;
    *word = 0;
    return set_error(ONEFFT_ERR_CUDA_BASE, "a pass-1 step waited too long for its pass 0 (code %u)", flag);
}

// Queue order of the step-wise uneven kernel: each transform of 2^13 .. 2^16 (largest first) as
// its pass-0 steps, its pass-1 steps placed at least kUnevenLagUnits units later (so they rarely
// wait, and the values between the passes of the transforms in flight stay in L2); then every
// smaller item whole.
static std::vector<UnevenUnit> uneven_units(const std::vector<UnevenItem> &items) {
    std::vector<UnevenUnit> units;
    std::vector<std::pair<int, size_t>> pending;  // (item, queue length after its pass 0)
    size_t head = 0;
    auto emit_pass1 = [&](int i) {
        const int steps = 1 << (items[i].log2n - 12);
        for (int k = 0; k < steps; ++k) units.push_back(UnevenUnit{i, steps + k});
    };
    for (int i = 0; i < (int)items.size(); ++i) {
        if (items[i].log2n < 13) continue;
        const int steps = 1 << (items[i].log2n - 12);
        for (int k = 0; k < steps; ++k) units.push_back(UnevenUnit{i, k});
        pending.emplace_back(i, units.size());
        while (head < pending.size() && units.size() - pending[head].second >= (size_t)kUnevenLagUnits)
            emit_pass1(pending[head++].first);
    }
    while (head < pending.size()) emit_pass1(pending[head++].first);
    for (int i = 0; i < (int)items.size(); ++i)
        if (items[i].log2n < 13) units.push_back(UnevenUnit{i, -1});
    return units;
}

static onefft_uneven *uneven_create(const onefft_desc *desc, size_t count, const int *split_choice);

extern "C" onefft_uneven *onefft_uneven_create(const onefft_desc *desc, size_t count) {
    t_last_error.clear();
    int tuned[kUnevenMaxLog2 + 1];
    for (int m = 0; m <= kUnevenMaxLog2; ++m) tuned[m] = uneven_tuned_split(m);
    return uneven_create(desc, count, tuned);
}

extern "C" onefft_uneven *onefft_uneven_create_split(const onefft_desc *desc, size_t count,
                                                     const int *split_choice) {
    t_last_error.clear();
    if (split_choice)
        for (int m = 13; m <= kUnevenMaxLog2; ++m)
            if (split_choice[m] < 0 || split_choice[m] >= kUnevenSplitChoices) {
                set_error(ONEFFT_ERR_ARG, "split choice %d for 2^%d out of range", split_choice[m], m);
                return nullptr;
            }
    if (!split_choice) return onefft_uneven_create(desc, count);
    return uneven_create(desc, count, split_choice);
}

static onefft_uneven *uneven_create(const onefft_desc *desc, size_t count, const int *split_choice) {
    if (!desc || count == 0 || count > (size_t)1 << 30) {
        set_error(ONEFFT_ERR_ARG, "invalid descriptor list");
        return nullptr;
    }
    // validate, then check that no two transforms overlap
    std::vector<size_t> by_offset(count);
    size_t span = 0;
    for (size_t i = 0; i < count; ++i) {
        const onefft_desc &d = desc[i];
        if (d.log2n < 0 || d.log2n > kUnevenMaxLog2 || (d.inverse != 0 && d.inverse != 1) || d.offset < 0 ||
            d.offset > ((int64_t)1 << 40)) {
            set_error(ONEFFT_ERR_ARG, "descriptor %zu invalid (log2n %d, inverse %d, offset %lld)", i, d.log2n,
                      d.inverse, (long long)d.offset);
            return nullptr;
        }
        span = std::max(span, (size_t)d.offset + ((size_t)1 << d.log2n));
        by_offset[i] = i;
    }
    std::sort(by_offset.begin(), by_offset.end(),
              [desc](size_t a, size_t b) { return desc[a].offset < desc[b].offset; });
    for (size_t i = 1; i < count; ++i) {
        const onefft_desc &p = desc[by_offset[i - 1]], &q = desc[by_offset[i]];
        if (p.offset + ((int64_t)1 << p.log2n) > q.offset) {
            set_error(ONEFFT_ERR_ARG, "transforms at offsets %lld and %lld overlap", (long long)p.offset,
                      (long long)q.offset);
            return nullptr;
        }
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        cuda_error(e, "no CUDA device");
        return nullptr;
    }
    onefft_uneven *u = new (std::nothrow) onefft_uneven();
    if (!u) {
        set_error(ONEFFT_ERR_SIZE, "out of host memory");
        return nullptr;
    }
    u->device = device;
    u->count = count;
    u->span = span;
    // largest transforms first, then by offset; equal sizes grouped into work items
    std::vector<onefft_desc> sorted(desc, desc + count);
    std::stable_sort(sorted.begin(), sorted.end(), [](const onefft_desc &a, const onefft_desc &b) {
        return a.log2n != b.log2n ? a.log2n > b.log2n : a.offset < b.offset;
    });
    std::vector<UnevenItem> items;
    for (size_t i = 0; i < count;) {
        const int m = sorted[i].log2n;
        const size_t cap = m <= 3 ? 256 : m <= 12 ? ((size_t)4096 >> m) : 1;
        size_t k = 0;
        while (i + k < count && sorted[i + k].log2n == m && k < cap) ++k;
        items.push_back(UnevenItem{m, (int)k, (int)i, 0});
        i += k;
    }
    // every size's split choice, used or not: it also selects the compiled kernel (uneven_kernel)
    for (int m = 13; m <= kUnevenMaxLog2; ++m) u->args.split[m] = split_choice[m];
    // tables of every size used: the plain single-kernel plan up to 2^12, the in-block two-pass
    // split beyond
    bool used[kUnevenMaxLog2 + 1] = {};
    for (const onefft_desc &d : sorted) used[d.log2n] = true;
    for (int m = 0; m <= kUnevenMaxLog2; ++m) {
        if (!used[m]) continue;
        if (m <= 12) {
            u->plans[m] = onefft_plan_create((size_t)1 << m);
        } else {
            const int len[2] = {uneven_split(m, split_choice[m], 0), uneven_split(m, split_choice[m], 1)};
            u->plans[m] = onefft_plan_create_tiles((size_t)1 << m, 2, len, nullptr, 0, 0);
        }
        if (!u->plans[m]) {
            onefft_uneven_destroy(u);
            set_error(ONEFFT_ERR_SIZE, "table build for 2^%d failed", m);
            return nullptr;
        }
        const onefft_plan *p = u->plans[m];
        u->args.stw[m][0] = p->stw[0];
        u->args.stw[m][1] = p->npass > 1 ? p->stw[1] : nullptr;
        u->args.tw_lo[m] = p->tw_lo;
        u->args.tw_hi[m] = p->tw_hi;
        u->args.lo_bits[m] = p->lo_bits;
    }
    const std::vector<UnevenUnit> units = uneven_units(items);
    const size_t desc_bytes = align256(count * sizeof(onefft_desc));
    const size_t item_bytes = align256(items.size() * sizeof(UnevenItem));
    const size_t unit_bytes = align256(units.size() * sizeof(UnevenUnit));
    // queue head, per item the pass-0 steps done, the abort word
    const size_t ctr_bytes = sizeof(int) + sizeof(unsigned) * (items.size() + 1);
    e = dev_alloc(&u->mem, desc_bytes + item_bytes + unit_bytes + align256(ctr_bytes));
    if (e != cudaSuccess) {
        u->mem = nullptr;
        onefft_uneven_destroy(u);
        set_error(ONEFFT_ERR_SIZE, "uneven batch allocation failed");
        return nullptr;
    }
    e = cudaHostAlloc((void **)&u->err_host, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e == cudaSuccess) {
        *(volatile unsigned *)u->err_host = 0;
        e = cudaHostGetDevicePointer((void **)&u->args.err, u->err_host, 0);
    } else {
        u->err_host = nullptr;
    }
    char *base = (char *)u->mem;
    u->args.desc = (const onefft_desc *)base;
    u->args.items = (const UnevenItem *)(base + desc_bytes);
    u->args.units = (const UnevenUnit *)(base + desc_bytes + item_bytes);
    u->args.nunits = (int)units.size();
    u->args.counter = (int *)(base + desc_bytes + item_bytes + unit_bytes);
    u->args.done = (unsigned *)(u->args.counter + 1);
    u->args.nitems = (int)items.size();
    if (e == cudaSuccess) e = cudaMemcpy(base, sorted.data(), count * sizeof(onefft_desc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(base + desc_bytes, items.data(), items.size() * sizeof(UnevenItem), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(base + desc_bytes + item_bytes, units.data(), units.size() * sizeof(UnevenUnit),
                       cudaMemcpyHostToDevice);
    // persistent grid: every block resident at once
    u->smem = uneven_smem_bytes();
    int per_sm = 0, sms = 0;
    if (e == cudaSuccess && u->smem > 48 * 1024)
        e = cudaFuncSetAttribute(uneven_kernel(u->args.split), cudaFuncAttributeMaxDynamicSharedMemorySize, u->smem);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, uneven_kernel(u->args.split), 256, u->smem);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    u->grid = std::max(1, std::min(per_sm * sms, (int)items.size()));
    // graph: zero the queue counter, the per-item step counters and the abort word, then the
    // persistent launch
    if (e == cudaSuccess) e = cudaGraphCreate(&u->graph, 0);
    cudaGraphNode_t mset = nullptr;
    if (e == cudaSuccess) {
        cudaMemsetParams mp{};
        mp.dst = u->args.counter;
        mp.value = 0;
        mp.elementSize = 4;
        mp.width = 2 + items.size();
        mp.height = 1;
        e = cudaGraphAddMemsetNode(&mset, u->graph, nullptr, 0, &mp);
    }
    if (e == cudaSuccess) {
        void *params[1] = {&u->args};
        cudaKernelNodeParams kp{};
        kp.func = (void *)uneven_kernel(u->args.split);
        kp.gridDim = dim3((unsigned)u->grid);
        kp.blockDim = dim3(256);
        kp.sharedMemBytes = (unsigned)u->smem;
        kp.kernelParams = params;
        e = cudaGraphAddKernelNode(&u->knode, u->graph, &mset, 1, &kp);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&u->exec, u->graph, 0);
    if (e != cudaSuccess) {
        onefft_uneven_destroy(u);
        cuda_error(e, "uneven batch setup");
        return nullptr;
    }
    return u;
}

extern "C" int onefft_uneven_execute(onefft_uneven *u, const float *d_in, float *d_out, void *stream) {
    t_last_error.clear();
    if (!u) return set_error(ONEFFT_ERR_ARG, "NULL batch");
    if (!d_in || !d_out) return set_error(ONEFFT_ERR_ARG, "NULL buffer");
    if (((uintptr_t)d_in | (uintptr_t)d_out) & 7) return set_error(ONEFFT_ERR_ARG, "device buffers must be 8-byte aligned");
    if (ranges_overlap(d_in, d_out, u->span * sizeof(float2))) return set_error(ONEFFT_ERR_ARG, "input and output overlap");
    cudaError_t e = cudaSuccess;
    if (u->args.in != (const float2 *)d_in || u->args.out != (float2 *)d_out) {
        u->args.in = (const float2 *)d_in;
        u->args.out = (float2 *)d_out;
        void *params[1] = {&u->args};
        cudaKernelNodeParams kp{};
        kp.func = (void *)uneven_kernel(u->args.split);
        kp.gridDim = dim3((unsigned)u->grid);
        kp.blockDim = dim3(256);
        kp.sharedMemBytes = (unsigned)u->smem;
        kp.kernelParams = params;
        e = cudaGraphExecKernelNodeSetParams(u->exec, u->knode, &kp);
    }
    if (e == cudaSuccess) {
        g_launches.fetch_add(1);
        e = cudaGraphLaunch(u->exec, (cudaStream_t)stream);
    }
    return e == cudaSuccess ? 0 : cuda_error(e, "uneven batch launch");
}

// ---- column transforms ------------------------------------------------------------------------
//
// One or two passes of the pass kernels over the whole n x cols matrix, seen as one array of
// n cols values whose element (j, b) sits at j cols + b:
//   one pass (n <= 2^12): transforms down the columns (stride cols), the larger transform's
//     factor and the column-layout store in the same kernel;
//   two passes n = 2^a 2^b: pass 0 transforms the top a bits of j (stride 2^b cols) with the
//     n-point four-step factor w_n^(j1 k0) (j1 = the low digit, column index >> log2 cols) and
//     writes column b's values as rows [b][j1][k0] of the work buffer, exactly the layout of a
//     two-pass plan's first pass for a batch of cols transforms; pass 1 transforms j1 in each
//     row block, multiplies by the larger transform's factor and writes the column layout.

struct onefft_columns {
    int device = 0;
    int m = 0, lb = 0, log_blk = 0, log2big = 0;
    int npass = 0, len[2] = {0, 0};
    unsigned long long col0 = 0;
    void *mem = nullptr;
    const float2 *stw[2] = {nullptr, nullptr};
    const double2 *tw_lo = nullptr, *tw_hi = nullptr;  // w_n (two passes)
    int lo_bits = 0;
    const double2 *big_lo = nullptr, *big_hi = nullptr;  // w_N (big_n > 0)
    int big_lo_bits = 0;
    float2 *work = nullptr;
    unsigned *err_host = nullptr, *err = nullptr;  // mapped pinned error word (TMA copy waits)
};

static bool pow2_log(unsigned long long x, int *l) {
    if (x == 0 || (x & (x - 1))) return false;
    int k = 0;
    while ((1ull << k) < x) ++k;
    *l = k;
    return true;
}

extern "C" onefft_columns *onefft_columns_create(size_t n, size_t cols, size_t blocks, unsigned long long big_n,
                                                 unsigned long long col0) {
    t_last_error.clear();
    int m, lb, lk, lbig = 0;
    if (!pow2_log(n, &m) || m < 4 || m > 24) {
        set_error(ONEFFT_ERR_SIZE, "columns: n=%zu is not a power of two in [16, 2^24]", n);
        return nullptr;
    }
    if (!pow2_log(cols, &lb) || lb < 4 || m + lb > 31) {
        set_error(ONEFFT_ERR_SIZE, "columns: cols=%zu is not a power of two >= 16 with n cols <= 2^31", cols);
        return nullptr;
    }
    if (!pow2_log(blocks, &lk) || lk > m) {
        set_error(ONEFFT_ERR_SIZE, "columns: blocks=%zu is not a power of two <= n", blocks);
        return nullptr;
    }
    if (big_n && (!pow2_log(big_n, &lbig) || lbig < m || lbig > 40 || col0 > (big_n >> m) ||
                  cols > (big_n >> m) - col0)) {
        set_error(ONEFFT_ERR_SIZE, "columns: big_n=%llu must be a power of two in [n, 2^40] with col0 + cols <= big_n / n",
                  big_n);
        return nullptr;
    }
    if (!big_n && col0) {
        set_error(ONEFFT_ERR_SIZE, "columns: col0 without big_n");
        return nullptr;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        cuda_error(e, "no CUDA device");
        return nullptr;
    }
    onefft_columns *c = new (std::nothrow) onefft_columns();
    if (!c) {
        set_error(ONEFFT_ERR_SIZE, "out of host memory");
        return nullptr;
    }
    c->device = device;
    c->m = m;
    c->lb = lb;
    c->log_blk = m - lk;
    c->log2big = lbig;
    c->col0 = col0;
    c->npass = m <= 12 ? 1 : 2;
    c->len[0] = c->npass == 1 ? m : (m + 1) / 2;
    c->len[1] = c->npass == 1 ? 0 : m / 2;
    // layout: stage tables, the w_n tables (two passes), the w_N tables, the work buffer
    size_t off[2] = {0, 0}, bytes = 0;
    for (int i = 0; i < c->npass; ++i) {
        off[i] = bytes;
        bytes = align256(bytes + sizeof(float2) * (size_t)stage_table_entries_host(c->len[i]));
    }
    size_t lo_off = 0, hi_off = 0, blo_off = 0, bhi_off = 0, work_off = 0;
    if (c->npass == 2) {
        c->lo_bits = m / 2;
        lo_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << c->lo_bits));
        hi_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << (m - c->lo_bits)));
    }
    if (lbig) {
        c->big_lo_bits = lbig / 2;
        blo_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << c->big_lo_bits));
        bhi_off = bytes;
        bytes = align256(bytes + sizeof(double2) * ((size_t)1 << (lbig - c->big_lo_bits)));
    }
    if (c->npass == 2) {
        work_off = bytes;
        bytes += sizeof(float2) << (m + lb);
    }
    e = dev_alloc(&c->mem, bytes);
    if (e != cudaSuccess) {
        delete c;
        cuda_error(e, "column transform allocation");
        set_error(ONEFFT_ERR_SIZE, "column transform allocation failed");
        return nullptr;
    }
    char *base = (char *)c->mem;
    e = cudaHostAlloc((void **)&c->err_host, sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable);
    if (e == cudaSuccess) {
        *(volatile unsigned *)c->err_host = 0;
        e = cudaHostGetDevicePointer((void **)&c->err, c->err_host, 0);
    } else {
        c->err_host = nullptr;
    }
    cudaStream_t s = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        for (int i = 0; i < c->npass && e == cudaSuccess; ++i) {
            c->stw[i] = (const float2 *)(base + off[i]);
            e = launch_stage_table((float2 *)(base + off[i]), c->len[i], s);
        }
        if (c->npass == 2 && e == cudaSuccess) {
            c->tw_lo = (const double2 *)(base + lo_off);
            c->tw_hi = (const double2 *)(base + hi_off);
            e = launch_big_table((double2 *)c->tw_lo, (double2 *)c->tw_hi, m, c->lo_bits, s);
        }
        if (lbig && e == cudaSuccess) {
            c->big_lo = (const double2 *)(base + blo_off);
            c->big_hi = (const double2 *)(base + bhi_off);
            e = launch_big_table((double2 *)c->big_lo, (double2 *)c->big_hi, lbig, c->big_lo_bits, s);
        }
        if (c->npass == 2) c->work = (float2 *)(base + work_off);
        cudaError_t e2 = cudaStreamSynchronize(s);
        if (e == cudaSuccess) e = e2;
        cudaStreamDestroy(s);
    }
    if (e != cudaSuccess) {
        cudaFree(c->mem);
        if (c->err_host) cudaFreeHost(c->err_host);
        delete c;
        cuda_error(e, "column transform table build");
        return nullptr;
    }
    return c;
}

extern "C" void onefft_columns_destroy(onefft_columns *c) {
    if (!c) return;
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != c->device) cudaSetDevice(c->device);
    cudaFree(c->mem);
    if (c->err_host) cudaFreeHost(c->err_host);
    if (cur >= 0 && cur != c->device) cudaSetDevice(cur);
    delete c;
}

extern "C" int onefft_columns_status(const onefft_columns *c) {
    t_last_error.clear();
    if (!c) return set_error(ONEFFT_ERR_ARG, "NULL column transform");
    if (!c->err_host) return 0;
    volatile unsigned *word = c->err_host;
    const unsigned flag = *word;
    if (!flag) return 0;
    *word = 0;
    return set_error(ONEFFT_ERR_CUDA_BASE, "a bulk tensor copy did not complete in time (code %u)", flag);
}

extern "C" int onefft_columns_execute(const onefft_columns *c, const float *d_in, float *d_out, int flags,
                                      void *stream) {
    t_last_error.clear();
    if (!c) return set_error(ONEFFT_ERR_ARG, "NULL column transform");
    if (!d_in || !d_out) return set_error(ONEFFT_ERR_ARG, "NULL buffer");
    if (((uintptr_t)d_in | (uintptr_t)d_out) & 7) return set_error(ONEFFT_ERR_ARG, "device buffers must be 8-byte aligned");
    if (flags & ~(ONEFFT_SWAP_IN | ONEFFT_SWAP_OUT)) return set_error(ONEFFT_ERR_ARG, "unknown flags %d", flags);
    const size_t bytes = sizeof(float2) << (c->m + c->lb);
    if (ranges_overlap(d_in, d_out, bytes)) return set_error(ONEFFT_ERR_ARG, "input and output overlap");
    int cur = -1;
    if (cudaGetDevice(&cur) != cudaSuccess || cur != c->device)
        return set_error(ONEFFT_ERR_ARG, "the column transform belongs to device %d, the current device is %d",
                         c->device, cur);
    const cudaStream_t s = (cudaStream_t)stream;
    // a pass runs through its bulk-tensor-copy tile when its length has one and what it reads is
    // 16-byte aligned (the work array always is)
    const bool in16 = ((uintptr_t)d_in & 15) == 0;
    auto run = [&](int mode, int len, const PassArgs &x, bool aligned) {
        g_launches.fetch_add(1);
        if (aligned && column_tma_log_c(len) >= 0) return launch_pass_columns_tma(mode, len, x, s);
        return launch_pass_columns(mode, len, x, s);
    };
    PassArgs a{};
    a.log2n = c->m + c->lb;
    a.tli = 31;
    a.err = c->err;
    a.swap_in = (flags & ONEFFT_SWAP_IN) ? 1 : 0;
    a.xlog_blk = c->log_blk;
    a.xlog_cols = c->lb;
    cudaError_t e;
    if (c->npass == 1) {
        a.in = (const float2 *)d_in;
        a.out = (float2 *)d_out;
        a.log_s = c->lb;
        a.stw = c->stw[0];
        a.swap_out = (flags & ONEFFT_SWAP_OUT) ? 1 : 0;
        a.tw_lo = c->big_lo;  // NULL: no factor
        a.tw_hi = c->big_hi;
        a.lo_bits = c->big_lo_bits;
        a.xlog2n = c->log2big;
        a.xcol0 = c->col0;
        a.colstore = 1;
        e = run(0, c->len[0], a, in16);
    } else {
        PassArgs p0 = a;
        p0.in = (const float2 *)d_in;
        p0.out = c->work;
        p0.log_s = c->len[1] + c->lb;
        p0.rev_b1 = c->len[1];
        p0.rev_b2 = c->lb;
        p0.stw = c->stw[0];
        p0.tw_lo = c->tw_lo;
        p0.tw_hi = c->tw_hi;
        p0.lo_bits = c->lo_bits;
        p0.xlog2n = c->m;
        p0.tw_shift = c->lb;
        e = run(0, c->len[0], p0, in16);
        if (e == cudaSuccess) {
            PassArgs p1 = a;
            p1.in = c->work;
            p1.out = (float2 *)d_out;
            p1.swap_in = 0;
            p1.swap_out = (flags & ONEFFT_SWAP_OUT) ? 1 : 0;
            p1.log_s = c->len[0];
            p1.stw = c->stw[1];
            p1.tw_lo = c->big_lo;
            p1.tw_hi = c->big_hi;
            p1.lo_bits = c->big_lo_bits;
            p1.xlog2n = c->log2big;
            p1.xcol0 = c->col0;
            p1.colstore = 1;
            e = run(2, c->len[1], p1, true);
        }
    }
    return e == cudaSuccess ? 0 : cuda_error(e, "column transform launch");
}
