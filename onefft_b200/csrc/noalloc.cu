// onefft_uneven_execute_noalloc: an uneven batch that allocates no device memory.
//
// onefft_uneven_create() allocates device memory for a batch (its sorted descriptors, work items
// and queue counter, and a plan's tables per size). Some callers cannot let a library do that:
// real-time threads that must never block in the allocator or meet an out-of-memory error
// after start-up, and applications that hand all device memory to their own arena or memory
// budget and forbid third-party cudaMalloc calls. This entry point runs the same persistent
// kernel (k_uneven, with the same tuned splits as onefft_uneven_create) with all of that state in
// one file-scope __device__ array instead:
//   - the twiddle tables of every size 2^4 .. 2^16, built by the first call on a device (and
//     again by the first call after that device's context was reset);
//   - up to kNoAllocMaxCount descriptors and work items, copied in by every call;
//   - the work-queue counter, zeroed by every call.
// Every call shares the array, so calls whose GPU work overlaps (other streams, or other
// threads' streams) race on it: the caller must order them, e.g. issue them on one stream.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <mutex>

#include "fft_device.cuh"
#include "fft_launch.h"
#include "onefft_cuda.h"
#include "uneven.h"

namespace ofb {

constexpr size_t kNoAllocScratchBytes = 384u << 10;  // 384 KiB per device
constexpr size_t kNoAllocMaxCount = 4096;            // descriptors per call
constexpr size_t kMaxDevices = 64;

// The scratch of the no-allocation path. In host code this name is only a handle for
// cudaGetSymbolAddress: its device address is looked up once per device and passed on.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

constexpr size_t align256c(size_t x) { return (x + 255) & ~(size_t)255; }

// log2 length of pass p of size 2^m in the scratch tables: one kernel up to 2^12, the tuned
// in-block split beyond (the split onefft_uneven_create uses).
constexpr int table_len(int m, int p) { return m <= 12 ? m : uneven_tuned_len(m, p); }

// Byte offsets of everything in the scratch: per size 2^4 .. 2^16 the stage tables of its passes
// and, for the two-pass sizes, the two FP64 tables of w_n (lo_bits = m / 2, as plan_build); then
// the descriptors, the work items and the queue counter. Computed at compile time, so the bound
// below is checked before any kernel can write into the array.
struct Layout {
    size_t stw[kUnevenMaxLog2 + 1][2];
    size_t lo[kUnevenMaxLog2 + 1];
    size_t hi[kUnevenMaxLog2 + 1];
    size_t desc, items, counter, total;
};

constexpr Layout make_layout() {
    Layout l{};
    size_t off = 0;
    for (int m = 4; m <= kUnevenMaxLog2; ++m) {
        for (int p = 0; p < (m <= 12 ? 1 : 2); ++p) {
            l.stw[m][p] = off;
            off = align256c(off + sizeof(float2) * (size_t)stage_table_entries(table_len(m, p)));
        }
        if (m > 12) {
            l.lo[m] = off;
            off = align256c(off + sizeof(double2) * ((size_t)1 << (m / 2)));
            l.hi[m] = off;
            off = align256c(off + sizeof(double2) * ((size_t)1 << (m - m / 2)));
        }
    }
    l.desc = off;
    off = align256c(off + sizeof(onefft_desc) * kNoAllocMaxCount);
    l.items = off;
    off = align256c(off + sizeof(UnevenItem) * kNoAllocMaxCount);
    l.counter = off;
    off = align256c(off + sizeof(int));
    l.total = off;
    return l;
}

constexpr Layout kLayout = make_layout();
static_assert(kLayout.total <= kNoAllocScratchBytes, "the no-allocation layout does not fit its array");

struct NoAllocDevice {
    bool ready = false;
    unsigned long long context = 0;  // id of the CUDA context the tables were built in
    UnevenArgs args{};               // table pointers into the scratch; desc/items/counter regions
    onefft_desc *desc = nullptr;
    UnevenItem *items = nullptr;
    int *counter = nullptr;
    const void *kernel = nullptr;
    int grid = 0;
    int smem = 0;
};

std::mutex g_noalloc_mutex;  // host-side staging below, and the per-device set-up
NoAllocDevice g_dev[kMaxDevices];
onefft_desc g_by_offset[kNoAllocMaxCount];
onefft_desc g_sorted[kNoAllocMaxCount];
UnevenItem g_items[kNoAllocMaxCount];

// reported through onefft_last_error() of the calling thread
int fail(int code, const char *msg) {
    record_error(msg);
    return code;
}

// A CUDA failure: cleared (so a non-sticky error does not surface in the caller's next check)
// and reported with the runtime's description.
int fail_cuda(cudaError_t e, const char *what) {
    cudaGetLastError();
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    record_error(buf);
    return ONEFFT_ERR_CUDA_BASE - (int)e;
}

// Unique id of the device's primary CUDA context, made current on this thread (cuCtxGetId), so
// that a context created after cudaDeviceReset, whose __device__ arrays start out empty, is
// noticed.
cudaError_t current_context_id(int device, unsigned long long *id) {
    using GetCurrent = CUresult (*)(CUcontext *);
    using GetId = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (GetCurrent)p;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (GetId)p;
    });
    if (!get_current || !get_id) return cudaErrorNotSupported;
    cudaError_t e = cudaSetDevice(device);  // makes the device's primary context current on this thread
    if (e != cudaSuccess) return e;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, id) != CUDA_SUCCESS) return cudaErrorNotSupported;
    return cudaSuccess;
}

// Builds every size's tables in the scratch, on `stream`, with `device` current. Called under
// g_noalloc_mutex, once per device and context.
cudaError_t setup(NoAllocDevice &d, int device, cudaStream_t stream) {
    unsigned char *base = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&base, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    d.ready = false;
    d.args = UnevenArgs{};
    for (int m = 4; m <= kUnevenMaxLog2; ++m) {
        for (int p = 0; p < (m <= 12 ? 1 : 2); ++p) {
            float2 *t = (float2 *)(base + kLayout.stw[m][p]);
            d.args.stw[m][p] = t;
            if ((e = launch_stage_table(t, table_len(m, p), stream)) != cudaSuccess) return e;
            g_launches.fetch_add(1);
        }
        if (m > 12) {
            double2 *lo = (double2 *)(base + kLayout.lo[m]), *hi = (double2 *)(base + kLayout.hi[m]);
            if ((e = launch_big_table(lo, hi, m, m / 2, stream)) != cudaSuccess) return e;
            g_launches.fetch_add(1);
            d.args.tw_lo[m] = lo;
            d.args.tw_hi[m] = hi;
            d.args.lo_bits[m] = m / 2;
            d.args.split[m] = uneven_tuned_split(m);
        }
    }
    d.desc = (onefft_desc *)(base + kLayout.desc);
    d.items = (UnevenItem *)(base + kLayout.items);
    d.counter = (int *)(base + kLayout.counter);
    d.args.desc = d.desc;
    d.args.items = d.items;
    d.args.counter = d.counter;
    d.kernel = uneven_kernel(d.args.split);  // the tuned kernel, as onefft_uneven_create
    d.smem = uneven_smem_bytes();
    if (d.smem > 48 * 1024 &&
        (e = cudaFuncSetAttribute(d.kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, d.smem)) != cudaSuccess)
        return e;
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, d.kernel, 256, d.smem)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) return e;
    d.grid = std::max(1, per_sm * sms);
    if ((e = cudaStreamSynchronize(stream)) != cudaSuccess) return e;
    d.ready = true;
    return cudaSuccess;
}

}  // namespace
}  // namespace ofb

using namespace ofb;

extern "C" int onefft_uneven_execute_noalloc(const onefft_desc *desc, size_t count, const float *d_in, float *d_out,
                                             void *stream) {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    record_error("");
    if (!desc || count == 0) return fail(ONEFFT_ERR_ARG, "empty descriptor list");
    if (count > kNoAllocMaxCount) return fail(ONEFFT_ERR_ARG, "more descriptors than the no-allocation limit (4096)");
    if (!d_in || !d_out || (((uintptr_t)d_in | (uintptr_t)d_out) & 7))
        return fail(ONEFFT_ERR_ARG, "device buffers must be non-NULL and 8-byte aligned");
    size_t span = 0;
    for (size_t i = 0; i < count; ++i) {
        const onefft_desc &d = desc[i];
        if (d.log2n < 0 || d.log2n > kUnevenMaxLog2 || (d.inverse != 0 && d.inverse != 1) || d.offset < 0 ||
            d.offset > ((int64_t)1 << 40))
            return fail(ONEFFT_ERR_ARG, "invalid descriptor");
        span = std::max(span, (size_t)d.offset + ((size_t)1 << d.log2n));
        g_by_offset[i] = d;
    }
    {
        const uintptr_t a = (uintptr_t)d_in, b = (uintptr_t)d_out, bytes = span * 8;
        if (a < b + bytes && b < a + bytes) return fail(ONEFFT_ERR_ARG, "input and output overlap");
    }
    // transforms must not overlap: check in offset order (std::sort works in place) ...
    std::sort(g_by_offset, g_by_offset + count,
              [](const onefft_desc &x, const onefft_desc &y) { return x.offset < y.offset; });
    for (size_t i = 1; i < count; ++i)
        if (g_by_offset[i - 1].offset + ((int64_t)1 << g_by_offset[i - 1].log2n) > g_by_offset[i].offset)
            return fail(ONEFFT_ERR_ARG, "transforms overlap");
    // ... then order largest first, by offset within a size (a counting sort into g_sorted, the
    // order onefft_uneven_create uses)
    size_t start[kUnevenMaxLog2 + 2] = {};
    for (size_t i = 0; i < count; ++i) ++start[kUnevenMaxLog2 - g_by_offset[i].log2n + 1];
    for (int k = 1; k <= kUnevenMaxLog2 + 1; ++k) start[k] += start[k - 1];
    for (size_t i = 0; i < count; ++i) g_sorted[start[kUnevenMaxLog2 - g_by_offset[i].log2n]++] = g_by_offset[i];
    int nitems = 0;
    for (size_t i = 0; i < count;) {
        const int m = g_sorted[i].log2n;
        const size_t cap = m <= 3 ? 256 : m <= 12 ? ((size_t)4096 >> m) : 1;
        size_t k = 0;
        while (i + k < count && g_sorted[i + k].log2n == m && k < cap) ++k;
        g_items[nitems++] = UnevenItem{m, (int)k, (int)i, 0};
        i += k;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail_cuda(e, "no CUDA device");
    if (device < 0 || (size_t)device >= kMaxDevices) return fail(ONEFFT_ERR_ARG, "device index out of range");
    unsigned long long context = 0;
    if ((e = current_context_id(device, &context)) != cudaSuccess)
        return fail_cuda(e, "no-allocation set-up: no context id");
    NoAllocDevice &dev = g_dev[device];
    cudaStream_t s = (cudaStream_t)stream;
    if (!dev.ready || dev.context != context) {
        if ((e = setup(dev, device, s)) != cudaSuccess) return fail_cuda(e, "no-allocation scratch set-up failed");
        dev.context = context;
    }
    UnevenArgs args = dev.args;
    args.in = (const float2 *)d_in;
    args.out = (float2 *)d_out;
    args.nitems = nitems;
    e = cudaMemcpyAsync(dev.desc, g_sorted, count * sizeof(onefft_desc), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dev.items, g_items, nitems * sizeof(UnevenItem), cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(dev.counter, 0, sizeof(int), s);
    if (e == cudaSuccess) {
        // a pageable-memory copy has read g_sorted / g_items when it returns, so the next call
        // may refill them; the GPU work itself is only enqueued
        void *params[1] = {&args};
        g_launches.fetch_add(1);
        e = cudaLaunchKernel(dev.kernel, dim3((unsigned)std::min(dev.grid, nitems)), dim3(256), params,
                             (size_t)dev.smem, s);
    }
    if (e != cudaSuccess) return fail_cuda(e, "no-allocation uneven batch failed");
    return 0;
}
