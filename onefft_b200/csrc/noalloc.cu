// onefft_uneven_execute_noalloc: an uneven batch that allocates no device memory.
//
// onefft_uneven_create() allocates device memory for a batch (its sorted descriptors, work items
// and queue counter, and a plan's tables per size). Some callers cannot let a library do that:
// real-time threads that must never block in the allocator or meet an out-of-memory error
// after start-up, and applications that hand all device memory to their own arena or memory
// budget and forbid third-party cudaMalloc calls. This entry point runs the same persistent
// kernel (k_uneven) with all of that state in one file-scope __device__ array instead:
//   - the twiddle tables of every size 2^4 .. 2^16, built once per device by the first call;
//   - up to kNoAllocMaxCount descriptors and work items, copied in by every call;
//   - the work-queue counter, zeroed by every call.
// Every call shares the array, so calls whose GPU work overlaps (other streams, or other
// threads' streams) race on it: the caller must order them, e.g. issue them on one stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <mutex>

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

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct NoAllocDevice {
    bool ready = false;
    UnevenArgs args{};  // table pointers into the scratch; desc/items/counter regions
    onefft_desc *desc = nullptr;
    UnevenItem *items = nullptr;
    int *counter = nullptr;
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

// Lays out the scratch and builds every size's tables in it, on `stream`, with `device`
// current. Called once per device, under g_noalloc_mutex.
cudaError_t setup(NoAllocDevice &d, int device, cudaStream_t stream) {
    unsigned char *base = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&base, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    size_t off = 0;
    for (int m = 4; m <= kUnevenMaxLog2; ++m) {
        const int passes = m <= 12 ? 1 : 2;
        for (int p = 0; p < passes; ++p) {
            const int l = m <= 12 ? m : uneven_split(m, 0, p);  // split choice 0 (args.split stays zero)
            d.args.stw[m][p] = (const float2 *)(base + off);
            if ((e = launch_stage_table((float2 *)(base + off), l, stream)) != cudaSuccess) return e;
            off = align256(off + sizeof(float2) * (size_t)stage_table_entries_host(l));
        }
        if (m > 12) {
            const int lo_bits = m / 2;  // as the plans' tables (plan_build)
            double2 *lo = (double2 *)(base + off);
            off = align256(off + sizeof(double2) * ((size_t)1 << lo_bits));
            double2 *hi = (double2 *)(base + off);
            off = align256(off + sizeof(double2) * ((size_t)1 << (m - lo_bits)));
            if ((e = launch_big_table(lo, hi, m, lo_bits, stream)) != cudaSuccess) return e;
            d.args.tw_lo[m] = lo;
            d.args.tw_hi[m] = hi;
            d.args.lo_bits[m] = lo_bits;
        }
    }
    d.desc = (onefft_desc *)(base + off);
    off = align256(off + sizeof(onefft_desc) * kNoAllocMaxCount);
    d.items = (UnevenItem *)(base + off);
    off = align256(off + sizeof(UnevenItem) * kNoAllocMaxCount);
    d.counter = (int *)(base + off);
    off = align256(off + sizeof(int));
    if (off > kNoAllocScratchBytes) return cudaErrorInvalidValue;  // layout exceeds the array
    d.args.desc = d.desc;
    d.args.items = d.items;
    d.args.counter = d.counter;
    d.smem = uneven_smem_bytes();
    int per_sm = 0, sms = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, uneven_kernel(nullptr), 256, d.smem)) != cudaSuccess)
        return e;
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
    if (e != cudaSuccess || device < 0 || (size_t)device >= kMaxDevices) return fail(ONEFFT_ERR_CUDA_BASE - (int)e, "no CUDA device");
    NoAllocDevice &dev = g_dev[device];
    cudaStream_t s = (cudaStream_t)stream;
    if (!dev.ready && (e = setup(dev, device, s)) != cudaSuccess)
        return fail(ONEFFT_ERR_CUDA_BASE - (int)e, "no-allocation scratch set-up failed");
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
        e = cudaLaunchKernel(uneven_kernel(nullptr), dim3((unsigned)std::min(dev.grid, nitems)), dim3(256), params,
                             (size_t)dev.smem, s);
    }
    if (e != cudaSuccess) return fail(ONEFFT_ERR_CUDA_BASE - (int)e, "no-allocation uneven batch failed");
    return 0;
}
