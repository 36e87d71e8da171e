// Internal launch interface between the C-ABI layer (onefft_api.cu) and the kernels
// (fft_kernels.cu). Nothing here is exported from the shared library.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace ofb {

// Raises a kernel's dynamic shared-memory limit to `bytes` on the calling thread's current
// device, once per device: the attribute belongs to each device's copy of the kernel, so a process
// that runs on several GPUs must set it on every one. `done` is the call site's own bit mask of
// devices already set (a function-local static of the launcher). Thread-safe.
inline cudaError_t smem_limit(const void* kernel, int bytes, std::atomic<unsigned long long>& done) {
    if (bytes <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = 1ull << (dev & 63);
    if (done.load(std::memory_order_acquire) & bit) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_acq_rel);
    return e;
}

// Arguments of one pass of the multi-pass decomposition (see k_pass in fft_kernels.cu).
struct PassArgs {
    const float2* in;
    float2* out;
    int log2n;       // transform size; consecutive transforms of a batch are 2^log2n apart
    int log_s;       // log2 of the element stride of this pass (first pass: log2(n / L0))
    int rev_b1;      // first pass: log2 L1, log2 L2 (0 for two passes) of the digit reversal
    int rev_b2;
    int swap_in;     // inverse: exchange re/im on load (first pass) / on store (last pass)
    int swap_out;
    const float2* stw;      // stage twiddles of this pass's tile length
    const double2* tw_lo;   // two-level FP64 tables of w_n
    const double2* tw_hi;
    int lo_bits;
    int l2_keep;     // store the intermediate array with L2 evict-last priority
    // Tile t of a launch starts at column
    //   col0 = ((outer_base + (t >> tli)) << outer_shift) + inner_base + ((t mod 2^tli) << log_c)
    // which lets a launch cover one chunk of the columns (tli = 31: col0 = t << log_c).
    int tli;
    int outer_shift;
    unsigned outer_base;
    unsigned inner_base;
    unsigned ntiles;  // grid size of the launch (tiles per transform)
    unsigned* err;    // plan's error word (mapped host memory): set by a kernel whose bounded wait ran out
    // pointwise weights (n complex values, NULL = none): the first pass multiplies input element
    // i by pre[i], the last pass output element i (natural order) by post[i]
    const float2* pre;
    const float2* post;
    // Column transforms (launch_pass_columns only; zero elsewhere). The launch covers one matrix
    // of 2^log2n values whose columns are 2^xlog_cols interleaved transforms:
    //  - tw_shift: the first pass's inter-pass factor of column col is F = xcol0 + (col >> tw_shift),
    //    its tables (tw_lo, tw_hi, lo_bits) those of w_(2^xlog2n); tw_lo NULL = no factor;
    //  - the last pass multiplies output k of transform h by w_(2^xlog2n)^((xcol0 + h) k);
    //  - colstore: output k of transform b goes to
    //    ((((k >> xlog_blk) << xlog_cols) + b) << xlog_blk) + (k mod 2^xlog_blk).
    int tw_shift;
    int xlog2n;
    unsigned long long xcol0;
    int colstore;
    int xlog_blk;
    int xlog_cols;
};

// Largest size handled by one kernel (k_tiny / k_batched).
constexpr int kMaxSingleLog2 = 14;

// log2 of the transforms per block of the one-kernel sizes: the default (4096-value tiles),
// and whether a width was compiled (the default, half and twice as many transforms per block, up
// to 8192 values; sizes 2^13 and 2^14 only one per block)
int batched_log_c(int log_l);
bool batched_log_c_supported(int log_l, int log_c);
int pass_log_c(int log_l);
bool pass_tile_supported(int log_l, int log_c);

// pre / post: optional pointwise weights of the input and output (n complex values each);
// log_c: transforms per block of k_batched (batched_log_c_supported; < 0 = the default; weighted
// calls always use the default)
cudaError_t launch_single_kernel(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                 int inverse, cudaStream_t stream, const float2* pre = nullptr,
                                 const float2* post = nullptr, int log_c = -1);
cudaError_t launch_pass(int mode, int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t stream);
// One pass (mode 0 first, 2 last) of a column transform (see the column fields of PassArgs), with
// the default tile width pass_log_c(log_l); one launch over the whole matrix of 2^a.log2n values
// (log2n <= 31, at least one tile).
cudaError_t launch_pass_columns(int mode, int log_l, const PassArgs& a, cudaStream_t stream);
// The same through the bulk-tensor-copy tiles (fft_tma.cu): tile width column_tma_log_c(log_l)
// (-1: none for this length); a.in 16-byte aligned; a.err set (an expired copy wait).
int column_tma_log_c(int log_l);
cudaError_t launch_pass_columns_tma(int mode, int log_l, const PassArgs& a, cudaStream_t stream);
// TMA-staged passes (fft_tma.cu): same arithmetic as launch_pass; 16-byte aligned buffers,
// batch <= 65535, shapes pass_tma_supported()
bool pass_tma_supported(int log_l, int log_c);
// Test hook: every first bounded wait of the TMA-staged kernels on the current device counts as
// expired while `on` (onefft_debug_expire_waits).
cudaError_t set_expire_waits(int on);
// Passes 0 and 1 of a three-pass transform (pass lengths 2^l0, 2^l1, 2^len2, tile widths 2^c0,
// 2^c1) in ONE persistent launch over chunks of 2^g last-digit columns, pass 1 trailing pass 0 by
// `lag` chunks (fft_tma.cu, k_pass01_fused). a0 / a1: the arguments of the chunked launches of
// passes 0 and 1 (ntiles = tiles per chunk; the per-chunk bases are ignored); one transform.
// ctr: 2 + 2^(len2 - g) zeroed words used by no concurrent launch (zero again afterwards).
bool pass01_fused_supported(int l0, int c0, int l1, int c1);
// One-kernel sizes 2^12 / 2^13 as a persistent kernel with one transform per block and the next
// transform's values arriving by one bulk copy while the current one computes (fft_tma.cu,
// k_batched_pipe); same bits as launch_single_kernel. `in` 16-byte aligned; err: the plan's error
// word (an expired copy wait).
bool batched_pipe_supported(int log2n);
cudaError_t launch_batched_pipe(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                int inverse, unsigned* err, cudaStream_t stream);
cudaError_t launch_pass01_fused(int l0, int c0, int l1, int c1, const PassArgs& a0, const PassArgs& a1, int g,
                                int len2, int lag, unsigned* ctr, cudaStream_t stream);
cudaError_t launch_pass_tma(int mode, int log_l, int log_c, const PassArgs& a, int batch, cudaStream_t stream);
// split-BF16 tensor-core variants (fft_tc.cu) of `terms` = 3 or 6 split products: n = 2^4 .. 2^14
// in one kernel; pass lengths 2^5 .. 2^12 with the default tile width pass_log_c()
cudaError_t launch_single_kernel_tc(int log2n, const float2* in, float2* out, long long batch, const float2* stw,
                                    int inverse, int terms, cudaStream_t stream);
cudaError_t launch_pass_tc(int mode, int log_l, const PassArgs& a, int batch, int terms, cudaStream_t stream);
// fused forward -> sum w^2 |y|^2 -> adjoint of 2 w^2 y, n = 2^4 .. 2^14 (fft_fused.cu)
cudaError_t launch_power_loss_grad(int log2n, const float2* x, const float* w, float2* grad, double* loss,
                                   long long batch, const float2* stw, cudaStream_t stream);
cudaError_t launch_stage_table(float2* dst, int log_l, cudaStream_t stream);
cudaError_t launch_big_table(double2* lo, double2* hi, int log2n, int lo_bits, cudaStream_t stream);
int stage_table_entries_host(int log_l);
// Sets the calling thread's onefft_last_error() message.
void record_error(const char *msg);
// Kernel launches issued through the library (onefft_debug_launch_count); every entry point that
// launches a kernel adds to it.
extern std::atomic<unsigned long long> g_launches;
cudaError_t launch_twiddle_probe(float2* dst, unsigned log2n, unsigned long long count, cudaStream_t stream);

}  // namespace ofb
