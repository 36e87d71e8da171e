// Internal interface of the persistent uneven-batch kernel (uneven.cu) and its host side
// (onefft_uneven_* in onefft_api.cu). Not exported from the shared library.
#pragma once

#include <cuda_runtime.h>

#include "onefft_cuda.h"

namespace ofb {

constexpr int kUnevenMaxLog2 = 16;

// One work item: `count` transforms of size 2^log2n at desc[first .. first + count).
struct UnevenItem {
    int log2n;
    int count;
    int first;
    int pad;
};

// Kernel arguments, passed by value (about 1 KiB).
struct UnevenArgs {
    const float2 *in;
    float2 *out;
    const onefft_desc *desc;  // sorted copy of the descriptors
    const UnevenItem *items;
    int nitems;
    int *counter;  // work queue head, zeroed before every launch
    const float2 *stw[kUnevenMaxLog2 + 1][2];  // stage tables: [m][0] single kernel / pass 0, [m][1] pass 1
    const double2 *tw_lo[kUnevenMaxLog2 + 1];
    const double2 *tw_hi[kUnevenMaxLog2 + 1];
    int lo_bits[kUnevenMaxLog2 + 1];
};

// Pass lengths (log2) of the two in-block passes for 13 <= m <= 16.
int uneven_split(int m, int pass);
// Dynamic shared memory of k_uneven, and the kernel itself (for graph nodes / occupancy).
int uneven_smem_bytes();
const void *uneven_kernel();

}  // namespace ofb
