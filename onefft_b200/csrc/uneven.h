// Internal interface of the persistent uneven-batch kernel (uneven.cu) and its host side
// (onefft_uneven_* in onefft_api.cu). Not exported from the shared library.
#pragma once

#include <cuda_runtime.h>

#include "onefft_cuda.h"

namespace ofb {

constexpr int kUnevenMaxLog2 = 16;
constexpr int kUnevenSplitChoices = 3;  // compiled two-pass splits per size 2^13 .. 2^16

// Two-pass splits (L0, L1) of the sizes one block handles, kUnevenSplitChoices per log2 n.
// Choice 0 is the plain path's split where it has one (2^15, 2^16), so that the batch reproduces
// the plain path bit for bit; the others are the candidates that onefft_b200/autotune.py times.
constexpr int kUnevenSplits[4][kUnevenSplitChoices][2] = {
    {{7, 6}, {6, 7}, {8, 5}},  // 2^13
    {{7, 7}, {8, 6}, {6, 8}},  // 2^14
    {{8, 7}, {7, 8}, {9, 6}},  // 2^15
    {{8, 8}, {9, 7}, {7, 9}},  // 2^16
};

// The split the batch uses per size 2^13 .. 2^16 unless told otherwise, measured by
// `python -m onefft_b200.autotune --uneven` on a B200 (2^25 values of one size per batch, half of
// them inverse): 2^13 (7,6) 183 us, (6,7) 216 us, (8,5) 158 us; 2^14 (7,7) 207 us, (8,6) 183 us,
// (6,8) 227 us; 2^15 (8,7) 206 us, (7,8) 221 us, (9,6) 239 us; 2^16 (8,8) 234 us, (9,7) 277 us,
// (7,9) 299 us.
constexpr int kUnevenTunedSplit[4] = {2, 1, 0, 0};

// Pass length (log2) of pass `pass` of the tuned split of 2^m, 13 <= m <= 16.
constexpr int uneven_tuned_len(int m, int pass) {
    return kUnevenSplits[m - 13][kUnevenTunedSplit[m - 13]][pass ? 1 : 0];
}

// One work item: `count` transforms of size 2^log2n at desc[first .. first + count).
struct UnevenItem {
    int log2n;
    int count;
    int first;
    int pad;
};

// One unit of the step-wise work queue: a small item whole (step < 0), or one step of 4096
// values of a transform of 2^13 .. 2^16: steps 0 .. 2^(m-12) - 1 of its pass 0, then as many of
// its pass 1.
struct UnevenUnit {
    int item;
    int step;
};

// Pass-1 units of a transform follow the last pass-0 unit of that transform by at least this many
// units in the queue: about the number of units the resident blocks run at once, so that pass
// 1 rarely waits, while the values between the passes of the transforms in flight (this many
// units of 32 KiB) stay far below the L2's 126 MB.
constexpr int kUnevenLagUnits = 1024;

// Kernel arguments, passed by value (about 1 KiB).
struct UnevenArgs {
    const float2 *in;
    float2 *out;
    const onefft_desc *desc;  // sorted copy of the descriptors
    const UnevenItem *items;
    int nitems;
    int *counter;  // work queue head, zeroed before every launch
    // Step-wise queue (NULL: every block runs whole items, the transforms of 2^13 .. 2^16 tile
    // after tile in one block): the units in queue order, and per item the pass-0 steps done,
    // followed by one abort word (all zeroed before every launch, like the counter).
    const UnevenUnit *units;
    int nunits;
    unsigned *done;
    unsigned *err;  // set when a pass-1 unit's bounded wait for its pass 0 ran out
    const float2 *stw[kUnevenMaxLog2 + 1][2];  // stage tables: [m][0] single kernel / pass 0, [m][1] pass 1
    const double2 *tw_lo[kUnevenMaxLog2 + 1];
    const double2 *tw_hi[kUnevenMaxLog2 + 1];
    int lo_bits[kUnevenMaxLog2 + 1];
    int split[kUnevenMaxLog2 + 1];  // 2^13 .. 2^16: which compiled split (0 .. kUnevenSplitChoices - 1)
};

// Pass lengths (log2) of the two in-block passes of split `choice` for 13 <= m <= 16 (0 for other
// m or choices).
int uneven_split(int m, int choice, int pass);
// The autotuned split choice of size 2^m (0 outside 13 .. 16).
int uneven_tuned_split(int m);
// Dynamic shared memory of k_uneven, and the kernel that runs split choices split[13 .. 16]
// (NULL: choice 0 everywhere), for graph nodes / launches / occupancy.
int uneven_smem_bytes();
const void *uneven_kernel(const int *split);

}  // namespace ofb
