// Split-BF16 tensor-core variant of the Stockham tile engine.
//
// Every radix-16 stage runs as a dense complex matrix product Y = F16 X on the tensor cores:
// 8 butterflies form the 16x8 operand X of one mma.sync m16n8k16 (bf16 in, FP32 accumulate).
// Each FP32 value v is split into hi = bf16(v) and lo = bf16(v - hi), and the product keeps the
// three terms F_hi X_hi + F_hi X_lo + F_lo X_hi (the dropped F_lo X_lo is ~2^-18 relative), for
// the real and imaginary parts: 12 MMAs per 8 butterflies. Twiddles before a stage and the last
// radix-2/4/8 stage (when log2 L is not a multiple of 4) stay in FP32. The representation error
// of one split product is ~2^-17, two orders of magnitude above FP32's rounding, so this variant
// is measured against the FP32 path's error bound and accepted only where it meets it.
#pragma once

#include <cuda_bf16.h>

#include "fft_device.cuh"

namespace ofb {

__device__ __forceinline__ unsigned pack_bf16(float lo_elem, float hi_elem) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo_elem, hi_elem);
    return *reinterpret_cast<unsigned*>(&p);
}

// v = hi + lo with hi = bf16(v), lo = bf16(v - hi)
__device__ __forceinline__ void split_bf16(float v, float& hi, float& lo) {
    hi = __bfloat162float(__float2bfloat16_rn(v));
    lo = v - hi;
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// A fragments of F16[p][q] = w_16^(p q) split in hi/lo: real, imaginary and negated imaginary
// parts. Lane l holds rows g = l/4, g+8 and columns 2t, 2t+1, 2t+8, 2t+9 (t = l%4) in the
// m16n8k16 row-major layout.
struct DftFrags {
    unsigned re_hi[4], re_lo[4], im_hi[4], im_lo[4], nim_hi[4], nim_lo[4];
};

__device__ __forceinline__ float2 w16(int k) {
    // w_16^k from exact constants (no libm), k mod 16
    const float c1 = kC8, s1 = kS8, r = kR2;
    const float cs[16] = {1.f, c1, r, s1, 0.f, -s1, -r, -c1, -1.f, -c1, -r, -s1, 0.f, s1, r, c1};
    const float sn[16] = {0.f, s1, r, c1, 1.f, c1, r, s1, 0.f, -s1, -r, -c1, -1.f, -c1, -r, -s1};
    k &= 15;
    return make_float2(cs[k], -sn[k]);
}

__device__ __forceinline__ void make_dft_frags(DftFrags& f, int lane) {
    const int g = lane >> 2, t = lane & 3;
    const int rows[4] = {g, g + 8, g, g + 8};
    const int cols[4] = {2 * t, 2 * t, 2 * t + 8, 2 * t + 8};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 w0 = w16(rows[i] * cols[i]), w1 = w16(rows[i] * (cols[i] + 1));
        float h0, l0, h1, l1;
        split_bf16(w0.x, h0, l0);
        split_bf16(w1.x, h1, l1);
        f.re_hi[i] = pack_bf16(h0, h1);
        f.re_lo[i] = pack_bf16(l0, l1);
        split_bf16(w0.y, h0, l0);
        split_bf16(w1.y, h1, l1);
        f.im_hi[i] = pack_bf16(h0, h1);
        f.im_lo[i] = pack_bf16(l0, l1);
        f.nim_hi[i] = pack_bf16(-h0, -h1);
        f.nim_lo[i] = pack_bf16(-l0, -l1);
    }
}

// One radix-16 stage S of a tile on the tensor cores, shared memory to shared memory.
// Butterfly beta (0 .. THREADS-1) is column c / lane j of the plain engine's thread beta:
// COL (LM = C): c = beta mod C, b = beta / C; ROW (LM = 1): b = beta mod T, c = beta / T.
// Element e of column c lives at slot spad(e LM + cofs(c)).
template <int LOG_L, int LOG_C, int LM, int S>
__device__ __forceinline__ void tc_stage(float2* smem, const float2* __restrict__ stw, const DftFrags& F, int tid) {
    using St = Stages<LOG_L>;
    constexpr int T = St::T, C = 1 << LOG_C;
    constexpr int LNS = St::log2_ns(S), NS = 1 << LNS;
    const int lane = tid & 31, warp_base = tid & ~31;
    const int t = lane & 3, nb = lane >> 2;
    float acc_r[4][4], acc_i[4][4];
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
        // inputs q = 2t, 2t+1, 2t+8, 2t+9 of butterfly beta = warp_base + 8 grp + nb
        const int beta = warp_base + 8 * grp + nb;
        const int c = LM == 1 ? beta >> (LOG_L - 4) : beta & (C - 1);
        const int b = LM == 1 ? beta & (T - 1) : beta >> LOG_C;
        const int cofs = LM == 1 ? c << LOG_L : c;
        const int qs[4] = {2 * t, 2 * t + 1, 2 * t + 8, 2 * t + 9};
        float xr_hi[4], xr_lo[4], xi_hi[4], xi_lo[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float2 x = smem[spad((b + qs[i] * T) * LM + cofs)];
            if (S > 0) {
                const int r = b & (NS - 1);
                if (qs[i] > 0) x = cmul(x, __ldg(stw + St::tw_offset(S) + (qs[i] - 1) * NS + r));
            }
            split_bf16(x.x, xr_hi[i], xr_lo[i]);
            split_bf16(x.y, xi_hi[i], xi_lo[i]);
        }
        const unsigned brh0 = pack_bf16(xr_hi[0], xr_hi[1]), brh1 = pack_bf16(xr_hi[2], xr_hi[3]);
        const unsigned brl0 = pack_bf16(xr_lo[0], xr_lo[1]), brl1 = pack_bf16(xr_lo[2], xr_lo[3]);
        const unsigned bih0 = pack_bf16(xi_hi[0], xi_hi[1]), bih1 = pack_bf16(xi_hi[2], xi_hi[3]);
        const unsigned bil0 = pack_bf16(xi_lo[0], xi_lo[1]), bil1 = pack_bf16(xi_lo[2], xi_lo[3]);
        float (&Dr)[4] = acc_r[grp];
        float (&Di)[4] = acc_i[grp];
#pragma unroll
        for (int i = 0; i < 4; ++i) Dr[i] = Di[i] = 0.f;
        // Yr = Fr Xr - Fi Xi, Yi = Fi Xr + Fr Xi, three split terms each; small terms first
        mma_bf16(Dr, F.re_lo, brh0, brh1);
        mma_bf16(Dr, F.re_hi, brl0, brl1);
        mma_bf16(Dr, F.nim_lo, bih0, bih1);
        mma_bf16(Dr, F.nim_hi, bil0, bil1);
        mma_bf16(Dr, F.re_hi, brh0, brh1);
        mma_bf16(Dr, F.nim_hi, bih0, bih1);
        mma_bf16(Di, F.im_lo, brh0, brh1);
        mma_bf16(Di, F.im_hi, brl0, brl1);
        mma_bf16(Di, F.re_lo, bih0, bih1);
        mma_bf16(Di, F.re_hi, bil0, bil1);
        mma_bf16(Di, F.im_hi, brh0, brh1);
        mma_bf16(Di, F.re_hi, bih0, bih1);
    }
    __syncthreads();  // every input of the stage has been read
#pragma unroll
    for (int grp = 0; grp < 4; ++grp) {
        // D fragment: rows p = nb, nb + 8; columns (butterflies) 2t, 2t+1 of the group
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int beta = warp_base + 8 * grp + 2 * t + h;
            const int c = LM == 1 ? beta >> (LOG_L - 4) : beta & (C - 1);
            const int b = LM == 1 ? beta & (T - 1) : beta >> LOG_C;
            const int cofs = LM == 1 ? c << LOG_L : c;
            const int e0 = ((b >> LNS) << (4 + LNS)) + (b & (NS - 1));
            smem[spad((e0 + nb * NS) * LM + cofs)] = make_float2(acc_r[grp][h], acc_i[grp][h]);
            smem[spad((e0 + (nb + 8) * NS) * LM + cofs)] = make_float2(acc_r[grp][2 + h], acc_i[grp][2 + h]);
        }
    }
    __syncthreads();
}

template <int LOG_L, int LOG_C, int LM, int S>
__device__ __forceinline__ void tc_stages(float2* smem, const float2* __restrict__ stw, const DftFrags& F, int tid) {
    if constexpr (S < Stages<LOG_L>::N16) {
        tc_stage<LOG_L, LOG_C, LM, S>(smem, stw, F, tid);
        tc_stages<LOG_L, LOG_C, LM, S + 1>(smem, stw, F, tid);
    }
}

// Same contract as tile_fft (v[k] = X[j + T k] in, Y[j + T k] out) with the radix-16 stages on
// the tensor cores. Needs L >= 16 and a block of whole warps (C L / 16 >= 32 threads).
template <int LOG_L, int LOG_C, int LM>
__device__ __forceinline__ void tile_fft_tc(float2 (&v)[16], int j, const float2* __restrict__ stw, float2* smem,
                                            int cofs, int tid) {
    using St = Stages<LOG_L>;
    DftFrags F;
    make_dft_frags(F, tid & 31);
    {
        float2* w = smem + spad(j * LM + cofs);
#pragma unroll
        for (int k = 0; k < 16; ++k) w[padc(k * St::T * LM)] = v[k];
    }
    __syncthreads();
    tc_stages<LOG_L, LOG_C, LM, 0>(smem, stw, F, tid);
    {
        const float2* r = smem + spad(j * LM + cofs);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = r[padc(k * St::T * LM)];
    }
    __syncthreads();
    if constexpr (St::REM != 0) stage_compute<LOG_L, St::COUNT - 1>(v, j, stw);
}

}  // namespace ofb
