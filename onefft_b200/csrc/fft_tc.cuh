// Split-BF16 tensor-core variants of the Stockham tile engine.
//
// Every radix-16 stage runs as a dense complex matrix product Y = F16 X on the tensor cores:
// 8 butterflies form the 16x8 operand X of one mma.sync m16n8k16 (bf16 in, FP32 accumulate).
// TERMS = 3: each FP32 value v is split into hi = bf16(v) and lo = bf16(v - hi), and the product
// keeps the three terms F_hi X_hi + F_hi X_lo + F_lo X_hi (the dropped F_lo X_lo is ~2^-16
// relative): 12 MMAs per 8 butterflies. TERMS = 6: three parts hi = bf16(v), mid = bf16(v - hi),
// lo = bf16(v - hi - mid) (24 significant bits, an FP32 value almost exactly), and the six terms
// of order up to 2^-16 (hh; hm, mh; hl, lh, mm), dropping those of 2^-24 and below, FP32's own
// rounding level: 24 MMAs per 8 butterflies. Terms are accumulated smallest first. Twiddles
// before a stage and the last radix-2/4/8 stage (when log2 L is not a multiple of 4) stay in
// FP32. Either variant is measured against the FP32 path's error bound and accepted only where
// it meets it.
#pragma once

#include <cuda_bf16.h>

#include "fft_device.cuh"

namespace ofb {

__device__ __forceinline__ unsigned pack_bf16(float lo_elem, float hi_elem) {
    __nv_bfloat162 p = __floats2bfloat162_rn(lo_elem, hi_elem);
    return *reinterpret_cast<unsigned*>(&p);
}

// v ~ sum of P bf16 parts: part 0 = bf16(v), part i = bf16(v - parts before it), each difference
// exact in FP32.
template <int P>
__device__ __forceinline__ void split_bf16(float v, float (&part)[P]) {
#pragma unroll
    for (int i = 0; i < P; ++i) {
        part[i] = __bfloat162float(__float2bfloat16_rn(v));
        v -= part[i];
    }
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Parts per value of a variant: 2 for three terms, 3 for six.
template <int TERMS>
constexpr int kParts = TERMS == 6 ? 3 : 2;

// A fragments of F16[p][q] = w_16^(p q) split in bf16 parts: real, imaginary and negated
// imaginary parts. Lane l holds rows g = l/4, g+8 and columns 2t, 2t+1, 2t+8, 2t+9 (t = l%4) in the
// m16n8k16 row-major layout.
template <int TERMS>
struct DftFrags {
    unsigned re[kParts<TERMS>][4], im[kParts<TERMS>][4], nim[kParts<TERMS>][4];
};

__device__ __forceinline__ float2 w16(int k) {
    // w_16^k from exact constants (no libm), k mod 16
    const float c1 = kC8, s1 = kS8, r = kR2;
    const float cs[16] = {1.f, c1, r, s1, 0.f, -s1, -r, -c1, -1.f, -c1, -r, -s1, 0.f, s1, r, c1};
    const float sn[16] = {0.f, s1, r, c1, 1.f, c1, r, s1, 0.f, -s1, -r, -c1, -1.f, -c1, -r, -s1};
    k &= 15;
    return make_float2(cs[k], -sn[k]);
}

template <int TERMS>
__device__ __forceinline__ void make_dft_frags(DftFrags<TERMS>& f, int lane) {
    constexpr int P = kParts<TERMS>;
    const int g = lane >> 2, t = lane & 3;
    const int rows[4] = {g, g + 8, g, g + 8};
    const int cols[4] = {2 * t, 2 * t, 2 * t + 8, 2 * t + 8};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float2 w0 = w16(rows[i] * cols[i]), w1 = w16(rows[i] * (cols[i] + 1));
        float r0[P], r1[P], i0[P], i1[P];
        split_bf16<P>(w0.x, r0);
        split_bf16<P>(w1.x, r1);
        split_bf16<P>(w0.y, i0);
        split_bf16<P>(w1.y, i1);
#pragma unroll
        for (int k = 0; k < P; ++k) {
            f.re[k][i] = pack_bf16(r0[k], r1[k]);
            f.im[k][i] = pack_bf16(i0[k], i1[k]);
            f.nim[k][i] = pack_bf16(-i0[k], -i1[k]);
        }
    }
}

// Yr += Fr Xr - Fi Xi and Yi += Fi Xr + Fr Xi with the variant's split terms, smallest first;
// xr[k] / xi[k] hold part k of the B fragment (two registers).
template <int TERMS>
__device__ __forceinline__ void tc_products(float (&Dr)[4], float (&Di)[4], const DftFrags<TERMS>& F,
                                            const unsigned (&xr)[kParts<TERMS>][2],
                                            const unsigned (&xi)[kParts<TERMS>][2]) {
#define OFB_TERM(D, FR, X, a, b) mma_bf16(D, F.FR[a], X[b][0], X[b][1])
    if constexpr (TERMS == 3) {
        OFB_TERM(Dr, re, xr, 1, 0); OFB_TERM(Dr, re, xr, 0, 1);
        OFB_TERM(Dr, nim, xi, 1, 0); OFB_TERM(Dr, nim, xi, 0, 1);
        OFB_TERM(Dr, re, xr, 0, 0); OFB_TERM(Dr, nim, xi, 0, 0);
        OFB_TERM(Di, im, xr, 1, 0); OFB_TERM(Di, im, xr, 0, 1);
        OFB_TERM(Di, re, xi, 1, 0); OFB_TERM(Di, re, xi, 0, 1);
        OFB_TERM(Di, im, xr, 0, 0); OFB_TERM(Di, re, xi, 0, 0);
    } else {
        // order 2^-16: lo hi, hi lo, mid mid
        OFB_TERM(Dr, re, xr, 2, 0); OFB_TERM(Dr, re, xr, 0, 2); OFB_TERM(Dr, re, xr, 1, 1);
        OFB_TERM(Dr, nim, xi, 2, 0); OFB_TERM(Dr, nim, xi, 0, 2); OFB_TERM(Dr, nim, xi, 1, 1);
        OFB_TERM(Di, im, xr, 2, 0); OFB_TERM(Di, im, xr, 0, 2); OFB_TERM(Di, im, xr, 1, 1);
        OFB_TERM(Di, re, xi, 2, 0); OFB_TERM(Di, re, xi, 0, 2); OFB_TERM(Di, re, xi, 1, 1);
        // order 2^-8: mid hi, hi mid
        OFB_TERM(Dr, re, xr, 1, 0); OFB_TERM(Dr, re, xr, 0, 1);
        OFB_TERM(Dr, nim, xi, 1, 0); OFB_TERM(Dr, nim, xi, 0, 1);
        OFB_TERM(Di, im, xr, 1, 0); OFB_TERM(Di, im, xr, 0, 1);
        OFB_TERM(Di, re, xi, 1, 0); OFB_TERM(Di, re, xi, 0, 1);
        // hi hi
        OFB_TERM(Dr, re, xr, 0, 0); OFB_TERM(Dr, nim, xi, 0, 0);
        OFB_TERM(Di, im, xr, 0, 0); OFB_TERM(Di, re, xi, 0, 0);
    }
#undef OFB_TERM
}

// One radix-16 stage S of a tile on the tensor cores, shared memory to shared memory.
// Butterfly beta (0 .. THREADS-1) is column c / lane j of the plain engine's thread beta:
// COL (LM = C): c = beta mod C, b = beta / C; ROW (LM = 1): b = beta mod T, c = beta / T.
// Element e of column c lives at slot spad(e LM + cofs(c)).
template <int LOG_L, int LOG_C, int LM, int S, int TERMS>
__device__ __forceinline__ void tc_stage(float2* smem, const float2* __restrict__ stw, const DftFrags<TERMS>& F,
                                         int tid) {
    constexpr int P = kParts<TERMS>;
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
        float xr_part[4][P], xi_part[4][P];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float2 x = smem[spad((b + qs[i] * T) * LM + cofs)];
            if (S > 0) {
                const int r = b & (NS - 1);
                if (qs[i] > 0) x = cmul(x, __ldg(stw + St::tw_offset(S) + (qs[i] - 1) * NS + r));
            }
            split_bf16<P>(x.x, xr_part[i]);
            split_bf16<P>(x.y, xi_part[i]);
        }
        unsigned xr[P][2], xi[P][2];
#pragma unroll
        for (int k = 0; k < P; ++k) {
            xr[k][0] = pack_bf16(xr_part[0][k], xr_part[1][k]);
            xr[k][1] = pack_bf16(xr_part[2][k], xr_part[3][k]);
            xi[k][0] = pack_bf16(xi_part[0][k], xi_part[1][k]);
            xi[k][1] = pack_bf16(xi_part[2][k], xi_part[3][k]);
        }
        float (&Dr)[4] = acc_r[grp];
        float (&Di)[4] = acc_i[grp];
#pragma unroll
        for (int i = 0; i < 4; ++i) Dr[i] = Di[i] = 0.f;
        tc_products<TERMS>(Dr, Di, F, xr, xi);
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

template <int LOG_L, int LOG_C, int LM, int S, int TERMS>
__device__ __forceinline__ void tc_stages(float2* smem, const float2* __restrict__ stw, const DftFrags<TERMS>& F,
                                          int tid) {
    if constexpr (S < Stages<LOG_L>::N16) {
        tc_stage<LOG_L, LOG_C, LM, S, TERMS>(smem, stw, F, tid);
        tc_stages<LOG_L, LOG_C, LM, S + 1, TERMS>(smem, stw, F, tid);
    }
}

// Same contract as tile_fft (v[k] = X[j + T k] in, Y[j + T k] out) with the radix-16 stages on
// the tensor cores, TERMS split products each. Needs L >= 16 and a block of whole warps
// (C L / 16 >= 32 threads).
template <int LOG_L, int LOG_C, int LM, int TERMS>
__device__ __forceinline__ void tile_fft_tc(float2 (&v)[16], int j, const float2* __restrict__ stw, float2* smem,
                                            int cofs, int tid) {
    using St = Stages<LOG_L>;
    DftFrags<TERMS> F;
    make_dft_frags<TERMS>(F, tid & 31);
    {
        float2* w = smem + spad(j * LM + cofs);
#pragma unroll
        for (int k = 0; k < 16; ++k) w[padc(k * St::T * LM)] = v[k];
    }
    __syncthreads();
    tc_stages<LOG_L, LOG_C, LM, 0, TERMS>(smem, stw, F, tid);
    {
        const float2* r = smem + spad(j * LM + cofs);
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = r[padc(k * St::T * LM)];
    }
    __syncthreads();
    if constexpr (St::REM != 0) stage_compute<LOG_L, St::COUNT - 1>(v, j, stw);
}

}  // namespace ofb
