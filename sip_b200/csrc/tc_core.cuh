// Tensor-core split-precision DFT stages ("tc" form).
//
// A length-256 transform is computed as 16 x 16: stage 1 runs 16-point DFTs
// over n2 for every n1 (x[n1 + 16 n2]), multiplies by W_256^{n1 k2}, stage 2
// runs 16-point DFTs over n1 for every k2, giving X[k2 + 16 k1].  Each
// stage is one real-embedded GEMM per 128 vectors,
//
//     D[v][o] = sum_i A[v][i] B[i][o],   i, o in [0, 32)
//     A[v] = (re x_0..x_15, im x_0..x_15),  D[v] = (re X_0..X_15, im X_0..X_15)
//     B = [[ Fr, Fi], [-Fi, Fr]],  F[n][k] = exp(SIGN 2 pi i n k / 16),
//
// on the 5th-generation tensor cores (tcgen05.mma kind::f16, BF16 operands,
// FP32 accumulation in tensor memory).  FP32 operands are split into three
// BF16 terms, x = x_hi + x_mid + x_lo (24 significant bits), and the six
// products of order <= 2 (hh, hm, mh, hl, mm, lh) are accumulated, so the
// stage keeps FP32 accuracy; a two-term split loses about 2^-16.
//
// Shared-memory operand layout (no swizzle, K-major): 8-row x 16-byte core
// matrices; core (i, j) (rows 8i.., K columns 8j..) at byte (i * KC + j) * 128
// with KC = 32 / 8 = 4 core matrices along K.  The leading-dimension byte
// offset (next core along K) is 128 and the stride-dimension byte offset
// (next 8-row group) is 512.
//
// Everything here is __host__ __device__ so the CPU harness can run the
// same layouts with a plain GEMM in place of the tensor cores.
#pragma once

#include <cuda_bf16.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include "fft_core.cuh"
#include "tile_io.cuh"

namespace sipfft {

constexpr int kTcK = 32;             // real-embedded K (and N) of a radix-16 stage
constexpr int kTcRows = 128;         // vectors per MMA (M)
constexpr int kTcTermBytes = kTcRows * kTcK * 2;  // one split term of A: 8 KB
constexpr int kTcBTermBytes = kTcK * kTcK * 2;    // one split term of B: 2 KB

// Byte offset of element (row, k) in a K-major core-matrix operand of 32 K.
SIP_HD constexpr int tc_off(int row, int k) {
    return (((row >> 3) * (kTcK / 8) + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1);
}

SIP_HD uint16_t tc_bf16_bits(float f) {
#if defined(__CUDA_ARCH__)
    return __bfloat16_as_ushort(__float2bfloat16_rn(f));
#else
    // round to nearest even on the float's bit pattern
    uint32_t u;
    memcpy(&u, &f, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return (uint16_t)(u >> 16);  // inf / nan
    const uint32_t lsb = (u >> 16) & 1u;
    u += 0x7fffu + lsb;
    return (uint16_t)(u >> 16);
#endif
}

SIP_HD float tc_bf16_float(uint16_t b) {
    const uint32_t u = (uint32_t)b << 16;
    float f;
#if defined(__CUDA_ARCH__)
    f = __uint_as_float(u);
#else
    memcpy(&f, &u, 4);
#endif
    return f;
}

// x = hi + mid + lo, each a bfloat16.
SIP_HD void tc_split3(float x, uint16_t& hi, uint16_t& mid, uint16_t& lo) {
    hi = tc_bf16_bits(x);
    const float r1 = x - tc_bf16_float(hi);
    mid = tc_bf16_bits(r1);
    const float r2 = r1 - tc_bf16_float(mid);
    lo = tc_bf16_bits(r2);
}

// Writes the three split terms of one 16-point complex vector (row `row` of
// the A operand block).  `a` points at term 0; terms are kTcTermBytes apart.
SIP_HD void tc_put_row(unsigned char* a, int row, const float2 (&x)[16]) {
    uint16_t h[kTcK], m[kTcK], l[kTcK];
#pragma unroll
    for (int n = 0; n < 16; ++n) {
        tc_split3(x[n].x, h[n], m[n], l[n]);
        tc_split3(x[n].y, h[16 + n], m[16 + n], l[16 + n]);
    }
#pragma unroll
    for (int j = 0; j < kTcK / 8; ++j) {
        const int off = tc_off(row, 8 * j);
        uint4 vh, vm, vl;
        vh.x = h[8 * j] | ((uint32_t)h[8 * j + 1] << 16);
        vh.y = h[8 * j + 2] | ((uint32_t)h[8 * j + 3] << 16);
        vh.z = h[8 * j + 4] | ((uint32_t)h[8 * j + 5] << 16);
        vh.w = h[8 * j + 6] | ((uint32_t)h[8 * j + 7] << 16);
        vm.x = m[8 * j] | ((uint32_t)m[8 * j + 1] << 16);
        vm.y = m[8 * j + 2] | ((uint32_t)m[8 * j + 3] << 16);
        vm.z = m[8 * j + 4] | ((uint32_t)m[8 * j + 5] << 16);
        vm.w = m[8 * j + 6] | ((uint32_t)m[8 * j + 7] << 16);
        vl.x = l[8 * j] | ((uint32_t)l[8 * j + 1] << 16);
        vl.y = l[8 * j + 2] | ((uint32_t)l[8 * j + 3] << 16);
        vl.z = l[8 * j + 4] | ((uint32_t)l[8 * j + 5] << 16);
        vl.w = l[8 * j + 6] | ((uint32_t)l[8 * j + 7] << 16);
        *reinterpret_cast<uint4*>(a + off) = vh;
        *reinterpret_cast<uint4*>(a + kTcTermBytes + off) = vm;
        *reinterpret_cast<uint4*>(a + 2 * kTcTermBytes + off) = vl;
    }
}

// The (A term, B term) pairs of the order <= 2 products, smallest first so
// that the FP32 accumulation adds the small terms before the large one.
constexpr int kTcProducts = 6;
SIP_HD constexpr int tc_a_term(int p) { return p == 0 ? 1 : p == 1 ? 2 : p == 2 ? 0 : p == 3 ? 1 : p == 4 ? 0 : 0; }
SIP_HD constexpr int tc_b_term(int p) { return p == 0 ? 1 : p == 1 ? 0 : p == 2 ? 2 : p == 3 ? 0 : p == 4 ? 1 : 0; }

// Host: the three split terms of B (K-major: row = output column o, K = i)
// for a DFT-16 of the given sign, in the core-matrix layout (3 x 2 KB).
inline void tc_make_b(int sign, uint16_t* out /* 3 * 32 * 32 */) {
    const double two_pi = 6.283185307179586476925286766559;
    for (int o = 0; o < kTcK; ++o)
        for (int i = 0; i < kTcK; ++i) {
            const int n = i & 15, k = o & 15;
            const double ang = sign * two_pi * (double)((n * k) % 16) / 16.0;
            const double fr = cos(ang), fi = sin(ang);
            double v;
            if (i < 16) v = o < 16 ? fr : fi;      // re x_n -> re X_k: Fr, -> im X_k: Fi
            else v = o < 16 ? -fi : fr;            // im x_n -> re X_k: -Fi, -> im X_k: Fr
            const uint16_t hb = tc_bf16_bits((float)v);
            const double r1 = v - tc_bf16_float(hb);
            const uint16_t mb = tc_bf16_bits((float)r1);
            const double r2 = r1 - tc_bf16_float(mb);
            const uint16_t lb = tc_bf16_bits((float)r2);
            const int off = tc_off(o, i) / 2;
            out[off] = hb;
            out[kTcK * kTcK + off] = mb;
            out[2 * kTcK * kTcK + off] = lb;
        }
}

// CPU stand-in for one M = 128, N = 32 stage: D = sum over the six products
// of A_term * B_term with K = 32 (used by the test harness only).
inline void tc_gemm_host(const unsigned char* a, const uint16_t* b, float* d /* 128 x 32 */) {
    for (int v = 0; v < kTcRows; ++v)
        for (int o = 0; o < kTcK; ++o) {
            float acc = 0.f;
            for (int p = 0; p < kTcProducts; ++p) {
                const unsigned char* at = a + tc_a_term(p) * kTcTermBytes;
                const uint16_t* bt = b + tc_b_term(p) * kTcK * kTcK;
                for (int i = 0; i < kTcK; ++i) {
                    const uint16_t av = *reinterpret_cast<const uint16_t*>(at + tc_off(v, i));
                    acc += tc_bf16_float(av) * tc_bf16_float(bt[tc_off(o, i) / 2]);
                }
            }
            d[v * kTcK + o] = acc;
        }
}

// ------------------------------------------------ tile phases (kernel + CPU harness)
constexpr int kTcP = 8;              // transforms of length 256 per tile
constexpr int kTcThreads = 128;      // = vectors per stage = MMA M
constexpr int kTcLD = 256 + 16 + 1;  // padded tile row (odd)

// Element n of transform q into the tile (adjacent-column or row input).
template <bool COLS_IN>
SIP_HD void tc_load_tile(int tid, const TileArgs& a, const TileCtx& c, float2* tile) {
    const float2* src = static_cast<const float2*>(a.src);
    const bool cj = (a.flags & TF_CONJ_IN) != 0;
    for (int f = tid; f < kTcP * 256; f += kTcThreads) {
        int q, n;
        if (COLS_IN) {
            n = f / kTcP;
            q = f - n * kTcP;
        } else {
            q = f >> 8;
            n = f & 255;
        }
        float2 v = make_float2(0.f, 0.f);
        if (q < c.cnt) v = maybe_conj(SIP_LDG(src + c.in_base + (long long)q * a.in_idist + (long long)n * a.in_stride), cj);
        tile[q * kTcLD + sidx(n)] = v;
    }
}

// Stage 1 vector of thread tid: (q, n1) = x[n1 + 16 n2], n2 < 16.
SIP_HD void tc_gather1(const float2* tile, int tid, float2 (&x)[16]) {
    const int q = tid >> 4, n1 = tid & 15;
#pragma unroll
    for (int n2 = 0; n2 < 16; ++n2) x[n2] = tile[q * kTcLD + sidx(n1 + 16 * n2)];
}

// Stage 1 result: Y[n1][k2] W_256^{n1 k2} stored at 16 n1 + k2.
template <int SIGN>
SIP_HD void tc_scatter1(float2* tile, int tid, const float (&r)[32], const float2* tw256) {
    const int q = tid >> 4, n1 = tid & 15;
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2)
        tile[q * kTcLD + sidx(16 * n1 + k2)] = c_tw<SIGN>(make_float2(r[k2], r[16 + k2]), SIP_LDG(tw256 + n1 * k2));
}

// Stage 2 vector of thread tid: (q, k2) = Y[16 n1 + k2], n1 < 16.
SIP_HD void tc_gather2(const float2* tile, int tid, float2 (&x)[16]) {
    const int q = tid >> 4, k2 = tid & 15;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) x[n1] = tile[q * kTcLD + sidx(16 * n1 + k2)];
}

// Stage 2 result: X[k2 + 16 k1].
SIP_HD void tc_scatter2(float2* tile, int tid, const float (&r)[32]) {
    const int q = tid >> 4, k2 = tid & 15;
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) tile[q * kTcLD + sidx(k2 + 16 * k1)] = make_float2(r[k1], r[16 + k1]);
}

// Element k of transform q out of the tile, with the four-step cross
// twiddle, scaling and conjugation of the generic kernel.
template <int SIGN, bool TW4, bool COLS_OUT>
SIP_HD void tc_store_tile(int tid, const TileArgs& a, const TileCtx& c, const float2* tile) {
    float2* dst = static_cast<float2*>(a.dst);
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    for (int f = tid; f < kTcP * 256; f += kTcThreads) {
        int q, k;
        if (COLS_OUT) {
            k = f / kTcP;
            q = f - k * kTcP;
        } else {
            q = f >> 8;
            k = f & 255;
        }
        if (q >= c.cnt) continue;
        float2 v = tile[q * kTcLD + sidx(k)];
        if (TW4) v = c_tw<SIGN>(v, cross_tw(a, (long long)(c.i0 + q) * k));
        if (sc) v = c_scale(v, a.scale);
        dst[c.out_base + (long long)q * a.out_idist + (long long)k * a.out_stride] = maybe_conj(v, cj);
    }
}

}  // namespace sipfft
