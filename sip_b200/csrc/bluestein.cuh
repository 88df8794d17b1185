// Bluestein's algorithm for lengths the radix passes cannot factor (a prime
// factor above 32): the DFT of length n becomes a cyclic convolution of
// length m >= 2n - 1 (m 2,3,5-smooth), run as the fused pulse-compression
// passes (OP_PC), between an element-wise pre pass and post pass:
//   c_j = exp(s i pi (j^2 mod 2n) / n)        (s = -1 forward, +1 inverse)
//   a_j = x_j c_j (j < n), 0 (n <= j < m)
//   y   = IFFT_m(FFT_m(a) . FFT_m(b)) / m,   b_j = conj(c_j), b_{m-j} = b_j
//   X_k = c_k y_k                              (k < n)
// since exp(s 2 pi i j k / n) = c_j c_k conj(c_{k-j}).  Odd-length R2C and
// C2R run the complex transform: the pre pass promotes real input, or
// expands a half spectrum to its Hermitian full length; the post pass keeps
// n/2 + 1 bins, or the real part.  Even real lengths run the half-length
// complex transform through Bluestein instead (the planner's real pre /
// post passes around a BLUE_C2C of n/2).  (Reference: the large-prime routes of
// core/fft/fft_api.cpp:84-132 send such lengths to a cube-tail / DFT core.)
#pragma once

#include "fft_core.cuh"

namespace sipfft {

enum BlueKind : int { BLUE_C2C = 0, BLUE_R2C = 1, BLUE_C2R = 2 };

struct BluesteinArgs {
    const void* src;
    void* dst;
    const float2* chirp;  // c_j, j < n
    long long n, m;       // transform and convolution lengths
    long long rows;
    long long in_pitch;   // input row pitch (float2 units; floats for R2C input)
    long long out_pitch;  // output row pitch (float2 units; floats for C2R output)
    int kind;             // BlueKind
    float scale = 1.0f;   // factor on the post pass's outputs
};

// Pre pass value a_j of row `row` (j < m).
SIP_HD float2 blue_pre_elem(const BluesteinArgs& a, long long row, long long j) {
    if (j >= a.n) return make_float2(0.f, 0.f);
    float2 x;
    if (a.kind == BLUE_C2C) {
        x = SIP_LDG(static_cast<const float2*>(a.src) + row * a.in_pitch + j);
    } else if (a.kind == BLUE_R2C) {
        x = make_float2(SIP_LDG(static_cast<const float*>(a.src) + row * a.in_pitch + j), 0.f);
    } else {
        // Hermitian extension of the half spectrum X[0..n/2]
        const float2* h = static_cast<const float2*>(a.src) + row * a.in_pitch;
        const long long half = a.n / 2;
        if (j <= half) {
            x = SIP_LDG(h + j);
            if (j == 0 || (2 * j == a.n)) x.y = 0.f;
        } else {
            const float2 v = SIP_LDG(h + (a.n - j));
            x = make_float2(v.x, -v.y);
        }
    }
    return c_mul(x, SIP_LDG(a.chirp + j));
}

// Post pass: output k of row `row` from the convolution row y (m values).
SIP_HD void blue_post_elem(const BluesteinArgs& a, long long row, long long k) {
    const float2* y = static_cast<const float2*>(a.src) + row * a.m;
    float2 v = c_mul(SIP_LDG(y + k), SIP_LDG(a.chirp + k));
    if (a.scale != 1.0f) v = c_scale(v, a.scale);
    if (a.kind == BLUE_C2R)
        static_cast<float*>(a.dst)[row * a.out_pitch + k] = v.x;
    else
        static_cast<float2*>(a.dst)[row * a.out_pitch + k] = v;
}

// Outputs per row of the post pass.
SIP_HD long long blue_out_count(const BluesteinArgs& a) { return a.kind == BLUE_R2C ? a.n / 2 + 1 : a.n; }

}  // namespace sipfft
