// Element-wise pre/post-processing passes of real transforms whose
// half-length complex FFT is longer than one tile (four-step lengths).
#pragma once

#include <cuda_runtime.h>

namespace sipfft {

struct RealPassArgs {
    const float2* src;
    float2* dst;
    const float2* tw;  // W_N^k, k in [0, m], N = 2m (forward values)
    long long m;       // half length
    long long rows;
    long long in_pitch, out_pitch;  // complex values per row
    int conj;          // post: conjugate the output; pre: conjugate the input
};

// R2C: X[k] = E[k] + W_N^k O[k] from the half-length spectrum Z (rows of m
// values), k in [0, m].
cudaError_t real_post(const RealPassArgs& a, cudaStream_t stream);

// C2R: Z[k] = E[k] + i W_N^{-k} D[k] from the half spectrum X (rows of
// m + 1 values), k in [0, m).
cudaError_t real_pre(const RealPassArgs& a, cudaStream_t stream);

}  // namespace sipfft
