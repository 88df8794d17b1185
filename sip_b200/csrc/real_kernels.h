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

// Element-wise passes of odd real lengths above one tile, where real rows
// 2p and 2p + 1 travel as complex row p (real_math.cuh pair_*_elem).
struct PairPassArgs {
    const void* src;
    void* dst;
    long long n;                    // real length (odd)
    long long rows;                 // real rows (the last pair may hold one)
    long long in_pitch, out_pitch;  // elements per row: float32 for real rows, complex64 otherwise
    int conj;                       // separate: conjugate the bins (R2C inverse); combine: conjugate the
                                    // input spectra (C2R forward)
};
// z[p][j] = x[2p][j] + i x[2p+1][j] (real rows in, complex rows out)
cudaError_t pair_pack(const PairPassArgs& a, cudaStream_t stream);
// bins k <= n/2 of real rows 2p, 2p+1 from complex spectrum row p
cudaError_t pair_separate(const PairPassArgs& a, cudaStream_t stream);
// complex spectrum row p from the half spectra of rows 2p, 2p+1
cudaError_t pair_combine(const PairPassArgs& a, cudaStream_t stream);
// real rows 2p, 2p+1 = Re, Im of complex row p
cudaError_t pair_split(const PairPassArgs& a, cudaStream_t stream);

}  // namespace sipfft
