// Bluestein pre/post passes and tables (bluestein.cu).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "bluestein.cuh"

namespace sipfft {

cudaError_t bluestein_pre(const BluesteinArgs& a, cudaStream_t stream);
cudaError_t bluestein_post(const BluesteinArgs& a, cudaStream_t stream);
// Queries both pass kernels, which loads their module under lazy loading
// (plan time, so that an exec does not load code).
cudaError_t bluestein_prepare();

// Chirp c_j = exp(sign i pi (j^2 mod 2n) / n), j < n (FP64, rounded once).
cudaError_t gen_chirp(float2* out, long long n, int sign, cudaStream_t stream);

// Convolution filter FFT_m(b), b_j = conj(c_j), b_{m-j} = b_j (j < n),
// computed on the host in FP64 and rounded once.
std::vector<float2> bluestein_filter(long long n, long long m, int sign);

// The sequence b itself on the device (FP64 phases rounded once), for
// filters of lengths too long for the host transform (device.cpp runs the
// library's own C2C of length m on it).
cudaError_t gen_blue_b(float2* out, long long n, long long m, int sign, cudaStream_t stream);

// Filters of length m above this are made on the GPU (FP32 transform of the
// FP64-made sequence) instead of by the host's FP64 transform, which takes
// seconds beyond it.
constexpr long long kHostBlueFilterMax = 1LL << 23;

// Smallest 2,3,5-smooth m >= 2n - 1.
long long bluestein_length(long long n);

}  // namespace sipfft
