// Batched 2-D fftshift / ifftshift kernel (shift.cu).
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"

namespace sipfft {

struct ShiftArgs {
    long long batch = 0, dist = 0;  // slices and the input distance between them (elements)
    int row = 0, col = 0;
    int sr = 0, sc = 0;             // row / column rotation of the output
    float scale = 1.0f;
    FastDiv div_per_row{}, div_row{};  // filled by shift_launch
};

cudaError_t shift_launch(const void* in, void* out, const ShiftArgs& a, cudaStream_t stream);

}  // namespace sipfft
