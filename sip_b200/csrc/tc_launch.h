// Host entry points of the tensor-core split-precision kernel (tc_kernel.cu).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "tile_io.cuh"

namespace sipfft {

int tc_smem_bytes();
int tc_tile_transforms();  // transforms of length 256 per tile
int tc_threads();
// Kernel for (sign, cross twiddle, adjacent-column input, adjacent-column output).
const void* tc_kernel(int sign, bool tw4, bool cols_in, bool cols_out);
cudaError_t tc_prepare(const void* fn, int* ctas_per_sm);
cudaError_t tc_launch(const void* fn, int grid, const TileArgs& args, const void* src, void* dst, const uint16_t* bmat,
                      const float2* tw256, cudaStream_t stream);
// Reads and clears the device error word (1 = a bounded wait ran out).
cudaError_t tc_take_error(unsigned* err);

}  // namespace sipfft
