// Host-side description of one tile-kernel launch and the entry points of
// tile_kernels.cu / twiddle.cu.
#pragma once

#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "tile_io.cuh"

namespace sipfft {

constexpr int kMaxTileThreads = 512;
// Opt-in shared memory per block on sm_100 (227 KB).
constexpr int kMaxTileSmem = 227 * 1024;

struct TileLaunch {
    int sign = -1;  // -1 forward, +1 inverse
    int e = 16;     // elements per thread (compiled variants: 16, 32)
    int op = OP_C2C;
    bool tw4 = false;
    int grid = 0;
    int block = 0;
    int smem_bytes = 0;
    const void* sk_fn = nullptr;  // size-specialized kernel (sk_configs.h), else the generic one
    TileArgs args{};  // src / dst are bound per exec
};

// Sets the dynamic shared-memory limit of the selected instantiation.
cudaError_t tile_prepare(int sign, int e, int op, bool tw4, int smem_bytes);

cudaError_t tile_launch(const TileLaunch& L, const void* src, void* dst, cudaStream_t stream);

// Raises the shared-memory limits of a size-specialized kernel and reports
// how many of its CTAs fit on one SM.
cudaError_t sk_prepare(const void* fn, int smem_bytes, int block, int* ctas_per_sm);

const void* tile_kernel_address(int sign, int e, int op, bool tw4);

// Twiddle tables, generated on the device in FP64 (sincospi) and rounded
// once to FP32.  All tables hold forward values exp(-2 pi i m / n).

// Stockham table for the pass list of `plan` (entries plan.N - 1 at most).
cudaError_t gen_stockham_twiddles(float2* out, const PlanDev& plan, int entries, cudaStream_t stream);

// Basis table of the size-specialized kernels (entries: basis_entries).
int basis_entries(const PlanDev& plan);
cudaError_t gen_basis_twiddles(float2* out, const PlanDev& plan, cudaStream_t stream);

// Split cross-twiddle table of four-step passes (tile_io.cuh cross_tw).
cudaError_t gen_split_twiddles(float2* out, long long n, int shift, cudaStream_t stream);

// out[k] = exp(-2 pi i k / n), k in [0, count).
cudaError_t gen_root_twiddles(float2* out, long long n, long long count, cudaStream_t stream);

}  // namespace sipfft
