#pragma once
// Shared-memory tile FFT kernels for sm_100a.
//
// One CTA takes one tile (P transforms of length N, see tile_io.cuh):
// coalesced global loads (16-byte vectors on contiguous tiles) into a
// padded shared-memory tile, all Stockham passes in shared memory with
// the butterflies in registers, and a coalesced store that fuses the
// real-transform post-process, the four-step cross twiddle, scaling and
// conjugation.  Each input value is read from HBM once and each output
// value written once, so the kernel is bounded by HBM bandwidth.
#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "tile_io.cuh"
#include "tile_launch.h"

namespace sipfft {

// The shared tile of every tile kernel.
extern __shared__ float2 sip_tile_smem[];

// One Stockham pass.  Kept out of line so that each radix gets its own
// register allocation instead of one allocation for the union of all
// radices of the dispatch switch.
template <int R, int SIGN, int S>
__device__ __noinline__ void gpu_pass(int tid, int T, int P, int N, int LD, const PassDesc pd,
                                      const float2* __restrict__ tw) {
    PassRegs<R, S> rg;
    pass_read<R, SIGN, S>(tid, T, P, N, sip_tile_smem, LD, pd, tw, rg);
    __syncthreads();
    pass_write<R, S>(tid, T, P, sip_tile_smem, LD, pd, rg);
    __syncthreads();
}

template <int SIGN, int E>
__device__ __forceinline__ void run_passes(int tid, int T, const TileArgs& a) {
    const PlanDev* plan = a.plan;
    const int npass = plan->npass;
    for (int i = 0; i < npass; ++i) {
        const PassDesc pd = plan->pass[i];
        switch (pd.R) {
#define SIP_PASS_CASE(R)                                                       \
    case R:                                                                    \
        if constexpr (R < 2 * E)                                               \
            gpu_pass<R, SIGN, cdiv(E, R)>(tid, T, a.P, a.N, a.LD, pd, a.tw);   \
        break;
            SIP_FFT_FOR_EACH_RADIX(SIP_PASS_CASE)
#undef SIP_PASS_CASE
            default:
                break;
        }
    }
}

// One tile of the generic kernel (also the work unit of the batch queue,
// queue.cu).  T is the block size; any T >= P N / E works.
template <int SIGN, int E, int OP, bool TW4>
__device__ __forceinline__ void tile_body(const TileArgs& a, int tile, int tid, int T) {
    float2* sm = sip_tile_smem;
    const TileCtx c = decode_tile(a, tile);
    if constexpr (OP == OP_C2C || OP == OP_PC) {
        load_c2c(tid, T, a, c, sm);
    } else if constexpr (OP == OP_R2C_HALF) {
        load_r2c_half(tid, T, a, c, sm);
    } else if constexpr (OP == OP_C2R_HALF) {
        load_c2r_half(tid, T, a, c, sm);
        __syncthreads();
        prep_c2r_half(tid, T, a, c, sm);
    } else if constexpr (OP == OP_R2C_PAIR) {
        load_r2c_pair(tid, T, a, c, sm);
    } else {
        load_c2r_pair(tid, T, a, c, sm);
    }
    __syncthreads();
    if constexpr (OP == OP_PC) {
        // forward FFT, filter, inverse FFT, all in shared memory
        run_passes<-1, E>(tid, T, a);
        mul_tile(tid, T, a, c, sm);
        __syncthreads();
        run_passes<1, E>(tid, T, a);
    } else {
        run_passes<SIGN, E>(tid, T, a);
    }
    if constexpr (OP == OP_C2C || OP == OP_PC) {
        store_c2c<SIGN, TW4>(tid, T, a, c, sm);
    } else if constexpr (OP == OP_R2C_HALF) {
        store_r2c_half(tid, T, a, c, sm);
    } else if constexpr (OP == OP_C2R_HALF) {
        store_c2r_half(tid, T, a, c, sm);
    } else if constexpr (OP == OP_R2C_PAIR) {
        store_r2c_pair(tid, T, a, c, sm);
    } else {
        store_c2r_pair(tid, T, a, c, sm);
    }
    __syncthreads();
}

template <int SIGN, int E, int OP, bool TW4>
__global__ void __launch_bounds__(kMaxTileThreads, 1) tile_fft_kernel(const TileArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x)
        tile_body<SIGN, E, OP, TW4>(a, tile, threadIdx.x, blockDim.x);
}

}  // namespace sipfft
