// Launches with programmatic dependent launch (PDL).
//
// A stream runs its kernels one after the other: normally the next kernel
// is launched only once the previous one has completed and its writes are
// flushed, so each small launch pays the launch latency on top of its own
// run time.  With the programmatic-stream-serialization attribute the next
// kernel is launched as soon as every CTA of the previous one has called
// grid_dep_launch() (fft_core.cuh), and its own CTAs wait in
// grid_dep_wait() until the previous kernel has completed: the launch
// overlaps the previous kernel's run, the data dependency is unchanged.
// Only kernels that call grid_dep_wait() before their first global-memory
// access are launched this way (the tile kernels and the element-wise real
// and Bluestein passes), and only small launches: a tile launch whose tiles
// fit one wave (every CTA one tile) or an element-wise pass of at most
// kPdlMaxValues values.  Small steps gain the overlapped launch (C2C 4096 x
// 256: 10.2 -> 8.7 us); persistent launches over many tiles measured 0.6-4 %
// slower with it (R2C 2^20 x 256).  SIP_FFT_PDL=0 turns it off.
#pragma once

#include <cuda_runtime.h>

namespace sipfft {

bool pdl_enabled();

constexpr long long kPdlMaxValues = 1LL << 22;

// `attr` must outlive the launch call that uses the returned configuration;
// `use`: the launch is small enough to gain from the attribute.
inline cudaLaunchConfig_t pdl_config(dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                     cudaLaunchAttribute* attr, bool use = true) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    attr->id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr->val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = use && pdl_enabled() ? 1 : 0;
    return cfg;
}

// Launches `fn(args...)` with the attribute when enabled and `values` (the
// element count the launch processes) is at most kPdlMaxValues.
template <typename... Params, typename... Args>
cudaError_t launch_pdl(void (*fn)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       long long values, Args&&... args) {
    cudaLaunchAttribute attr;
    cudaLaunchConfig_t cfg = pdl_config(grid, block, smem, stream, &attr, values <= kPdlMaxValues);
    return cudaLaunchKernelEx(&cfg, fn, static_cast<Args&&>(args)...);
}

}  // namespace sipfft
