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
// and Bluestein passes).  SIP_FFT_PDL=0 turns it off.
#pragma once

#include <cuda_runtime.h>

namespace sipfft {

bool pdl_enabled();

// `attr` must outlive the launch call that uses the returned configuration.
inline cudaLaunchConfig_t pdl_config(dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                                     cudaLaunchAttribute* attr) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    attr->id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr->val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cfg;
}

// Launches `fn(args...)` with the attribute (when enabled).
template <typename... Params, typename... Args>
cudaError_t launch_pdl(void (*fn)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args) {
    cudaLaunchAttribute attr;
    cudaLaunchConfig_t cfg = pdl_config(grid, block, smem, stream, &attr);
    return cudaLaunchKernelEx(&cfg, fn, static_cast<Args&&>(args)...);
}

}  // namespace sipfft
