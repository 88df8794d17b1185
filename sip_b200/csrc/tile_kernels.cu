// Host-side dispatch of the tile kernels compiled in tile_inst.cu.
#include <cuda_runtime.h>

#include <cstdlib>

#include "launch_attr.h"
#include "tile_launch.h"

namespace sipfft {

using KernelFn = void (*)(const TileArgs);

KernelFn tile_pick_fwd_e16(int op, bool tw4);
KernelFn tile_pick_fwd_e32(int op, bool tw4);
KernelFn tile_pick_inv_e16(int op, bool tw4);
KernelFn tile_pick_inv_e32(int op, bool tw4);

namespace {

KernelFn pick_kernel(int sign, int e, int op, bool tw4) {
    if (sign < 0) {
        if (e == 16) return tile_pick_fwd_e16(op, tw4);
        if (e == 32) return tile_pick_fwd_e32(op, tw4);
    } else {
        if (e == 16) return tile_pick_inv_e16(op, tw4);
        if (e == 32) return tile_pick_inv_e32(op, tw4);
    }
    return nullptr;
}

}  // namespace

// The dynamic shared-memory ceiling is an attribute of the kernel function,
// shared by every plan that launches it, so it is raised once to the
// per-block maximum rather than set to one plan's tile size.
cudaError_t tile_prepare(int sign, int e, int op, bool tw4, int smem_bytes) {
    KernelFn fn = pick_kernel(sign, e, op, tw4);
    if (fn == nullptr) return cudaErrorInvalidValue;
    if (smem_bytes > kMaxTileSmem) return cudaErrorInvalidValue;
    return cudaFuncSetAttribute(reinterpret_cast<const void*>(fn), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                kMaxTileSmem);
}

// Read at every launch, so that a process can compare both forms.
bool pdl_enabled() {
    const char* e = std::getenv("SIP_FFT_PDL");
    return e == nullptr || std::atoi(e) != 0;
}

// Both kernel families wait for the previous kernel of the stream before
// touching global memory (grid_dep_wait), so both launch with PDL when the
// launch is one wave of tiles.
cudaError_t tile_launch(const TileLaunch& L, const void* src, void* dst, cudaStream_t stream) {
    TileArgs a = L.args;
    a.src = src;
    a.dst = dst;
    const void* fn = L.sk_fn;
    if (fn == nullptr) fn = reinterpret_cast<const void*>(pick_kernel(L.sign, L.e, L.op, L.tw4));
    if (fn == nullptr) return cudaErrorInvalidValue;
    void* params[] = {&a};
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t cfg =
        pdl_config(dim3(L.grid), dim3(L.block), (size_t)L.smem_bytes, stream, &attr, a.ntiles <= L.grid);
    return cudaLaunchKernelExC(&cfg, fn, params);
}

cudaError_t sk_prepare(const void* fn, int smem_bytes, int block, int* ctas_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, block, (size_t)smem_bytes);
}

const void* tile_kernel_address(int sign, int e, int op, bool tw4) {
    return reinterpret_cast<const void*>(pick_kernel(sign, e, op, tw4));
}

}  // namespace sipfft
