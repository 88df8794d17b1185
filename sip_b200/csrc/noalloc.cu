// C2C execution whose scratch lives in a fixed device array of this file
// instead of a caller-bound workspace (sipFftExecC2CNoAlloc, api.cpp).
//
// Some callers cannot allocate device memory at the point where they run a
// transform: a real-time signal chain in which a cudaMalloc or cudaFree
// would synchronise the device and stall its other streams, or a host whose
// GPU memory is already handed out by another framework's pool or reserved
// up front under a fixed budget.  For them this path runs the passes of a
// planned C2C transform (the same kernels as the ordinary exec) with the
// four-step intermediate in `g_na_scratch`, a static device array that the
// CUDA runtime reserves on every GPU that loads the library and keeps until
// the process exits, in place of the bound workspace.  The plan's twiddle
// tables were made with the plan.  The path calls no cudaMalloc, cudaFree or
// other allocating routine.
//
// In host code `g_na_scratch` only stands in for the device array; its
// device address comes from cudaGetSymbolAddress, looked up once per device
// by the first call on that device, with that device current.  That lookup
// may load the module, so the first call on a device should come before any
// stream capture.  The array keeps whatever the last call left in it, and
// nothing in it has to start at zero: the first pass writes every element of
// the intermediate before the second pass reads it, so no clearing is done.
// All calls share the one array per device, so calls whose kernels overlap
// on the GPU (streams not ordered against each other, or several host
// threads) race; order them, for example by issuing them on one stream.
#include <cuda_runtime.h>

#include <cstdio>
#include <exception>

#include "noalloc.h"

namespace sipfft {

namespace {

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

constexpr int kNaMaxDevices = 64;

// Device address of g_na_scratch per device (null until the first call).
void* g_na_base[kNaMaxDevices] = {};

}  // namespace

int noalloc_exec(const FftPlan& p, const void* in, void* out) {
    int device = -1;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess || device < 0 || device >= kNaMaxDevices) {
        std::fprintf(stderr, "[sip_b200] no-alloc exec: no usable current device (%s)\n", cudaGetErrorString(e));
        return kNaInternal;
    }
    if (g_na_base[device] == nullptr) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_na_scratch);
        if (e != cudaSuccess || ptr == nullptr) {
            std::fprintf(stderr, "[sip_b200] no-alloc exec: cudaGetSymbolAddress of the static scratch failed: %s\n",
                         cudaGetErrorString(e));
            return kNaInternal;
        }
        g_na_base[device] = ptr;
    }
    try {
        launch_steps(p, in, out, g_na_base[device]);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "[sip_b200] no-alloc exec failed: %s\n", ex.what());
        return kNaInternal;
    }
    return kNaOk;
}

}  // namespace sipfft
