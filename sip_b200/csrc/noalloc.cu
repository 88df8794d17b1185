// C2C execution whose scratch lives in a fixed device array of this file
// instead of a caller-bound workspace (sipFftExecC2CNoAlloc, api.cpp).
//
// Some callers cannot allocate device memory at the point where they run a
// transform: a real-time signal chain in which a cudaMalloc or cudaFree
// would synchronise the device and stall its other streams, or a host whose
// GPU memory is already handed out by another framework's pool or reserved
// up front under a fixed budget.  For them this path runs the passes of a
// planned C2C transform (the same kernels as the ordinary exec) with the
// four-step intermediate in `g_na_scratch`, a static device array of this
// file, in place of the bound workspace.  The path calls no cudaMalloc,
// cudaFree or other allocating routine.
//
// When the array is reserved: CUDA loads modules lazily by default (12.2 and
// later), and this file's module holds no kernel, so the array is reserved
// on a device when its address is first looked up there.  That lookup
// (cudaGetSymbolAddress, with the plan's device current) is done while an
// eligible plan is prepared on its device, i.e. inside MakePlan, which
// allocates the plan's tables anyway; the address is kept in the plan and
// the exec call only reads it.  Once reserved, the array stays until the
// process exits (or the device is reset: cudaDeviceReset invalidates every
// plan made before it, this address included, so make new plans after one).
// MakePlan should therefore come before any stream capture; the exec call
// itself does no set-up.
//
// In host code `g_na_scratch` only stands in for the device array; its
// device address is the one cudaGetSymbolAddress returns.  The array keeps
// whatever the last call left in it, and nothing in it has to start at zero:
// the first pass writes every element of the intermediate before the second
// pass reads it, so no clearing is done.  All calls share the one array per
// device, so calls whose kernels overlap on the GPU (streams not ordered
// against each other, or several host threads) race; order them, for
// example by issuing them on one stream.
#include <cuda_runtime.h>

#include <cstdio>
#include <exception>

#include "noalloc.h"

namespace sipfft {

namespace {

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

}  // namespace

bool noalloc_eligible(const FftPlan& p) {
    return p.type == AsdSip::ASCEND_FFT_C2C && p.compute_mode == kComputeFp32 && p.workspace_need <= kNaScratchBytes;
}

void noalloc_resolve(FftPlan& p) {
    p.noalloc_scratch = nullptr;
    if (!noalloc_eligible(p)) return;
    void* ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_na_scratch) != cudaSuccess) {
        (void)cudaGetLastError();  // leave no sticky error for the caller's next call
        return;
    }
    p.noalloc_scratch = ptr;
}

int noalloc_exec(const FftPlan& p, const void* in, void* out) {
    if (p.noalloc_scratch == nullptr) {
        std::fprintf(stderr,
                     "[sip_b200] no-alloc exec: the static scratch's device address was not resolved when the plan "
                     "was prepared on its device\n");
        return kNaInternal;
    }
    try {
        launch_steps(p, in, out, p.noalloc_scratch);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "[sip_b200] no-alloc exec failed: %s\n", ex.what());
        return kNaInternal;
    }
    return kNaOk;
}

}  // namespace sipfft
