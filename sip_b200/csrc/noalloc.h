// C2C execution with scratch in a static device array (noalloc.cu).
#pragma once

#include <cstddef>

#include "plan.h"

namespace sipfft {

// Static scratch per device: the intermediate of two-pass (four-step) plans,
// at most 32 MiB, i.e. batch x length <= 4,194,304 complex points.
constexpr size_t kNaScratchBytes = size_t(32) << 20;

enum : int { kNaOk = 0, kNaInternal = 1 };

// Whether a plan can run through noalloc_exec (FP32 C2C, workspace need
// within the static array).
bool noalloc_eligible(const FftPlan& p);

// Resolves the static array's device address on the current device into
// p.noalloc_scratch (cudaGetSymbolAddress).  Called while an eligible plan
// is prepared on its device, which is where the module holding the array is
// loaded and the array reserved under lazy module loading, so that the exec
// call itself neither loads nor reserves anything.  Leaves the address null
// (and the no-alloc exec then fails with a message) if the lookup fails.
void noalloc_resolve(FftPlan& p);

// Runs every step of a validated plan (device tables ready, scratch address
// resolved) on the plan's stream and the current device, with the static
// scratch in place of the workspace.  Returns kNaOk or kNaInternal (message
// on stderr).
int noalloc_exec(const FftPlan& p, const void* in, void* out);

}  // namespace sipfft
