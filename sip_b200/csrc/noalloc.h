// C2C execution with scratch in a static device array (noalloc.cu).
#pragma once

#include <cstddef>

#include "plan.h"

namespace sipfft {

// Static scratch per device: the intermediate of two-pass (four-step) plans,
// at most 32 MiB, i.e. batch x length <= 4,194,304 complex points.
constexpr size_t kNaScratchBytes = size_t(32) << 20;

enum : int { kNaOk = 0, kNaInternal = 1 };

// Runs every step of a validated plan (FP32 C2C, device tables ready,
// workspace need <= kNaScratchBytes) on the plan's stream and the current
// device, with the static scratch in place of the workspace.  Returns kNaOk
// or kNaInternal (message on stderr).
int noalloc_exec(const FftPlan& p, const void* in, void* out);

}  // namespace sipfft
