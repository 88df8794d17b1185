// Registry of the compiled size-specialized tile kernels (sk_configs.h).
#pragma once

#include <vector>

#include "sk_modes.h"

namespace sipfft {

struct SkEntry {
    int n, P, T, op, mode, sign;
    bool tw4;
    bool twb;  // basis pass twiddles (else the full Stockham table)
    int flags = 1;  // the configuration's TWB bits (sk_kernel.cuh SK_TW_BASIS, SK_TW_SMEM, SK_MIRROR_PAIR)
    int stages;
    std::vector<int> radices;
    int LD;
    int smem;        // dynamic shared memory per CTA (bytes)
    const void* fn;  // kernel (library) or CPU runner (test harness)
    int order = 0;   // position in the SIP_SK_CONFIGS list
    int minb = 0;    // CTAs-per-SM register target (__launch_bounds__)
    bool jit = false;  // compiled at run time (jit.cpp); fn is set by sk_jit_load
};

// The `variant`-th entry compiled for (op, mode, sign, tw4, n) in
// SIP_SK_CONFIGS order (0: the default); the default when that variant is
// not compiled; nullptr when no entry is.
const SkEntry* sk_find(int op, int mode, int sign, bool tw4, int n, int variant = 0);

// The first compiled entry for (op, mode, sign, tw4, n) whose TWB bits
// include all of `flags`; nullptr if none.
const SkEntry* sk_find_flags(int op, int mode, int sign, bool tw4, int n, int flags);

// The first compiled variant of `e`'s kernel (same op, mode, sign, tw4, n
// and transforms per tile) with more threads per tile; nullptr if none.
const SkEntry* sk_find_wider(const SkEntry* e);

const std::vector<SkEntry>& sk_registry();

// Run-time specialization (jit.cpp): an entry for a configuration that
// sk_configs.h does not compile, chosen from (op, mode, n, transforms) and
// compiled by NVRTC (loaded when the plan is first prepared on a device).
// Not yet compiled: `sync` compiles it now, else it is compiled in the
// background and nullptr returned (the generic kernel runs this step; plans
// made later get the entry).  nullptr also when no configuration fits or
// NVRTC is not available.
const SkEntry* sk_jit_entry(int op, int mode, int sign, bool tw4, int n, long long transforms, bool sync);
bool sk_jit_available();
// Waits up to timeout_ms for the background compilations; true when none is left.
bool sk_jit_wait(long long timeout_ms);

}  // namespace sipfft
