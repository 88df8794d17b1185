// Run-time specialization of the size-specialized tile kernels.
//
// sk_configs.h compiles sk kernels for a fixed list of lengths; every other
// length would run on the generic tile kernel, whose pass loop dispatches
// on the radix at run time.  For those lengths the planner can instead
// pick an sk configuration here (radices, transforms per tile, threads,
// stages, register target) and have NVRTC compile sk_fft_kernel<that
// configuration> from the library's own kernel headers, embedded in the
// library at build time.  Compilation happens once per configuration and
// process, and the cubin is kept in an on-disk cache (SIP_FFT_JIT_CACHE, default
// $HOME/.cache/sip_fft_jit) keyed by a hash of the source, the headers, the
// options and the NVRTC version.  The configuration is chosen and compiled
// when the plan is made (CPU work; the compiler's register report rejects
// configurations that spill) and loaded when the plan is first prepared on
// a device.  NVRTC is loaded with dlopen; without it no run-time entry is
// offered and the generic kernel runs.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "sk_registry.h"

namespace sipfft {

struct JitCfg {
    int op = 0, mode = 0, sign = -1;
    bool tw4 = false;
    int n = 0, P = 1, T = 32, stages = 2, minb = 1;
    std::vector<int> radices;
    int LD = 0, smem = 0;
    int twb = 1;  // SkCfg TWB bits: SK_TW_BASIS (else the full Stockham table), SK_TW_SMEM, SK_MIRROR_PAIR
};

// Host-side configuration for at most `values` values per thread and pass
// (0: SIP_FFT_JIT_E or 32), with the radices in the given order (null: the
// cheapest factorization, largest radix first); no CUDA or NVRTC calls.
bool sk_jit_choose(int op, int mode, int sign, bool tw4, int n, long long transforms, JitCfg* out, int values = 0,
                   const std::vector<int>* order = nullptr);

// The configuration the planner uses: candidates of sk_jit_choose compiled
// in turn (32, 16, 48 values per thread) until one has no register spills
// (else the fewest spilled bytes).  Compiles on the CPU; false with a
// message when nothing compiles.
bool sk_jit_select(int op, int mode, int sign, bool tw4, int n, long long transforms, JitCfg* out,
                   std::string* err);

// The NVRTC source and the kernel's name expression for a configuration.
std::string sk_jit_source();
std::string sk_jit_name_expr(const JitCfg& c);

// Compiles a configuration to a cubin (through the process and disk
// caches) with its spilled bytes; returns false with the compiler log in
// *err on failure.
bool sk_jit_compile(const JitCfg& c, std::vector<char>* cubin, std::string* lowered, std::string* err, int* spill);

// Compiles and loads the kernel of a run-time entry (from sk_jit_entry)
// and stores it in the entry; returns the kernel.  Throws PlanError when
// compilation or loading fails.
const void* sk_jit_load(const SkEntry* e);

}  // namespace sipfft
