/*
 * Extensions of the B200 FFT C ABI beyond the reference's fft_api.h.
 * None of these has a counterpart in the reference; they exist for
 * bindings that do not build aclTensor descriptors and for tooling.
 */
#ifndef SIP_B200_FFT_EXT_H
#define SIP_B200_FFT_EXT_H

#include <cstddef>

#include "fft_api.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Executes a planned handle on raw device pointers laid out as the
 * reference's tensors would be (contiguous, batch outermost).  Performs
 * every check of asdFftExecC2C/R2C/C2R except the tensor shape match. */
AsdSip::AspbStatus sipFftExecRaw(AsdSip::asdFftHandle handle, const void* input, void* output);

/* Writes a JSON description of the plan's kernel steps into buf (always
 * NUL-terminated when cap > 0) and the full length + 1 into *needed. */
AsdSip::AspbStatus sipFftDescribePlan(AsdSip::asdFftHandle handle, char* buf, size_t cap, size_t* needed);

/* Library version string. */
const char* sipFftVersion(void);

#ifdef __cplusplus
}
#endif

#endif
