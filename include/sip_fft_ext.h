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

/* Compute form of the next MakePlan on this handle (call after Create, before
 * MakePlan):
 *   SIP_FFT_COMPUTE_FP32     0  FP32 Stockham passes (default; the drop-in path)
 *   SIP_FFT_COMPUTE_TC_SPLIT 1  passes of length 256 run as two radix-16
 *                               DFT-matrix GEMM stages on the tensor cores, BF16
 *                               operands split in three terms (hi + mid + lo),
 *                               FP32 accumulation; other passes stay FP32.
 * Returns INVALID_PARAM for an unknown mode or an already planned handle. */
#define SIP_FFT_COMPUTE_FP32 0
#define SIP_FFT_COMPUTE_TC_SPLIT 1
AsdSip::AspbStatus sipFftSetComputeMode(AsdSip::asdFftHandle handle, int mode);

/* Reads and clears the device error word: bit 0 = a tensor-core kernel's
 * bounded wait ran out (its results are invalid).  0 after a clean run. */
AsdSip::AspbStatus sipFftTakeDeviceErrors(unsigned* errors);

/* Library version string. */
const char* sipFftVersion(void);

#ifdef __cplusplus
}
#endif

#endif
