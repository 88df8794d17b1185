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

/* Executes a planned 1-D or pulse-compression handle on its first `rows`
 * transforms only (1 <= rows <= the plan's batch), with the intermediate in
 * `workspace` when it is not NULL (at least the plan's workspace size; NULL:
 * the bound workspace, under the usual workspace protocol).  Lets a caller
 * keep one resident plan per length and run requests of any smaller batch
 * through it (the serving loop does).  API_NOT_SUPPORT for multi-D plans and
 * plans with steps that cannot be limited to rows (Bluestein lengths, odd
 * real lengths above one tile, the cluster and tensor-core forms). */
AsdSip::AspbStatus sipFftExecRawRows(AsdSip::asdFftHandle handle, long long rows, const void* input, void* output,
                                     void* workspace);

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

/* Planner hints for the next MakePlan on this handle (after Create, before
 * MakePlan); 0 restores the planner default.  Explicit hints disable the
 * tune cache (file named by the SIP_FFT_TUNE_CACHE environment variable,
 * written by sip_b200.autotune).  */
#define SIP_FFT_HINT_TILE_TRANSFORMS 1  /* transforms per tile */
#define SIP_FFT_HINT_ELEMS_PER_THREAD 2 /* 16 or 32 */
#define SIP_FFT_HINT_GENERIC_ONLY 3     /* 1: runtime-radix tile kernels only */
#define SIP_FFT_HINT_RADIX_ORDER 4      /* 0: descending radices, 1: ascending */
#define SIP_FFT_HINT_REAL_FUSED 5       /* real lengths above one tile: 0 default (R2C fused,
                                           C2R pre-process pass), 1 fuse both, 2 fuse neither */
#define SIP_FFT_HINT_SK_VARIANT 6       /* which compiled size-specialized kernel variant: -1
                                           (default) automatic (the first, or for a row step of
                                           less than one wave of tiles the variant with more
                                           threads per tile where one is compiled); 0..15 that
                                           variant (a step without it uses its first) */
#define SIP_FFT_HINT_RUNTIME_COMPILE 7  /* steps of a length without a compiled size-specialized
                                           kernel: 0 default (steps of >= 2^18 values use one compiled
                                           with NVRTC; a configuration not yet compiled is compiled in
                                           the background and this plan runs the generic kernel),
                                           1 always, compiled at MakePlan, 2 never (generic kernel) */
AsdSip::AspbStatus sipFftSetPlanHint(AsdSip::asdFftHandle handle, int key, int value);

/* Waits up to timeout_ms for the run-time kernel compilations started in
 * the background by MakePlan; ACL_SUCCESS when none is left, else
 * ACL_ERROR_INTERNAL_ERROR.  No counterpart in the reference.  */
AsdSip::AspbStatus sipFftJitWait(long long timeout_ms);

/* Compiles (no GPU needed) the run-time specialized kernel the planner
 * would choose for one tile step: op 0 C2C, 1 R2C half-length, 2 C2R
 * half-length, 3 R2C row pairs, 4 C2R row pairs; mode 0 rows, 1 columns,
 * 2 rows in / columns out; sign -1 or +1; tw4 1 for the four-step cross
 * twiddle; n the tile transform length; transforms the step's count.
 * ACL_SUCCESS when it compiled (or was in the cache), ACL_ERROR_API_NOT_SUPPORT
 * when no run-time configuration fits or NVRTC is missing,
 * ACL_ERROR_INTERNAL_ERROR when compilation failed.  No counterpart in the
 * reference (a diagnostic of this library's run-time compiler).  */
AsdSip::AspbStatus sipFftJitCompileCheck(int op, int mode, int sign, int tw4, int n, long long transforms);

/* fftshift / ifftshift fused into the transform's output store (after
 * Create, before MakePlan; C2C 1-D and 2-D plans): mode 1 rotates every
 * output slice as asdFftShift does ((n+1)/2 per axis), mode 2 as
 * asdIfftShift (n/2 per axis), each value times `scale`; mode 0 turns it
 * off.  1-D slices are 1 x N; 2-D slices are X x Y, and the plan then needs
 * a workspace of batch * X * Y * 8 bytes.  Saves the separate shift pass the
 * reference runs (core/fft/fftshift.cpp). */
#define SIP_FFT_SHIFT_NONE 0
#define SIP_FFT_SHIFT_FFTSHIFT 1
#define SIP_FFT_SHIFT_IFFTSHIFT 2
AsdSip::AspbStatus sipFftSetOutputShift(AsdSip::asdFftHandle handle, int mode, double scale);

/* Pulse compression (matched filtering): plans y = IFFT(FFT(x) * F) for
 * `batch` complex64 rows of length n, with F the filter spectrum (n complex64
 * values in device memory, owned by the caller and read at exec time).
 * Execute with asdFftExecC2C or sipFftExecRaw ((batch, n) in and out).  Up to
 * n = 16384 the whole chain is one kernel (one HBM read and write); above it,
 * three passes (forward column pass, fused row FFT-multiply-IFFT pass,
 * inverse column pass) with a workspace of batch * n * 8 bytes.  Flags:
 * SIP_FFT_PULSE_CONJ_FILTER multiplies by conj(F) (F = the spectrum of the
 * transmitted pulse); SIP_FFT_PULSE_SCALE scales by 1/n.  The reference
 * composes this from asdFftExecC2C and asdMul (include/base_api.h). */
#define SIP_FFT_PULSE_CONJ_FILTER 1
#define SIP_FFT_PULSE_SCALE 2
AsdSip::AspbStatus sipFftMakePlanPulse1D(AsdSip::asdFftHandle handle, int64_t n, int64_t batch, const void* filter,
                                         int flags);

/* Batched execution: the passes of many planned handles (generic tile
 * kernels: plan them with SIP_FFT_HINT_GENERIC_ONLY) run in one persistent
 * work-queue launch per pass index, replayed from a captured CUDA graph when
 * the batch's wave structure repeats.  Add binds the operands; Exec enqueues
 * on `stream` (cudaStream_t); Clear empties the batch for reuse.  Exec runs
 * on a non-null stream.  SetGate makes the launch wait for *device_flag != 0
 * (at most poll_limit <= 2^24 polls per CTA, then bit 1 of the status word is
 * set and the launch does no work); TakeStatus reads and clears the status
 * word.  Only plans whose passes are all tile passes are accepted (C2C of any
 * length, real transforms up to one tile per row); others give
 * ACL_ERROR_API_NOT_SUPPORT.  The batch keeps pointers into the added plans'
 * device tables: a plan must stay alive until every exec it was added to has
 * completed.  None of these has a counterpart in the reference. */
typedef void* sipFftBatch;
AsdSip::AspbStatus sipFftBatchCreate(sipFftBatch* batch);
AsdSip::AspbStatus sipFftBatchDestroy(sipFftBatch batch);
AsdSip::AspbStatus sipFftBatchClear(sipFftBatch batch);
AsdSip::AspbStatus sipFftBatchAdd(sipFftBatch batch, AsdSip::asdFftHandle handle, const void* input, void* output);
/* As sipFftBatchAdd for the first `rows` rows of the plan's batch
 * (1 <= rows <= batch), with the plan's workspace for those rows at
 * `workspace` (rows * (workspace size / batch) bytes; may be null when the
 * plan needs none), so one plan of the largest batch serves requests of any
 * smaller batch, each with its own workspace.  C2C and pulse plans only. */
AsdSip::AspbStatus sipFftBatchAddRows(sipFftBatch batch, AsdSip::asdFftHandle handle, const void* input, void* output,
                                      int64_t rows, void* workspace);
AsdSip::AspbStatus sipFftBatchExec(sipFftBatch batch, void* stream);
AsdSip::AspbStatus sipFftBatchSetGate(sipFftBatch batch, const unsigned* device_flag, long long poll_limit);
AsdSip::AspbStatus sipFftBatchUseGraphs(sipFftBatch batch, int enable);
AsdSip::AspbStatus sipFftBatchTakeStatus(sipFftBatch batch, unsigned* status);

/* Runs a planned C2C handle (FP32 compute form) with the same kernels as
 * the ordinary exec but allocates nothing: the intermediate of two-pass
 * (four-step) plans goes to a static device array of the library, 32 MiB on
 * every GPU that loads it, instead of the bound workspace, which is not
 * needed.  It is for callers that cannot allocate device memory while they
 * run, such as a real-time signal chain where cudaMalloc/cudaFree would
 * synchronise the device and stall its other streams, or a host whose GPU
 * memory belongs to another pool or a fixed budget.  A plan whose workspace
 * would exceed 32 MiB (batch x length > 4,194,304 complex points for a
 * two-pass length) gives ACL_ERROR_INVALID_PARAM with a message; a non-C2C
 * or tensor-core plan gives ACL_ERROR_API_NOT_SUPPORT.  Runs on the plan's
 * device and stream.  The array's device address is looked up
 * (cudaGetSymbolAddress) when MakePlan prepares an eligible plan on its
 * device; under CUDA's default lazy module loading that is also when the
 * array is reserved, so the exec call itself loads and reserves nothing.
 * Make the plan before any stream capture, and make new plans after a
 * cudaDeviceReset.  Every call shares the array, so calls whose kernels
 * overlap on the GPU race: order them, e.g. on one stream.  No counterpart
 * in the reference. */
AsdSip::AspbStatus sipFftExecC2CNoAlloc(AsdSip::asdFftHandle handle, const void* input, void* output);

/* Library version string. */
const char* sipFftVersion(void);

#ifdef __cplusplus
}
#endif

#endif
