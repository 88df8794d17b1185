/*
 * FFT plan/exec C ABI of the B200 FFT library (drop-in for hicann/sip's
 * include/fft_api.h).
 *
 * Every declaration below keeps the reference's name, argument order,
 * types and enum values, so code written against the reference compiles
 * and links unchanged.  The functions are declared inside `extern "C"`
 * and `namespace AsdSip`, which leaves the exported symbols unmangled;
 * C++ reference parameters (`asdFftHandle&`, `size_t&`, `asdFftType&`)
 * travel as pointers at the ABI level.
 *
 * Reference interface replaced, entry by entry (reference include/fft_api.h):
 *   asdFftCreate            :50   -> sip_b200/csrc/api.cpp
 *   asdFftSetStream         :53   (stream = cudaStream_t)
 *   asdFftMakePlan1D        :57
 *   asdFftIstftMakePlan     :61   (ISTFT is outside this library: API_NOT_SUPPORT)
 *   asdFftExecC2C           :67
 *   asdFftExecC2CSeparated  :70   (planar real/imag layout)
 *   asdFftExecC2R           :74
 *   asdFftExecR2C           :77
 *   asdFftExecIstft         :79   (API_NOT_SUPPORT)
 *   asdFftDestroy           :83
 *   asdFftMakePlan2D        :85
 *   asdFftMakePlan3D        :88
 *   asdFftGetWorkspaceSize  :91
 *   asdFftSetWorkspace      :93
 *   asdFftSynchronize       :95
 *   asdFftGetType           :97
 *   asdFftShift             :109
 *   asdIfftShift            :125
 *
 * Semantics (reference docs/en/API_Reference/FFT/FFT_1D.md:29): forward
 * uses exp(-2*pi*i*j*k/N), inverse exp(+2*pi*i*j*k/N); no transform is
 * normalised.  R2C with INVERSE returns conj(rfft(x)); C2R with FORWARD
 * returns the hfft of the half spectrum.
 */
#ifndef ASDSIP_FFT_API_H
#define ASDSIP_FFT_API_H

#include "utils/aspb_status.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aclTensor aclTensor;

namespace AsdSip {
typedef void* asdFftHandle;

enum asdFftStatus { SUCCESS = 0, FAILED = 1 };

enum asdFftType {
    ASCEND_FFT_C2C = 0x10,
    ASCEND_FFT_C2R = 0x11,
    ASCEND_FFT_R2C = 0x12,
    ASCEND_STFT_C2C = 0x20,
    ASCEND_STFT_C2R = 0x21,
    ASCEND_STFT_R2C = 0x22,
    ASCEND_FFT_C2C_SEP = 0x30
};

enum asdFftDirection {
    ASCEND_FFT_FORWARD = 0x10,
    ASCEND_FFT_INVERSE = 0x11,
};

enum asdFft1dDimType {
    ASCEND_FFT_HORIZONTAL = 0x10,
    ASCEND_FFT_VERTICAL = 0x11,
};

/* Allocates an empty handle; the plan is made by one MakePlan call. */
AsdSip::AspbStatus asdFftCreate(asdFftHandle& handle);

/* Binds a CUDA stream (cudaStream_t) to the handle.  NULL is rejected. */
AsdSip::AspbStatus asdFftSetStream(asdFftHandle handle, void* stream);

/* 1D plan of `batchSize` transforms of length `fftSize`.  A handle can be
 * planned once.  HORIZONTAL tensors are (batchSize, fftSize). */
AsdSip::AspbStatus asdFftMakePlan1D(asdFftHandle handle, int64_t fftSize, asdFftType fftType, asdFftDirection direction,
                                    int64_t batchSize,
                                    asdFft1dDimType dimType = asdFft1dDimType::ASCEND_FFT_HORIZONTAL);

AspbStatus asdFftIstftMakePlan(asdFftHandle handle, const aclTensor* input, const int64_t nFft,
                               const int64_t hopLengthOpt, const int64_t winLengthOpt, const bool center = true,
                               const bool normalized = false, const bool onesidedOpt = false, int64_t lengthOpt = 0,
                               const bool returnComplex = true);

/* complex64 -> complex64. */
AsdSip::AspbStatus asdFftExecC2C(asdFftHandle handle, const aclTensor* input, const aclTensor* output);

/* complex transform on planar float32 real/imag tensors. */
AsdSip::AspbStatus asdFftExecC2CSeparated(asdFftHandle handle, const aclTensor* inputReal, const aclTensor* inputImag,
                                          const aclTensor* outputReal, const aclTensor* outputImag);

/* complex64 half spectrum (..., N/2+1) -> float32 (..., N). */
AsdSip::AspbStatus asdFftExecC2R(asdFftHandle handle, const aclTensor* input, const aclTensor* output);

/* float32 (..., N) -> complex64 half spectrum (..., N/2+1). */
AsdSip::AspbStatus asdFftExecR2C(asdFftHandle handle, const aclTensor* input, const aclTensor* output);

AspbStatus asdFftExecIstft(asdFftHandle handle, const aclTensor* input, const aclTensor* windowOpt,
                           const aclTensor* output);

/* Releases the handle and its plan; device tables shared with other plans
 * stay alive until their last user is destroyed. */
AsdSip::AspbStatus asdFftDestroy(asdFftHandle handle);

AsdSip::AspbStatus asdFftMakePlan2D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, asdFftType fftType,
                                    asdFftDirection direction, int32_t batchSize);

AspbStatus asdFftMakePlan3D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, int64_t fftSizeZ,
                            asdFftType fftType, asdFftDirection direction, int32_t batchSize);

/* Bytes of device scratch the plan needs (0 when it needs none).  A plan
 * that needs scratch must have this queried before exec. */
AsdSip::AspbStatus asdFftGetWorkspaceSize(asdFftHandle handle, size_t& workspaceSize);

AsdSip::AspbStatus asdFftSetWorkspace(asdFftHandle handle, void* workspace);

/* Blocks until the bound stream drains. */
AsdSip::AspbStatus asdFftSynchronize(asdFftHandle handle);

AsdSip::AspbStatus asdFftGetType(asdFftHandle handle, asdFftType& fftType);

/* output[s][(r + (row+1)/2) % row][(c + (col+1)/2) % col] = input[s][r][c]
 * for `batch` complex64 slices of row x col; slice s of the input starts at
 * element s*dist (dist <= 0 means row*col). */
AsdSip::AspbStatus asdFftShift(int64_t row, int64_t col, int64_t batch, int64_t dist, const aclTensor* input,
                               aclTensor* output, void* stream, void* workspace = nullptr);

/* output[s][(r + row/2) % row][(c + col/2) % col] = scale * input[s][r][c]. */
AsdSip::AspbStatus asdIfftShift(int64_t row, int64_t col, int64_t batch, int64_t dist, double scale,
                                const aclTensor* input, aclTensor* output, void* stream, void* workspace = nullptr);
}  // namespace AsdSip

#ifdef __cplusplus
}
#endif

#endif
