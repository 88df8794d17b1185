/*
 * Minimal stand-in for the CANN tensor descriptor used by the FFT C ABI.
 *
 * The reference passes tensors as opaque `aclTensor*` created by CANN's
 * aclCreateTensor and inspected with aclGetViewShape / aclGetDataType
 * (reference core/fft/fft_api.cpp:1575-1587).  CANN does not exist on a
 * CUDA machine, so this library exports the four C functions the FFT path
 * needs, with CANN's signatures, over a small struct holding the view
 * shape, strides, dtype and a device pointer.  Code that created tensors
 * with CANN keeps compiling against this header unchanged.
 *
 * Data-type values follow CANN's aclDataType numbering (ACL_FLOAT = 0,
 * ACL_COMPLEX64 = 16), which is also the numbering the reference's test
 * fixtures store in their .bin headers.
 */
#ifndef SIP_B200_ACL_TENSOR_H
#define SIP_B200_ACL_TENSOR_H

#include <cstddef>
#include <cstdint>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct aclTensor aclTensor;

typedef enum {
    ACL_DT_UNDEFINED = -1,
    ACL_FLOAT = 0,
    ACL_FLOAT16 = 1,
    ACL_INT8 = 2,
    ACL_INT32 = 3,
    ACL_UINT8 = 4,
    ACL_INT16 = 6,
    ACL_UINT16 = 7,
    ACL_UINT32 = 8,
    ACL_INT64 = 9,
    ACL_UINT64 = 10,
    ACL_DOUBLE = 11,
    ACL_BOOL = 12,
    ACL_COMPLEX64 = 16,
    ACL_COMPLEX128 = 17,
    ACL_BF16 = 27
} aclDataType;

typedef enum {
    ACL_FORMAT_UNDEFINED = -1,
    ACL_FORMAT_NCHW = 0,
    ACL_FORMAT_NHWC = 1,
    ACL_FORMAT_ND = 2
} aclFormat;

/* Creates a descriptor.  `tensorData` is a device pointer owned by the
 * caller; the descriptor never frees it.  Returns NULL on invalid input
 * (negative dims, NULL dims with viewDimsNum > 0, more than 8 dims). */
aclTensor* aclCreateTensor(const int64_t* viewDims, uint64_t viewDimsNum, aclDataType dataType,
                           const int64_t* stride, int64_t offset, aclFormat format, const int64_t* storageDims,
                           uint64_t storageDimsNum, void* tensorData);

/* Frees a descriptor created by aclCreateTensor (NULL is accepted). */
int aclDestroyTensor(const aclTensor* tensor);

/* Returns a newly allocated (new[]) copy of the view shape; the caller
 * releases it with delete[] (or aclFreeViewShape from C). */
int aclGetViewShape(const aclTensor* tensor, int64_t** viewDims, uint64_t* viewDimsNum);

int aclGetDataType(const aclTensor* tensor, aclDataType* dataType);

/* C-callable release for the array returned by aclGetViewShape. */
void aclFreeViewShape(int64_t* viewDims);

/* Device address of element 0 of the view (storage pointer + offset). */
void* aclGetTensorData(const aclTensor* tensor);

#ifdef __cplusplus
}
#endif

#endif
