// aclTensor stand-in: the four CANN tensor functions the FFT ABI consumes
// (reference core/fft/fft_api.cpp:1575-1587 uses aclGetViewShape and
// aclGetDataType; callers build tensors with aclCreateTensor).
#include "acl_tensor.h"

#include <cstring>
#include <new>

struct aclTensor {
    int64_t dims[8];
    int64_t strides[8];
    uint64_t ndim;
    aclDataType dtype;
    aclFormat format;
    int64_t offset;
    void* data;
};

namespace {

size_t elem_bytes(aclDataType t) {
    switch (t) {
        case ACL_FLOAT: case ACL_INT32: case ACL_UINT32: return 4;
        case ACL_FLOAT16: case ACL_BF16: case ACL_INT16: case ACL_UINT16: return 2;
        case ACL_INT8: case ACL_UINT8: case ACL_BOOL: return 1;
        case ACL_DOUBLE: case ACL_INT64: case ACL_UINT64: case ACL_COMPLEX64: return 8;
        case ACL_COMPLEX128: return 16;
        default: return 0;
    }
}

}  // namespace

extern "C" {

aclTensor* aclCreateTensor(const int64_t* viewDims, uint64_t viewDimsNum, aclDataType dataType,
                           const int64_t* stride, int64_t offset, aclFormat format, const int64_t* storageDims,
                           uint64_t storageDimsNum, void* tensorData) {
    (void)storageDims;
    (void)storageDimsNum;
    if (viewDimsNum > 8 || (viewDimsNum > 0 && viewDims == nullptr)) return nullptr;
    for (uint64_t i = 0; i < viewDimsNum; ++i)
        if (viewDims[i] < 0) return nullptr;
    aclTensor* t = new (std::nothrow) aclTensor;
    if (t == nullptr) return nullptr;
    std::memset(t, 0, sizeof(*t));
    t->ndim = viewDimsNum;
    int64_t run = 1;
    for (int64_t i = (int64_t)viewDimsNum - 1; i >= 0; --i) {
        t->dims[i] = viewDims[i];
        t->strides[i] = stride != nullptr ? stride[i] : run;
        run *= viewDims[i] > 0 ? viewDims[i] : 1;
    }
    t->dtype = dataType;
    t->format = format;
    t->offset = offset;
    t->data = tensorData;
    return t;
}

int aclDestroyTensor(const aclTensor* tensor) {
    delete tensor;
    return 0;
}

int aclGetViewShape(const aclTensor* tensor, int64_t** viewDims, uint64_t* viewDimsNum) {
    if (tensor == nullptr || viewDims == nullptr || viewDimsNum == nullptr) return 100000;
    int64_t* out = new (std::nothrow) int64_t[tensor->ndim > 0 ? tensor->ndim : 1];
    if (out == nullptr) return 100000;
    for (uint64_t i = 0; i < tensor->ndim; ++i) out[i] = tensor->dims[i];
    *viewDims = out;
    *viewDimsNum = tensor->ndim;
    return 0;
}

int aclGetDataType(const aclTensor* tensor, aclDataType* dataType) {
    if (tensor == nullptr || dataType == nullptr) return 100000;
    *dataType = tensor->dtype;
    return 0;
}

void aclFreeViewShape(int64_t* viewDims) { delete[] viewDims; }

void* aclGetTensorData(const aclTensor* tensor) {
    if (tensor == nullptr || tensor->data == nullptr) return nullptr;
    return static_cast<char*>(tensor->data) + tensor->offset * (int64_t)elem_bytes(tensor->dtype);
}

}  // extern "C"
