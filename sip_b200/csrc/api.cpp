// C ABI of the B200 FFT library (include/fft_api.h, include/sip_fft_ext.h).
//
// Validation order, status codes and the workspace protocol follow the
// reference's public functions in core/fft/fft_api.cpp (asdFftCreate
// :1047, asdFftSetStream :1067, asdFftMakePlan1D :1124, asdFftMakePlan2D
// :1245, asdFftMakePlan3D :1292, asdFftGetWorkspaceSize :1339,
// asdFftSetWorkspace :1361, asdFftSynchronize :1376, asdFftGetType :1392,
// asdFftExecV2 :1446, tensor matching :1512-1750, asdFftExecC2C/C2R/R2C
// :1752-1844).  Every call holds one process-wide mutex, as the reference's
// fft_mtx does; no exception crosses the ABI.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>

#include "acl_tensor.h"
#include "fft_api.h"
#include "jit.h"
#include "plan.h"
#include "sip_fft_ext.h"
#include "noalloc.h"
#include "queue.h"
#include "shift.h"
#include "tc_launch.h"

using namespace AsdSip;
using sipfft::FftPlan;
using sipfft::PlanError;

namespace {

std::mutex g_mu;
std::unordered_map<void*, std::unique_ptr<FftPlan>> g_plans;

constexpr int64_t kMaxFftSize = int64_t(1) << 27;

FftPlan* find_plan(asdFftHandle h) {
    auto it = g_plans.find(h);
    return it == g_plans.end() ? nullptr : it->second.get();
}

bool trace_enabled() {
    const char* t = std::getenv("ASDSIP_FFT_PLAN_TRACE");
    return t != nullptr && std::strcmp(t, "1") == 0;
}

bool device_present() {
    int n = 0;
    return cudaGetDeviceCount(&n) == cudaSuccess && n > 0;
}

// Builds the kernel steps and, when a GPU is present, the device tables.
// Any failure leaves the plan uninitialised; the reference reports plan
// construction failures as INVALID_PARAM (fft_api.cpp:1181-1187).
AspbStatus finish_plan(FftPlan& plan) {
    try {
        if (!plan.hints_explicit) sipfft::apply_tune_cache(plan);
        sipfft::build_steps(plan);
        if (device_present()) sipfft::prepare_device(plan);
    } catch (const std::exception& e) {
        plan.steps.clear();
        plan.resources_ready = false;
        std::fprintf(stderr, "[sip_b200] make plan failed: %s\n", e.what());
        return ACL_ERROR_INVALID_PARAM;
    }
    plan.initialized = true;
    if (trace_enabled()) std::fprintf(stderr, "ASDSIP_FFT_PLAN %s\n", sipfft::describe(plan).c_str());
    return ACL_SUCCESS;
}

AspbStatus check_direction(asdFftDirection d) {
    return (d == ASCEND_FFT_FORWARD || d == ASCEND_FFT_INVERSE) ? ACL_SUCCESS : ACL_ERROR_INVALID_PARAM;
}

// ---------------------------------------------------------- tensor match
struct View {
    std::vector<int64_t> dims;
    aclDataType dtype = ACL_DT_UNDEFINED;
    bool ok = false;
};

View view_of(const aclTensor* t) {
    View v;
    if (t == nullptr) return v;
    int64_t* dims = nullptr;
    uint64_t n = 0;
    if (aclGetViewShape(t, &dims, &n) != 0) {
        delete[] dims;
        return v;
    }
    v.dims.assign(dims, dims + n);
    delete[] dims;
    if (aclGetDataType(t, &v.dtype) != 0) return v;
    v.ok = true;
    return v;
}

// Element count of a view, or -1 when a dimension is negative or the product
// overflows int64.
int64_t view_elems(const View& v) {
    int64_t e = 1;
    for (int64_t d : v.dims) {
        if (d < 0) return -1;
        if (d != 0 && e > std::numeric_limits<int64_t>::max() / d) return -1;
        e *= d;
    }
    return e;
}

// asdFftShift / asdIfftShift with the reference's checks
// (core/fft/fftshift.cpp:27-140, core/fft/ifftshift.cpp): positive sizes,
// no int64 overflow, dist <= 0 meaning row * col and 0 < dist < row * col
// rejected, complex64 tensors holding at least (batch - 1) * dist + row * col
// input and batch * row * col output elements.  In addition overlapping
// input and output are rejected (the rotation is not in-place safe) and
// sizes beyond int32 per axis are not supported.
AspbStatus run_shift(int64_t row, int64_t col, int64_t batch, int64_t dist, double scale, bool inverse,
                     const aclTensor* input, aclTensor* output, void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    constexpr int64_t kMax = std::numeric_limits<int64_t>::max();
    if (row <= 0 || col <= 0 || batch <= 0) return ACL_ERROR_INVALID_PARAM;
    if (row > kMax / col) return ACL_ERROR_INVALID_PARAM;
    const int64_t slice = row * col;
    if (dist <= 0) {
        dist = slice;
    } else if (dist < slice) {
        return ACL_ERROR_INVALID_PARAM;
    }
    const View vi = view_of(input), vo = view_of(output);
    if (!vi.ok || !vo.ok) return ACL_ERROR_INVALID_PARAM;
    if (vi.dtype != ACL_COMPLEX64 || vo.dtype != ACL_COMPLEX64) return ACL_ERROR_UNSUPPORTED_DATA_TYPE;
    if (batch - 1 > (kMax - slice) / dist) return ACL_ERROR_INVALID_PARAM;
    if (batch > kMax / slice) return ACL_ERROR_INVALID_PARAM;
    const int64_t need_in = (batch - 1) * dist + slice, need_out = batch * slice;
    const int64_t have_in = view_elems(vi), have_out = view_elems(vo);
    if (have_in < need_in || have_out < need_out) return ACL_ERROR_INVALID_PARAM;
    if (row > std::numeric_limits<int32_t>::max() || col > std::numeric_limits<int32_t>::max())
        return ACL_ERROR_API_NOT_SUPPORT;
    const char* ib = static_cast<const char*>(aclGetTensorData(input));
    char* ob = static_cast<char*>(aclGetTensorData(output));
    if (ib == nullptr || ob == nullptr) return ACL_ERROR_INVALID_PARAM;
    if (ib < ob + need_out * 8 && ob < ib + need_in * 8) return ACL_ERROR_INVALID_PARAM;
    if (!device_present()) return ACL_ERROR_INTERNAL_ERROR;
    sipfft::ShiftArgs a;
    a.batch = batch;
    a.dist = dist;
    a.row = (int)row;
    a.col = (int)col;
    a.sr = (int)(inverse ? row / 2 : (row + 1) / 2);
    a.sc = (int)(inverse ? col / 2 : (col + 1) / 2);
    a.scale = (float)scale;
    const cudaError_t e = sipfft::shift_launch(ib, ob, a, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        std::fprintf(stderr, "[sip_b200] shift launch failed: %s\n", cudaGetErrorString(e));
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

// Product of the leading dims [0, count) equals the plan's batch.
bool leading_is_batch(const std::vector<int64_t>& dims, size_t count, int64_t batch) {
    int64_t e = 1;
    for (size_t i = 0; i < count; ++i) {
        if (dims[i] <= 0 || e > batch / dims[i]) return false;
        e *= dims[i];
    }
    return e == batch;
}

// Trailing dims equal the plan's sizes, the last one replaced by
// last_override when >= 0; leading extent equals batch.
bool match_shape(const FftPlan& p, const View& v, int64_t last_override) {
    const size_t nd = p.sizes.size();
    if (v.dims.size() < nd) return false;
    const size_t lead = v.dims.size() - nd;
    for (size_t i = 0; i < nd; ++i) {
        int64_t want = p.sizes[i];
        if (i == nd - 1 && last_override >= 0) want = last_override;
        if (v.dims[lead + i] != want) return false;
    }
    return leading_is_batch(v.dims, lead, p.batch);
}

// Reference matchC2C_ (fft_api.cpp:1568-1618): 1D tensors have rank 2,
// (batch, N); a batch-1 plan also accepts (N, 1).
bool match_c2c(const FftPlan& p, const aclTensor* t) {
    View v = view_of(t);
    if (!v.ok || v.dtype != ACL_COMPLEX64) return false;
    if (p.sizes.size() == 1) {
        if (v.dims.size() != 2) return false;
        if (p.batch == 1) return (v.dims[0] == 1 && v.dims[1] == p.sizes[0]) || (v.dims[0] == p.sizes[0] && v.dims[1] == 1);
        return v.dims[0] == p.batch && v.dims[1] == p.sizes[0];
    }
    return match_shape(p, v, -1);
}

// Half-spectrum side (reference matchC2R_, fft_api.cpp:1620-1674).
bool match_spectrum(const FftPlan& p, const aclTensor* t) {
    View v = view_of(t);
    if (!v.ok || v.dtype != ACL_COMPLEX64) return false;
    return match_shape(p, v, p.sizes.back() / 2 + 1);
}

// Real side (reference matchR2C_, fft_api.cpp:1676-1718).
bool match_real(const FftPlan& p, const aclTensor* t) {
    View v = view_of(t);
    if (!v.ok || v.dtype != ACL_FLOAT) return false;
    return match_shape(p, v, -1);
}

// --------------------------------------------------------------- exec
size_t operand_bytes(const FftPlan& p, bool input) {
    int64_t rows = p.batch;
    for (size_t i = 0; i + 1 < p.sizes.size(); ++i) rows *= p.sizes[i];
    const int64_t n = p.sizes.back();
    const size_t real_b = (size_t)(rows * n * 4);
    const size_t spec_b = (size_t)(rows * (n / 2 + 1) * 8);
    switch (p.type) {
        case ASCEND_FFT_R2C: return input ? real_b : spec_b;
        case ASCEND_FFT_C2R: return input ? spec_b : real_b;
        default: return (size_t)(rows * n * 8);
    }
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int want) {
        if (want < 0) return;
        if (cudaGetDevice(&prev) == cudaSuccess && prev != want) cudaSetDevice(want);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Reference asdFftExecV2 + CheckWorkspaceBinding (fft_api.cpp:1020-1032,
// 1446-1511).
AspbStatus exec_plan(FftPlan& p, const void* in, void* out) {
    if (!p.initialized) return ACL_ERROR_INVALID_PARAM;
    const bool ws_required = p.workspace_need > 0;
    if (ws_required && p.workspace == nullptr) {
        std::fprintf(stderr, "[sip_b200] workspace has not been set\n");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    if (ws_required && p.workspace_recorded == 0) {
        std::fprintf(stderr, "[sip_b200] call asdFftGetWorkspaceSize before exec\n");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (in == nullptr || out == nullptr) return ACL_ERROR_INTERNAL_ERROR;
    // Input and output must be separate, or exactly aliased for C2C plans
    // (every C2C plan reads a tile before it writes the same tile).
    const char* ib = static_cast<const char*>(in);
    const char* ob = static_cast<const char*>(out);
    const size_t isz = operand_bytes(p, true), osz = operand_bytes(p, false);
    const bool overlap = ib < ob + osz && ob < ib + isz;
    if (overlap && !(ib == ob && p.type == ASCEND_FFT_C2C)) {
        std::fprintf(stderr, "[sip_b200] input and output overlap\n");
        return ACL_ERROR_INVALID_PARAM;
    }
    try {
        if (!p.resources_ready) {
            if (!device_present()) return ACL_ERROR_INTERNAL_ERROR;
            sipfft::prepare_device(p);
        }
        DeviceGuard g(p.device);
        sipfft::launch_steps(p, in, out, p.workspace);
    } catch (const PlanError& e) {
        std::fprintf(stderr, "[sip_b200] exec failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] exec failed: %s\n", e.what());
        return ACL_ERROR_INVALID_PARAM;
    }
    return ACL_SUCCESS;
}

AspbStatus exec_tensors(asdFftHandle handle, asdFftType want, const aclTensor* input, const aclTensor* output) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || !p->initialized) return ACL_ERROR_INVALID_PARAM;
    if (p->type != want) return ACL_ERROR_INVALID_PARAM;
    bool ok_in = false, ok_out = false;
    switch (want) {
        case ASCEND_FFT_C2C:
            ok_in = match_c2c(*p, input);
            ok_out = match_c2c(*p, output);
            break;
        case ASCEND_FFT_R2C:
            ok_in = match_real(*p, input);
            ok_out = match_spectrum(*p, output);
            break;
        case ASCEND_FFT_C2R:
            ok_in = match_spectrum(*p, input);
            ok_out = match_real(*p, output);
            break;
        default:
            break;
    }
    if (!ok_in || !ok_out) {
        std::fprintf(stderr, "[sip_b200] tensor does not match the plan\n");
        return ACL_ERROR_INVALID_PARAM;
    }
    return exec_plan(*p, aclGetTensorData(input), aclGetTensorData(output));
}

}  // namespace

extern "C" {

namespace AsdSip {

AspbStatus asdFftCreate(asdFftHandle& handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    try {
        auto plan = std::make_unique<FftPlan>();
        void* key = plan.get();
        g_plans.emplace(key, std::move(plan));
        handle = key;
    } catch (const std::exception&) {
        handle = nullptr;
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus asdFftSetStream(asdFftHandle handle, void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (stream == nullptr) return ACL_ERROR_INVALID_PARAM;
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    p->stream = stream;
    return ACL_SUCCESS;
}

AspbStatus asdFftMakePlan1D(asdFftHandle handle, int64_t fftSize, asdFftType fftType, asdFftDirection direction,
                            int64_t batchSize, asdFft1dDimType dimType) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    if (fftSize <= 0 || fftSize > kMaxFftSize) return ACL_ERROR_INVALID_PARAM;
    if (batchSize <= 0 || batchSize > (int64_t)std::numeric_limits<int32_t>::max()) return ACL_ERROR_INVALID_PARAM;
    if (fftType != ASCEND_FFT_C2C && fftType != ASCEND_FFT_C2R && fftType != ASCEND_FFT_R2C &&
        fftType != ASCEND_FFT_C2C_SEP)
        return ACL_ERROR_INVALID_PARAM;
    if (check_direction(direction) != ACL_SUCCESS) return ACL_ERROR_INVALID_PARAM;
    if (p->initialized) return ACL_ERROR_INVALID_PARAM;
    if (dimType != ASCEND_FFT_HORIZONTAL && dimType != ASCEND_FFT_VERTICAL) return ACL_ERROR_INVALID_PARAM;
    // Vertical batches are rejected as on the reference's Ascend 950 route
    // (fft_api.cpp:1111-1116); strided layouts are not part of this ABI.
    if (dimType == ASCEND_FFT_VERTICAL && batchSize > 1) return ACL_ERROR_API_NOT_SUPPORT;
    p->type = fftType;
    p->direction = direction;
    p->sizes = {fftSize};
    p->batch = batchSize;
    p->vertical = dimType == ASCEND_FFT_VERTICAL;
    if (fftType == ASCEND_FFT_C2C_SEP) p->type = ASCEND_FFT_C2C_SEP;
    return finish_plan(*p);
}

AspbStatus asdFftIstftMakePlan(asdFftHandle handle, const aclTensor* input, const int64_t nFft,
                               const int64_t hopLengthOpt, const int64_t winLengthOpt, const bool center,
                               const bool normalized, const bool onesidedOpt, int64_t lengthOpt,
                               const bool returnComplex) {
    (void)handle; (void)input; (void)nFft; (void)hopLengthOpt; (void)winLengthOpt; (void)center;
    (void)normalized; (void)onesidedOpt; (void)lengthOpt; (void)returnComplex;
    return ACL_ERROR_API_NOT_SUPPORT;
}

AspbStatus asdFftExecC2C(asdFftHandle handle, const aclTensor* input, const aclTensor* output) {
    return exec_tensors(handle, ASCEND_FFT_C2C, input, output);
}

// Separated real / imaginary float planes (reference fft_api.cpp:1912-1985):
// the four views must have equal shapes (else INTERNAL_ERROR) and FLOAT
// dtype (else OP_INPUT_NOT_MATCH); the trailing dims must equal the plan's
// sizes and the leading ones its batch (else INVALID_PARAM).
AspbStatus asdFftExecC2CSeparated(asdFftHandle handle, const aclTensor* inputReal, const aclTensor* inputImag,
                                  const aclTensor* outputReal, const aclTensor* outputImag) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    const View v[4] = {view_of(inputReal), view_of(inputImag), view_of(outputReal), view_of(outputImag)};
    for (const View& x : v)
        if (!x.ok) return ACL_ERROR_INVALID_PARAM;
    for (int i = 1; i < 4; ++i)
        if (v[i].dims != v[0].dims) return ACL_ERROR_INTERNAL_ERROR;
    for (const View& x : v)
        if (x.dtype != ACL_FLOAT) return ACL_ERROR_OP_INPUT_NOT_MATCH;
    if (!p->initialized) return ACL_ERROR_INVALID_PARAM;
    if (p->type != ASCEND_FFT_C2C_SEP) return ACL_ERROR_INVALID_PARAM;
    const auto& d = v[0].dims;
    if (d.size() < p->sizes.size()) return ACL_ERROR_INVALID_PARAM;
    const size_t lead = d.size() - p->sizes.size();
    for (size_t i = 0; i < p->sizes.size(); ++i)
        if (d[lead + i] != p->sizes[i]) return ACL_ERROR_INVALID_PARAM;
    if (!leading_is_batch(d, lead, p->batch)) return ACL_ERROR_INVALID_PARAM;
    const void* ptr[4] = {aclGetTensorData(inputReal), aclGetTensorData(inputImag), aclGetTensorData(outputReal),
                          aclGetTensorData(outputImag)};
    for (const void* q : ptr)
        if (q == nullptr) return ACL_ERROR_INVALID_PARAM;
    // outputs must not partially overlap the inputs or each other
    const size_t bytes = (size_t)p->batch * (size_t)p->sizes[0] * 4;
    auto overlap = [&](const void* a, const void* b) {
        const char* x = static_cast<const char*>(a);
        const char* y = static_cast<const char*>(b);
        return x < y + bytes && y < x + bytes;
    };
    if (overlap(ptr[2], ptr[3]) || (overlap(ptr[0], ptr[2]) && ptr[0] != ptr[2]) ||
        (overlap(ptr[1], ptr[3]) && ptr[1] != ptr[3]) || overlap(ptr[0], ptr[3]) || overlap(ptr[1], ptr[2]))
        return ACL_ERROR_INVALID_PARAM;
    try {
        if (!p->resources_ready) {
            if (!device_present()) return ACL_ERROR_INTERNAL_ERROR;
            sipfft::prepare_device(*p);
        }
        DeviceGuard g(p->device);
        sipfft::launch_separated(*p, static_cast<const float*>(ptr[0]), static_cast<const float*>(ptr[1]),
                                 static_cast<float*>(const_cast<void*>(ptr[2])),
                                 static_cast<float*>(const_cast<void*>(ptr[3])));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] separated exec failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus asdFftExecC2R(asdFftHandle handle, const aclTensor* input, const aclTensor* output) {
    return exec_tensors(handle, ASCEND_FFT_C2R, input, output);
}

AspbStatus asdFftExecR2C(asdFftHandle handle, const aclTensor* input, const aclTensor* output) {
    return exec_tensors(handle, ASCEND_FFT_R2C, input, output);
}

AspbStatus asdFftExecIstft(asdFftHandle handle, const aclTensor* input, const aclTensor* windowOpt,
                           const aclTensor* output) {
    (void)handle; (void)input; (void)windowOpt; (void)output;
    return ACL_ERROR_API_NOT_SUPPORT;
}

AspbStatus asdFftDestroy(asdFftHandle handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_plans.find(handle);
    if (it == g_plans.end()) return ACL_ERROR_INVALID_PARAM;
    g_plans.erase(it);
    return ACL_SUCCESS;
}

namespace {
AspbStatus common_check(asdFftHandle handle, std::initializer_list<int64_t> sizes, int64_t batch) {
    if (find_plan(handle) == nullptr) return ACL_ERROR_INVALID_PARAM;
    for (int64_t s : sizes)
        if (s <= 0 || s > kMaxFftSize) return ACL_ERROR_INVALID_PARAM;
    if (batch <= 0) return ACL_ERROR_INVALID_PARAM;
    return ACL_SUCCESS;
}
}  // namespace

AspbStatus asdFftMakePlan2D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, asdFftType fftType,
                            asdFftDirection direction, int32_t batchSize) {
    std::lock_guard<std::mutex> lk(g_mu);
    AspbStatus st = common_check(handle, {fftSizeX, fftSizeY}, batchSize);
    if (st != ACL_SUCCESS) return st;
    if (fftType != ASCEND_FFT_C2C && fftType != ASCEND_FFT_C2R && fftType != ASCEND_FFT_R2C)
        return ACL_ERROR_INVALID_PARAM;
    if (check_direction(direction) != ACL_SUCCESS) return ACL_ERROR_INVALID_PARAM;
    FftPlan* p = find_plan(handle);
    if (p->initialized) return ACL_ERROR_INVALID_PARAM;
    p->type = fftType;
    p->direction = direction;
    p->sizes = {fftSizeX, fftSizeY};
    p->batch = batchSize;
    return finish_plan(*p);
}

AspbStatus asdFftMakePlan3D(asdFftHandle handle, int64_t fftSizeX, int64_t fftSizeY, int64_t fftSizeZ,
                            asdFftType fftType, asdFftDirection direction, int32_t batchSize) {
    std::lock_guard<std::mutex> lk(g_mu);
    AspbStatus st = common_check(handle, {fftSizeX, fftSizeY, fftSizeZ}, batchSize);
    if (st != ACL_SUCCESS) return st;
    if (fftType != ASCEND_FFT_C2C && fftType != ASCEND_FFT_C2R && fftType != ASCEND_FFT_R2C &&
        fftType != ASCEND_FFT_C2C_SEP)
        return ACL_ERROR_INVALID_PARAM;
    if (check_direction(direction) != ACL_SUCCESS) return ACL_ERROR_INVALID_PARAM;
    FftPlan* p = find_plan(handle);
    if (p->initialized) return ACL_ERROR_INVALID_PARAM;
    p->type = fftType;
    p->direction = direction;
    p->sizes = {fftSizeX, fftSizeY, fftSizeZ};
    p->batch = batchSize;
    return finish_plan(*p);
}

AspbStatus asdFftGetWorkspaceSize(asdFftHandle handle, size_t& workspaceSize) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    workspaceSize = p->workspace_need;
    p->workspace_recorded = p->workspace_need;
    return ACL_SUCCESS;
}

AspbStatus asdFftSetWorkspace(asdFftHandle handle, void* workspace) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    p->workspace = workspace;
    return ACL_SUCCESS;
}

AspbStatus asdFftSynchronize(asdFftHandle handle) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INTERNAL_ERROR;
    if (cudaStreamSynchronize(static_cast<cudaStream_t>(p->stream)) != cudaSuccess) return ACL_ERROR_INTERNAL_ERROR;
    return ACL_SUCCESS;
}

AspbStatus asdFftGetType(asdFftHandle handle, asdFftType& fftType) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INTERNAL_ERROR;
    fftType = p->type;
    return ACL_SUCCESS;
}

AspbStatus asdFftShift(int64_t row, int64_t col, int64_t batch, int64_t dist, const aclTensor* input,
                       aclTensor* output, void* stream, void* workspace) {
    (void)workspace;
    return run_shift(row, col, batch, dist, 1.0, false, input, output, stream);
}

AspbStatus asdIfftShift(int64_t row, int64_t col, int64_t batch, int64_t dist, double scale, const aclTensor* input,
                        aclTensor* output, void* stream, void* workspace) {
    (void)workspace;
    return run_shift(row, col, batch, dist, scale, true, input, output, stream);
}

}  // namespace AsdSip

AspbStatus sipFftExecRaw(asdFftHandle handle, const void* input, void* output) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    return exec_plan(*p, input, output);
}

AspbStatus sipFftExecRawRows(asdFftHandle handle, long long rows, const void* input, void* output,
                             void* workspace) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || !p->initialized || rows < 1 || rows > p->batch) return ACL_ERROR_INVALID_PARAM;
    if (!sipfft::rows_exec_supported(*p)) return ACL_ERROR_API_NOT_SUPPORT;
    void* ws = workspace != nullptr ? workspace : p->workspace;
    if (p->workspace_need > 0) {
        if (ws == nullptr) {
            std::fprintf(stderr, "[sip_b200] workspace has not been set\n");
            return ACL_ERROR_INTERNAL_ERROR;
        }
        if (workspace == nullptr && p->workspace_recorded == 0) {
            std::fprintf(stderr, "[sip_b200] call asdFftGetWorkspaceSize before exec\n");
            return ACL_ERROR_INVALID_PARAM;
        }
    }
    if (input == nullptr || output == nullptr) return ACL_ERROR_INTERNAL_ERROR;
    const char* ib = static_cast<const char*>(input);
    const char* ob = static_cast<const char*>(output);
    const size_t isz = operand_bytes(*p, true) / (size_t)p->batch * (size_t)rows;
    const size_t osz = operand_bytes(*p, false) / (size_t)p->batch * (size_t)rows;
    const bool overlap = ib < ob + osz && ob < ib + isz;
    if (overlap && !(ib == ob && p->type == ASCEND_FFT_C2C)) {
        std::fprintf(stderr, "[sip_b200] input and output overlap\n");
        return ACL_ERROR_INVALID_PARAM;
    }
    try {
        if (!p->resources_ready) {
            if (!device_present()) return ACL_ERROR_INTERNAL_ERROR;
            sipfft::prepare_device(*p);
        }
        DeviceGuard g(p->device);
        sipfft::launch_rows(*p, rows, input, output, ws);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] exec failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftDescribePlan(asdFftHandle handle, char* buf, size_t cap, size_t* needed) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr) return ACL_ERROR_INVALID_PARAM;
    const std::string s = sipfft::describe(*p);
    if (needed != nullptr) *needed = s.size() + 1;
    if (buf != nullptr && cap > 0) {
        const size_t n = s.size() < cap - 1 ? s.size() : cap - 1;
        std::memcpy(buf, s.data(), n);
        buf[n] = '\0';
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftSetComputeMode(asdFftHandle handle, int mode) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || p->initialized) return ACL_ERROR_INVALID_PARAM;
    if (mode != sipfft::kComputeFp32 && mode != sipfft::kComputeTcSplit) return ACL_ERROR_INVALID_PARAM;
    p->compute_mode = mode;
    return ACL_SUCCESS;
}

AspbStatus sipFftTakeDeviceErrors(unsigned* errors) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (errors == nullptr) return ACL_ERROR_INVALID_PARAM;
    *errors = 0;
    if (!device_present()) return ACL_SUCCESS;
    return sipfft::tc_take_error(errors) == cudaSuccess ? ACL_SUCCESS : ACL_ERROR_INTERNAL_ERROR;
}

AspbStatus sipFftJitCompileCheck(int op, int mode, int sign, int tw4, int n, long long transforms) {
    sipfft::JitCfg c;
    if (!sipfft::sk_jit_available() || !sipfft::sk_jit_choose(op, mode, sign, tw4 != 0, n, transforms, &c))
        return ACL_ERROR_API_NOT_SUPPORT;
    std::string err;
    if (!sipfft::sk_jit_select(op, mode, sign, tw4 != 0, n, transforms, &c, &err)) {
        std::fprintf(stderr, "sipFftJitCompileCheck: %s\n", err.c_str());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftJitWait(long long timeout_ms) {
    if (timeout_ms < 0) return ACL_ERROR_INVALID_PARAM;
    return sipfft::sk_jit_wait(timeout_ms) ? ACL_SUCCESS : ACL_ERROR_INTERNAL_ERROR;
}

AspbStatus sipFftSetPlanHint(asdFftHandle handle, int key, int value) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || p->initialized) return ACL_ERROR_INVALID_PARAM;
    switch (key) {
        case SIP_FFT_HINT_TILE_TRANSFORMS:
            if (value < 0 || value > 4096) return ACL_ERROR_INVALID_PARAM;
            p->hint_p = value;
            break;
        case SIP_FFT_HINT_ELEMS_PER_THREAD:
            if (value != 0 && value != 16 && value != 32) return ACL_ERROR_INVALID_PARAM;
            p->hint_e = value;
            break;
        case SIP_FFT_HINT_GENERIC_ONLY:
            if (value != 0 && value != 1) return ACL_ERROR_INVALID_PARAM;
            p->hint_generic = value;
            break;
        case SIP_FFT_HINT_RADIX_ORDER:
            if (value != 0 && value != 1) return ACL_ERROR_INVALID_PARAM;
            p->hint_order = value;
            break;
        case SIP_FFT_HINT_REAL_FUSED:
            if (value < 0 || value > 2) return ACL_ERROR_INVALID_PARAM;
            p->hint_real_fused = value;
            break;
        case SIP_FFT_HINT_SK_VARIANT:
            if (value < -1 || value > 15) return ACL_ERROR_INVALID_PARAM;
            p->hint_sk_variant = value;
            break;
        case SIP_FFT_HINT_RUNTIME_COMPILE:
            if (value < 0 || value > 2) return ACL_ERROR_INVALID_PARAM;
            p->hint_jit = value;
            break;
        default:
            return ACL_ERROR_INVALID_PARAM;
    }
    p->hints_explicit = true;
    return ACL_SUCCESS;
}

// ------------------------------------------------------------------ batch
// Upper bound of a gate wait (polls per CTA), so a flag that is never set
// ends the launch within seconds.
constexpr long long kMaxGatePolls = 1LL << 24;

AspbStatus sipFftBatchCreate(sipFftBatch* batch) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr) return ACL_ERROR_INVALID_PARAM;
    if (!device_present()) return ACL_ERROR_INTERNAL_ERROR;
    try {
        *batch = sipfft::batch_create();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] batch create failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchDestroy(sipFftBatch batch) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr) return ACL_ERROR_INVALID_PARAM;
    sipfft::batch_destroy(static_cast<sipfft::Batch*>(batch));
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchClear(sipFftBatch batch) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr) return ACL_ERROR_INVALID_PARAM;
    sipfft::batch_clear(static_cast<sipfft::Batch*>(batch));
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchAdd(sipFftBatch batch, asdFftHandle handle, const void* input, void* output) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (batch == nullptr || p == nullptr || !p->initialized || input == nullptr || output == nullptr)
        return ACL_ERROR_INVALID_PARAM;
    if (p->workspace_need > 0 && (p->workspace == nullptr || p->workspace_recorded == 0)) return ACL_ERROR_INVALID_PARAM;
    try {
        if (!p->resources_ready) sipfft::prepare_device(*p);
        if (!sipfft::batch_add(static_cast<sipfft::Batch*>(batch), *p, input, output)) return ACL_ERROR_API_NOT_SUPPORT;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] batch add failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchAddRows(sipFftBatch batch, asdFftHandle handle, const void* input, void* output, int64_t rows,
                              void* workspace) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (batch == nullptr || p == nullptr || !p->initialized || input == nullptr || output == nullptr)
        return ACL_ERROR_INVALID_PARAM;
    if (rows < 1 || rows > p->batch) return ACL_ERROR_INVALID_PARAM;
    if (p->workspace_need > 0 && workspace == nullptr) return ACL_ERROR_INVALID_PARAM;
    try {
        if (!p->resources_ready) sipfft::prepare_device(*p);
        if (!sipfft::batch_add_rows(static_cast<sipfft::Batch*>(batch), *p, input, output, rows, workspace))
            return ACL_ERROR_API_NOT_SUPPORT;
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] batch add failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchExec(sipFftBatch batch, void* stream) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr || stream == nullptr) return ACL_ERROR_INVALID_PARAM;
    auto* b = static_cast<sipfft::Batch*>(batch);
    try {
        sipfft::batch_exec(b, static_cast<cudaStream_t>(stream));
    } catch (const std::exception& e) {
        std::fprintf(stderr, "[sip_b200] batch exec failed: %s\n", e.what());
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchSetGate(sipFftBatch batch, const unsigned* device_flag, long long poll_limit) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr || poll_limit < 0 || poll_limit > kMaxGatePolls) return ACL_ERROR_INVALID_PARAM;
    sipfft::batch_set_gate(static_cast<sipfft::Batch*>(batch), device_flag, poll_limit);
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchUseGraphs(sipFftBatch batch, int enable) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr) return ACL_ERROR_INVALID_PARAM;
    sipfft::batch_use_graphs(static_cast<sipfft::Batch*>(batch), enable != 0);
    return ACL_SUCCESS;
}

AspbStatus sipFftBatchTakeStatus(sipFftBatch batch, unsigned* status) {
    std::lock_guard<std::mutex> lk(g_mu);
    if (batch == nullptr || status == nullptr) return ACL_ERROR_INVALID_PARAM;
    try {
        *status = sipfft::batch_take_status(static_cast<sipfft::Batch*>(batch));
    } catch (const std::exception&) {
        return ACL_ERROR_INTERNAL_ERROR;
    }
    return ACL_SUCCESS;
}

AspbStatus sipFftSetOutputShift(asdFftHandle handle, int mode, double scale) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || p->initialized || mode < 0 || mode > 2) return ACL_ERROR_INVALID_PARAM;
    p->out_shift = mode;
    p->out_scale = scale;
    return ACL_SUCCESS;
}

AspbStatus sipFftMakePlanPulse1D(asdFftHandle handle, int64_t fftSize, int64_t batchSize, const void* filter,
                                 int flags) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || p->initialized || filter == nullptr) return ACL_ERROR_INVALID_PARAM;
    if (fftSize <= 0 || fftSize > kMaxFftSize) return ACL_ERROR_INVALID_PARAM;
    if (batchSize <= 0 || batchSize > (int64_t)std::numeric_limits<int32_t>::max()) return ACL_ERROR_INVALID_PARAM;
    if ((flags & ~(sipfft::kPulseConj | sipfft::kPulseScale)) != 0) return ACL_ERROR_INVALID_PARAM;
    p->type = ASCEND_FFT_C2C;
    p->direction = ASCEND_FFT_FORWARD;
    p->sizes = {fftSize};
    p->batch = batchSize;
    p->pulse = true;
    p->pulse_filter = filter;
    p->pulse_flags = flags;
    return finish_plan(*p);
}

// Runs a planned C2C handle with its scratch in the library's static device
// array (noalloc.cu) instead of the bound workspace, for callers that must
// not allocate device memory while they run.  Validation happens before any
// CUDA call; a plan needing more scratch than the array holds is rejected.
AspbStatus sipFftExecC2CNoAlloc(asdFftHandle handle, const void* input, void* output) {
    std::lock_guard<std::mutex> lk(g_mu);
    FftPlan* p = find_plan(handle);
    if (p == nullptr || !p->initialized || input == nullptr || output == nullptr) return ACL_ERROR_INVALID_PARAM;
    if (p->type != ASCEND_FFT_C2C || p->compute_mode != sipfft::kComputeFp32) {
        std::fprintf(stderr, "[sip_b200] no-alloc exec: only FP32 C2C plans are supported\n");
        return ACL_ERROR_API_NOT_SUPPORT;
    }
    if (p->workspace_need > sipfft::kNaScratchBytes) {
        std::fprintf(stderr,
                     "[sip_b200] no-alloc exec: the plan needs %zu bytes of scratch; the static scratch holds at "
                     "most %zu bytes (batch x length <= %zu complex points)\n",
                     (size_t)p->workspace_need, sipfft::kNaScratchBytes, sipfft::kNaScratchBytes / 8);
        return ACL_ERROR_INVALID_PARAM;
    }
    const char* ib = static_cast<const char*>(input);
    const char* ob = static_cast<const char*>(output);
    const size_t isz = operand_bytes(*p, true), osz = operand_bytes(*p, false);
    if (ib != ob && ib < ob + osz && ob < ib + isz) {
        std::fprintf(stderr, "[sip_b200] input and output overlap\n");
        return ACL_ERROR_INVALID_PARAM;
    }
    if (!device_present() || !p->resources_ready || p->noalloc_scratch == nullptr) {
        std::fprintf(stderr,
                     "[sip_b200] no-alloc exec: the plan was not prepared on a device (no GPU at plan time, or the "
                     "static scratch could not be looked up)\n");
        return ACL_ERROR_INTERNAL_ERROR;
    }
    DeviceGuard g(p->device);
    return sipfft::noalloc_exec(*p, input, output) == sipfft::kNaOk ? ACL_SUCCESS : ACL_ERROR_INTERNAL_ERROR;
}

const char* sipFftVersion(void) { return "sip_b200-fft 0.1.0"; }

}  // extern "C"
