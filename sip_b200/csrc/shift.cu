// fftshift / ifftshift of batched 2-D complex64 slices (asdFftShift,
// asdIfftShift; reference core/fft/fftshift.cpp, core/fft/ifftshift.cpp and
// the kernels ops/fft/fftshift, ops/fft/ifftshift):
//   out[s][(r + sr) % row][(c + sc) % col] = scale * in[s * dist + r * col + c]
// with (sr, sc) = ((row + 1) / 2, (col + 1) / 2) for fftshift and
// (row / 2, col / 2) for ifftshift.
//
// HBM-bound permuted copy: each thread produces kShiftVec consecutive output
// elements of one output row (coalesced stores) from at most two contiguous
// input runs (the row's rotation point), so both sides stream.  Index
// division uses FastDiv when every index fits 32 bits.
#include <cuda_runtime.h>

#include "fft_core.cuh"
#include "shift.h"

namespace sipfft {

namespace {

constexpr int kShiftVec = 4;
constexpr int kShiftBlock = 256;

template <bool SCALE, bool FAST>
__global__ void __launch_bounds__(kShiftBlock) k_shift(const float2* __restrict__ in, float2* __restrict__ out,
                                                      ShiftArgs a) {
    // one work item = kShiftVec consecutive output elements of one output row
    const long long per_row = (a.col + kShiftVec - 1) / kShiftVec;
    const long long items = (long long)a.batch * a.row * per_row;
    for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < items;
         it += (long long)gridDim.x * blockDim.x) {
        long long orow_all, chunk;
        if (FAST) {
            orow_all = fd_div(a.div_per_row, (uint32_t)it);
            chunk = it - orow_all * per_row;
        } else {
            orow_all = it / per_row;
            chunk = it - orow_all * per_row;
        }
        long long s, orow;
        if (FAST) {
            s = fd_div(a.div_row, (uint32_t)orow_all);
            orow = orow_all - s * a.row;
        } else {
            s = orow_all / a.row;
            orow = orow_all - s * a.row;
        }
        long long irow = orow - a.sr;
        if (irow < 0) irow += a.row;
        const float2* src = in + s * a.dist + irow * a.col;
        float2* dst = out + (s * a.row + orow) * a.col;
        const int c0 = (int)(chunk * kShiftVec);
        int ic = c0 - a.sc;
        if (ic < 0) ic += a.col;
#pragma unroll
        for (int v = 0; v < kShiftVec; ++v) {
            const int oc = c0 + v;
            if (oc < a.col) {
                float2 x = __ldcs(src + ic);
                if (SCALE) x = make_float2(x.x * a.scale, x.y * a.scale);
                __stcs(dst + oc, x);
            }
            if (++ic == a.col) ic = 0;
        }
    }
}

}  // namespace

cudaError_t shift_launch(const void* in, void* out, const ShiftArgs& args, cudaStream_t stream) {
    ShiftArgs a = args;
    const long long per_row = (a.col + kShiftVec - 1) / kShiftVec;
    const long long items = (long long)a.batch * a.row * per_row;
    if (items == 0) return cudaSuccess;
    const bool fast = items < (1LL << 31) && (long long)a.batch * a.row < (1LL << 31);
    if (fast) {
        a.div_per_row = make_fastdiv((uint32_t)per_row);
        a.div_row = make_fastdiv((uint32_t)a.row);
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long want = (items + kShiftBlock - 1) / kShiftBlock;
    const int grid = (int)(want < (long long)sms * 16 ? want : (long long)sms * 16);
    const auto* i = static_cast<const float2*>(in);
    auto* o = static_cast<float2*>(out);
    const bool sc = a.scale != 1.0f;
    if (fast) {
        if (sc) k_shift<true, true><<<grid, kShiftBlock, 0, stream>>>(i, o, a);
        else k_shift<false, true><<<grid, kShiftBlock, 0, stream>>>(i, o, a);
    } else {
        if (sc) k_shift<true, false><<<grid, kShiftBlock, 0, stream>>>(i, o, a);
        else k_shift<false, false><<<grid, kShiftBlock, 0, stream>>>(i, o, a);
    }
    return cudaGetLastError();
}

}  // namespace sipfft
