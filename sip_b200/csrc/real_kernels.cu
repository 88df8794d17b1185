// Real-transform pre/post passes for lengths beyond one tile (element
// formulas in real_math.cuh).
#include "real_kernels.h"

#include "real_math.cuh"

namespace sipfft {

namespace {

// One thread per pair (k, m - k), k in [0, m/2]: each value and each
// twiddle is read once (the mirror's twiddle follows from W_{2m}^k).
__global__ void k_real_post(const RealPassArgs a) {
    const long long pairs = a.m / 2 + 1;
    const bool cj = a.conj != 0;
    for (long long row = blockIdx.y; row < a.rows; row += gridDim.y) {
        const float2* z = a.src + row * a.in_pitch;
        float2* x = a.dst + row * a.out_pitch;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < pairs;
             k += (long long)gridDim.x * blockDim.x) {
            const long long km = a.m - k;
            if (k > 0 && k < km) {
                real_post_pair(z, k, a.m, a.tw, cj, x + k, x + km);
            } else {
                x[k] = real_post_elem(z, k, a.m, a.tw, cj);
                if (km != k) x[km] = real_post_elem(z, km, a.m, a.tw, cj);
            }
        }
    }
}

__global__ void k_real_pre(const RealPassArgs a) {
    const long long pairs = a.m / 2 + 1;
    const bool cj = a.conj != 0;
    for (long long row = blockIdx.y; row < a.rows; row += gridDim.y) {
        const float2* x = a.src + row * a.in_pitch;
        float2* z = a.dst + row * a.out_pitch;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < pairs;
             k += (long long)gridDim.x * blockDim.x) {
            const long long km = a.m - k;
            if (k > 0 && k < km) {
                real_pre_pair(x, k, a.m, a.tw, cj, z + k, z + km);
            } else {
                z[k] = real_pre_elem(x, k, a.m, a.tw, cj);
                if (km != k && km < a.m) z[km] = real_pre_elem(x, km, a.m, a.tw, cj);
            }
        }
    }
}

dim3 grid_for(long long per_row, long long rows, int block) {
    long long gx = (per_row + block - 1) / block;
    if (gx > 4096) gx = 4096;
    long long gy = rows < 65535 ? rows : 65535;
    return dim3((unsigned)gx, (unsigned)gy, 1);
}

}  // namespace

cudaError_t real_post(const RealPassArgs& a, cudaStream_t stream) {
    k_real_post<<<grid_for(a.m / 2 + 1, a.rows, 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t real_pre(const RealPassArgs& a, cudaStream_t stream) {
    k_real_pre<<<grid_for(a.m / 2 + 1, a.rows, 256), 256, 0, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace sipfft
