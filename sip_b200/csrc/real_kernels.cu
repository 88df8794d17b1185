// Real-transform pre/post passes for lengths beyond one tile (element
// formulas in real_math.cuh).  Launched with programmatic dependent launch
// (launch_attr.h): each kernel waits for the previous one before its first
// global-memory access.
#include "real_kernels.h"

#include "launch_attr.h"

#include "real_math.cuh"

namespace sipfft {

namespace {

// One thread per pair (k, m - k), k in [0, m/2]: each value and each
// twiddle is read once (the mirror's twiddle follows from W_{2m}^k).
__global__ void k_real_post(const RealPassArgs a) {
    grid_dep_wait();
    grid_dep_launch();
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
    grid_dep_wait();
    grid_dep_launch();
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

__global__ void k_pair_pack(const PairPassArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const long long pairs = (a.rows + 1) / 2;
    for (long long p = blockIdx.y; p < pairs; p += gridDim.y) {
        const float* xa = static_cast<const float*>(a.src) + 2 * p * a.in_pitch;
        const float* xb = 2 * p + 1 < a.rows ? xa + a.in_pitch : nullptr;
        float2* z = static_cast<float2*>(a.dst) + p * a.out_pitch;
        for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < a.n;
             j += (long long)gridDim.x * blockDim.x)
            z[j] = make_float2(__ldg(xa + j), xb != nullptr ? __ldg(xb + j) : 0.f);
    }
}

__global__ void k_pair_separate(const PairPassArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const long long pairs = (a.rows + 1) / 2;
    const bool cj = a.conj != 0;
    for (long long p = blockIdx.y; p < pairs; p += gridDim.y) {
        const float2* z = static_cast<const float2*>(a.src) + p * a.in_pitch;
        float2* outa = static_cast<float2*>(a.dst) + 2 * p * a.out_pitch;
        float2* outb = 2 * p + 1 < a.rows ? outa + a.out_pitch : nullptr;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; 2 * k <= a.n;
             k += (long long)gridDim.x * blockDim.x) {
            float2 xa, xb;
            pair_separate_elem(z, k, a.n, cj, &xa, &xb);
            outa[k] = xa;
            if (outb != nullptr) outb[k] = xb;
        }
    }
}

__global__ void k_pair_combine(const PairPassArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const long long pairs = (a.rows + 1) / 2;
    const bool fwd = a.conj != 0;
    for (long long p = blockIdx.y; p < pairs; p += gridDim.y) {
        const float2* xa = static_cast<const float2*>(a.src) + 2 * p * a.in_pitch;
        const float2* xb = 2 * p + 1 < a.rows ? xa + a.in_pitch : nullptr;
        float2* z = static_cast<float2*>(a.dst) + p * a.out_pitch;
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < a.n;
             k += (long long)gridDim.x * blockDim.x)
            z[k] = pair_combine_elem(xa, xb, k, a.n, fwd);
    }
}

__global__ void k_pair_split(const PairPassArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const long long pairs = (a.rows + 1) / 2;
    for (long long p = blockIdx.y; p < pairs; p += gridDim.y) {
        const float2* z = static_cast<const float2*>(a.src) + p * a.in_pitch;
        float* outa = static_cast<float*>(a.dst) + 2 * p * a.out_pitch;
        float* outb = 2 * p + 1 < a.rows ? outa + a.out_pitch : nullptr;
        for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < a.n;
             j += (long long)gridDim.x * blockDim.x) {
            const float2 v = __ldg(z + j);
            outa[j] = v.x;
            if (outb != nullptr) outb[j] = v.y;
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
    return launch_pdl(k_real_post, grid_for(a.m / 2 + 1, a.rows, 256), dim3(256), 0, stream, a.m * a.rows, a);
}

cudaError_t real_pre(const RealPassArgs& a, cudaStream_t stream) {
    return launch_pdl(k_real_pre, grid_for(a.m / 2 + 1, a.rows, 256), dim3(256), 0, stream, a.m * a.rows, a);
}

cudaError_t pair_pack(const PairPassArgs& a, cudaStream_t stream) {
    return launch_pdl(k_pair_pack, grid_for(a.n, (a.rows + 1) / 2, 256), dim3(256), 0, stream, a.n * a.rows, a);
}

cudaError_t pair_separate(const PairPassArgs& a, cudaStream_t stream) {
    return launch_pdl(k_pair_separate, grid_for(a.n / 2 + 1, (a.rows + 1) / 2, 256), dim3(256), 0, stream, a.n * a.rows, a);
}

cudaError_t pair_combine(const PairPassArgs& a, cudaStream_t stream) {
    return launch_pdl(k_pair_combine, grid_for(a.n, (a.rows + 1) / 2, 256), dim3(256), 0, stream, a.n * a.rows, a);
}

cudaError_t pair_split(const PairPassArgs& a, cudaStream_t stream) {
    return launch_pdl(k_pair_split, grid_for(a.n, (a.rows + 1) / 2, 256), dim3(256), 0, stream, a.n * a.rows, a);
}

}  // namespace sipfft
