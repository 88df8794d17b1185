// Bluestein pre/post passes and the chirp table (bluestein.cuh).  The pre
// and post passes launch with programmatic dependent launch (launch_attr.h).
#include "bluestein.h"

#include "launch_attr.h"

namespace sipfft {

namespace {

constexpr int kBlueBlock = 256;

__global__ void k_blue_pre(const BluesteinArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    float2* dst = static_cast<float2*>(a.dst);
    for (long long row = blockIdx.y; row < a.rows; row += gridDim.y)
        for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < a.m;
             j += (long long)gridDim.x * blockDim.x)
            dst[row * a.m + j] = blue_pre_elem(a, row, j);
}

__global__ void k_blue_post(const BluesteinArgs a) {
    grid_dep_wait();
    grid_dep_launch();
    const long long cnt = blue_out_count(a);
    for (long long row = blockIdx.y; row < a.rows; row += gridDim.y)
        for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < cnt;
             k += (long long)gridDim.x * blockDim.x)
            blue_post_elem(a, row, k);
}

__global__ void k_chirp(float2* out, long long n, int sign) {
    for (long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x; j < n;
         j += (long long)gridDim.x * blockDim.x) {
        const long long q = (j * j) % (2 * n);  // exact phase index: exp(i pi q / n)
        double s, c;
        sincospi((double)q / (double)n, &s, &c);
        out[j] = make_float2((float)c, (float)(sign * s));
    }
}

// The convolution sequence of the Bluestein filter: b_j = conj(c_j) for
// j < n and b_{m-j} = b_j for 0 < j < n, zero elsewhere (m >= 2n - 1); the
// filter is its length-m FFT.  FP64 phases, rounded once.
__global__ void k_blue_b(float2* out, long long n, long long m, int sign) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < m;
         i += (long long)gridDim.x * blockDim.x) {
        const long long j = i < n ? i : (i > m - n ? m - i : -1);
        if (j < 0) {
            out[i] = make_float2(0.f, 0.f);
            continue;
        }
        const long long q = (j * j) % (2 * n);
        double s, c;
        sincospi((double)q / (double)n, &s, &c);
        out[i] = make_float2((float)c, (float)(-sign * s));
    }
}

dim3 grid2(long long per_row, long long rows) {
    long long gx = (per_row + kBlueBlock - 1) / kBlueBlock;
    if (gx > 4096) gx = 4096;
    const long long gy = rows < 65535 ? rows : 65535;
    return dim3((unsigned)gx, (unsigned)gy, 1);
}

}  // namespace

cudaError_t bluestein_prepare() {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, k_blue_pre);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_blue_post);
    return e;
}

cudaError_t bluestein_pre(const BluesteinArgs& a, cudaStream_t stream) {
    return launch_pdl(k_blue_pre, grid2(a.m, a.rows), dim3(kBlueBlock), 0, stream, a.m * a.rows, a);
}

cudaError_t bluestein_post(const BluesteinArgs& a, cudaStream_t stream) {
    return launch_pdl(k_blue_post, grid2(blue_out_count(a), a.rows), dim3(kBlueBlock), 0, stream,
                      blue_out_count(a) * a.rows, a);
}

cudaError_t gen_blue_b(float2* out, long long n, long long m, int sign, cudaStream_t stream) {
    long long g = (m + kBlueBlock - 1) / kBlueBlock;
    if (g > 65535) g = 65535;
    k_blue_b<<<(unsigned)g, kBlueBlock, 0, stream>>>(out, n, m, sign);
    return cudaGetLastError();
}

cudaError_t gen_chirp(float2* out, long long n, int sign, cudaStream_t stream) {
    long long blocks = (n + kBlueBlock - 1) / kBlueBlock;
    if (blocks > 65535) blocks = 65535;
    k_chirp<<<(unsigned)blocks, kBlueBlock, 0, stream>>>(out, n, sign);
    return cudaGetLastError();
}

}  // namespace sipfft
