// Twiddle-table generation on the device.
//
// Angles are formed from exact integers (m, n) and evaluated with FP64
// sincospi, then rounded once to FP32, following the reference's
// FP64-then-round coefficient builders
// (ops/include/params/fft_real_stockham.h:77-111,
// ops/fft/c2c/fft_regbase/fft_regbase/large/fft_c2c_coefficients.h:17-90).
#include <cuda_runtime.h>

#include "tile_launch.h"

namespace sipfft {

namespace {

__device__ __forceinline__ float2 root_fwd(long long m, long long n) {
    m %= n;
    if (m < 0) m += n;
    double s, c;
    sincospi(2.0 * (double)m / (double)n, &s, &c);
    return make_float2((float)c, (float)(-s));
}

__global__ void k_stockham_tw(float2* out, const PlanDev plan, int entries) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= entries) return;
    for (int p = 0; p < plan.npass; ++p) {
        const PassDesc& pd = plan.pass[p];
        if (pd.L <= 1) continue;
        const int cnt = pd.L * (pd.R - 1);
        if (i >= pd.tw && i < pd.tw + cnt) {
            const int off = i - pd.tw;  // twiddle-major: entry (r - 1) L + k
            const int r = off / pd.L + 1;
            const int k = off - (r - 1) * pd.L;
            out[i] = root_fwd((long long)r * k, (long long)pd.L * pd.R);
            return;
        }
    }
}

// Basis table (fft_core.cuh basis_split): per pass with span L > 1, the L
// values of W_{LR}^{r k} (k < L) for r = 1..a-1, then of W_{LR}^{a h k} for
// h = 1..R/a-1; twiddle-major, so the consecutive k of a warp's butterflies
// read consecutive entries.
__global__ void k_basis_tw(float2* out, const PlanDev plan, int entries) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= entries) return;
    int off = 0;
    for (int p = 0; p < plan.npass; ++p) {
        const PassDesc& pd = plan.pass[p];
        if (pd.L <= 1) continue;
        const int bc = basis_count(pd.R);
        const int cnt = pd.L * bc;
        if (i < off + cnt) {
            const int t = (i - off) / pd.L;  // twiddle-major: entry t L + k
            const int k = (i - off) - t * pd.L;
            const int a = basis_split(pd.R);
            const long long r = t < a - 1 ? t + 1 : (long long)a * (t - (a - 1) + 1);
            out[i] = root_fwd(r * k, (long long)pd.L * pd.R);
            return;
        }
        off += cnt;
    }
}

__global__ void k_root_tw(float2* out, long long n, long long count) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = root_fwd(i, n);
}

// Split cross-twiddle table: [W_n^lo, lo < B][W_n^{hi B}, hi < ceil(n/B)].
__global__ void k_split_tw(float2* out, long long n, long long B, long long count) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = root_fwd(i < B ? i : (i - B) * B, n);
}

}  // namespace

cudaError_t gen_split_twiddles(float2* out, long long n, int shift, cudaStream_t stream) {
    const long long B = 1LL << shift;
    const long long count = B + (n + B - 1) / B;
    const int block = 256;
    k_split_tw<<<(unsigned)((count + block - 1) / block), block, 0, stream>>>(out, n, B, count);
    return cudaGetLastError();
}

cudaError_t gen_stockham_twiddles(float2* out, const PlanDev& plan, int entries, cudaStream_t stream) {
    if (entries <= 0) return cudaSuccess;
    const int block = 256;
    k_stockham_tw<<<(entries + block - 1) / block, block, 0, stream>>>(out, plan, entries);
    return cudaGetLastError();
}

int basis_entries(const PlanDev& plan) {
    int n = 0;
    for (int p = 0; p < plan.npass; ++p)
        if (plan.pass[p].L > 1) n += plan.pass[p].L * basis_count(plan.pass[p].R);
    return n;
}

cudaError_t gen_basis_twiddles(float2* out, const PlanDev& plan, cudaStream_t stream) {
    const int entries = basis_entries(plan);
    if (entries <= 0) return cudaSuccess;
    const int block = 256;
    k_basis_tw<<<(entries + block - 1) / block, block, 0, stream>>>(out, plan, entries);
    return cudaGetLastError();
}

cudaError_t gen_root_twiddles(float2* out, long long n, long long count, cudaStream_t stream) {
    if (count <= 0) return cudaSuccess;
    const int block = 256;
    long long blocks = (count + block - 1) / block;
    if (blocks > 65535LL * 16) blocks = 65535LL * 16;
    k_root_tw<<<(unsigned)blocks, block, 0, stream>>>(out, n, count);
    return cudaGetLastError();
}

}  // namespace sipfft
