// Tensor-core split-precision length-256 tile kernel (tcgen05, sm_100a).
//
// One CTA of 128 threads takes tiles of 8 transforms of length 256 (the
// passes of the 65536 = 256 x 256 four-step).  Each of the two radix-16
// stages (tc_core.cuh) is 128 vectors x 16 points: every thread gathers one
// vector from the shared tile, splits it into three BF16 terms and writes
// row `tid` of the A operand; one elected thread issues the 12 MMAs
// (6 products x 2 K-halves, M = 128, N = 32, K = 16) into a 32-column
// tensor-memory accumulator and commits them to an mbarrier; after a
// bounded wait each thread reads its row back with tcgen05.ld (32x32b) and
// applies the W_256 twiddle (stage 1) or keeps the result (stage 2).  Loads,
// stores, the four-step cross twiddle and scaling follow the generic tile
// kernel (tile_io.cuh).  Waits never spin forever: after kTcWaitLimit
// polls the kernel records an error in sip_tc_error, releases its tensor
// memory and returns.
#include <cuda_runtime.h>

#include "tc_core.cuh"
#include "tc_launch.h"
#include "tile_io.cuh"

namespace sipfft {

__device__ unsigned int sip_tc_error = 0;

namespace {

constexpr long long kTcWaitLimit = 1LL << 26;

struct TcSmem {
    alignas(1024) unsigned char a[3 * kTcTermBytes];    // A operand: hi, mid, lo (24 KB)
    alignas(1024) unsigned char b[3 * kTcBTermBytes];   // B operand: hi, mid, lo (6 KB)
    alignas(16) float2 tile[kTcP * kTcLD];              // 17.5 KB
    alignas(8) unsigned long long mbar;
    unsigned int tmem_base;
    int abort;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

// No-swizzle K-major descriptor: LBO = 128 B (next core matrix along K),
// SBO = 512 B (next 8-row group), version 1.
__device__ __forceinline__ unsigned long long tc_desc(unsigned addr) {
    unsigned long long d = 0;
    d |= (unsigned long long)((addr & 0x3FFFF) >> 4);
    d |= (unsigned long long)(128 >> 4) << 16;
    d |= (unsigned long long)(512 >> 4) << 32;
    d |= 1ULL << 46;
    return d;
}

// kind::f16 instruction descriptor: D F32, A/B BF16, both K-major, N = 32, M = 128.
constexpr unsigned kTcIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ void tc_mma(unsigned tmem_d, unsigned long long da, unsigned long long db, bool accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(kTcIdesc), "r"((unsigned)accum));
}

// Returns false when the bounded wait ran out.
__device__ __forceinline__ bool mbar_wait(unsigned addr, unsigned parity) {
    for (long long i = 0; i < kTcWaitLimit; ++i) {
        unsigned ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// One radix-16 stage over the 128 vectors in A; returns false on a wait timeout.
__device__ __forceinline__ bool tc_stage(TcSmem& s, unsigned& phase, float (&r)[32]) {
    const int tid = threadIdx.x;
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
        const unsigned a0 = smem_u32(s.a), b0 = smem_u32(s.b);
        bool acc = false;
#pragma unroll
        for (int p = 0; p < kTcProducts; ++p)
#pragma unroll
            for (int kk = 0; kk < 2; ++kk) {
                tc_mma(s.tmem_base, tc_desc(a0 + tc_a_term(p) * kTcTermBytes + kk * 256),
                       tc_desc(b0 + tc_b_term(p) * kTcBTermBytes + kk * 256), acc);
                acc = true;
            }
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                         smem_u32(&s.mbar))
                     : "memory");
    }
    const bool ok = mbar_wait(smem_u32(&s.mbar), phase);
    phase ^= 1u;
    if (!ok) return false;
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    const unsigned taddr = s.tmem_base + ((unsigned)((tid >> 5) * 32) << 16);
    unsigned v[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) r[i] = __uint_as_float(v[i]);
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    return true;
}

template <int SIGN, bool TW4, bool COLS_IN, bool COLS_OUT>
__global__ void __launch_bounds__(kTcThreads) tc_fft256_kernel(const TileArgs a, const uint16_t* __restrict__ bmat,
                                                               const float2* __restrict__ tw256) {
    extern __shared__ unsigned char tc_raw[];
    TcSmem& s = *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(tc_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x;
    const int warp = tid >> 5;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 32;\n" ::"r"(smem_u32(&s.tmem_base))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(&s.mbar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        s.abort = 0;
    }
    for (int i = tid; i < 3 * kTcBTermBytes / 16; i += kTcThreads)
        reinterpret_cast<uint4*>(s.b)[i] = reinterpret_cast<const uint4*>(bmat)[i];
    asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
    unsigned phase = 0;

    for (int tile = blockIdx.x; tile < a.ntiles && !s.abort; tile += gridDim.x) {
        const TileCtx c = decode_tile(a, tile);
        tc_load_tile<COLS_IN>(tid, a, c, s.tile);
        __syncthreads();
        {
            float2 x[16];
            tc_gather1(s.tile, tid, x);
            tc_put_row(s.a, tid, x);
            float r[32];
            if (!tc_stage(s, phase, r)) s.abort = 1;
            __syncthreads();
            if (s.abort) break;
            tc_scatter1<SIGN>(s.tile, tid, r, tw256);
        }
        __syncthreads();
        {
            float2 x[16];
            tc_gather2(s.tile, tid, x);
            tc_put_row(s.a, tid, x);
            float r[32];
            if (!tc_stage(s, phase, r)) s.abort = 1;
            __syncthreads();
            if (s.abort) break;
            tc_scatter2(s.tile, tid, r);
        }
        __syncthreads();
        tc_store_tile<SIGN, TW4, COLS_OUT>(tid, a, c, s.tile);
        __syncthreads();
    }
    if (s.abort && tid == 0) {
        atomicOr(&sip_tc_error, 1u);
        // let MMAs still in flight land before the tensor memory is released
        mbar_wait(smem_u32(&s.mbar), phase);
    }
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 32;\n" ::"r"(s.tmem_base) : "memory");
}

using TcFn = void (*)(const TileArgs, const uint16_t*, const float2*);

template <int SIGN>
TcFn pick(bool tw4, bool cols_in, bool cols_out) {
    if (tw4) return tc_fft256_kernel<SIGN, true, true, true>;
    if (cols_in && cols_out) return tc_fft256_kernel<SIGN, false, true, true>;
    if (!cols_in && cols_out) return tc_fft256_kernel<SIGN, false, false, true>;
    return tc_fft256_kernel<SIGN, false, false, false>;
}

}  // namespace

int tc_smem_bytes() { return (int)sizeof(TcSmem) + 1024; }

int tc_tile_transforms() { return kTcP; }

int tc_threads() { return kTcThreads; }

const void* tc_kernel(int sign, bool tw4, bool cols_in, bool cols_out) {
    return reinterpret_cast<const void*>(sign < 0 ? pick<-1>(tw4, cols_in, cols_out) : pick<1>(tw4, cols_in, cols_out));
}

cudaError_t tc_prepare(const void* fn, int* ctas_per_sm) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, tc_smem_bytes());
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, fn, kTcThreads, (size_t)tc_smem_bytes());
}

cudaError_t tc_launch(const void* fn, int grid, const TileArgs& args, const void* src, void* dst, const uint16_t* bmat,
                      const float2* tw256, cudaStream_t stream) {
    TileArgs a = args;
    a.src = src;
    a.dst = dst;
    void* params[] = {&a, const_cast<uint16_t**>(&bmat), const_cast<float2**>(&tw256)};
    return cudaLaunchKernel(fn, dim3(grid), dim3(kTcThreads), params, (size_t)tc_smem_bytes(), stream);
}

cudaError_t tc_take_error(unsigned* err) {
    unsigned zero = 0;
    cudaError_t e = cudaMemcpyFromSymbol(err, sip_tc_error, sizeof(unsigned));
    if (e != cudaSuccess) return e;
    return cudaMemcpyToSymbol(sip_tc_error, &zero, sizeof(unsigned));
}

}  // namespace sipfft
