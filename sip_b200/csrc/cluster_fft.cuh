// Cluster four-step: one C2C transform of N = N1 x N2 points spread over a
// thread-block cluster of C CTAs that exchange through distributed shared
// memory (DSMEM), one kernel, one HBM round trip.
//
// For batches too small to fill the GPU with one CTA per transform (C2C
// 4096 x 256: 256 CTAs on 148 SMs, each waiting on its own 32 KB load), the
// transform is split C ways.  With x viewed as [N1][N2] (x[i1 N2 + i2]):
//   pass A  CTA r: the N1-point FFTs of columns i2 in [r PA, (r+1) PA),
//           PA = N2 / C, read from HBM (runs of PA adjacent columns), the
//           result Y[k1][i2] kept in its shared memory as rows [k1][PA];
//   cluster barrier;
//   pass B  CTA r: rows k1 in [r PB, (r+1) PB), PB = N1 / C: Y[k1][i2] for
//           every i2 gathered from the cluster's shared memories (PA
//           contiguous values per peer CTA), times the cross twiddle
//           W_N^{i2 k1}, the N2-point FFTs, and X[k1 + N1 k2] stored with
//           PB adjacent outputs per k2;
//   (a second cluster barrier after the gather: no CTA leaves while a peer
//   may still read its rows).
// The radix passes are the size-specialized kernel's (sk_kernel.cuh): pass A
// is an SK_COLS configuration whose last pass writes the row layout here,
// pass B an SK_ROWS_T configuration whose pass 0 reads the gathered rows.
// The four-step algebra is that of the library's two-kernel four-step
// (plan.cpp add_c2c_1d; the reference's fft_c2c_large.cpp:199-235).
//
// Phase functions take the cluster's shared-memory pointers as an array so
// that the CPU harness (tests/native/tile_emu.cpp) runs them rank by rank.
#pragma once

#include "sk_kernel.cuh"

namespace sipfft {

template <class KA_, class KB_, int C_>
struct ClCfg {
    using KA = KA_;  // SkCfg<N1, PA, T, OP_C2C, SK_COLS, SIGN, false, ...>
    using KB = KB_;  // SkCfg<N2, PB, T, OP_C2C, SK_ROWS_T, SIGN, false, ...>
    static constexpr int C = C_;
    static constexpr int N1 = KA::N, N2 = KB::N, N = N1 * N2;
    static constexpr int PA = N2 / C, PB = N1 / C;
    static constexpr int T = KA::T;
    static constexpr int SIGN = KA::SIGN;
    // shared memory: pass A tile | rows [k1][PA] of Y | pass B tile
    static constexpr int ROWS_OFF = KA::BUF;
    static constexpr int B_OFF = KA::BUF + (N1 * PA + 1) / 2 * 2;
    static constexpr int SMEM_VALUES = B_OFF + KB::BUF;
    static_assert(N2 % C == 0 && N1 % C == 0, "both lengths split over the cluster");
    static_assert(KA::P == PA && KB::P == PB, "tile widths follow the cluster split");
    static_assert(KA::MODE == SK_COLS && KB::MODE == SK_ROWS_T && KA::OP == OP_C2C && KB::OP == OP_C2C,
                  "pass A reads columns, pass B writes the transposed rows");
    static_assert(KB::T == T && KB::SIGN == SIGN && !KA::TW4 && !KB::TW4 && !KA::SPLIT && !KB::SPLIT,
                  "one block shape and direction; the cross twiddle is applied in the gather");
    static_assert(!KA::TWS && !KB::TWS, "pass twiddles through the read-only cache");
};

// The last pass of A writes element k1 of column q to rows[k1 * PA + q]
// (consecutive threads: consecutive columns).
template <class CC, int PASS>
SIP_HD void cl_pass_a_write_rows(int tid, float2* rows, const typename SkPass<typename CC::KA, PASS>::Regs& rg) {
    using SP = SkPass<typename CC::KA, PASS>;
    static_assert(SP::LAST, "the last pass of A");
#pragma unroll
    for (int s = 0; s < SP::S; ++s) {
        const int b = tid + s * CC::T;
        if (SP::TOTAL % CC::T != 0 && b >= SP::TOTAL) continue;
        int q, j;
        SP::butterfly_index(b, q, j);
#pragma unroll
        for (int r = 0; r < SP::R; ++r) rows[(j + r * SP::NR) * CC::PA + q] = rg.v[s][r];  // L = NR here
    }
}

// Pass B's input: row k1 = r PB + q of the gathered Y, element i2 = n, from
// peer n / PA (`peer(p)`: that CTA's rows), times the cross twiddle; written
// in the row layout of KB's staging ([q][n]).  Consecutive threads read
// consecutive values of one peer's row.
template <class CC, class Peer>
SIP_HD void cl_gather(int tid, const TileArgs& b, int rank, Peer peer, float2* stage) {
    constexpr int TOTAL = CC::PB * CC::N2;
    for (int f = tid; f < TOTAL; f += CC::T) {
        const int q = f / CC::N2;
        const int n = f - q * CC::N2;
        const int k1 = rank * CC::PB + q;
        const float2 y = peer(n / CC::PA)[k1 * CC::PA + n % CC::PA];
        stage[q * CC::N2 + n] = c_tw<CC::SIGN>(y, cross_tw(b, (long long)n * k1));
    }
}

}  // namespace sipfft

#if defined(__CUDACC__) && !defined(__CUDACC_RTC__)
#include <cooperative_groups.h>

namespace sipfft {

template <class CC, int PASS>
__device__ __forceinline__ void cl_run_a(int tid, const TileArgs& a, const TileCtx& c, float2* buf, float2* rows) {
    using SP = SkPass<typename CC::KA, PASS>;
    typename SP::Regs rg;
    SP::read(tid, a, c, buf, rg);
    __syncthreads();
    if constexpr (SP::LAST) {
        cl_pass_a_write_rows<CC, PASS>(tid, rows, rg);
    } else {
        SP::write_smem(tid, buf, rg);
        __syncthreads();
        cl_run_a<CC, PASS + 1>(tid, a, c, buf, rows);
    }
}

// One cluster per transform: grid = transforms x C CTAs, cluster dimension C.
template <class CC>
__global__ void __launch_bounds__(CC::T) cluster_fft_kernel(const TileArgs a, const TileArgs b) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    const int tid = threadIdx.x;
    const int rank = (int)cluster.block_rank();
    const long long tr = blockIdx.x / CC::C;
    float2* abuf = sk_smem;
    float2* rows = sk_smem + CC::ROWS_OFF;
    float2* bbuf = sk_smem + CC::B_OFF;
    // pass A: columns [rank PA, (rank + 1) PA) of transform tr
    TileCtx ca;
    ca.i0 = rank * CC::PA;
    ca.cnt = CC::PA;
    ca.in_base = tr * CC::N + ca.i0;
    ca.out_base = 0;
    sk_stage<typename CC::KA>(tid, a, ca, abuf);
    sk_commit();
    sk_wait<0>();
    __syncthreads();
    cl_run_a<CC, 0>(tid, a, ca, abuf, rows);
    cluster.sync();
    // pass B: rows [rank PB, (rank + 1) PB)
    cl_gather<CC>(tid, b, rank, [&](int p) -> const float2* { return cluster.map_shared_rank(rows, p); }, bbuf);
    // after this barrier no CTA reads another's rows any more, so each may
    // finish and leave on its own
    cluster.sync();
    TileCtx cb;
    cb.i0 = rank * CC::PB;
    cb.cnt = CC::PB;
    cb.in_base = 0;
    cb.out_base = tr * CC::N + cb.i0;
    sk_run<typename CC::KB, 0>(tid, b, cb, bbuf);
}

}  // namespace sipfft
#endif
