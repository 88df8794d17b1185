// The cluster four-step configurations compiled into the library (and run by
// the CPU harness).
#pragma once

#include "cluster_fft.cuh"

namespace sipfft {

template <int N1, int PA, int T, int SIGN, int... R>
using ClA = SkCfg<N1, PA, T, OP_C2C, SK_COLS, SIGN, false, 1, SK_TW_BASIS, R...>;
template <int N2, int PB, int T, int SIGN, int... R>
using ClB = SkCfg<N2, PB, T, OP_C2C, SK_ROWS_T, SIGN, false, 1, SK_TW_BASIS, R...>;

// 1024 = 32 x 32 on 2 CTAs, 4096 = 64 x 64 on 4, 8192 = 64 x 128 on 4
template <int SIGN> using Cl1024 = ClCfg<ClA<32, 16, 128, SIGN, 4, 8>, ClB<32, 16, 128, SIGN, 4, 8>, 2>;
template <int SIGN> using Cl4096 = ClCfg<ClA<64, 16, 128, SIGN, 8, 8>, ClB<64, 16, 128, SIGN, 8, 8>, 4>;
template <int SIGN> using Cl8192 = ClCfg<ClA<64, 32, 256, SIGN, 8, 8>, ClB<128, 16, 256, SIGN, 8, 16>, 4>;

#define SIP_CL_CONFIGS(X) X(Cl1024<-1>) X(Cl1024<1>) X(Cl4096<-1>) X(Cl4096<1>) X(Cl8192<-1>) X(Cl8192<1>)

}  // namespace sipfft
