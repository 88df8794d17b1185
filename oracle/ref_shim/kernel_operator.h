// Qualifier shim that lets the reference's SIMT Stockham header
// (ops/fft/real/fft_stockham/fft_stockham/kernel/arch35/vendor/
// fft_stockham_mix.h) compile as plain C++ for the oracle: address-space
// and launch qualifiers become nothing, a vector-function call runs its
// body once with one thread (every thread loop then covers all indices),
// and barriers are no-ops.  Test infrastructure only.
#pragma once
#define __simt_vf__
#define __aicore__
#define __gm__
#define __ubuf__
#define __launch_bounds__(x)

struct RefDim3 {
    int x, y, z;
    RefDim3(int a = 1, int b = 1, int c = 1) : x(a), y(b), z(c) {}
};
using dim3 = RefDim3;
inline RefDim3 threadIdx{0, 0, 0};
inline RefDim3 blockDim{1, 1, 1};

enum RefPipe { PIPE_V = 0, PIPE_ALL = 1 };
namespace AscendC {
template <int P>
inline void PipeBarrier() {}
}  // namespace AscendC
inline void asc_syncthreads() {}

template <auto F, class... A>
inline void asc_vf_call(RefDim3, A... args) {
    F(args...);
}
