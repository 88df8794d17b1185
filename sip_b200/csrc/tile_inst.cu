// Instantiations of the tile kernels for one (sign, elements-per-thread)
// pair.  The build compiles this file once per pair (-DSIP_INST_SIGN,
// -DSIP_INST_E) so the variants compile in parallel.
#include "tile_kernel_impl.cuh"

#ifndef SIP_INST_SIGN
#error "SIP_INST_SIGN must be defined"
#endif
#ifndef SIP_INST_E
#error "SIP_INST_E must be defined"
#endif

#define SIP_CAT2(a, b) a##b
#define SIP_CAT(a, b) SIP_CAT2(a, b)
#if SIP_INST_SIGN < 0
#define SIP_INST_NAME SIP_CAT(tile_pick_fwd_e, SIP_INST_E)
#else
#define SIP_INST_NAME SIP_CAT(tile_pick_inv_e, SIP_INST_E)
#endif

namespace sipfft {

using KernelFn = void (*)(const TileArgs);

// Real ops run a fixed sign (R2C forward, C2R inverse) and conjugate on
// load or store for the other direction; the four-step cross twiddle
// exists for C2C only.
KernelFn SIP_INST_NAME(int op, bool tw4) {
    constexpr int S = SIP_INST_SIGN;
    constexpr int E = SIP_INST_E;
    switch (op) {
        case OP_C2C:
            return tw4 ? tile_fft_kernel<S, E, OP_C2C, true> : tile_fft_kernel<S, E, OP_C2C, false>;
#if SIP_INST_SIGN < 0
        case OP_R2C_HALF:
            return tile_fft_kernel<S, E, OP_R2C_HALF, false>;
        case OP_R2C_PAIR:
            return tile_fft_kernel<S, E, OP_R2C_PAIR, false>;
#else
        case OP_C2R_HALF:
            return tile_fft_kernel<S, E, OP_C2R_HALF, false>;
        case OP_C2R_PAIR:
            return tile_fft_kernel<S, E, OP_C2R_PAIR, false>;
        case OP_PC:  // runs both FFT directions; instantiated once, under sign +1
            return tw4 ? tile_fft_kernel<S, E, OP_PC, true> : tile_fft_kernel<S, E, OP_PC, false>;
#endif
        default:
            return nullptr;
    }
}

}  // namespace sipfft
