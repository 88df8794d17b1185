// Tile modes of the size-specialized kernels (sk_kernel.cuh).  Free of host
// headers so that the runtime compiler (jit.cpp) can include it.
#pragma once

namespace sipfft {

enum SkMode : int {
    SK_ROWS = 0,    // transforms are contiguous rows; the tile is one contiguous run
    SK_COLS = 1,    // transforms are adjacent columns (in_idist = out_idist = 1)
    SK_ROWS_T = 2,  // contiguous rows in, adjacent columns out (four-step pass B)
};

// Bits of a configuration's TWB parameter (SkCfg):
//   SK_TW_BASIS     pass twiddles from the basis table (fewer loads, one
//                   product more) instead of the full Stockham table;
//   SK_TW_SMEM      the pass twiddle table and the real pre/post-process
//                   twiddles are copied to shared memory once per
//                   persistent CTA and read from there;
//   SK_MIRROR_PAIR  real tiles: the last pass of an R2C (first pass of a
//                   C2R) gives each thread butterfly u and its mirror
//                   NR - u, so that the post-process (pre-process) runs on
//                   registers (sk_pair_last_r2c, SkPairFirstC2R); in the
//                   real four-step's pass B, butterfly j of a row and
//                   butterfly NR - 1 - j of its mirror row
//                   (sk_pair_last_r2c_4b);
//   SK_SPLIT_PASS0  pass 0 reads the staging buffer and writes the work
//                   layout into the other buffer, one butterfly (pair) at a
//                   time instead of all of them across a barrier; the next
//                   tile is staged after pass 0 (overlapping the later
//                   passes) instead of before it.
enum : int { SK_TW_BASIS = 1, SK_TW_SMEM = 2, SK_MIRROR_PAIR = 4, SK_SPLIT_PASS0 = 8 };

}  // namespace sipfft
