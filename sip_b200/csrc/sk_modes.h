// Tile modes of the size-specialized kernels (sk_kernel.cuh).  Free of host
// headers so that the runtime compiler (jit.cpp) can include it.
#pragma once

namespace sipfft {

enum SkMode : int {
    SK_ROWS = 0,    // transforms are contiguous rows; the tile is one contiguous run
    SK_COLS = 1,    // transforms are adjacent columns (in_idist = out_idist = 1)
    SK_ROWS_T = 2,  // contiguous rows in, adjacent columns out (four-step pass B)
};

}  // namespace sipfft
