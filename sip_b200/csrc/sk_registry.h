// Registry of the compiled size-specialized tile kernels (sk_configs.h).
#pragma once

#include <vector>

namespace sipfft {

enum SkMode : int {
    SK_ROWS = 0,    // transforms are contiguous rows; the tile is one contiguous run
    SK_COLS = 1,    // transforms are adjacent columns (in_idist = out_idist = 1)
    SK_ROWS_T = 2,  // contiguous rows in, adjacent columns out (four-step pass B)
};

struct SkEntry {
    int n, P, T, op, mode, sign;
    bool tw4;
    bool twb;  // basis pass twiddles (else the full Stockham table)
    int stages;
    std::vector<int> radices;
    int LD;
    int smem;        // dynamic shared memory per CTA (bytes)
    const void* fn;  // kernel (library) or CPU runner (test harness)
    int order = 0;   // position in the SIP_SK_CONFIGS list
};

// The `variant`-th entry compiled for (op, mode, sign, tw4, n) in
// SIP_SK_CONFIGS order (0: the default); the default when that variant is
// not compiled; nullptr when no entry is.
const SkEntry* sk_find(int op, int mode, int sign, bool tw4, int n, int variant = 0);

const std::vector<SkEntry>& sk_registry();

}  // namespace sipfft
