// Size-specialized tile FFT kernels ("sk").
//
// Same algorithm as the generic tile kernel (fft_core.cuh passes,
// tile_io.cuh operand layouts) with every size known at compile time:
// transform length N, radix sequence, transforms per tile P, threads T,
// operation and tile mode.  All index arithmetic folds to constants or
// shifts, each pass is inlined with exactly its own registers, and the
// kernel is persistent with a two-stage shared-memory pipeline:
//
//   stage(it+1): cp.async 16/8/4-byte copies of the next tile's input into
//                the other buffer (issued before the current tile's passes)
//   pass 0:      reads the staged tile in its input layout (applying the
//                real-transform pre-processing on the fly), writes the padded
//                work layout
//   pass 1..m-2: shared memory -> registers -> shared memory
//   pass m-1:    registers -> global memory (coalesced), or -> shared memory
//                followed by the real-transform post-process for R2C
//
// Phase functions are __host__ __device__ and take (tid, T) so the CPU
// harness (tests/native/tile_emu.cpp) runs them thread by thread.
#pragma once

#include "fft_core.cuh"
#include "sk_modes.h"
#include "tile_io.cuh"

namespace sipfft {

// Tile layout of a configuration as plain functions of its parameters, so
// that the runtime compiler's host side (jit.cpp) sizes a tile exactly as
// SkCfg does.  Odd first radices write conflict-free unpadded; even ones
// need a pad slot every max(16, R0) values (radix-32 strides need one per 32).
SIP_HD constexpr int sk_pad_group(int r0) { return r0 > 16 ? r0 : 16; }
SIP_HD constexpr int sk_index(int n, int r0) { return r0 % 2 == 0 ? n + n / sk_pad_group(r0) : n; }
// Work-layout pitch: element n of transform q at q * LD + sk_index(n), LD odd.
SIP_HD constexpr int sk_pitch(int n, int r0) {
    return ((sk_index(n - 1, r0) + 1) & 1) ? sk_index(n - 1, r0) + 1 : sk_index(n - 1, r0) + 2;
}
// The TWB bits (SK_TW_BASIS, SK_TW_SMEM, SK_MIRROR_PAIR, SK_SPLIT_PASS0) are
// defined in sk_modes.h.

SIP_HD constexpr int sk_twcount(int r, bool basis) { return basis ? basis_count(r) : r - 1; }
// Entries per table row of pass p in shared memory: all L values k of the
// span, or k <= L/2 for the mirrored last pass of an R2C tile (its butterfly
// pairs read only those).
SIP_HD constexpr int sk_tws_stride(int op, int flags, int p, int np, int L) {
    return ((flags & SK_MIRROR_PAIR) && (op == OP_R2C_HALF || op == OP_R2C_PAIR) && p == np - 1) ? L / 2 + 1 : L;
}
// Real pre/post-process twiddles W_{2M}^k staged in shared memory (k < count).
SIP_HD constexpr int sk_tw2s(int op, int n, int r0, int rlast, int flags) {
    return !(flags & SK_TW_SMEM) ? 0
         : op == OP_R2C_HALF ? ((flags & SK_MIRROR_PAIR) ? n / rlast / 2 + 1 : n / 2 + 1)
         : op == OP_C2R_HALF ? ((flags & SK_MIRROR_PAIR) ? n / r0 / 2 + 1 : n / r0)
         : 0;
}
// Complex values of shared memory the staged twiddles take (even count).
SIP_HD constexpr int sk_tws_values(int op, int n, const int* rs, int np, int flags) {
    int total = 0, L = 1;
    for (int p = 0; p < np; ++p) {
        if (L > 1) total += sk_twcount(rs[p], (flags & SK_TW_BASIS) != 0) * sk_tws_stride(op, flags, p, np, L);
        L *= rs[p];
    }
    total += sk_tw2s(op, n, rs[0], rs[np - 1], flags);
    return (flags & SK_TW_SMEM) ? (total + 1) / 2 * 2 : 0;
}

// Staged input values (complex64 units) per tile.
SIP_HD constexpr int sk_stage_values(int op, int p, int n) {
    return op == OP_C2R_HALF ? p * (n + 1)
         : op == OP_R2C_4B ? p * n
         : op == OP_C2R_4A ? (p + 2) * n  // sk_c2r4a_at: each row H columns, then a span of H + 2
         : op == OP_C2R_PAIR ? p * (n + 1)
         : p * n;  // R2C pair: 2P rows of N floats = P*N complex slots
}
// Complex values per buffer, rounded up to an even count so that the
// second buffer starts on a 16-byte boundary (cp.async 16-byte copies).
SIP_HD constexpr int sk_buffer_values(int op, int p, int n, int r0) {
    return ((sk_stage_values(op, p, n) > p * sk_pitch(n, r0) ? sk_stage_values(op, p, n) : p * sk_pitch(n, r0)) + 1) /
           2 * 2;
}

template <int N_, int P_, int T_, int OP_, int MODE_, int SIGN_, bool TW4_, int MINB_, int TWB_, int... Rs>
struct SkCfg {
    static constexpr int N = N_;
    static constexpr int P = P_;
    static constexpr int T = T_;
    static constexpr int OP = OP_;
    static constexpr int MODE = MODE_;
    static constexpr int SIGN = SIGN_;
    static constexpr bool TW4 = TW4_;
    static constexpr int NP = sizeof...(Rs);

    static constexpr int radix(int p) {
        constexpr int r[] = {Rs...};
        return r[p];
    }
    static constexpr int span(int p) {  // product of the radices before pass p
        int l = 1;
        for (int i = 0; i < p; ++i) l *= radix(i);
        return l;
    }
    // Pass twiddles: SK_TW_BASIS reads the basis table (fft_core.cuh
    // basis_split: fewer loads, one extra product), else the full
    // Stockham table (one load per twiddle, fewer instructions).
    static constexpr int FLAGS = TWB_;
    static constexpr bool TWB = (TWB_ & SK_TW_BASIS) != 0;
    static constexpr bool TWS = (TWB_ & SK_TW_SMEM) != 0;
    static constexpr bool MPAIR = (TWB_ & SK_MIRROR_PAIR) != 0;
    static constexpr bool SPLIT = (TWB_ & SK_SPLIT_PASS0) != 0;
    // The configuration's own operation (SkView below re-labels OP for the
    // halves of a pulse tile; the staged twiddle layout follows CFG_OP).
    static constexpr int CFG_OP = OP_;
    static constexpr int twcount(int r) { return TWB ? basis_count(r) : r - 1; }
    static constexpr int twoff(int p) {  // offset of pass p in the twiddle table
        int off = 0;
        for (int i = 0; i < p; ++i)
            if (span(i) > 1) off += span(i) * twcount(radix(i));
        return off;
    }
    static constexpr int tw_entries() { return twoff(NP); }
    static constexpr int idx(int n) { return sk_index(n, radix(0)); }
    static constexpr bool colmap(int p) {
        return MODE == SK_COLS || (MODE == SK_ROWS_T && p == NP - 1 && OP == OP_C2C);
    }
    // Mirrored-tile ops: slots [0, H) hold rows / columns c*H + q of the first
    // half, slots [H, 2H) their mirrors (sk_mirror_*).
    static constexpr bool MIRROR = OP == OP_R2C_4B || OP == OP_C2R_4A;
    static constexpr int H = P / 2;
    static constexpr int slots(int p) { return (P * (N / radix(p)) + T - 1) / T; }

    static constexpr int LD = sk_pitch(N, radix(0));
    static constexpr int STAGE = sk_stage_values(OP, P, N);
    static constexpr int BUF = sk_buffer_values(OP, P, N, radix(0));
    // Staged twiddles (SK_TW_SMEM): per pass p with span > 1, twcount rows
    // of tws_stride(p) entries from tws_off(p), then TW2S real twiddles.
    static constexpr int tws_stride(int p) { return sk_tws_stride(CFG_OP, FLAGS, p, NP, span(p)); }
    static constexpr int tws_off(int p) {
        int off = 0;
        for (int i = 0; i < p; ++i)
            if (span(i) > 1) off += twcount(radix(i)) * tws_stride(i);
        return off;
    }
    static constexpr int TW2_OFF = tws_off(NP);
    static constexpr int TW2S = sk_tw2s(CFG_OP, N, radix(0), radix(NP - 1), FLAGS);
    static constexpr int TWSM = TWS ? (TW2_OFF + TW2S + 1) / 2 * 2 : 0;
    static constexpr int SMEM = 2 * BUF * 8 + TWSM * 8;
    // CTAs per SM the shared memory allows with two stages (228 KB per SM,
    // 1 KB reserved per CTA); used as the register-allocation target.
    static constexpr int smem_ctas(int stages) {
        const int per = stages * BUF * 8 + 1024;
        const int n = (228 * 1024) / per;
        return n < 1 ? 1 : n;
    }
    // Minimum resident CTAs per SM (register-allocation target), chosen
    // per configuration so that the kernel does not spill.
    static constexpr int MINB = MINB_;
    // Pass 0 reads the staged input (false) or the work layout (true: the
    // inverse half of a pulse-compression tile, SkView below).
    static constexpr bool WORK_IN = false;

    static_assert(span(NP) == N, "radices must multiply to N");
    static_assert(!(TW4 && OP != OP_C2C && OP != OP_PC), "cross twiddles are C2C / pulse only");
    static_assert(!MPAIR || ((((OP == OP_R2C_HALF || OP == OP_C2R_HALF || OP == OP_R2C_PAIR || OP == OP_C2R_PAIR) &&
                               MODE == SK_ROWS) ||
                              (OP == OP_R2C_4B && MODE == SK_ROWS_T) || (OP == OP_C2R_4A && MODE == SK_COLS)) &&
                             NP >= 2),
                  "mirrored butterfly pairs: real rows, or mirrored four-step rows, of two or more passes");
    static_assert(!MPAIR || (OP != OP_R2C_HALF && OP != OP_R2C_PAIR) || SIGN < 0,
                  "R2C tiles run the forward transform");
    static_assert(!MPAIR || (OP != OP_C2R_HALF && OP != OP_C2R_PAIR) || SIGN > 0,
                  "C2R tiles run the inverse transform");
    static_assert(!SPLIT || (NP >= 2 && OP != OP_PC), "a split pass 0 needs a later pass, and no pulse tile");
    static constexpr int rad_list[] = {Rs...};
    static_assert(TWSM == sk_tws_values(OP_, N_, rad_list, NP, TWB_), "staged twiddle layout");
};

// A configuration seen with another operation, direction and pass-0 source:
// the two halves of an OP_PC tile run the same radix passes as
// SkView<K, OP_PC, -1, false> (forward, staged input, last pass to shared
// memory) and SkView<K, OP_C2C, +1, true> (inverse, from the work layout,
// last pass to global memory with the C2C epilogue).
template <class K, int OP_, int SIGN_, bool WORK_IN_>
struct SkView : K {
    static constexpr int OP = OP_;
    static constexpr int SIGN = SIGN_;
    static constexpr bool WORK_IN = WORK_IN_;
};

// ------------------------------------------------------------ twiddles
// Entry t (1-based row of the basis or full table) at span index k of pass
// PASS: from shared memory (SK_TW_SMEM) or through the read-only cache.
template <class K, int PASS>
SIP_HD float2 sk_ptw(const TileArgs& a, const TileCtx& c, int t, int k) {
    if constexpr (K::TWS)
        return c.tws[K::tws_off(PASS) + (t - 1) * K::tws_stride(PASS) + k];
    else
        return SIP_LDG(a.tw + K::twoff(PASS) + (t - 1) * K::span(PASS) + k);
}

// Real pre/post-process twiddle W_{2M}^k (the tile's tw2 root table).
template <class K>
SIP_HD float2 sk_tw2(const TileArgs& a, const TileCtx& c, int k) {
    if constexpr (K::TWS && K::TW2S > 0)
        return c.tws[K::TW2_OFF + k];
    else
        return SIP_LDG(a.tw2 + k);
}

// w[r] = W_{L R}^{r k} for 1 <= r < R (forward values; w[0] is unused):
// one table load each, or basis products W^{r_lo k} W^{a r_hi k}.
template <class K, int PASS, int R>
SIP_HD void sk_pass_twiddles(const TileArgs& a, const TileCtx& c, int k, float2 (&w)[R]) {
    if constexpr (!K::TWB) {
#pragma unroll
        for (int r = 1; r < R; ++r) w[r] = sk_ptw<K, PASS>(a, c, r, k);
    } else {
        constexpr int A = basis_split(R);
        float2 lo[A], hi[R / A];
        lo[0] = make_float2(1.f, 0.f);
        hi[0] = make_float2(1.f, 0.f);
#pragma unroll
        for (int t = 1; t < A; ++t) lo[t] = sk_ptw<K, PASS>(a, c, t, k);
#pragma unroll
        for (int t = 1; t < R / A; ++t) hi[t] = sk_ptw<K, PASS>(a, c, A - 1 + t, k);
#pragma unroll
        for (int r = 1; r < R; ++r) {
            const int rl = r % A, rh = r / A;
            w[r] = rh == 0 ? lo[rl] : rl == 0 ? hi[rh] : c_mul(lo[rl], hi[rh]);
        }
    }
}

// Copies the pass twiddles of passes P0.. and the real twiddles to shared
// memory (once per persistent CTA; a barrier follows before the first use).
template <class K, int P0>
SIP_HD void sk_load_tws_pass(int tid, const TileArgs& a, float2* tws) {
    if constexpr (P0 < K::NP) {
        if constexpr (K::span(P0) > 1) {
            constexpr int L = K::span(P0), ST = K::tws_stride(P0);
            constexpr int TOTAL = K::twcount(K::radix(P0)) * ST;
            for (int i = tid; i < TOTAL; i += K::T) {
                const int t = i / ST, k = i - t * ST;
                tws[K::tws_off(P0) + i] = a.tw[K::twoff(P0) + t * L + k];
            }
        }
        sk_load_tws_pass<K, P0 + 1>(tid, a, tws);
    }
}

template <class K>
SIP_HD void sk_load_tws(int tid, const TileArgs& a, float2* tws) {
    if constexpr (K::TWS) {
        sk_load_tws_pass<K, 1>(tid, a, tws);
        for (int k = tid; k < K::TW2S; k += K::T) tws[K::TW2_OFF + k] = a.tw2[k];
    }
}

// Column index of slot q of a C2R_4A tile (-1 when the slot is unused).
template <class K>
SIP_HD int sk_c2r4a_col(const TileArgs& a, int i0, int cnt, int q) {
    const int qq = q < K::H ? q : q - K::H;
    if (qq >= cnt) return -1;
    const int col0 = i0 + qq;
    if (q < K::H) return col0;
    if (col0 == 0 || 2 * col0 == a.n_other) return -1;
    return a.n_other - col0;
}

// ------------------------------------------------------------ staging
// Copies the tile's input into `stage` (byte-exact image of the input
// layout: rows [q][n] for the row modes, [n][q] for SK_COLS).
SIP_HD void sk_copy_run(int tid, int T, float2* stage_base, int stage_off_bytes, const char* src, long long bytes) {
    char* dst = reinterpret_cast<char*>(stage_base) + stage_off_bytes;
    const uintptr_t a = reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst) | (uintptr_t)bytes;
    const int g = (a & 15) == 0 ? 16 : (a & 7) == 0 ? 8 : 4;
    const long long chunks = bytes / g;
    for (long long c = tid; c < chunks; c += T) {
#if defined(__CUDA_ARCH__)
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst + c * g);
        if (g == 16)
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src + c * g));
        else if (g == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src + c * g));
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src + c * g));
#else
        for (int b = 0; b < g; ++b) dst[c * g + b] = src[c * g + b];
#endif
    }
}

template <class K>
SIP_HD void sk_stage(int tid, const TileArgs& a, const TileCtx& c, float2* stage) {
    constexpr int T = K::T;
    const char* src = static_cast<const char*>(a.src);
    if constexpr (K::MODE == SK_COLS && !K::MIRROR) {
        // [n][q]: one run of cnt adjacent columns per element index n
        const char* base = src + c.in_base * 8;
        const long long pitch = a.in_stride * 8;
        const uintptr_t align = reinterpret_cast<uintptr_t>(base) | (uintptr_t)pitch | (uintptr_t)(c.cnt * 8) |
                                reinterpret_cast<uintptr_t>(stage) | (uintptr_t)(K::P * 8);
        const int g = (align & 15) == 0 ? 16 : 8;
        const int cpr = c.cnt * 8 / g;  // chunks per run
        const int total = K::N * cpr;
        char* dst = reinterpret_cast<char*>(stage);
        for (int ch = tid; ch < total; ch += T) {
            const int n = ch / cpr;
            const int cc = ch - n * cpr;
            const char* s = base + n * pitch + cc * g;
            char* d = dst + n * (K::P * 8) + cc * g;
#if defined(__CUDA_ARCH__)
            const unsigned da = (unsigned)__cvta_generic_to_shared(d);
            if (g == 16)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(da), "l"(s));
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(da), "l"(s));
#else
            for (int b = 0; b < g; ++b) d[b] = s[b];
#endif
        }
    } else if constexpr (K::OP == OP_R2C_4B) {
        // rows k1 = i0 + q (slot q) and N1 - k1 (slot H + q) of Y, N values each
        const int n1 = a.n_other;
        const char* ybase = src + (c.in_base - (long long)c.i0 * K::N) * 8;  // row 0 of this batch row
        // 16-byte copies when the rows are 16-byte aligned (a workspace from
        // cudaMalloc), 8-byte copies otherwise
        const int g = ((reinterpret_cast<uintptr_t>(ybase) | reinterpret_cast<uintptr_t>(stage)) & 15) == 0 ? 16 : 8;
        const int cpr = K::N * 8 / g;  // chunks per row
        for (int ch = tid; ch < K::P * cpr; ch += T) {
            const int slot = ch / cpr;
            const int cc = ch - slot * cpr;
            const int q = slot < K::H ? slot : slot - K::H;
            const int k1 = c.i0 + q;
            if (q >= c.cnt) continue;
            int row = k1;
            if (slot >= K::H) {
                if (k1 == 0 || 2 * k1 == n1) continue;  // self-mirrored rows
                row = n1 - k1;
            }
            const char* s = ybase + (long long)row * K::N * 8 + cc * g;
            char* d = reinterpret_cast<char*>(stage) + slot * K::N * 8 + cc * g;
#if defined(__CUDA_ARCH__)
            const unsigned da = (unsigned)__cvta_generic_to_shared(d);
            if (g == 16)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(da), "l"(s));
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(da), "l"(s));
#else
            for (int b = 0; b < g; ++b) d[b] = s[b];
#endif
        }
    } else if constexpr (K::OP == OP_C2R_4A) {
        // Row n1 of the tile: the H columns i0 .. i0 + H - 1 (one run) and
        // the span of mirror columns N2 - i0 - H .. N2 - i0 + 1 (one run of
        // H + 2; of H for i0 = 0, whose mirror of column 0 is column 0
        // itself), in 16-byte copies when the batch row is 16-byte aligned
        // (sk_c2r4a_at reads them).  Columns past the tile's count stay
        // inside the row and are not used.
        static_assert(K::H % 2 == 0, "mirror spans start on an even column");
        constexpr int SP = K::P + 2;
        const int n2c = a.n_other;
        const char* xbase = src + (c.in_base - c.i0) * 8;  // X[0] of this batch row
        const int g = ((reinterpret_cast<uintptr_t>(xbase) & 15) == 0 && n2c % 2 == 0) ? 16 : 8;
        const int ms0 = n2c - c.i0 - K::H;
        const int cf = K::H * 8 / g;
        const int cm = (c.i0 == 0 ? K::H : K::H + 2) * 8 / g;
        const int per = cf + cm;
        for (int ch = tid; ch < K::N * per; ch += T) {
            const int n1 = ch / per;
            int k = ch - n1 * per;
            const char* s;
            char* d;
            if (k < cf) {
                s = xbase + ((long long)n1 * n2c + c.i0) * 8 + k * g;
                d = reinterpret_cast<char*>(stage) + (n1 * SP) * 8 + k * g;
            } else {
                k -= cf;
                s = xbase + ((long long)n1 * n2c + ms0) * 8 + k * g;
                d = reinterpret_cast<char*>(stage) + (n1 * SP + K::H) * 8 + k * g;
            }
#if defined(__CUDA_ARCH__)
            const unsigned da = (unsigned)__cvta_generic_to_shared(d);
            if (g == 16)
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(da), "l"(s));
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(da), "l"(s));
#else
            for (int b = 0; b < g; ++b) d[b] = s[b];
#endif
        }
    } else if constexpr (K::OP == OP_R2C_PAIR) {
        const int r0 = 2 * c.i0;
        const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
        sk_copy_run(tid, T, stage, 0, src + (long long)r0 * a.in_idist * 4, (long long)nrows * K::N * 4);
    } else if constexpr (K::OP == OP_C2R_PAIR) {
        const int r0 = 2 * c.i0;
        const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
        sk_copy_run(tid, T, stage, 0, src + (long long)r0 * a.in_idist * 8, (long long)nrows * (K::N / 2 + 1) * 8);
    } else {
        int rowlen = K::OP == OP_C2R_HALF ? K::N + 1 : K::N;
        if (K::OP == OP_PC && (a.flags & TF_BLUE)) rowlen = a.n_other;
        sk_copy_run(tid, T, stage, 0, src + c.in_base * 8, (long long)c.cnt * rowlen * 8);
    }
}

// The partner of the last real row of an odd batch is zero (pair ops).
template <class K>
SIP_HD void sk_zero_missing(int tid, const TileArgs& a, const TileCtx& c, float2* stage) {
    if constexpr (K::OP == OP_R2C_PAIR || K::OP == OP_C2R_PAIR) {
        const int r0 = 2 * c.i0;
        const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
        if (nrows & 1) {
            if constexpr (K::OP == OP_R2C_PAIR) {
                float* s = reinterpret_cast<float*>(stage) + (long long)nrows * K::N;
                for (int n = tid; n < K::N; n += K::T) s[n] = 0.f;
            } else {
                float2* s = stage + (long long)nrows * (K::N / 2 + 1);
                for (int n = tid; n < K::N / 2 + 1; n += K::T) s[n] = make_float2(0.f, 0.f);
            }
        }
    }
}

// Staged element of row n1 in slot `slot`: columns i0 + q at [0, H), the
// mirror column N2 - (i0 + q) of slot H + q at 2H - q of the mirror span.
template <class K>
SIP_HD float2 sk_c2r4a_at(const float2* stage, int n1, int slot) {
    const float2* row = stage + n1 * (K::P + 2);
    return slot < K::H ? row[slot] : row[3 * K::H - slot];
}

// C2R_4A pass-0 input: Z[k] = E + i W_{2M}^{+k} D, k = n1 N2 + n2, from X[k]
// and X[M-k] (M = N1 N2; the partner sits in the mirror column, row
// N1-1-n1, or in the same column for n2 = 0 and n2 = N2/2; X[M] itself is
// read from global memory).  The split table a.tw2 holds W_{2M}.
template <class K>
SIP_HD float2 sk_c2r4a_input(const TileArgs& a, const TileCtx& c, const float2* stage, int slot, int n1) {
    const int n2c = a.n_other;
    const int col = sk_c2r4a_col<K>(a, c.i0, c.cnt, slot);
    if (col < 0) return make_float2(0.f, 0.f);
    const long long M = (long long)K::N * n2c;
    const bool cj = (a.flags & TF_CONJ_IN) != 0;
    float2 x = maybe_conj(sk_c2r4a_at<K>(stage, n1, slot), cj);
    float2 y;
    if (col == 0) {
        if (n1 == 0) {
            const float2* xrow = static_cast<const float2*>(a.src) + (c.in_base - c.i0);
            const float ny = SIP_LDG(xrow + M).x;
            return make_float2(0.5f * (x.x + ny), 0.5f * (x.x - ny));
        }
        y = sk_c2r4a_at<K>(stage, K::N - n1, slot);
    } else if (2 * col == n2c) {
        y = sk_c2r4a_at<K>(stage, K::N - 1 - n1, slot);
    } else {
        const int ms = slot < K::H ? slot + K::H : slot - K::H;
        y = sk_c2r4a_at<K>(stage, K::N - 1 - n1, ms);
    }
    y = maybe_conj(y, cj);
    const long long kk = (long long)n1 * n2c + col;
    const float2 e = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
    const float2 d = make_float2(0.5f * (x.x - y.x), 0.5f * (x.y + y.y));
    const float2 od = c_mulc(d, cross_tw(a, kk));
    return make_float2(e.x - od.y, e.y + od.x);
}

// Value n of transform q as pass 0 reads it from the staged input.
template <class K>
SIP_HD float2 sk_input(const TileArgs& a, const TileCtx& c, const float2* stage, int q, int n) {
    constexpr int N = K::N;
    if constexpr (K::OP == OP_PC) {
        if (a.flags & TF_BLUE) {  // Bluestein: chirp times the input, zero padded
            const int nb = a.n_other;
            return n < nb ? c_mul(stage[q * nb + n], SIP_LDG(a.tw2 + n)) : make_float2(0.f, 0.f);
        }
        return stage[q * N + n];
    } else if constexpr (K::OP == OP_C2C) {
        const float2 v = K::MODE == SK_COLS ? stage[n * K::P + q] : stage[q * N + n];
        return maybe_conj(v, (a.flags & TF_CONJ_IN) != 0);
    } else if constexpr (K::OP == OP_R2C_HALF || K::OP == OP_R2C_4B) {
        return stage[q * N + n];
    } else if constexpr (K::OP == OP_C2R_4A) {
        return sk_c2r4a_input<K>(a, c, stage, q, n);
    } else if constexpr (K::OP == OP_R2C_PAIR) {
        const float* s = reinterpret_cast<const float*>(stage);
        return make_float2(s[(2 * q) * N + n], s[(2 * q + 1) * N + n]);
    } else if constexpr (K::OP == OP_C2R_HALF) {
        // Z[n] = E + i W_{2M}^{+n} D from X[n], X[M-n] (DC / Nyquist use real parts only)
        const float2* row = stage + q * (N + 1);
        const bool cj = (a.flags & TF_CONJ_IN) != 0;
        if (n == 0) {
            const float dc = row[0].x, ny = row[N].x;
            return make_float2(0.5f * (dc + ny), 0.5f * (dc - ny));
        }
        const float2 x = maybe_conj(row[n], cj), y = maybe_conj(row[N - n], cj);
        const float2 e = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
        const float2 d = make_float2(0.5f * (x.x - y.x), 0.5f * (x.y + y.y));
        const float2 od = c_mulc(d, sk_tw2<K>(a, c, n));
        return make_float2(e.x - od.y, e.y + od.x);
    } else {  // OP_C2R_PAIR
        constexpr int H = N / 2 + 1;
        const int kk = n <= N / 2 ? n : N - n;
        float2 xa = stage[(2 * q) * H + kk];
        float2 xb = stage[(2 * q + 1) * H + kk];
        if (kk == 0 || 2 * kk == N) {
            xa.y = 0.f;
            xb.y = 0.f;
        }
        if ((n > N / 2) != ((a.flags & TF_CONJ_IN) != 0)) {
            xa.y = -xa.y;
            xb.y = -xb.y;
        }
        return make_float2(xa.x - xb.y, xa.y + xb.x);
    }
}

// Compile-time loop: f(SkIC<I>{}) for I in [B, E), so that the index can be a
// template argument (the compile-time roots of tw_const).
template <int V>
struct SkIC {
    static constexpr int value = V;
};
template <int I, int E, class F>
SIP_HD void sk_static_for(F&& f) {
    if constexpr (I < E) {
        f(SkIC<I>{});
        sk_static_for<I + 1, E>(f);
    }
}

// ------------------------------------------------------------- passes
template <class K, int PASS>
struct SkPass {
    static constexpr int R = K::radix(PASS);
    static constexpr int L = K::span(PASS);
    static constexpr int NR = K::N / R;
    static constexpr int S = K::slots(PASS);
    static constexpr int TOTAL = K::P * NR;
    static constexpr bool COL = K::colmap(PASS);
    static constexpr bool LAST = PASS == K::NP - 1;
    using Regs = PassRegs<R, S>;

    SIP_HD static void butterfly_index(int b, int& q, int& j) {
        if (COL) {
            q = b % K::P;
            j = b / K::P;
        } else {
            q = b / NR;
            j = b % NR;
        }
    }

    // Reads (pass 0: from the staged input) and transforms butterfly slot s
    // of this thread; false when the slot has no butterfly.
    SIP_HD static bool read_slot(int tid, int s, const TileArgs& a, const TileCtx& c, const float2* buf,
                                 float2 (&v)[R]) {
        const int b = tid + s * K::T;
        if (TOTAL % K::T != 0 && b >= TOTAL) return false;
        int q, j;
        butterfly_index(b, q, j);
        if constexpr (PASS == 0 && !K::WORK_IN && K::OP == OP_C2R_HALF) {
            // C2R pre-process: the twiddle of element n = j + r NR is
            // W_{2M}^{j + r NR} = W_{2M}^j W_{2R}^r, one table entry per
            // butterfly times compile-time constants
            const float2 wj = sk_tw2<K>(a, c, j);
            const float2* row = buf + q * (K::N + 1);
            const bool cj = (a.flags & TF_CONJ_IN) != 0;
            sk_static_for<0, R>([&](auto ic) {
                constexpr int r = decltype(ic)::value;
                const int n = j + r * NR;
                if (n == 0) {
                    const float dc = row[0].x, ny = row[K::N].x;
                    v[r] = make_float2(0.5f * (dc + ny), 0.5f * (dc - ny));
                } else {
                    const float2 x = maybe_conj(row[n], cj), y = maybe_conj(row[K::N - n], cj);
                    const float2 e = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
                    const float2 d = make_float2(0.5f * (x.x - y.x), 0.5f * (x.y + y.y));
                    const float2 od = c_mulc(d, tw_const<2 * R, r, -1>(wj));
                    v[r] = make_float2(e.x - od.y, e.y + od.x);
                }
            });
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                if constexpr (PASS == 0 && !K::WORK_IN)
                    v[r] = sk_input<K>(a, c, buf, q, j + r * NR);
                else
                    v[r] = buf[q * K::LD + K::idx(j + r * NR)];
            }
        }
        if constexpr (L > 1) {
            // twiddle-major tables: consecutive k of a warp read consecutive
            // entries
            float2 w[R];
            sk_pass_twiddles<K, PASS>(a, c, j % L, w);
#pragma unroll
            for (int r = 1; r < R; ++r) v[r] = c_tw<K::SIGN>(v[r], w[r]);
        }
        dft<R, K::SIGN>(v);
        return true;
    }

    // Writes butterfly slot s to the padded work layout.
    SIP_HD static void write_slot(int tid, int s, float2* buf, const float2 (&v)[R]) {
        const int b = tid + s * K::T;
        if (TOTAL % K::T != 0 && b >= TOTAL) return;
        int q, j;
        butterfly_index(b, q, j);
        const int o = (j / L) * L * R + j % L;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[q * K::LD + K::idx(o + r * L)] = v[r];
    }

    SIP_HD static void read(int tid, const TileArgs& a, const TileCtx& c, const float2* buf, Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) read_slot(tid, s, a, c, buf, rg.v[s]);
    }

    // Writes to the padded work layout (all passes except a global-storing last one).
    SIP_HD static void write_smem(int tid, float2* buf, const Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) write_slot(tid, s, buf, rg.v[s]);
    }

    // Last pass straight to global memory: element k = j + r N/R of transform q.
    SIP_HD static void write_global(int tid, const TileArgs& a, const TileCtx& c, const Regs& rg) {
        static_assert(LAST, "global store from the last pass only");
        const bool sc = (a.flags & TF_SCALE) != 0;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int b = tid + s * K::T;
            if (TOTAL % K::T == 0 || b < TOTAL) {
                int q, j;
                butterfly_index(b, q, j);
                if (!K::MIRROR && q >= c.cnt) continue;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int k = j + r * NR;
                    float2 v = rg.v[s][r];
                    if constexpr (K::OP == OP_C2C) {
                        if constexpr (K::WORK_IN) {  // inverse half of a pulse tile
                            if (a.flags & TF_BLUE) {  // Bluestein: outputs k < n_other times the chirp
                                if (k >= a.n_other) continue;
                                v = c_mul(v, SIP_LDG(a.tw2 + k));
                            }
                        }
                        if constexpr (K::TW4) v = c_tw<K::SIGN>(v, cross_tw(a, (long long)(c.i0 + q) * k));
                        if (sc) v = c_scale(v, a.scale);
                        v = maybe_conj(v, (a.flags & TF_CONJ_OUT) != 0);
                        static_cast<float2*>(a.dst)[c.out_base + (long long)q * a.out_idist + (long long)k * a.out_stride] = v;
                    } else if constexpr (K::OP == OP_C2R_4A) {
                        const int col = sk_c2r4a_col<K>(a, c.i0, c.cnt, q);
                        if (col < 0) continue;
                        v = c_tw<K::SIGN>(v, cross_tw(a, 2LL * col * k));
                        if (sc) v = c_scale(v, a.scale);
                        static_cast<float2*>(a.dst)[c.out_base - c.i0 + col + (long long)k * a.out_stride] = v;
                    } else if constexpr (K::OP == OP_C2R_HALF) {
                        const float f = 2.0f * (sc ? a.scale : 1.0f);
                        static_cast<float2*>(a.dst)[c.out_base + (long long)q * a.out_idist + k] = c_scale(v, f);
                    } else if constexpr (K::OP == OP_C2R_PAIR) {
                        const float f = sc ? a.scale : 1.0f;
                        const int row = 2 * (c.i0 + q);
                        float* d = static_cast<float*>(a.dst);
                        d[(long long)row * a.out_idist + k] = v.x * f;
                        if (row + 1 < a.rows) d[(long long)(row + 1) * a.out_idist + k] = v.y * f;
                    }
                }
            }
        }
    }
};

template <class K>
constexpr bool sk_last_to_smem() {
    return ((K::OP == OP_R2C_HALF || K::OP == OP_R2C_PAIR || K::OP == OP_R2C_4B) && !K::MPAIR) || K::OP == OP_PC;
}

// R2C value X[k] from Z[k] and Z[M-k] (formula of tile_io.cuh
// store_r2c_half) with W_{2M}^k from the split table.
SIP_HD float2 sk_r2c_value(const TileArgs& a, float2 z, float2 zm, long long k) {
    const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
    float2 x = c_add(ev, c_mul(cross_tw(a, k), od));
    if (a.flags & TF_SCALE) x = c_scale(x, a.scale);
    return maybe_conj(x, (a.flags & TF_CONJ_OUT) != 0);
}

// X[k] and X[M - k] from Z[k], Z[M - k] with one twiddle: X[M - k] =
// conj(ev - W od) since W_{2M}^{M-k} = -conj(W_{2M}^k).
SIP_HD void sk_r2c_pair(const TileArgs& a, float2 z, float2 zm, long long k, float2* xk, float2* xmk) {
    const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
    const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
    const float2 t = c_mul(cross_tw(a, k), od);
    float2 x = c_add(ev, t);
    float2 y = make_float2(ev.x - t.x, t.y - ev.y);
    if (a.flags & TF_SCALE) {
        x = c_scale(x, a.scale);
        y = c_scale(y, a.scale);
    }
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    *xk = maybe_conj(x, cj);
    *xmk = maybe_conj(y, cj);
}

// R2C post-process from the work layout (formulas of tile_io.cuh
// store_r2c_half / store_r2c_pair), coalesced over the output rows.
template <class K>
SIP_HD void sk_post(int tid, const TileArgs& a, const TileCtx& c, const float2* buf) {
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    float2* dst = static_cast<float2*>(a.dst);
    if constexpr (K::OP == OP_R2C_HALF) {
        // one thread per pair (k, M - k), k in [0, M/2]: Z[k], Z[M - k] and
        // W_{2M}^k are read once; X[M - k] = conj(ev - W od) follows from
        // W_{2M}^{M-k} = -conj(W_{2M}^k).  k = 0 also gives X[M].
        constexpr int M = K::N, U = M / 2 + 1;
        const int total = c.cnt * U;
        for (int f = tid; f < total; f += K::T) {
            const int q = f / U;
            const int k = f - q * U;
            const float2* row = buf + q * K::LD;
            float2* out = dst + c.out_base + (long long)q * a.out_idist;
            const float2 z = row[K::idx(k)];
            const float2 zm = row[K::idx(k == 0 ? 0 : M - k)];
            const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            const float2 t = c_mul(sk_tw2<K>(a, c, k), od);
            float2 x = c_add(ev, t);
            if (sc) x = c_scale(x, a.scale);
            out[k] = maybe_conj(x, cj);
            if (k == 0) {  // X[M] = Re z0 - Im z0 (W_{2M}^M = -1)
                float2 xm = make_float2(ev.x - t.x, ev.y - t.y);
                if (sc) xm = c_scale(xm, a.scale);
                out[M] = maybe_conj(xm, cj);
            } else if (2 * k != M) {
                float2 xm = make_float2(ev.x - t.x, t.y - ev.y);
                if (sc) xm = c_scale(xm, a.scale);
                out[M - k] = maybe_conj(xm, cj);
            }
        }
    } else if constexpr (K::OP == OP_R2C_4B) {
        // rows k1 = i0 + q (slot q) and N1 - k1 (slot H + q) -> X[k1 + N1 k2]
        // and X[(N1 - k1) + N1 (N2 - 1 - k2)]; row 0 and row N1/2 pair with
        // themselves, row 0 also produces X[M].
        constexpr int N2 = K::N;
        const int N1 = a.n_other;
        const long long M = (long long)N1 * N2;
        float2* x = dst + (c.out_base - c.i0);
        for (int f = tid; f < K::H * N2; f += K::T) {
            const int q = f % K::H;
            const int k2 = f / K::H;
            if (q >= c.cnt) continue;
            const int k1 = c.i0 + q;
            const float2* rq = buf + q * K::LD;
            const float2* rm = buf + (K::H + q) * K::LD;
            const long long kk = k1 + (long long)N1 * k2;
            const float2 z = rq[K::idx(k2)];
            if (k1 == 0) {
                x[kk] = sk_r2c_value(a, z, rq[K::idx(k2 == 0 ? 0 : N2 - k2)], kk);
                if (k2 == 0) x[M] = sk_r2c_value(a, z, z, M);
            } else if (2 * k1 == N1) {
                x[kk] = sk_r2c_value(a, z, rq[K::idx(N2 - 1 - k2)], kk);
            } else {
                const float2 zm = rm[K::idx(N2 - 1 - k2)];
                sk_r2c_pair(a, z, zm, kk, x + kk, x + (M - kk));
            }
        }
    } else if constexpr (K::OP == OP_R2C_PAIR) {
        // one thread per bin k of a complex row: Z[k] and Z[N - k] give bin k
        // of both real rows (x_a = Re part, x_b = Im part of the packed row)
        constexpr int N = K::N, H = N / 2 + 1;
        const int r0 = 2 * c.i0;
        const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
        const int total = ((nrows + 1) >> 1) * H;
        for (int f = tid; f < total; f += K::T) {
            const int q = f / H;
            const int k = f - q * H;
            const float2* row = buf + q * K::LD;
            const float2 z = row[K::idx(k)];
            const float2 zm = row[K::idx(k == 0 ? 0 : N - k)];
            float2 xa = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            float2 xb = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            if (sc) {
                xa = c_scale(xa, a.scale);
                xb = c_scale(xb, a.scale);
            }
            const long long ra = r0 + 2 * q;
            dst[ra * a.out_idist + k] = maybe_conj(xa, cj);
            if (2 * q + 1 < nrows) dst[(ra + 1) * a.out_idist + k] = maybe_conj(xb, cj);
        }
    }
}

// ------------------------------------------------ mirrored butterfly pairs
// SK_MIRROR_PAIR for real half-length tiles of length M (the complex FFT
// of the packed row).  In a pass of radix R with NR = M / R butterflies and
// span NR (the last pass; the first pass reads the same index set), the
// elements of butterfly u are u + r NR and those of butterfly NR - u are
// their mirrors: M - (u + r NR) = (NR - u) + (R - 1 - r) NR, and for u = 0
// the mirror of r NR is (R - r) NR in the same butterfly (u = NR / 2 is its
// own mirror when NR is even).  One thread takes the pair (u, NR - u), u in
// [0, NR / 2], so each R2C output pair X[k], X[M - k] (each C2R input pair)
// meets in its registers: the post-process stores to global memory without
// another shared-memory round trip, and the pre-process reads every bin once.
// The mirror's pass twiddles W_M^{r (NR - u)} = W_R^r conj(W_M^{r u}) and the
// real twiddles W_{2M}^{u + r NR} = W_{2M}^u W_{2R}^r need table entries of
// u only, times compile-time constants.

// Last pass of an R2C_HALF tile, post-process fused, output to global memory.
template <class K>
SIP_HD void sk_pair_last_r2c(int tid, const TileArgs& a, const TileCtx& c, const float2* buf) {
    constexpr int PASS = K::NP - 1;
    constexpr int R = K::radix(PASS);
    constexpr int M = K::N;
    constexpr int NR = M / R;
    constexpr int U = NR / 2 + 1;
    constexpr int TOTAL = K::P * U;
    constexpr int S = (TOTAL + K::T - 1) / K::T;
    static_assert(K::span(PASS) == NR, "the last pass spans N / R");
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    float2* dst = static_cast<float2*>(a.dst);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) break;
        const int q = f / U;
        const int u = f - q * U;
        if (q >= c.cnt) continue;
        const bool mirror = u != 0 && 2 * u != NR;  // NR - u is another butterfly
        const float2* row = buf + q * K::LD;
        float2 A[R], B[R];
#pragma unroll
        for (int r = 0; r < R; ++r) A[r] = row[K::idx(u + r * NR)];
        if (mirror) {
#pragma unroll
            for (int r = 0; r < R; ++r) B[r] = row[K::idx(NR - u + r * NR)];
        }
        if (u != 0) {
            float2 w[R];
            sk_pass_twiddles<K, PASS>(a, c, u, w);
#pragma unroll
            for (int r = 1; r < R; ++r) A[r] = c_tw<K::SIGN>(A[r], w[r]);
            if (mirror)
                sk_static_for<1, R>([&](auto ic) {
                    constexpr int r = decltype(ic)::value;
                    B[r] = tw_const<R, r, K::SIGN>(c_tw<-K::SIGN>(B[r], w[r]));
                });
        }
        dft<R, K::SIGN>(A);
        if (mirror) dft<R, K::SIGN>(B);
        const float2 w2u = sk_tw2<K>(a, c, u);
        float2* out = dst + c.out_base + (long long)q * a.out_idist;
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            const int k = u + r * NR;
            const float2 z = A[r];
            const float2 zm = mirror ? B[R - 1 - r] : (u == 0 ? A[(R - r) % R] : A[R - 1 - r]);
            const float2 w2 = tw_const<2 * R, r, -1>(w2u);  // W_{2M}^k
            const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            const float2 t = c_mul(w2, od);
            float2 x = c_add(ev, t);
            float2 y = make_float2(ev.x - t.x, t.y - ev.y);  // X[M - k]
            if (sc) {
                x = c_scale(x, a.scale);
                y = c_scale(y, a.scale);
            }
            out[k] = maybe_conj(x, cj);
            // X[M - k] belongs to this thread when the mirror is another
            // butterfly; for u = 0 only X[M] (r = 0) is not stored as some X[k]
            if (mirror || (u == 0 && r == 0)) out[M - k] = maybe_conj(y, cj);
        });
    }
}

// Last pass of an R2C_4B tile (pass B of a real four-step: rows k1 = i0 + q
// in slots [0, H), their mirror rows N1 - k1 in slots [H, 2H)), post-process
// fused, output to global memory.  With NR = N2 / R, element r of butterfly
// j of row k1 is bin k2 = j + r NR, output index kk = k1 + N1 k2, whose
// mirror M - kk = (N1 - k1) + N1 (N2 - 1 - k2) is element R - 1 - r of
// butterfly NR - 1 - j of row N1 - k1.  One thread takes the unit (q, j):
// butterfly j of slot q and butterfly NR - 1 - j of slot H + q, and stores
// X[kk] and X[M - kk] for its R elements.  The two rows that are their own
// mirror take the partner butterfly from their own slot and store X[kk]
// only (the mirror bin is another unit's X[kk']): k1 = N1 / 2 (butterfly
// NR - 1 - j, element R - 1 - r) and k1 = 0 (bin N2 - k2: butterfly NR - j,
// element R - 1 - r, or for j = 0 element R - r of butterfly 0; the unit
// j = 0 also stores X[M]).  W_{2M}^{kk} = W_{2M}^{k1 + N1 j} W_{2R}^r: one
// split-table twiddle per unit times compile-time constants.
template <class K>
SIP_HD void sk_pair_last_r2c_4b(int tid, const TileArgs& a, const TileCtx& c, const float2* buf) {
    constexpr int PASS = K::NP - 1;
    constexpr int R = K::radix(PASS);
    constexpr int N2 = K::N;
    constexpr int NR = N2 / R;
    constexpr int H = K::H;
    constexpr int TOTAL = H * NR;
    constexpr int S = (TOTAL + K::T - 1) / K::T;
    static_assert(K::span(PASS) == NR, "the last pass spans N / R");
    const int N1 = a.n_other;
    const long long M = (long long)N1 * N2;
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    float2* x = static_cast<float2*>(a.dst) + (c.out_base - c.i0);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) break;
        const int q = f % H;  // consecutive threads: adjacent rows, so stores run along k1
        const int j = f / H;
        if (q >= c.cnt) continue;
        const int k1 = c.i0 + q;
        const bool row0 = k1 == 0, half = 2 * k1 == N1, self = row0 || half;
        const int jb = row0 ? (NR - j) % NR : NR - 1 - j;
        const float2* ra = buf + q * K::LD;
        const float2* rb = buf + (self ? q : H + q) * K::LD;
        float2 A[R], B[R];
#pragma unroll
        for (int r = 0; r < R; ++r) A[r] = ra[K::idx(j + r * NR)];
        if (j != 0) {
            float2 w[R];
            sk_pass_twiddles<K, PASS>(a, c, j, w);
#pragma unroll
            for (int r = 1; r < R; ++r) A[r] = c_tw<K::SIGN>(A[r], w[r]);
        }
        dft<R, K::SIGN>(A);
#pragma unroll
        for (int r = 0; r < R; ++r) B[r] = rb[K::idx(jb + r * NR)];
        if (jb != 0) {
            float2 w[R];
            sk_pass_twiddles<K, PASS>(a, c, jb, w);
#pragma unroll
            for (int r = 1; r < R; ++r) B[r] = c_tw<K::SIGN>(B[r], w[r]);
        }
        dft<R, K::SIGN>(B);
        const float2 w0 = cross_tw(a, k1 + (long long)N1 * j);  // W_{2M}^{k1 + N1 j}
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            const long long kk = k1 + (long long)N1 * (j + r * NR);
            const float2 z = A[r];
            const float2 zm = (row0 && j == 0) ? A[(R - r) % R] : B[R - 1 - r];
            const float2 w2 = tw_const<2 * R, r, -1>(w0);  // W_{2M}^{kk}
            const float2 ev = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            const float2 od = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            const float2 t = c_mul(w2, od);
            float2 xk = c_add(ev, t);
            float2 xm = make_float2(ev.x - t.x, t.y - ev.y);  // X[M - kk]; X[M] for kk = 0
            if (sc) {
                xk = c_scale(xk, a.scale);
                xm = c_scale(xm, a.scale);
            }
            x[kk] = maybe_conj(xk, cj);
            if (!self) x[M - kk] = maybe_conj(xm, cj);
            if (row0 && j == 0 && r == 0) x[M] = maybe_conj(xm, cj);
        });
    }
}

// First pass of a C2R_HALF tile from the staged bins X[0..M], pre-process
// fused: Z[n] = E + i W_{2M}^{+n} D and Z[M - n] from X[n], X[M - n].
template <class K>
struct SkPairFirstC2R {
    static constexpr int R = K::radix(0);
    static constexpr int M = K::N;
    static constexpr int NR = M / R;
    static constexpr int U = NR / 2 + 1;
    static constexpr int TOTAL = K::P * U;
    static constexpr int S = (TOTAL + K::T - 1) / K::T;
    struct Regs {
        float2 a[S][R], b[S][R];
    };

    // Z[n], Z[M - n] from x = X[n], y = X[M - n] and w = W_{2M}^n.
    SIP_HD static void prep(float2 x, float2 y, float2 w, float2& zn, float2& zm) {
        const float2 e = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
        const float2 d = make_float2(0.5f * (x.x - y.x), 0.5f * (x.y + y.y));
        const float2 od = c_mulc(d, w);
        zn = make_float2(e.x - od.y, e.y + od.x);
        zm = make_float2(e.x + od.y, od.x - e.y);
    }

    // Unit slot s of this thread: butterflies u (into A) and NR - u (into B),
    // pre-processed and transformed; false when the slot has no unit.
    SIP_HD static bool read_slot(int tid, int s, const TileArgs& a, const TileCtx& c, const float2* stage,
                                 float2 (&A)[R], float2 (&B)[R]) {
        const bool cj = (a.flags & TF_CONJ_IN) != 0;
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) return false;
        const int q = f / U;
        const int u = f - q * U;
        const float2* row = stage + q * (M + 1);
        const float2 wu = sk_tw2<K>(a, c, u);
        // One code path for every unit: element r of butterfly u is Z[n] from
        // (X[n], X[M - n]), n = u + r NR, and the same pair gives element
        // R - 1 - r of the mirror butterfly.  For u = 0 (and u = NR / 2) the
        // mirror is the butterfly itself, whose elements all come out of the
        // Z[n] side (each of its bins is read twice there); X[0] and X[M] enter
        // with their imaginary parts ignored, which turns the formula into
        // Z[0] = ((X0 + XM) / 2, (X0 - XM) / 2).
        const bool mirror = u != 0 && 2 * u != NR;
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            const int n = u + r * NR;
            float2 x = maybe_conj(row[n], cj), y = maybe_conj(row[M - n], cj);
            if (n == 0) {
                x.y = 0.f;
                y.y = 0.f;
            }
            prep(x, y, tw_const<2 * R, r, -1>(wu), A[r], B[R - 1 - r]);
        });
        if (mirror) dft<R, K::SIGN>(B);
        dft<R, K::SIGN>(A);
        return true;
    }

    // Pass 0 has span 1: butterfly j writes element r to j R + r.
    SIP_HD static void write_slot(int tid, int s, float2* buf, const float2 (&A)[R], const float2 (&B)[R]) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) return;
        const int q = f / U;
        const int u = f - q * U;
        float2* row = buf + q * K::LD;
#pragma unroll
        for (int r = 0; r < R; ++r) row[K::idx(u * R + r)] = A[r];
        if (u != 0 && 2 * u != NR) {
#pragma unroll
            for (int r = 0; r < R; ++r) row[K::idx((NR - u) * R + r)] = B[r];
        }
    }

    SIP_HD static void read(int tid, const TileArgs& a, const TileCtx& c, const float2* stage, Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) read_slot(tid, s, a, c, stage, rg.a[s], rg.b[s]);
    }

    SIP_HD static void write_smem(int tid, float2* buf, const Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) write_slot(tid, s, buf, rg.a[s], rg.b[s]);
    }
};

// Last pass of an R2C_PAIR tile (real rows 2q and 2q + 1 packed as one
// complex row Z of odd length N), the bin separation fused: bin b <= (N-1)/2
// of the two rows is (Z[b] + conj Z[N-b]) / 2 and (Z[b] - conj Z[N-b]) / 2i.
// For each element k of butterfly u the stored bin is min(k, N - k); its
// partner is the mirror butterfly's element R - 1 - r (u = 0: element R - r
// of the same butterfly, which stores only k = r NR <= (N-1)/2).
template <class K>
SIP_HD void sk_pair_last_r2c_rows(int tid, const TileArgs& a, const TileCtx& c, const float2* buf) {
    constexpr int PASS = K::NP - 1;
    constexpr int R = K::radix(PASS);
    constexpr int N = K::N;
    constexpr int NR = N / R;
    constexpr int U = NR / 2 + 1;
    constexpr int TOTAL = K::P * U;
    constexpr int S = (TOTAL + K::T - 1) / K::T;
    static_assert(N % 2 == 1 && K::span(PASS) == NR, "odd lengths; the last pass spans N / R");
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    float2* dst = static_cast<float2*>(a.dst);
    const int r0 = 2 * c.i0;
    const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) break;
        const int q = f / U;
        const int u = f - q * U;
        if (2 * q >= nrows) continue;
        const bool mirror = u != 0;  // NR is odd: no butterfly is its own mirror but u = 0
        const float2* row = buf + q * K::LD;
        float2 A[R], B[R];
#pragma unroll
        for (int r = 0; r < R; ++r) A[r] = row[K::idx(u + r * NR)];
        if (mirror) {
#pragma unroll
            for (int r = 0; r < R; ++r) B[r] = row[K::idx(NR - u + r * NR)];
            float2 w[R];
            sk_pass_twiddles<K, PASS>(a, c, u, w);
#pragma unroll
            for (int r = 1; r < R; ++r) A[r] = c_tw<K::SIGN>(A[r], w[r]);
            sk_static_for<1, R>([&](auto ic) {
                constexpr int r = decltype(ic)::value;
                B[r] = tw_const<R, r, K::SIGN>(c_tw<-K::SIGN>(B[r], w[r]));
            });
            dft<R, K::SIGN>(B);
        }
        dft<R, K::SIGN>(A);
        const long long ra = r0 + 2 * q;
        float2* outa = dst + ra * a.out_idist;
        float2* outb = outa + a.out_idist;
        const bool second = 2 * q + 1 < nrows;
        auto store = [&](int b, float2 z, float2 zm) {
            float2 xa = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
            float2 xb = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
            if (sc) {
                xa = c_scale(xa, a.scale);
                xb = c_scale(xb, a.scale);
            }
            outa[b] = maybe_conj(xa, cj);
            if (second) outb[b] = maybe_conj(xb, cj);
        };
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            if (mirror) {
                const int k = u + r * NR;
                if (2 * k < N) store(k, A[r], B[R - 1 - r]);
                else store(N - k, B[R - 1 - r], A[r]);
            } else if constexpr (2 * r * NR < N) {
                store(r * NR, A[r], A[(R - r) % R]);
            }
        });
    }
}

// Pass 0 of a C2R_4A tile (pass A of a real four-step: columns n2 = i0 + q
// in slots [0, H), their mirror columns N2 - n2 in slots [H, 2H)), the
// pre-process fused on mirrored butterfly pairs.  Bin n = n1 N2 + n2 of the
// half spectrum pairs with M - n = (N1 - 1 - n1) N2 + (N2 - n2): with NR =
// N1 / R, element r of butterfly j of column n2 (row n1 = j + r NR) pairs
// with element R - 1 - r of butterfly NR - 1 - j of the mirror column.  One
// thread takes the unit (q, j), reads both bins of each pair once, and
// forms Z[n] = E + i W_{2M}^{+n} D and Z[M - n] from them with one
// split-table twiddle W_{2M}^{j N2 + n2} per unit times the constants
// W_{2R}^r, then runs both butterflies.  The columns that are their own
// mirror (n2 = 0: rows n1 and N1 - n1, with X[M] for n1 = 0; n2 = N2 / 2:
// rows n1 and N1 - 1 - n1) read the partner bin from their own slot and
// form Z[n] only: every butterfly of such a column is some unit's first.
template <class K>
struct SkPairFirstC2R4A {
    static constexpr int R = K::radix(0);
    static constexpr int N1 = K::N;
    static constexpr int NR = N1 / R;
    static constexpr int H = K::H;
    static constexpr int TOTAL = H * NR;
    static constexpr int S = (TOTAL + K::T - 1) / K::T;
    static_assert(K::span(1) == R, "pass 0 has span 1");
    struct Regs {
        float2 a[S][R], b[S][R];
    };

    SIP_HD static bool unit(int tid, int s, const TileCtx& c, int& q, int& j) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) return false;
        q = f % H;  // consecutive threads: adjacent columns (contiguous in the staged rows)
        j = f / H;
        return q < c.cnt;
    }

    SIP_HD static bool read_slot(int tid, int s, const TileArgs& a, const TileCtx& c, const float2* stage,
                                 float2 (&A)[R], float2 (&B)[R]) {
        int q, j;
        if (!unit(tid, s, c, q, j)) return false;
        const int n2c = a.n_other;
        const int col = c.i0 + q;
        const bool col0 = col == 0, half = 2 * col == n2c, self = col0 || half;
        const bool cj = (a.flags & TF_CONJ_IN) != 0;
        const float2 w0 = cross_tw(a, (long long)j * n2c + col);  // W_{2M}^{j N2 + n2}
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            const int n1 = j + r * NR;
            const float2 x = maybe_conj(sk_c2r4a_at<K>(stage, n1, q), cj);
            if (col0 && n1 == 0) {  // Z[0] from the real parts of X[0] and X[M]
                const float2* xrow = static_cast<const float2*>(a.src) + (c.in_base - c.i0);
                const float ny = SIP_LDG(xrow + (long long)N1 * n2c).x;
                A[r] = make_float2(0.5f * (x.x + ny), 0.5f * (x.x - ny));
                return;
            }
            const int prow = col0 ? N1 - n1 : N1 - 1 - n1;
            const float2 y = maybe_conj(sk_c2r4a_at<K>(stage, prow, self ? q : H + q), cj);
            const float2 w = tw_const<2 * R, r, -1>(w0);  // W_{2M}^{n}
            const float2 e = make_float2(0.5f * (x.x + y.x), 0.5f * (x.y - y.y));
            const float2 d = make_float2(0.5f * (x.x - y.x), 0.5f * (x.y + y.y));
            const float2 od = c_mulc(d, w);
            A[r] = make_float2(e.x - od.y, e.y + od.x);           // Z[n]
            B[R - 1 - r] = make_float2(e.x + od.y, od.x - e.y);   // Z[M - n]
        });
        dft<R, K::SIGN>(A);
        if (!self) dft<R, K::SIGN>(B);
        return true;
    }

    // Pass 0 has span 1: butterfly j writes element r to j R + r.
    SIP_HD static void write_slot(int tid, int s, const TileArgs& a, const TileCtx& c, float2* buf,
                                  const float2 (&A)[R], const float2 (&B)[R]) {
        int q, j;
        if (!unit(tid, s, c, q, j)) return;
        const int col = c.i0 + q;
        float2* ra = buf + q * K::LD;
#pragma unroll
        for (int r = 0; r < R; ++r) ra[K::idx(j * R + r)] = A[r];
        if (col != 0 && 2 * col != a.n_other) {
            float2* rb = buf + (H + q) * K::LD;
            const int jb = NR - 1 - j;
#pragma unroll
            for (int r = 0; r < R; ++r) rb[K::idx(jb * R + r)] = B[r];
        }
    }

    SIP_HD static void read(int tid, const TileArgs& a, const TileCtx& c, const float2* stage, Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) read_slot(tid, s, a, c, stage, rg.a[s], rg.b[s]);
    }

    SIP_HD static void write_smem(int tid, const TileArgs& a, const TileCtx& c, float2* buf, const Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) write_slot(tid, s, a, c, buf, rg.a[s], rg.b[s]);
    }
};


// First pass of a C2R_PAIR tile from the staged spectra of real rows 2q and
// 2q + 1 (N/2 + 1 bins each): Z[n] = Xa[n] + i Xb[n] with the Hermitian
// halves, every staged bin read once (for bin m and its mirror N - m).
template <class K>
struct SkPairFirstC2RRows {
    static constexpr int R = K::radix(0);
    static constexpr int N = K::N;
    static constexpr int H = N / 2 + 1;
    static constexpr int NR = N / R;
    static constexpr int U = NR / 2 + 1;
    static constexpr int TOTAL = K::P * U;
    static constexpr int S = (TOTAL + K::T - 1) / K::T;
    static_assert(N % 2 == 1, "odd lengths");

    // Z[m] (lo) and Z[N - m] (hi) from bin m of both rows, m <= N/2.
    SIP_HD static void bins(const float2* sa, const float2* sb, int m, bool fwd, float2& lo, float2& hi) {
        float2 xa = sa[m], xb = sb[m];
        if (m == 0) {
            xa.y = 0.f;
            xb.y = 0.f;
        }
        const float2 plain = make_float2(xa.x - xb.y, xa.y + xb.x);    // Xa + i Xb
        const float2 mirr = make_float2(xa.x + xb.y, xb.x - xa.y);     // conj(Xa) + i conj(Xb)
        lo = fwd ? mirr : plain;
        hi = fwd ? plain : mirr;
    }

    SIP_HD static bool read_slot(int tid, int s, const TileArgs& a, const TileCtx& c, const float2* stage,
                                 float2 (&A)[R], float2 (&B)[R]) {
        const bool fwd = (a.flags & TF_CONJ_IN) != 0;
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) return false;
        const int q = f / U;
        const int u = f - q * U;
        const float2* sa = stage + (2 * q) * H;
        const float2* sb = sa + H;
        // one code path for every unit (u = 0 is its own mirror: B unused)
        sk_static_for<0, R>([&](auto ic) {
            constexpr int r = decltype(ic)::value;
            const int n = u + r * NR;
            const bool low = 2 * n < N;
            float2 lo, hi;
            bins(sa, sb, low ? n : N - n, fwd, lo, hi);
            A[r] = low ? lo : hi;
            B[R - 1 - r] = low ? hi : lo;
        });
        if (u != 0) dft<R, K::SIGN>(B);
        dft<R, K::SIGN>(A);
        return true;
    }

    SIP_HD static void write_slot(int tid, int s, float2* buf, const float2 (&A)[R], const float2 (&B)[R]) {
        const int f = tid + s * K::T;
        if (TOTAL % K::T != 0 && f >= TOTAL) return;
        const int q = f / U;
        const int u = f - q * U;
        float2* row = buf + q * K::LD;
#pragma unroll
        for (int r = 0; r < R; ++r) row[K::idx(u * R + r)] = A[r];
        if (u != 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) row[K::idx((NR - u) * R + r)] = B[r];
        }
    }

    struct Regs {
        float2 a[S][R], b[S][R];
    };

    SIP_HD static void read(int tid, const TileArgs& a, const TileCtx& c, const float2* stage, Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) read_slot(tid, s, a, c, stage, rg.a[s], rg.b[s]);
    }

    SIP_HD static void write_smem(int tid, float2* buf, const Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) write_slot(tid, s, buf, rg.a[s], rg.b[s]);
    }
};

// Type selection without the standard library (the run-time compiler has none).
template <bool B, class T, class F>
struct SkPick {
    using type = T;
};
template <class T, class F>
struct SkPick<false, T, F> {
    using type = F;
};

// Pass 0 of a SK_SPLIT_PASS0 tile: from the staging buffer `stage` into the
// work layout of the other buffer `work`, one slot at a time (no barrier
// between reading and writing, so only one slot's values are live).
template <class K>
SIP_HD void sk_pass0_split(int tid, const TileArgs& a, const TileCtx& c, const float2* stage, float2* work) {
    if constexpr (K::MPAIR && (K::OP == OP_C2R_HALF || K::OP == OP_C2R_PAIR)) {
        using PP = typename SkPick<K::OP == OP_C2R_HALF, SkPairFirstC2R<K>, SkPairFirstC2RRows<K>>::type;
#pragma unroll
        for (int s = 0; s < PP::S; ++s) {
            float2 A[PP::R], B[PP::R];
            if (PP::read_slot(tid, s, a, c, stage, A, B)) PP::write_slot(tid, s, work, A, B);
        }
    } else {
        using SP = SkPass<K, 0>;
#pragma unroll
        for (int s = 0; s < SP::S; ++s) {
            float2 v[SP::R];
            if (SP::read_slot(tid, s, a, c, stage, v)) SP::write_slot(tid, s, work, v);
        }
    }
}

// OP_PC: the spectra in the work layout times the filter spectrum, element
// k of transform q times mul[(i0 + q) * mul_pitch_p + k * mul_pitch_k]
// (conjugated under TF_MUL_CONJ), as tile_io.cuh mul_tile.
template <class K>
SIP_HD void sk_mul(int tid, const TileArgs& a, const TileCtx& c, float2* buf) {
    const bool cj = (a.flags & TF_MUL_CONJ) != 0;
    const int total = c.cnt * K::N;
    // B filter values per thread in flight at once: the filter comes from
    // L2, and one load per iteration would wait out its latency each time
    constexpr int B = 8;
    for (int f0 = tid; f0 < total; f0 += B * K::T) {
        float2 m[B];
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const int f = f0 + i * K::T;
            if (f < total) {
                const int q = f / K::N;
                const int k = f - q * K::N;
                m[i] = SIP_LDG(a.mul + (long long)(c.i0 + q) * a.mul_pitch_p + (long long)k * a.mul_pitch_k);
            }
        }
#pragma unroll
        for (int i = 0; i < B; ++i) {
            const int f = f0 + i * K::T;
            if (f < total) {
                const int q = f / K::N;
                const int k = f - q * K::N;
                float2& v = buf[q * K::LD + K::idx(k)];
                v = c_mul(v, maybe_conj(m[i], cj));
            }
        }
    }
}

}  // namespace sipfft

// ------------------------------------------------------------ kernel
#if defined(__CUDACC__)
namespace sipfft {

extern __shared__ __align__(16) float2 sk_smem[];

__device__ __forceinline__ void sk_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void sk_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <class K, int PASS>
__device__ __forceinline__ void sk_run(int tid, const TileArgs& a, const TileCtx& c, float2* buf) {
    using SP = SkPass<K, PASS>;
    if constexpr (K::MPAIR && K::OP == OP_R2C_HALF && SP::LAST) {
        sk_pair_last_r2c<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_R2C_PAIR && SP::LAST) {
        sk_pair_last_r2c_rows<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_R2C_4B && SP::LAST) {
        sk_pair_last_r2c_4b<K>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && K::OP == OP_C2R_4A && PASS == 0) {
        using PP = SkPairFirstC2R4A<K>;
        typename PP::Regs rg;
        PP::read(tid, a, c, buf, rg);
        __syncthreads();
        PP::write_smem(tid, a, c, buf, rg);
        __syncthreads();
        sk_run<K, 1>(tid, a, c, buf);
    } else if constexpr (K::MPAIR && (K::OP == OP_C2R_HALF || K::OP == OP_C2R_PAIR) && PASS == 0) {
        using PP = typename SkPick<K::OP == OP_C2R_HALF, SkPairFirstC2R<K>, SkPairFirstC2RRows<K>>::type;
        typename PP::Regs rg;
        PP::read(tid, a, c, buf, rg);
        __syncthreads();
        PP::write_smem(tid, buf, rg);
        __syncthreads();
        sk_run<K, 1>(tid, a, c, buf);
    } else {
        typename SP::Regs rg;
        SP::read(tid, a, c, buf, rg);
        if constexpr (SP::LAST && !sk_last_to_smem<K>()) {
            SP::write_global(tid, a, c, rg);
        } else {
            __syncthreads();
            SP::write_smem(tid, buf, rg);
            __syncthreads();
            if constexpr (!SP::LAST) sk_run<K, PASS + 1>(tid, a, c, buf);
        }
    }
}

// One half of a pulse-compression tile.  SIP_SK_PC_SPLIT = 1 keeps each
// half out of line, so that it gets its own register allocation instead of
// one for both halves and the filter between them.
#ifndef SIP_SK_PC_SPLIT
#define SIP_SK_PC_SPLIT 0
#endif
template <class KV>
#if SIP_SK_PC_SPLIT
__device__ __noinline__
#else
__device__ __forceinline__
#endif
void sk_half(int tid, const TileArgs& a, const TileCtx& c, float2* buf) {
    sk_run<KV, 0>(tid, a, c, buf);
}

// STAGES = 2: the next tile is staged while the current one is transformed;
// STAGES = 1: one buffer (tiles too large to double), overlap comes from
// several CTAs per SM.
template <class K, int STAGES>
__global__ void __launch_bounds__(K::T, K::MINB) sk_fft_kernel(const TileArgs a) {
    const int tid = threadIdx.x;
    float2* bufs[2] = {sk_smem, sk_smem + (STAGES == 2 ? K::BUF : 0)};
    int tile = blockIdx.x;
    grid_dep_wait();
    grid_dep_launch();
    if (tile >= a.ntiles) return;
    // staged twiddles after the buffers (the barrier before pass 0 of the
    // first tile orders the copy before any use)
    float2* tws = sk_smem + (STAGES == 2 ? 2 : 1) * K::BUF;
    sk_load_tws<K>(tid, a, tws);
    if constexpr (K::SPLIT) {
        // buffers: bufs[0] stages the input, bufs[1] holds the work layout
        static_assert(STAGES == 2, "a split pass 0 needs the staging and the work buffer");
        sk_stage<K>(tid, a, decode_tile(a, tile), bufs[0]);
        sk_commit();
        for (; tile < a.ntiles; tile += gridDim.x) {
            TileCtx c = decode_tile(a, tile);
            if constexpr (K::TWS) c.tws = tws;
            sk_wait<0>();
            __syncthreads();
            if constexpr (K::OP == OP_R2C_PAIR || K::OP == OP_C2R_PAIR) {
                sk_zero_missing<K>(tid, a, c, bufs[0]);
                __syncthreads();
            }
            sk_pass0_split<K>(tid, a, c, bufs[0], bufs[1]);
            __syncthreads();
            const int next = tile + gridDim.x;
            if (next < a.ntiles) sk_stage<K>(tid, a, decode_tile(a, next), bufs[0]);
            sk_commit();
            sk_run<K, 1>(tid, a, c, bufs[1]);
            if constexpr (sk_last_to_smem<K>()) sk_post<K>(tid, a, c, bufs[1]);
            __syncthreads();
        }
        return;
    }
    if (STAGES == 2) {
        sk_stage<K>(tid, a, decode_tile(a, tile), bufs[0]);
        sk_commit();
    }
    for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
        float2* cur = bufs[it & 1];
        TileCtx c = decode_tile(a, tile);
        if constexpr (K::TWS) c.tws = tws;
        if (STAGES == 2) {
            const int next = tile + gridDim.x;
            if (next < a.ntiles) sk_stage<K>(tid, a, decode_tile(a, next), bufs[(it + 1) & 1]);
            sk_commit();
            sk_wait<1>();
        } else {
            sk_stage<K>(tid, a, c, cur);
            sk_commit();
            sk_wait<0>();
        }
        __syncthreads();
        if constexpr (K::OP == OP_R2C_PAIR || K::OP == OP_C2R_PAIR) {
            sk_zero_missing<K>(tid, a, c, cur);
            __syncthreads();
        }
        if constexpr (K::OP == OP_PC) {
            // forward FFT, filter, inverse FFT, all in shared memory.  The
            // butterfly indices and addresses depend on the thread index
            // alone; opaque copies of it per tile and half keep the
            // compiler from hoisting them out of the tile loop (fewer
            // spills: 240 against 328 bytes per thread for 4320 points as
            // 18 x 16 x 15 on 288 threads)
            int tid_fwd = tid;
            asm volatile("" : "+r"(tid_fwd));
            sk_half<SkView<K, OP_PC, -1, false>>(tid_fwd, a, c, cur);
            sk_mul<K>(tid_fwd, a, c, cur);
            __syncthreads();
            int tid_inv = tid;
            asm volatile("" : "+r"(tid_inv));
            sk_half<SkView<K, OP_C2C, 1, true>>(tid_inv, a, c, cur);
            __syncthreads();
            continue;
        }
        sk_run<K, 0>(tid, a, c, cur);
        if constexpr (sk_last_to_smem<K>()) sk_post<K>(tid, a, c, cur);
        __syncthreads();
    }
}

}  // namespace sipfft
#endif
