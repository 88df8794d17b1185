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
// Staged input values (complex64 units) per tile.
SIP_HD constexpr int sk_stage_values(int op, int p, int n) {
    return op == OP_C2R_HALF ? p * (n + 1)
         : (op == OP_R2C_4B || op == OP_C2R_4A) ? p * n
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
    // Pass twiddles: TWB = 1 reads the basis table (fft_core.cuh
    // basis_split: fewer loads, one extra product), TWB = 0 the full
    // Stockham table (one load per twiddle, fewer instructions).
    static constexpr bool TWB = TWB_ != 0;
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
    static constexpr int SMEM = 2 * BUF * 8;
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
    static_assert(OP != OP_C2C || MODE != SK_COLS || true, "");
    static_assert(!(TW4 && OP != OP_C2C && OP != OP_PC), "cross twiddles are C2C / pulse only");
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
        // element n1 of columns n2 = i0 + q (slot q) and N2 - n2 (slot H + q);
        // each thread keeps one slot and walks the rows
        static_assert(T % K::P == 0, "C2R_4A staging maps threads to slots");
        const int n2c = a.n_other;
        const char* xbase = src + (c.in_base - c.i0) * 8;  // X[0] of this batch row
        const int slot = tid % K::P;
        const int col = sk_c2r4a_col<K>(a, c.i0, c.cnt, slot);
        if (col >= 0) {
            const char* s = xbase + (long long)col * 8;
            char* d = reinterpret_cast<char*>(stage) + slot * 8;
            for (int n1 = tid / K::P; n1 < K::N; n1 += T / K::P) {
#if defined(__CUDA_ARCH__)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                                 (unsigned)__cvta_generic_to_shared(d + n1 * K::P * 8)),
                             "l"(s + (long long)n1 * n2c * 8));
#else
                for (int b = 0; b < 8; ++b) d[n1 * K::P * 8 + b] = s[(long long)n1 * n2c * 8 + b];
#endif
            }
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
    float2 x = maybe_conj(stage[n1 * K::P + slot], cj);
    float2 y;
    if (col == 0) {
        if (n1 == 0) {
            const float2* xrow = static_cast<const float2*>(a.src) + (c.in_base - c.i0);
            const float ny = SIP_LDG(xrow + M).x;
            return make_float2(0.5f * (x.x + ny), 0.5f * (x.x - ny));
        }
        y = stage[(K::N - n1) * K::P + slot];
    } else if (2 * col == n2c) {
        y = stage[(K::N - 1 - n1) * K::P + slot];
    } else {
        const int ms = slot < K::H ? slot + K::H : slot - K::H;
        y = stage[(K::N - 1 - n1) * K::P + ms];
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
        const float2 od = c_mulc(d, SIP_LDG(a.tw2 + n));
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

    // Reads (pass 0: from the staged input) and transforms this thread's butterflies.
    SIP_HD static void read(int tid, const TileArgs& a, const TileCtx& c, const float2* buf, Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int b = tid + s * K::T;
            if (TOTAL % K::T == 0 || b < TOTAL) {
                int q, j;
                butterfly_index(b, q, j);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if constexpr (PASS == 0 && !K::WORK_IN)
                        rg.v[s][r] = sk_input<K>(a, c, buf, q, j + r * NR);
                    else
                        rg.v[s][r] = buf[q * K::LD + K::idx(j + r * NR)];
                }
                if constexpr (L > 1 && !K::TWB) {
                    const int k = j % L;
                    const float2* w = a.tw + K::twoff(PASS) + k;  // twiddle-major table
#pragma unroll
                    for (int r = 1; r < R; ++r) rg.v[s][r] = c_tw<K::SIGN>(rg.v[s][r], SIP_LDG(w + (r - 1) * L));
                } else if constexpr (L > 1) {
                    // basis twiddles: W^{r k} = W^{r_lo k} W^{a r_hi k}
                    constexpr int A = basis_split(R);
                    const int k = j % L;
                    const float2* w = a.tw + K::twoff(PASS) + k;  // twiddle-major table
                    float2 lo[A], hi[R / A];
                    lo[0] = make_float2(1.f, 0.f);
                    hi[0] = make_float2(1.f, 0.f);
#pragma unroll
                    for (int t = 1; t < A; ++t) lo[t] = SIP_LDG(w + (t - 1) * L);
#pragma unroll
                    for (int t = 1; t < R / A; ++t) hi[t] = SIP_LDG(w + (A - 1 + t - 1) * L);
#pragma unroll
                    for (int r = 1; r < R; ++r) {
                        const int rl = r % A, rh = r / A;
                        const float2 t = rh == 0 ? lo[rl] : rl == 0 ? hi[rh] : c_mul(lo[rl], hi[rh]);
                        rg.v[s][r] = c_tw<K::SIGN>(rg.v[s][r], t);
                    }
                }
                dft<R, K::SIGN>(rg.v[s]);
            }
        }
    }

    // Writes to the padded work layout (all passes except a global-storing last one).
    SIP_HD static void write_smem(int tid, float2* buf, const Regs& rg) {
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const int b = tid + s * K::T;
            if (TOTAL % K::T == 0 || b < TOTAL) {
                int q, j;
                butterfly_index(b, q, j);
                const int o = (j / L) * L * R + j % L;
#pragma unroll
                for (int r = 0; r < R; ++r) buf[q * K::LD + K::idx(o + r * L)] = rg.v[s][r];
            }
        }
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
    return K::OP == OP_R2C_HALF || K::OP == OP_R2C_PAIR || K::OP == OP_R2C_4B || K::OP == OP_PC;
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
            const float2 t = c_mul(SIP_LDG(a.tw2 + k), od);
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

// OP_PC: the spectra in the work layout times the filter spectrum, element
// k of transform q times mul[(i0 + q) * mul_pitch_p + k * mul_pitch_k]
// (conjugated under TF_MUL_CONJ), as tile_io.cuh mul_tile.
template <class K>
SIP_HD void sk_mul(int tid, const TileArgs& a, const TileCtx& c, float2* buf) {
    const bool cj = (a.flags & TF_MUL_CONJ) != 0;
    const int total = c.cnt * K::N;
    for (int f = tid; f < total; f += K::T) {
        const int q = f / K::N;
        const int k = f - q * K::N;
        const float2 m = SIP_LDG(a.mul + (long long)(c.i0 + q) * a.mul_pitch_p + (long long)k * a.mul_pitch_k);
        float2& v = buf[q * K::LD + K::idx(k)];
        v = c_mul(v, maybe_conj(m, cj));
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
    if (tile >= a.ntiles) return;
    if (STAGES == 2) {
        sk_stage<K>(tid, a, decode_tile(a, tile), bufs[0]);
        sk_commit();
    }
    for (int it = 0; tile < a.ntiles; ++it, tile += gridDim.x) {
        float2* cur = bufs[it & 1];
        const TileCtx c = decode_tile(a, tile);
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
            // forward FFT, filter, inverse FFT, all in shared memory
            sk_half<SkView<K, OP_PC, -1, false>>(tid, a, c, cur);
            sk_mul<K>(tid, a, c, cur);
            __syncthreads();
            // the inverse half's butterfly indices and addresses equal the
            // forward half's; an opaque copy of the thread index keeps the
            // compiler from holding them in registers across both halves
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
