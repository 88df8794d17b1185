// Tile loads and stores of the FFT kernels.
//
// A tile is P transforms of length N held in shared memory (layout of
// fft_core.cuh: element n of transform p at p * LD + sidx(n)).  Each
// kernel launch processes tiles; a tile index decodes to an "outer" index
// o and a first "inner" transform i0, so one descriptor covers
//   rows of a batch          (outer = 1, inner = rows, idist = row pitch),
//   columns of a 2D/3D axis  (inner = columns, idist = 1, stride = pitch),
//   four-step passes         (column pass with twiddles, row pass with a
//                             transposed store).
// Element (p, n) of the tile is read from src[in_base + p * in_idist +
// n * in_stride] and written to dst[out_base + p * out_idist + k *
// out_stride] (complex64 units for complex operands, float32 units for
// real operands).
//
// Real transforms follow the reference's even/odd treatment
// (ops/fft/real/fft_stockham/fft_stockham/kernel/arch35/
// fft_real_stockham_r2c.cpp:28-124 and fft_real_stockham_c2r.cpp:23-110):
//   even N: N reals are read as N/2 complex values, a length-N/2 complex
//           FFT runs, and a post-process with W_N^k forms the N/2+1 bins
//           (C2R: pre-process, inverse FFT, unpack with factor 2);
//   odd N:  two real rows form one complex row (x_a + i x_b) of length N;
//           the bins of each row are separated with Z[k] and conj(Z[N-k]).
// The imaginary parts of the DC bin (and the Nyquist bin for even N) of a
// C2R input are ignored, which is what numpy.fft.irfft / hfft do.
#pragma once

#include "fft_core.cuh"

namespace sipfft {

enum TileOp : int {
    OP_C2C = 0,
    OP_R2C_HALF = 1,
    OP_C2R_HALF = 2,
    OP_R2C_PAIR = 3,
    OP_C2R_PAIR = 4,
    // Large real lengths (half length M = n_other x N beyond one tile), fused
    // into the four-step passes with mirrored tiles (size-specialized only):
    OP_R2C_4B = 5,  // pass B: rows k1 and N1-k1 of Y, R2C post-process -> X
    OP_C2R_4A = 6,  // pass A: columns n2 and N2-n2 of X, C2R pre-process, column FFT, cross twiddle -> Y
    // Pulse compression of each tile row in shared memory: forward FFT,
    // multiply bin k of transform i0 + p by mul[(i0 + p) * mul_pitch_p +
    // k * mul_pitch_k] (conjugated with TF_MUL_CONJ), inverse FFT, then the
    // C2C store (cross twiddle with TW4, scaling with TF_SCALE).
    OP_PC = 7,
};

enum TileFlags : int {
    TF_CONJ_IN = 1,   // conjugate every loaded value (C2R forward = hfft)
    TF_CONJ_OUT = 2,  // conjugate every stored value (R2C inverse)
    TF_SCALE = 4,     // multiply stored values by `scale`
    TF_MUL = 8,       // multiply stored value k of transform i0 + p by
                      // mul[(i0 + p) * mul_pitch_p + k * mul_pitch_k] (C2C)
    TF_MUL_CONJ = 16, // use conj(mul[...]) (TF_MUL and OP_PC)
    TF_PLANAR_IN = 32,   // C2C input as two float planes: src (real), src_im (imaginary)
    TF_PLANAR_OUT = 64,  // C2C output as two float planes: dst (real), dst_im (imaginary)
    TF_SHIFT_OUT = 128,  // C2C output rotated per slice of sh_rows x sh_cols (fftshift epilogue)
    TF_BLUE = 256,    // OP_PC as Bluestein's whole transform (size-specialized tiles only): rows
                      // of n_other values in and out, times the chirp tw2[j] on load (zero
                      // padded to N) and tw2[k] on store, outputs k < n_other only
};

struct TileArgs {
    const PlanDev* plan;     // device copy of the pass list
    const float2* tw;        // Stockham twiddles
    const float2* tw2;       // W_N^k table (real pre/post-process) or W_Ntot^m (four-step)
    const void* src;
    void* dst;
    long long in_odist, in_idist, in_stride;
    long long out_odist, out_idist, out_stride;
    int N;                   // FFT length of each tile transform
    int P;                   // transforms per tile
    int LD;                  // shared-memory row pitch (complex values)
    int inner;               // transforms per outer index
    int tiles_per_outer;
    int ntiles;
    int rows;                // real rows (pair ops)
    int flags;
    int tw4_shift;           // four-step cross twiddles: split base B = 2^tw4_shift
    int n_other;             // OP_R2C_4B: rows N1 of Y; OP_C2R_4A: columns N2 of X
    const float2* mul;       // TF_MUL spectrum (e.g. a matched filter)
    const float* src_im;     // TF_PLANAR_IN imaginary plane
    float* dst_im;           // TF_PLANAR_OUT imaginary plane
    long long sh_slice;      // TF_SHIFT_OUT: elements per slice (sh_rows x sh_cols)
    int sh_rows, sh_cols;    //   slice shape
    int sh_r, sh_c;          //   row / column rotation
    FastDiv div_sh_cols;     //   / sh_cols
    long long mul_pitch_p, mul_pitch_k;
    float scale;
    FastDiv div_n;           // / N
    FastDiv div_p;           // / P
    FastDiv div_h;           // / (N/2+1) or / (N+1) for the half ops
    FastDiv div_tpo;         // / tiles_per_outer
};

struct TileCtx {
    int cnt;   // transforms present in this tile (<= P)
    int i0;    // inner index of transform 0
    long long in_base, out_base;
    // Twiddle tables staged in shared memory by the size-specialized kernels
    // that keep them there (SK_TW_SMEM); null otherwise.
    const float2* tws = nullptr;
};

SIP_HD TileCtx decode_tile(const TileArgs& a, int tile) {
    TileCtx c;
    const int o = (int)fd_div(a.div_tpo, (uint32_t)tile);
    const int it = tile - o * a.tiles_per_outer;
    c.i0 = it * a.P;
    c.cnt = a.inner - c.i0 < a.P ? a.inner - c.i0 : a.P;
    c.in_base = (long long)o * a.in_odist + (long long)c.i0 * a.in_idist;
    c.out_base = (long long)o * a.out_odist + (long long)c.i0 * a.out_idist;
    return c;
}

SIP_HD float2 maybe_conj(float2 v, bool cj) { return cj ? make_float2(v.x, -v.y) : v; }

// ------------------------------------------------------------- C2C load
SIP_HD void load_c2c(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    if (a.flags & TF_PLANAR_IN) {
        // separated real / imaginary planes (asdFftExecC2CSeparated)
        const float* re = static_cast<const float*>(a.src);
        const int total = c.cnt * a.N;
        for (int f = tid; f < total; f += T) {
            const int p = (int)fd_div(a.div_n, (uint32_t)f);
            const int n = f - p * a.N;
            const long long i = c.in_base + (long long)p * a.in_idist + (long long)n * a.in_stride;
            sm[p * a.LD + sidx(n)] = make_float2(SIP_LDG(re + i), SIP_LDG(a.src_im + i));
        }
        return;
    }
    const float2* src = static_cast<const float2*>(a.src);
    const int N = a.N, P = a.P, LD = a.LD;
    const bool cj = (a.flags & TF_CONJ_IN) != 0;
    if (a.in_stride == 1 && a.in_idist == N) {
        // The tile is one contiguous run of cnt * N values.
        const float2* base = src + c.in_base;
        const int count = c.cnt * N;
        int f0 = 0;
        if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) {
            if (tid == 0) sm[sidx(0)] = maybe_conj(SIP_LDG(base), cj);
            f0 = 1;
        }
        const int pairs = (count - f0) >> 1;
        const float4* b4 = reinterpret_cast<const float4*>(base + f0);
        for (int q = tid; q < pairs; q += T) {
            const float4 v = SIP_LDG(b4 + q);
            const int f = f0 + 2 * q;
            int p = (int)fd_div(a.div_n, (uint32_t)f);
            int n = f - p * N;
            sm[p * LD + sidx(n)] = maybe_conj(make_float2(v.x, v.y), cj);
            if (++n == N) { n = 0; ++p; }
            sm[p * LD + sidx(n)] = maybe_conj(make_float2(v.z, v.w), cj);
        }
        const int tail = f0 + 2 * pairs;
        if (tail < count && tid == T - 1) {
            const int p = (int)fd_div(a.div_n, (uint32_t)tail);
            sm[p * LD + sidx(tail - p * N)] = maybe_conj(SIP_LDG(base + tail), cj);
        }
    } else if (a.in_idist == 1) {
        // Adjacent transforms are adjacent in memory (columns): consecutive
        // threads take consecutive transforms of the same element index.
        const int total = P * N;
        for (int f = tid; f < total; f += T) {
            const int n = (int)fd_div(a.div_p, (uint32_t)f);
            const int p = f - n * P;
            if (p < c.cnt)
                sm[p * LD + sidx(n)] = maybe_conj(SIP_LDG(src + c.in_base + p + (long long)n * a.in_stride), cj);
        }
    } else {
        const int total = c.cnt * N;
        for (int f = tid; f < total; f += T) {
            const int p = (int)fd_div(a.div_n, (uint32_t)f);
            const int n = f - p * N;
            sm[p * LD + sidx(n)] =
                maybe_conj(SIP_LDG(src + c.in_base + (long long)p * a.in_idist + (long long)n * a.in_stride), cj);
        }
    }
}

// Four-step cross twiddle W_N^m from the split table a.tw2:
// [W_N^lo for lo < B][W_N^{hi B} for hi < ceil(N/B)], B = 2^tw4_shift,
// m = hi B + lo.  Both halves are a few KB and stay in L1; the product of two
// correctly rounded values is within about one ulp.
SIP_HD float2 cross_tw(const TileArgs& a, long long m) {
    const long long B = 1LL << a.tw4_shift;
    const float2 lo = SIP_LDG(a.tw2 + (m & (B - 1)));
    const float2 hi = SIP_LDG(a.tw2 + B + (m >> a.tw4_shift));
    return c_mul(lo, hi);
}

// TF_SHIFT_OUT: position of output element f (flat index into the output
// array of slices) after rotating its slice by (sh_r, sh_c), the layout of
// asdFftShift / asdIfftShift applied to the transform's output.
SIP_HD long long shifted_index(const TileArgs& a, long long f) {
    const long long s = f / a.sh_slice;
    const int rem = (int)(f - s * a.sh_slice);
    const int row = (int)fd_div(a.div_sh_cols, (uint32_t)rem);
    const int col = rem - row * a.sh_cols;
    int r2 = row + a.sh_r;
    if (r2 >= a.sh_rows) r2 -= a.sh_rows;
    int c2 = col + a.sh_c;
    if (c2 >= a.sh_cols) c2 -= a.sh_cols;
    return s * a.sh_slice + (long long)r2 * a.sh_cols + c2;
}

// ------------------------------------------------------------ C2C store
// TW4: multiply element k of transform p by W_N^{(i0 + p) k} (the four-step
// cross twiddle).
template <int SIGN, bool TW4>
SIP_HD float2 c2c_out_value(const TileArgs& a, const TileCtx& c, const float2* sm, int p, int n) {
    float2 v = sm[p * a.LD + sidx(n)];
    if (TW4) v = c_tw<SIGN>(v, cross_tw(a, (long long)(c.i0 + p) * n));
    if (a.flags & TF_MUL) {
        const float2 m = SIP_LDG(a.mul + (long long)(c.i0 + p) * a.mul_pitch_p + (long long)n * a.mul_pitch_k);
        v = c_mul(v, maybe_conj(m, (a.flags & TF_MUL_CONJ) != 0));
    }
    if (a.flags & TF_SCALE) v = c_scale(v, a.scale);
    return maybe_conj(v, (a.flags & TF_CONJ_OUT) != 0);
}

template <int SIGN, bool TW4>
SIP_HD void store_c2c(int tid, int T, const TileArgs& a, const TileCtx& c, const float2* sm) {
    float2* dst = static_cast<float2*>(a.dst);
    const int N = a.N, P = a.P;
#define SIP_C2C_VALUE(p_, n_) c2c_out_value<SIGN, TW4>(a, c, sm, (p_), (n_))
    if (a.flags & TF_SHIFT_OUT) {
        const int total = c.cnt * N;
        for (int f = tid; f < total; f += T) {
            const int p = (int)fd_div(a.div_n, (uint32_t)f);
            const int n = f - p * N;
            const long long i = c.out_base + (long long)p * a.out_idist + (long long)n * a.out_stride;
            dst[shifted_index(a, i)] = SIP_C2C_VALUE(p, n);
        }
        return;
    }
    if (a.flags & TF_PLANAR_OUT) {
        float* re = static_cast<float*>(a.dst);
        const int total = c.cnt * N;
        for (int f = tid; f < total; f += T) {
            const int p = (int)fd_div(a.div_n, (uint32_t)f);
            const int n = f - p * N;
            const long long i = c.out_base + (long long)p * a.out_idist + (long long)n * a.out_stride;
            const float2 v = SIP_C2C_VALUE(p, n);
            re[i] = v.x;
            a.dst_im[i] = v.y;
        }
        return;
    }
    if (a.out_stride == 1 && a.out_idist == N) {
        float2* base = dst + c.out_base;
        const int count = c.cnt * N;
        int f0 = 0;
        if ((reinterpret_cast<uintptr_t>(base) & 15) != 0) {
            if (tid == 0) base[0] = SIP_C2C_VALUE(0, 0);
            f0 = 1;
        }
        const int pairs = (count - f0) >> 1;
        float4* b4 = reinterpret_cast<float4*>(base + f0);
        for (int q = tid; q < pairs; q += T) {
            const int f = f0 + 2 * q;
            int p = (int)fd_div(a.div_n, (uint32_t)f);
            int n = f - p * N;
            const float2 v0 = SIP_C2C_VALUE(p, n);
            if (++n == N) { n = 0; ++p; }
            const float2 v1 = SIP_C2C_VALUE(p, n);
            b4[q] = make_float4(v0.x, v0.y, v1.x, v1.y);
        }
        const int tail = f0 + 2 * pairs;
        if (tail < count && tid == T - 1) {
            const int p = (int)fd_div(a.div_n, (uint32_t)tail);
            base[tail] = SIP_C2C_VALUE(p, tail - p * N);
        }
    } else if (a.out_idist == 1) {
        const int total = P * N;
        for (int f = tid; f < total; f += T) {
            const int n = (int)fd_div(a.div_p, (uint32_t)f);
            const int p = f - n * P;
            if (p < c.cnt) dst[c.out_base + p + (long long)n * a.out_stride] = SIP_C2C_VALUE(p, n);
        }
    } else {
        const int total = c.cnt * N;
        for (int f = tid; f < total; f += T) {
            const int p = (int)fd_div(a.div_n, (uint32_t)f);
            const int n = f - p * N;
            dst[c.out_base + (long long)p * a.out_idist + (long long)n * a.out_stride] = SIP_C2C_VALUE(p, n);
        }
    }
}

#undef SIP_C2C_VALUE

// OP_PC: multiplies the spectra held in the tile by the filter spectrum
// (every element of the tile's transforms, between the two FFTs).
SIP_HD void mul_tile(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    const int N = a.N;
    const bool cj = (a.flags & TF_MUL_CONJ) != 0;
    const int total = c.cnt * N;
    for (int f = tid; f < total; f += T) {
        const int p = (int)fd_div(a.div_n, (uint32_t)f);
        const int n = f - p * N;
        const float2 m = SIP_LDG(a.mul + (long long)(c.i0 + p) * a.mul_pitch_p + (long long)n * a.mul_pitch_k);
        float2& v = sm[p * a.LD + sidx(n)];
        v = c_mul(v, maybe_conj(m, cj));
    }
}

// ------------------------------------------------- R2C, even N (half length)
// Input: rows of 2M reals read as M complex values (row pitch in_idist in
// complex units).  Output: rows of M+1 bins (pitch out_idist).
// X[k] = E[k] + W_{2M}^k O[k], E = (Z[k] + conj Z[M-k]) / 2,
// O = (Z[k] - conj Z[M-k]) / 2i, indices mod M; a.tw2[k] = W_{2M}^k.
SIP_HD void load_r2c_half(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    load_c2c(tid, T, a, c, sm);
}

SIP_HD void store_r2c_half(int tid, int T, const TileArgs& a, const TileCtx& c, const float2* sm) {
    float2* dst = static_cast<float2*>(a.dst);
    const int M = a.N, LD = a.LD, H = M + 1;
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    const int total = c.cnt * H;
    for (int f = tid; f < total; f += T) {
        const int p = (int)fd_div(a.div_h, (uint32_t)f);
        const int k = f - p * H;
        const float2* row = sm + p * LD;
        const float2 z = row[sidx(k == M ? 0 : k)];
        const float2 zm = row[sidx(k == 0 ? 0 : M - k)];
        const float2 b = make_float2(zm.x, -zm.y);
        const float2 ev = make_float2(0.5f * (z.x + b.x), 0.5f * (z.y + b.y));
        const float2 od = make_float2(0.5f * (z.y - b.y), -0.5f * (z.x - b.x));
        float2 x = c_add(ev, c_mul(SIP_LDG(a.tw2 + k), od));
        if (sc) x = c_scale(x, a.scale);
        dst[c.out_base + (long long)p * a.out_idist + k] = maybe_conj(x, cj);
    }
}

// ------------------------------------------------- C2R, even N (half length)
// Raw bins X[0..M] are loaded, then pairs (k, M-k) are pre-processed in
// shared memory into Z (length M, inverse FFT); each output pair of reals
// is 2 z[n].
SIP_HD void load_c2r_half(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    const float2* src = static_cast<const float2*>(a.src);
    const int M = a.N, LD = a.LD, H = M + 1;
    const bool cj = (a.flags & TF_CONJ_IN) != 0;
    const int total = c.cnt * H;
    for (int f = tid; f < total; f += T) {
        const int p = (int)fd_div(a.div_h, (uint32_t)f);
        const int k = f - p * H;
        sm[p * LD + sidx(k)] = maybe_conj(SIP_LDG(src + c.in_base + (long long)p * a.in_idist + k), cj);
    }
}

SIP_HD void prep_c2r_half(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    const int M = a.N, LD = a.LD, Q = M / 2 + 1;
    const int total = c.cnt * Q;
    for (int f = tid; f < total; f += T) {
        const int p = f / Q;
        const int k = f - p * Q;
        float2* row = sm + p * LD;
        if (k == 0) {
            const float dc = row[sidx(0)].x, ny = row[sidx(M)].x;
            row[sidx(0)] = make_float2(0.5f * (dc + ny), 0.5f * (dc - ny));
            continue;
        }
        const int kk = M - k;
        const float2 x = row[sidx(k)], y = row[sidx(kk)];
        const float2 b = make_float2(y.x, -y.y);
        const float2 e = make_float2(0.5f * (x.x + b.x), 0.5f * (x.y + b.y));
        const float2 d = make_float2(0.5f * (x.x - b.x), 0.5f * (x.y - b.y));
        const float2 od = c_mulc(d, SIP_LDG(a.tw2 + k));  // W_{2M}^{+k} d
        row[sidx(k)] = make_float2(e.x - od.y, e.y + od.x);
        if (kk != k) row[sidx(kk)] = make_float2(e.x + od.y, od.x - e.y);
    }
}

SIP_HD void store_c2r_half(int tid, int T, const TileArgs& a, const TileCtx& c, const float2* sm) {
    // Output rows of 2M reals written as M complex pairs (pitch out_idist).
    float2* dst = static_cast<float2*>(a.dst);
    const int M = a.N, LD = a.LD;
    const float s = 2.0f * ((a.flags & TF_SCALE) ? a.scale : 1.0f);
    const int total = c.cnt * M;
    for (int f = tid; f < total; f += T) {
        const int p = (int)fd_div(a.div_n, (uint32_t)f);
        const int n = f - p * M;
        dst[c.out_base + (long long)p * a.out_idist + n] = c_scale(sm[p * LD + sidx(n)], s);
    }
}

// ------------------------------------------------ R2C / C2R, two rows per FFT
// Transform p of a tile carries real rows 2 (i0 + p) and 2 (i0 + p) + 1 of
// a.rows rows; row r starts at r * in_idist (r * out_idist) elements, in
// float32 units for the real side and complex64 units for the spectrum.
SIP_HD void load_r2c_pair(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    const float* src = static_cast<const float*>(a.src);
    const int N = a.N, LD = a.LD;
    const int r0 = 2 * c.i0;
    const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
    const int total = nrows * N;
    for (int f = tid; f < total; f += T) {
        const int rl = (int)fd_div(a.div_n, (uint32_t)f);
        const int n = f - rl * N;
        float* slot = reinterpret_cast<float*>(sm + (rl >> 1) * LD + sidx(n));
        slot[rl & 1] = SIP_LDG(src + (long long)(r0 + rl) * a.in_idist + n);
    }
    if (nrows & 1) {
        // odd batch: the partner of the last row is zero
        float2* row = sm + (nrows >> 1) * LD;
        for (int n = tid; n < N; n += T) row[sidx(n)].y = 0.f;
    }
}

SIP_HD void store_r2c_pair(int tid, int T, const TileArgs& a, const TileCtx& c, const float2* sm) {
    float2* dst = static_cast<float2*>(a.dst);
    const int N = a.N, LD = a.LD, H = N / 2 + 1;
    const bool cj = (a.flags & TF_CONJ_OUT) != 0;
    const bool sc = (a.flags & TF_SCALE) != 0;
    const int r0 = 2 * c.i0;
    const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
    const int total = nrows * H;
    for (int f = tid; f < total; f += T) {
        const int rl = (int)fd_div(a.div_h, (uint32_t)f);
        const int k = f - rl * H;
        const float2* row = sm + (rl >> 1) * LD;
        const float2 z = row[sidx(k)];
        const float2 zm = row[sidx(k == 0 ? 0 : N - k)];
        float2 x;
        if ((rl & 1) == 0)
            x = make_float2(0.5f * (z.x + zm.x), 0.5f * (z.y - zm.y));
        else
            x = make_float2(0.5f * (z.y + zm.y), -0.5f * (z.x - zm.x));
        if (sc) x = c_scale(x, a.scale);
        dst[(long long)(r0 + rl) * a.out_idist + k] = maybe_conj(x, cj);
    }
}

SIP_HD void load_c2r_pair(int tid, int T, const TileArgs& a, const TileCtx& c, float2* sm) {
    const float2* src = static_cast<const float2*>(a.src);
    const int N = a.N, LD = a.LD, half = N / 2;
    const bool fwd = (a.flags & TF_CONJ_IN) != 0;
    const int r0 = 2 * c.i0;
    const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
    const int total = c.cnt * N;
    for (int f = tid; f < total; f += T) {
        const int p = (int)fd_div(a.div_n, (uint32_t)f);
        const int k = f - p * N;
        const int kk = k <= half ? k : N - k;
        const long long ra = (long long)(r0 + 2 * p) * a.in_idist + kk;
        float2 xa = SIP_LDG(src + ra);
        float2 xb = (2 * p + 1 < nrows) ? SIP_LDG(src + ra + a.in_idist) : make_float2(0.f, 0.f);
        if (kk == 0 || 2 * kk == N) {
            xa.y = 0.f;
            xb.y = 0.f;
        }
        if ((k > half) != fwd) {
            xa.y = -xa.y;
            xb.y = -xb.y;
        }
        sm[p * LD + sidx(k)] = make_float2(xa.x - xb.y, xa.y + xb.x);
    }
}

SIP_HD void store_c2r_pair(int tid, int T, const TileArgs& a, const TileCtx& c, const float2* sm) {
    float* dst = static_cast<float*>(a.dst);
    const int N = a.N, LD = a.LD;
    const float s = (a.flags & TF_SCALE) ? a.scale : 1.0f;
    const int r0 = 2 * c.i0;
    const int nrows = (a.rows - r0) < 2 * c.cnt ? (a.rows - r0) : 2 * c.cnt;
    const int total = nrows * N;
    for (int f = tid; f < total; f += T) {
        const int rl = (int)fd_div(a.div_n, (uint32_t)f);
        const int n = f - rl * N;
        const float2 z = sm[(rl >> 1) * LD + sidx(n)];
        dst[(long long)(r0 + rl) * a.out_idist + n] = ((rl & 1) ? z.y : z.x) * s;
    }
}

}  // namespace sipfft
