// Core arithmetic of the B200 FFT kernels: complex helpers, compile-time
// trigonometric constants, in-register DFT butterflies for radices
// 2..32, exact fast integer division, and one Stockham pass over a tile
// held in shared memory.
//
// Everything here is __host__ __device__ so that the same index and
// butterfly code can be driven phase by phase on the CPU by the test
// harness (tests/native/tile_emu.cu) without a GPU.
//
// Stage algebra (self-sorting DIT Stockham, the scheme the reference's
// ops/fft/real/fft_stockham/.../vendor/fft_stockham_mix.h:1218-1267 runs
// one global-memory stage at a time; here all stages of a transform run
// in shared memory): for a transform of length N = R_0 R_1 ... R_{m-1},
// pass p has radix R = R_p and span L = R_0 ... R_{p-1}.  Butterfly j in
// [0, N/R) reads x[j + r N/R] (r < R), multiplies element r by
// W_{L R}^{r (j mod L)}, runs an R-point DFT and writes element r to
// (j / L) L R + (j mod L) + r L.  After the last pass the data is in
// natural order.
#pragma once

#if defined(__CUDACC_RTC__)
// Runtime compilation (jit.cpp): the compiler provides the vector types.
typedef unsigned int uint32_t;
typedef unsigned long long uint64_t;
typedef unsigned long long uintptr_t;
#else
#include <cuda_runtime.h>
#include <stdint.h>
#endif

#if defined(__CUDACC__)
#define SIP_HD __host__ __device__ __forceinline__
#else
#define SIP_HD inline
#endif

#if defined(__CUDA_ARCH__)
#define SIP_LDG(p) __ldg(p)
#else
#define SIP_LDG(p) (*(p))
#endif

namespace sipfft {

// ------------------------------------------- programmatic dependent launch
// A kernel launched with the programmatic-stream-serialization attribute
// (launch_attr.h) may start while the previous kernel of its stream still
// runs.  grid_dep_wait() returns once that kernel has completed and its
// memory operations are visible, so every such kernel calls it before its
// first global-memory access.  grid_dep_launch() lets the stream's next
// kernel of that kind start launching; it waits in turn.  Both do nothing
// in a kernel launched without the attribute, and on the host.
SIP_HD void grid_dep_wait() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
#endif
}
SIP_HD void grid_dep_launch() {
#if defined(__CUDA_ARCH__) && __CUDA_ARCH__ >= 900
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
#endif
}

// ---------------------------------------------------------------- complex
SIP_HD float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
SIP_HD float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
SIP_HD float2 c_mul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
SIP_HD float2 c_mulc(float2 a, float2 b) { return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
SIP_HD float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
SIP_HD float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
// Twiddle tables hold forward (exp(-i theta)) values; the inverse sign uses
// their conjugate.
template <int SIGN>
SIP_HD float2 c_tw(float2 a, float2 w) { return SIGN < 0 ? c_mul(a, w) : c_mulc(a, w); }
// a * (SIGN * i)
template <int SIGN>
SIP_HD float2 c_mul_si(float2 a) { return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x); }

// ------------------------------------------------- compile-time cos / sin
// cos(2 pi m / n) and sin(2 pi m / n) in double precision, evaluated by the
// compiler.  The angle is reduced exactly with integer arithmetic to a
// quadrant plus an offset in [0, pi/4], where a Taylor series of 12 terms
// is accurate to well below one double ulp.
constexpr double kHalfPi = 1.57079632679489661923132169163975;

constexpr double cx_sin_small(double x) {
    double x2 = x * x, term = x, sum = x;
    for (int i = 1; i < 12; ++i) {
        term *= -x2 / double((2 * i) * (2 * i + 1));
        sum += term;
    }
    return sum;
}
constexpr double cx_cos_small(double x) {
    double x2 = x * x, term = 1.0, sum = 1.0;
    for (int i = 1; i < 12; ++i) {
        term *= -x2 / double((2 * i - 1) * (2 * i));
        sum += term;
    }
    return sum;
}
// which = 0 -> cos, 1 -> sin
constexpr double cx_trig2pi(long long m, long long n, int which) {
    m = ((m % n) + n) % n;
    const long long t = 4 * m;
    const long long q = t / n;  // quadrant
    const long long r = t - q * n;
    double ca = 0, sa = 0;
    if (2 * r <= n) {
        const double a = kHalfPi * double(r) / double(n);
        ca = cx_cos_small(a);
        sa = cx_sin_small(a);
    } else {
        const double b = kHalfPi * double(n - r) / double(n);
        ca = cx_sin_small(b);
        sa = cx_cos_small(b);
    }
    double c = 0, s = 0;
    switch (q) {
        case 0: c = ca; s = sa; break;
        case 1: c = -sa; s = ca; break;
        case 2: c = -ca; s = -sa; break;
        default: c = sa; s = -ca; break;
    }
    return which == 0 ? c : s;
}

constexpr bool cx_is_prime(int n) {
    if (n < 2) return false;
    for (int d = 2; d * d <= n; ++d)
        if (n % d == 0) return false;
    return true;
}
constexpr int cx_split(int n) {
    // outer factor of a composite radix: 4 when it divides (radix-4 cores
    // are cheapest), else the smallest prime factor.
    if (n % 4 == 0 && n > 4) return 4;
    for (int d = 2; d * d <= n; ++d)
        if (n % d == 0) return d;
    return n;
}

// a * W_R^M with W_R = exp(SIGN * 2 pi i / R); exact forms for multiples
// of 1/8 turn, a complex multiply by a folded constant otherwise.
template <int R, int M, int SIGN>
SIP_HD float2 tw_const(float2 a) {
    constexpr int m = ((M % R) + R) % R;
    if constexpr (m == 0) {
        return a;
    } else if constexpr (2 * m == R) {
        return make_float2(-a.x, -a.y);
    } else if constexpr (4 * m == R) {
        return c_mul_si<SIGN>(a);
    } else if constexpr (4 * m == 3 * R) {
        return c_mul_si<-SIGN>(a);
    } else if constexpr ((8 * m) % R == 0) {
        constexpr float h = 0.70710678118654752440f;
        constexpr int e = (8 * m) / R;  // odd eighth: 1, 3, 5, 7
        constexpr float cr = (e == 1 || e == 7) ? h : -h;
        constexpr float ci = (e == 1 || e == 3) ? h : -h;  // sin sign before SIGN
        constexpr float si = SIGN < 0 ? -ci : ci;
        return make_float2(a.x * cr - a.y * si, a.x * si + a.y * cr);
    } else {
        constexpr float c = float(cx_trig2pi(m, R, 0));
        constexpr float s = float(SIGN * cx_trig2pi(m, R, 1));
        return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
    }
}

// ------------------------------------------------------------ butterflies
template <int R, int SIGN>
SIP_HD void dft(float2 (&v)[R]);

template <int SIGN>
SIP_HD void dft2(float2 (&v)[2]) {
    const float2 a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
}

template <int SIGN>
SIP_HD void dft4(float2 (&v)[4]) {
    const float2 s02 = c_add(v[0], v[2]), d02 = c_sub(v[0], v[2]);
    const float2 s13 = c_add(v[1], v[3]), d13 = c_mul_si<SIGN>(c_sub(v[1], v[3]));
    v[0] = c_add(s02, s13);
    v[2] = c_sub(s02, s13);
    v[1] = c_add(d02, d13);
    v[3] = c_sub(d02, d13);
}

// Odd prime R: pairs (n, R-n) share cos terms and carry opposite sin terms,
// X[k] = x0 + sum_n a_n cos(2 pi n k / R) + SIGN i sum_n b_n sin(2 pi n k / R)
// with a_n = x_n + x_{R-n}, b_n = x_n - x_{R-n}.  The constants are template
// arguments of the recursion, so they are folded at compile time.
template <int R, int K, int Nn, int H>
SIP_HD void prime_acc(const float2 (&a)[H], const float2 (&b)[H], float2& A, float2& B) {
    if constexpr (Nn <= H) {
        constexpr float c = float(cx_trig2pi((long long)Nn * K, R, 0));
        constexpr float s = float(cx_trig2pi((long long)Nn * K, R, 1));
        A.x += a[Nn - 1].x * c;
        A.y += a[Nn - 1].y * c;
        B.x += b[Nn - 1].x * s;
        B.y += b[Nn - 1].y * s;
        prime_acc<R, K, Nn + 1, H>(a, b, A, B);
    }
}

template <int R, int SIGN, int K, int H>
SIP_HD void prime_out(float2 (&v)[R], const float2 (&a)[H], const float2 (&b)[H], float2 x0) {
    if constexpr (K <= H) {
        float2 A = x0, B = make_float2(0.f, 0.f);
        prime_acc<R, K, 1, H>(a, b, A, B);
        const float2 iB = c_mul_si<SIGN>(B);
        v[K] = c_add(A, iB);
        v[R - K] = c_sub(A, iB);
        prime_out<R, SIGN, K + 1, H>(v, a, b, x0);
    }
}

template <int R, int SIGN>
SIP_HD void dft_prime(float2 (&v)[R]) {
    constexpr int H = (R - 1) / 2;
    float2 a[H], b[H];
    float2 sum = v[0];
#pragma unroll
    for (int n = 1; n <= H; ++n) {
        a[n - 1] = c_add(v[n], v[R - n]);
        b[n - 1] = c_sub(v[n], v[R - n]);
        sum = c_add(sum, a[n - 1]);
    }
    const float2 x0 = v[0];
    prime_out<R, SIGN, 1, H>(v, a, b, x0);
    v[0] = sum;
}

// Composite R = A * B (Cooley-Tukey inside the registers): inputs at
// n1 + A n2, B-point DFTs over n2, twiddle W_R^{n1 k2}, A-point DFTs over
// n1; output X[B k1 + k2] lands at k1 + A k2 and is permuted back to
// natural order at compile time.
template <int R, int SIGN>
SIP_HD void dft(float2 (&v)[R]);

template <int R, int A, int B, int SIGN, int N1, int K2>
SIP_HD void comp_twiddle(float2 (&v)[R], const float2 (&t)[B]) {
    if constexpr (K2 < B) {
        v[N1 + A * K2] = tw_const<R, N1 * K2, SIGN>(t[K2]);
        comp_twiddle<R, A, B, SIGN, N1, K2 + 1>(v, t);
    }
}

template <int R, int A, int B, int SIGN, int N1>
SIP_HD void comp_inner(float2 (&v)[R]) {
    if constexpr (N1 < A) {
        float2 t[B];
#pragma unroll
        for (int n2 = 0; n2 < B; ++n2) t[n2] = v[N1 + A * n2];
        dft<B, SIGN>(t);
        comp_twiddle<R, A, B, SIGN, N1, 0>(v, t);
        comp_inner<R, A, B, SIGN, N1 + 1>(v);
    }
}

template <int R, int SIGN>
SIP_HD void dft_composite(float2 (&v)[R]) {
    constexpr int A = cx_split(R);
    constexpr int B = R / A;
    comp_inner<R, A, B, SIGN, 0>(v);
    float2 out[R];
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) {
        float2 t[A];
#pragma unroll
        for (int n1 = 0; n1 < A; ++n1) t[n1] = v[n1 + A * k2];
        dft<A, SIGN>(t);
#pragma unroll
        for (int k1 = 0; k1 < A; ++k1) out[B * k1 + k2] = t[k1];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = out[i];
}

template <int R, int SIGN>
SIP_HD void dft(float2 (&v)[R]) {
    if constexpr (R == 1) {
    } else if constexpr (R == 2) {
        dft2<SIGN>(v);
    } else if constexpr (R == 4) {
        dft4<SIGN>(v);
    } else if constexpr (cx_is_prime(R)) {
        dft_prime<R, SIGN>(v);
    } else {
        dft_composite<R, SIGN>(v);
    }
}

// ------------------------------------------------------- fast division
// Exact unsigned division by a runtime constant d (1 <= d < 2^31) for any
// 32-bit dividend: q = (mulhi(m, n) + n) >> s with s = ceil(log2 d) and
// m = floor(2^32 (2^s - d) / d) + 1 (the round-up method of Granlund and
// Montgomery, "Division by invariant integers using multiplication", 1994).
struct FastDiv {
    uint32_t d;
    uint32_t m;
    uint32_t s;
};

inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f{d, 0, 0};
    uint32_t s = 0;
    while ((1ull << s) < d) ++s;
    f.s = s;
    f.m = (uint32_t)(((1ull << 32) * ((1ull << s) - d)) / d + 1);
    return f;
}

SIP_HD uint32_t fd_div(const FastDiv& f, uint32_t n) {
#if defined(__CUDA_ARCH__)
    const uint32_t hi = __umulhi(f.m, n);
#else
    const uint32_t hi = (uint32_t)(((uint64_t)f.m * n) >> 32);
#endif
    return (uint32_t)(((uint64_t)hi + n) >> f.s);
}

// ------------------------------------------------------------ tile layout
// Element n of transform p of a tile lives at p * LD + n + n / 16: one pad
// slot per 16 complex values spreads the strided writes of the early
// passes over distinct shared-memory bank pairs.
SIP_HD constexpr int sidx(int n) { return n + (n >> 4); }

constexpr int kMaxPasses = 12;

struct PassDesc {
    int R;       // radix
    int L;       // product of the radices of the earlier passes
    int tw;      // offset of this pass's twiddles in the Stockham table
    FastDiv nr;  // division by N / R
    FastDiv l;   // division by L
};

struct PlanDev {
    int N;      // transform length
    int npass;  // number of passes
    PassDesc pass[kMaxPasses];
};

// Registers one thread carries between the read and write halves of a pass.
template <int R, int S>
struct PassRegs {
    float2 v[S][R];
};

constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Read half of a pass: gather the butterflies this thread owns (butterfly
// b = tid + s T over all P transforms of the tile), twiddle, transform.
// `tw` is the plan's Stockham table of forward twiddles: for a pass with
// span L > 1, entry pd.tw + (r-1) L + k is W_{L R}^{r k} (twiddle-major, so
// the consecutive k of a warp read consecutive entries).
template <int R, int SIGN, int S>
SIP_HD void pass_read(int tid, int T, int P, int N, const float2* sm, int LD, const PassDesc& pd,
                      const float2* __restrict__ tw, PassRegs<R, S>& rg) {
    const int NR = (int)pd.nr.d;
    const int total = P * NR;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int b = tid + s * T;
        if (b < total) {
            const int p = (int)fd_div(pd.nr, (uint32_t)b);
            const int j = b - p * NR;
            const float2* row = sm + p * LD;
#pragma unroll
            for (int r = 0; r < R; ++r) rg.v[s][r] = row[sidx(j + r * NR)];
            if (pd.L > 1) {
                const int k = j - (int)fd_div(pd.l, (uint32_t)j) * pd.L;
                const float2* w = tw + pd.tw + k;
#pragma unroll
                for (int r = 1; r < R; ++r) rg.v[s][r] = c_tw<SIGN>(rg.v[s][r], SIP_LDG(w + (r - 1) * pd.L));
            }
            dft<R, SIGN>(rg.v[s]);
        }
    }
    (void)N;
}

// Write half of a pass: scatter the transformed butterflies to their
// self-sorted positions.
template <int R, int S>
SIP_HD void pass_write(int tid, int T, int P, float2* sm, int LD, const PassDesc& pd, const PassRegs<R, S>& rg) {
    const int NR = (int)pd.nr.d;
    const int total = P * NR;
#pragma unroll
    for (int s = 0; s < S; ++s) {
        const int b = tid + s * T;
        if (b < total) {
            const int p = (int)fd_div(pd.nr, (uint32_t)b);
            const int j = b - p * NR;
            const int g = (int)fd_div(pd.l, (uint32_t)j);
            const int k = j - g * pd.L;
            const int o = g * pd.L * R + k;
            float2* row = sm + p * LD;
#pragma unroll
            for (int r = 0; r < R; ++r) row[sidx(o + r * pd.L)] = rg.v[s][r];
        }
    }
}

// Twiddle basis of a radix: a pass with span L > 1 needs W^{r k} for
// r < R.  Writing r = r_lo + a r_hi (r_lo < a), the "basis" table holds, per
// k, the a - 1 values W^{r_lo k} followed by the R/a - 1 values
// W^{a r_hi k}; every other twiddle is one product of two table entries.
// a is the divisor of R that minimises the entry count (R itself for a
// prime, which degenerates to the full table).
constexpr int basis_split(int R) {
    int best = R, cost = R - 1;
    for (int d = 2; d < R; ++d)
        if (R % d == 0 && (d - 1) + (R / d - 1) < cost) {
            cost = (d - 1) + (R / d - 1);
            best = d;
        }
    return best;
}
constexpr int basis_count(int R) {
    const int a = basis_split(R);
    return (a - 1) + (R / a - 1);
}

// The radices a plan may use; every entry has a compiled pass.
#define SIP_FFT_FOR_EACH_RADIX(X) \
    X(2) X(3) X(4) X(5) X(7) X(8) X(9) X(10) X(11) X(13) X(15) X(16) X(17) X(19) X(23) X(25) X(27) X(29) X(31) X(32)

inline bool radix_supported(int r) {
    switch (r) {
#define SIP_CASE_(R) case R:
        SIP_FFT_FOR_EACH_RADIX(SIP_CASE_)
#undef SIP_CASE_
        return true;
        default:
            return false;
    }
}

}  // namespace sipfft
