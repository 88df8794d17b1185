// Element formulas of the real-transform pre/post passes for lengths
// beyond one tile, shared by real_kernels.cu and the CPU test harness.
// They are the formulas of the fused tile stores/loads in tile_io.cuh,
// after the reference's fft_real_stockham_r2c.cpp:60-105 (post-process)
// and fft_real_stockham_c2r.cpp:73-100 (even pre-process).
#pragma once

#include "fft_core.cuh"

namespace sipfft {

// X[k], k in [0, m], from the half-length spectrum row z (m values).
SIP_HD float2 real_post_elem(const float2* z, long long k, long long m, const float2* tw, bool conj) {
    const float2 zk = SIP_LDG(z + (k == m ? 0 : k));
    const float2 zm = SIP_LDG(z + (k == 0 ? 0 : m - k));
    const float2 b = make_float2(zm.x, -zm.y);
    const float2 ev = make_float2(0.5f * (zk.x + b.x), 0.5f * (zk.y + b.y));
    const float2 od = make_float2(0.5f * (zk.y - b.y), -0.5f * (zk.x - b.x));
    float2 v = c_add(ev, c_mul(SIP_LDG(tw + k), od));
    if (conj) v.y = -v.y;
    return v;
}

// Z[k], k in [0, m), from the half spectrum row x (m + 1 values).
SIP_HD float2 real_pre_elem(const float2* x, long long k, long long m, const float2* tw, bool conj) {
    if (k == 0) {
        const float dc = SIP_LDG(x).x, ny = SIP_LDG(x + m).x;
        return make_float2(0.5f * (dc + ny), 0.5f * (dc - ny));
    }
    float2 xv = SIP_LDG(x + k), yv = SIP_LDG(x + m - k);
    if (conj) {
        xv.y = -xv.y;
        yv.y = -yv.y;
    }
    const float2 b = make_float2(yv.x, -yv.y);
    const float2 e = make_float2(0.5f * (xv.x + b.x), 0.5f * (xv.y + b.y));
    const float2 d = make_float2(0.5f * (xv.x - b.x), 0.5f * (xv.y - b.y));
    const float2 od = c_mulc(d, SIP_LDG(tw + k));
    return make_float2(e.x - od.y, e.y + od.x);
}

// X[k] and X[m - k] for 0 < k < m - k: one read of z[k], z[m - k] and
// W_{2m}^k; the mirror uses W_{2m}^{m-k} = -conj(W_{2m}^k), so
// X[m - k] = conj(ev - W od) where X[k] = ev + W od.
SIP_HD void real_post_pair(const float2* z, long long k, long long m, const float2* tw, bool conj, float2* xk,
                           float2* xmk) {
    const float2 zk = SIP_LDG(z + k);
    const float2 zm = SIP_LDG(z + m - k);
    const float2 b = make_float2(zm.x, -zm.y);
    const float2 ev = make_float2(0.5f * (zk.x + b.x), 0.5f * (zk.y + b.y));
    const float2 od = make_float2(0.5f * (zk.y - b.y), -0.5f * (zk.x - b.x));
    const float2 t = c_mul(SIP_LDG(tw + k), od);
    float2 v = c_add(ev, t);
    float2 w = make_float2(ev.x - t.x, -(ev.y - t.y));
    if (conj) {
        v.y = -v.y;
        w.y = -w.y;
    }
    *xk = v;
    *xmk = w;
}

// Z[k] and Z[m - k] for 0 < k < m - k from x[k], x[m - k] and W_{2m}^k:
// with Z[k] = e + i W^{-k} d (e, d from x[k] and conj x[m - k]), the mirror
// is Z[m - k] = conj(e) + conj(i W^{-k} d) (its e is conj(e), its d is
// -conj(d), and W^{-(m-k)} = -conj(W^{-k})).
SIP_HD void real_pre_pair(const float2* x, long long k, long long m, const float2* tw, bool conj, float2* zk,
                          float2* zmk) {
    float2 xv = SIP_LDG(x + k), yv = SIP_LDG(x + m - k);
    if (conj) {
        xv.y = -xv.y;
        yv.y = -yv.y;
    }
    const float2 b = make_float2(yv.x, -yv.y);
    const float2 e = make_float2(0.5f * (xv.x + b.x), 0.5f * (xv.y + b.y));
    const float2 d = make_float2(0.5f * (xv.x - b.x), 0.5f * (xv.y - b.y));
    const float2 od = c_mulc(d, SIP_LDG(tw + k));
    *zk = make_float2(e.x - od.y, e.y + od.x);
    *zmk = make_float2(e.x + od.y, -e.y + od.x);
}

// ---------------------------------------- odd real lengths above one tile
// Two real rows travel as one complex row z = x_a + i x_b of length n
// (the two-rows-per-transform packing of tile_io.cuh load_r2c_pair /
// store_r2c_pair, applied to whole rows around the complex four-step).

// Bin k <= n/2 of rows a and b from Z = FFT(z): (Z[k] + conj Z[n-k]) / 2 and
// (Z[k] - conj Z[n-k]) / 2i, conjugated for the inverse direction.
SIP_HD void pair_separate_elem(const float2* z, long long k, long long n, bool conj, float2* xa, float2* xb) {
    const float2 zk = SIP_LDG(z + k), zm = SIP_LDG(z + (k == 0 ? 0 : n - k));
    float2 a = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    float2 b = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    if (conj) {
        a.y = -a.y;
        b.y = -b.y;
    }
    *xa = a;
    *xb = b;
}

// Z[k], k < n, of the complex row that carries the spectra of rows a and b
// (half spectra of n/2 + 1 bins; xb null: a zero row): Xa[k] + i Xb[k] with
// the Hermitian halves, the DC bin's imaginary parts ignored; `fwd`
// (C2R forward, hfft) conjugates the input spectra.
SIP_HD float2 pair_combine_elem(const float2* xa, const float2* xb, long long k, long long n, bool fwd) {
    const long long kk = 2 * k <= n ? k : n - k;
    float2 a = SIP_LDG(xa + kk);
    float2 b = xb != nullptr ? SIP_LDG(xb + kk) : make_float2(0.f, 0.f);
    if (kk == 0) {
        a.y = 0.f;
        b.y = 0.f;
    }
    if ((2 * k > n) != fwd) {
        a.y = -a.y;
        b.y = -b.y;
    }
    return make_float2(a.x - b.y, a.y + b.x);
}

}  // namespace sipfft
