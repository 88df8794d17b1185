// Host parts of Bluestein's algorithm (bluestein.cuh): the convolution
// length and the FP64 convolution filter, computed with a self-sorting
// Stockham FFT over the radices 4, 2, 3, 5 on the host.
#include <cmath>
#include <complex>
#include <stdexcept>
#include <vector>

#include "bluestein.h"

namespace sipfft {

namespace {

using cd = std::complex<double>;

bool smooth235(long long m) {
    for (long long p : {2LL, 3LL, 5LL})
        while (m % p == 0) m /= p;
    return m == 1;
}

// Forward DFT (exp(-2 pi i jk / n)) of x, n 2,3,5-smooth.
void fft_host(std::vector<cd>& x) {
    const long long n = (long long)x.size();
    std::vector<int> radices;
    long long r = n;
    while (r % 4 == 0) {
        radices.push_back(4);
        r /= 4;
    }
    for (int p : {2, 3, 5})
        while (r % p == 0) {
            radices.push_back(p);
            r /= p;
        }
    if (r != 1) throw std::invalid_argument("length is not 2,3,5-smooth");
    std::vector<cd> y(n);
    long long L = 1;
    const double two_pi = 2.0 * 3.14159265358979323846264338327950288;
    for (int R : radices) {
        const long long nr = n / R;
        for (long long j = 0; j < nr; ++j) {
            const long long k = j % L;
            cd v[5];
            for (int q = 0; q < R; ++q) {
                const long long e = (long long)q * k % (L * R);
                const cd w = std::polar(1.0, -two_pi * (double)e / (double)(L * R));
                v[q] = x[j + q * nr] * w;
            }
            const long long base = (j / L) * L * R + k;
            for (int o = 0; o < R; ++o) {
                cd s = 0;
                for (int q = 0; q < R; ++q) s += v[q] * std::polar(1.0, -two_pi * (double)((q * o) % R) / R);
                y[base + o * L] = s;
            }
        }
        x.swap(y);
        L *= R;
    }
}

}  // namespace

long long bluestein_length(long long n) {
    long long m = 2 * n - 1;
    while (!smooth235(m)) ++m;
    return m;
}

std::vector<float2> bluestein_filter(long long n, long long m, int sign) {
    std::vector<cd> b(m, cd(0, 0));
    const double pi = 3.14159265358979323846264338327950288;
    for (long long j = 0; j < n; ++j) {
        const long long q = (j * j) % (2 * n);
        const cd c = std::polar(1.0, sign * pi * (double)q / (double)n);
        b[j] = std::conj(c);
        if (j > 0) b[m - j] = std::conj(c);
    }
    fft_host(b);
    std::vector<float2> out(m);
    for (long long i = 0; i < m; ++i) out[i] = make_float2((float)b[i].real(), (float)b[i].imag());
    return out;
}

}  // namespace sipfft
