/*
 * ORACLE — CPU restatement of the reference's FFT arithmetic.  Test
 * infrastructure only: the tests, __graft_entry__.smoke() and bench.py's
 * CPU-baseline / reference arm use it as the checker and the timed CPU
 * baseline; the library never calls it.
 *
 * What it restates (hicann/sip paths, relative to the reference root):
 *   - self-sorting DIT mixed-radix Stockham stage:
 *       ops/fft/real/fft_stockham/fft_stockham/kernel/arch35/vendor/
 *       fft_stockham_mix.h:1089-1200 (stockhamForwardGeneral: for block,
 *       q < radix, j < prev, out[block*len + q*prev + j] =
 *       sum_p dft[q][p] * tw[p][j] * in[block*prev + j + p*part])
 *       driven stage by stage as in runStockhamForward :1218-1267;
 *   - coefficient layouts: ops/include/params/fft_real_stockham.h:77-111
 *       (dft[q*r+p] = exp(sign 2 pi i p q / r), tw[p*prev+j] =
 *       exp(sign 2 pi i p j / len), real twiddles exp(sign 2 pi i k / N),
 *       FP64 angles rounded once to float), radix order 2,3,5,7 ascending
 *       (fft_real_stockham.h:47-55), extended here to any prime factor;
 *   - R2C: pack / post-process / odd zero-imaginary pack + truncate,
 *       fft_real_stockham_r2c.cpp:28-124;
 *   - C2R: Hermitian expand / even pre-process / unpack x2 / store real,
 *       fft_real_stockham_c2r.cpp:23-110.
 * The float entry points keep the reference's FP32 arithmetic (float
 * tables, float accumulation); the double entry points are the FP64
 * oracle.  Rows are split over `orc_set_threads` POSIX threads.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_TWO_PI 6.283185307179586476925286766559

static int g_threads = 1;

void orc_set_threads(int n) { g_threads = n < 1 ? 1 : n; }
int orc_get_threads(void) { return g_threads; }

/* ---------------------------------------------------------------- LCG */
/* Deterministic inputs of the reference's unit tests:
 * tests/ut/framework/test_util/float_util.h:23-36 (state = state *
 * 1664525 + 1013904223; value = lo + state * 2^-32 * (hi - lo), in
 * float) seeded with 2026 (tests/ut/framework/test_util/util.cpp:324).
 * Complex tensors draw the real then the imaginary part (util.cpp:335). */
void orc_lcg_uniform(uint32_t* state, float lo, float hi, int64_t count, float* out) {
    const float inv = 1.0f / 4294967296.0f;
    uint32_t s = *state;
    for (int64_t i = 0; i < count; ++i) {
        s = s * 1664525u + 1013904223u;
        out[i] = lo + ((float)s * inv) * (hi - lo);
    }
    *state = s;
}

/* ----------------------------------------------------------- factoring */
static int orc_radices(int64_t n, int* out) {
    int cnt = 0;
    static const int first[4] = {2, 3, 5, 7};
    for (int i = 0; i < 4; ++i)
        while (n % first[i] == 0) {
            out[cnt++] = first[i];
            n /= first[i];
        }
    for (int64_t p = 11; p * p <= n; p += 2)
        while (n % p == 0) {
            out[cnt++] = (int)p;
            n /= p;
        }
    if (n > 1) out[cnt++] = (int)n;
    return cnt;
}

/* Stockham over one row for element type T (float or double). */
#define ORC_DEFINE_STOCKHAM(T, SUF)                                                                         \
    static void orc_stockham_row_##SUF(int64_t n, int sign, const int* radices, int nr, const T* dft_all,   \
                                       const T* tw_all, T* ws0, T* ws1, T** result) {                        \
        int64_t len = 1, twoff = 0, dftoff = 0;                                                              \
        T* src = ws0;                                                                                        \
        T* dst = ws1;                                                                                        \
        (void)sign;                                                                                          \
        for (int s = 0; s < nr; ++s) {                                                                       \
            const int64_t r = radices[s], prev = len;                                                        \
            len *= r;                                                                                        \
            const int64_t part = n / r, blocks = n / len;                                                    \
            const T* dft = dft_all + 2 * dftoff;                                                             \
            const T* tw = tw_all + 2 * twoff;                                                                \
            for (int64_t block = 0; block < blocks; ++block)                                                 \
                for (int64_t q = 0; q < r; ++q)                                                              \
                    for (int64_t j = 0; j < prev; ++j) {                                                     \
                        T re = 0, im = 0;                                                                    \
                        int64_t in_idx = block * prev + j;                                                   \
                        for (int64_t p = 0; p < r; ++p, in_idx += part) {                                    \
                            const T xr = src[2 * in_idx], xi = src[2 * in_idx + 1];                          \
                            T br = xr, bi = xi;                                                              \
                            if (p > 0) {                                                                     \
                                const T twr = tw[2 * (p * prev + j)], twi = tw[2 * (p * prev + j) + 1];      \
                                br = xr * twr - xi * twi;                                                    \
                                bi = xr * twi + xi * twr;                                                    \
                                const T dr = dft[2 * (q * r + p)], di = dft[2 * (q * r + p) + 1];            \
                                re += br * dr - bi * di;                                                     \
                                im += br * di + bi * dr;                                                     \
                            } else {                                                                         \
                                re += br;                                                                    \
                                im += bi;                                                                    \
                            }                                                                                \
                        }                                                                                    \
                        const int64_t y = block * len + q * prev + j;                                        \
                        dst[2 * y] = re;                                                                     \
                        dst[2 * y + 1] = im;                                                                 \
                    }                                                                                        \
            twoff += r * prev;                                                                               \
            dftoff += r * r;                                                                                 \
            T* t = src;                                                                                      \
            src = dst;                                                                                       \
            dst = t;                                                                                         \
        }                                                                                                    \
        *result = src;                                                                                       \
    }                                                                                                        \
    /* dft / tw tables of fft_real_stockham.h:77-111 (FP64 angle, rounded to T). */                         \
    static void orc_tables_##SUF(int64_t n, int sign, const int* radices, int nr, T** dft, T** tw) {        \
        int64_t dn = 0, tn = 0, prev = 1;                                                                    \
        for (int s = 0; s < nr; ++s) {                                                                       \
            dn += (int64_t)radices[s] * radices[s];                                                          \
            tn += (int64_t)radices[s] * prev;                                                                \
            prev *= radices[s];                                                                              \
        }                                                                                                    \
        *dft = (T*)malloc(sizeof(T) * 2 * (dn > 0 ? dn : 1));                                                \
        *tw = (T*)malloc(sizeof(T) * 2 * (tn > 0 ? tn : 1));                                                 \
        int64_t di = 0, ti = 0;                                                                              \
        prev = 1;                                                                                            \
        for (int s = 0; s < nr; ++s) {                                                                       \
            const int64_t r = radices[s], len = prev * r;                                                    \
            for (int64_t q = 0; q < r; ++q)                                                                  \
                for (int64_t p = 0; p < r; ++p) {                                                            \
                    const double a = sign * ORC_TWO_PI * (double)((p * q) % r) / (double)r;                  \
                    (*dft)[di++] = (T)cos(a);                                                                \
                    (*dft)[di++] = (T)sin(a);                                                                \
                }                                                                                            \
            for (int64_t p = 0; p < r; ++p)                                                                  \
                for (int64_t j = 0; j < prev; ++j) {                                                         \
                    const double a = sign * ORC_TWO_PI * (double)p * (double)j / (double)len;                \
                    (*tw)[ti++] = (T)cos(a);                                                                 \
                    (*tw)[ti++] = (T)sin(a);                                                                 \
                }                                                                                            \
            prev = len;                                                                                      \
        }                                                                                                    \
    }

ORC_DEFINE_STOCKHAM(float, f32)
ORC_DEFINE_STOCKHAM(double, f64)

/* ------------------------------------------------------------ threading */
typedef struct {
    void (*row_fn)(void* ctx, int64_t row, void* scratch);
    void* ctx;
    int64_t rows;
    size_t scratch_bytes;
    int64_t next;
    pthread_mutex_t mu;
} orc_pool_t;

static void* orc_worker(void* arg) {
    orc_pool_t* p = (orc_pool_t*)arg;
    void* scratch = malloc(p->scratch_bytes > 0 ? p->scratch_bytes : 1);
    for (;;) {
        pthread_mutex_lock(&p->mu);
        const int64_t row = p->next++;
        pthread_mutex_unlock(&p->mu);
        if (row >= p->rows) break;
        p->row_fn(p->ctx, row, scratch);
    }
    free(scratch);
    return NULL;
}

static void orc_for_rows(int64_t rows, size_t scratch_bytes, void (*fn)(void*, int64_t, void*), void* ctx) {
    orc_pool_t pool;
    pool.row_fn = fn;
    pool.ctx = ctx;
    pool.rows = rows;
    pool.scratch_bytes = scratch_bytes;
    pool.next = 0;
    pthread_mutex_init(&pool.mu, NULL);
    int nt = g_threads;
    if (nt > rows) nt = (int)(rows > 0 ? rows : 1);
    if (nt <= 1) {
        orc_worker(&pool);
    } else {
        pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nt);
        for (int i = 0; i < nt; ++i) pthread_create(&th[i], NULL, orc_worker, &pool);
        for (int i = 0; i < nt; ++i) pthread_join(th[i], NULL);
        free(th);
    }
    pthread_mutex_destroy(&pool.mu);
}

/* ------------------------------------------------------------------ C2C */
#define ORC_DEFINE_C2C(T, SUF)                                                                             \
    typedef struct {                                                                                       \
        int64_t n;                                                                                         \
        int sign;                                                                                          \
        int radices[64];                                                                                   \
        int nr;                                                                                            \
        T *dft, *tw;                                                                                       \
        const T* in;                                                                                       \
        T* out;                                                                                            \
    } orc_c2c_ctx_##SUF;                                                                                   \
    static void orc_c2c_row_##SUF(void* vctx, int64_t row, void* scratch) {                               \
        orc_c2c_ctx_##SUF* c = (orc_c2c_ctx_##SUF*)vctx;                                                   \
        T* ws0 = (T*)scratch;                                                                              \
        T* ws1 = ws0 + 2 * c->n;                                                                           \
        memcpy(ws0, c->in + 2 * row * c->n, sizeof(T) * 2 * c->n);                                         \
        T* res;                                                                                            \
        orc_stockham_row_##SUF(c->n, c->sign, c->radices, c->nr, c->dft, c->tw, ws0, ws1, &res);           \
        memcpy(c->out + 2 * row * c->n, res, sizeof(T) * 2 * c->n);                                        \
    }                                                                                                      \
    /* Unnormalised complex DFT of `batch` interleaved rows; inverse selects exp(+2 pi i jk / n). */      \
    int orc_c2c_##SUF(int64_t n, int inverse, int64_t batch, const T* in, T* out) {                        \
        orc_c2c_ctx_##SUF c;                                                                               \
        c.n = n;                                                                                           \
        c.sign = inverse ? 1 : -1;                                                                         \
        c.nr = orc_radices(n, c.radices);                                                                  \
        orc_tables_##SUF(n, c.sign, c.radices, c.nr, &c.dft, &c.tw);                                       \
        c.in = in;                                                                                         \
        c.out = out;                                                                                       \
        orc_for_rows(batch, sizeof(T) * 4 * (size_t)n, orc_c2c_row_##SUF, &c);                             \
        free(c.dft);                                                                                       \
        free(c.tw);                                                                                        \
        return 0;                                                                                          \
    }

ORC_DEFINE_C2C(float, f32)
ORC_DEFINE_C2C(double, f64)

/* ------------------------------------------------------------------ R2C */
#define ORC_DEFINE_REAL(T, SUF)                                                                            \
    typedef struct {                                                                                       \
        int64_t n, m;                                                                                      \
        int sign;                                                                                          \
        int radices[64];                                                                                   \
        int nr;                                                                                            \
        T *dft, *tw, *rtw;                                                                                 \
        const T* in;                                                                                       \
        T* out;                                                                                            \
    } orc_real_ctx_##SUF;                                                                                  \
    static T* orc_real_twiddles_##SUF(int64_t n, int64_t count, int sign) {                                \
        T* t = (T*)malloc(sizeof(T) * 2 * (count > 0 ? count : 1));                                        \
        for (int64_t k = 0; k < count; ++k) {                                                              \
            const double a = sign * ORC_TWO_PI * (double)k / (double)n;                                    \
            t[2 * k] = (T)cos(a);                                                                          \
            t[2 * k + 1] = (T)sin(a);                                                                      \
        }                                                                                                  \
        return t;                                                                                          \
    }                                                                                                      \
    /* r2c.cpp:28-124: even N packs pairs, odd N zero-imaginary pack. */                                  \
    static void orc_r2c_row_##SUF(void* vctx, int64_t row, void* scratch) {                               \
        orc_real_ctx_##SUF* c = (orc_real_ctx_##SUF*)vctx;                                                 \
        const int64_t n = c->n, m = c->m, h = n / 2 + 1;                                                   \
        T* ws0 = (T*)scratch;                                                                              \
        T* ws1 = ws0 + 2 * m;                                                                              \
        const T* x = c->in + row * n;                                                                      \
        T* out = c->out + 2 * row * h;                                                                     \
        if (n % 2 == 0) {                                                                                  \
            memcpy(ws0, x, sizeof(T) * n);                                                                 \
        } else {                                                                                           \
            for (int64_t i = 0; i < n; ++i) {                                                              \
                ws0[2 * i] = x[i];                                                                         \
                ws0[2 * i + 1] = 0;                                                                        \
            }                                                                                              \
        }                                                                                                  \
        T* z;                                                                                              \
        orc_stockham_row_##SUF(m, c->sign, c->radices, c->nr, c->dft, c->tw, ws0, ws1, &z);                \
        if (n % 2 == 1) {                                                                                  \
            memcpy(out, z, sizeof(T) * 2 * h);                                                             \
            return;                                                                                        \
        }                                                                                                  \
        for (int64_t k = 0; k < h; ++k) {                                                                  \
            if (k == 0) {                                                                                  \
                out[0] = z[0] + z[1];                                                                      \
                out[1] = 0;                                                                                \
            } else if (k == m) {                                                                           \
                out[2 * k] = z[0] - z[1];                                                                  \
                out[2 * k + 1] = 0;                                                                        \
            } else {                                                                                       \
                const T zr = z[2 * k], zi = z[2 * k + 1];                                                  \
                const T nr_ = z[2 * (m - k)], ni = -z[2 * (m - k) + 1];                                    \
                const T er = (zr + nr_) * (T)0.5, ei = (zi + ni) * (T)0.5;                                 \
                const T orr = (zi - ni) * (T)0.5, oi = (nr_ - zr) * (T)0.5;                                \
                const T wr = c->rtw[2 * k], wi = c->rtw[2 * k + 1];                                        \
                out[2 * k] = er + (wr * orr - wi * oi);                                                    \
                out[2 * k + 1] = ei + (wr * oi + wi * orr);                                                \
            }                                                                                              \
        }                                                                                                  \
    }                                                                                                      \
    /* rfft (forward) or conj(rfft) (inverse) of `batch` rows of n reals -> n/2+1 bins. */                \
    int orc_r2c_##SUF(int64_t n, int inverse, int64_t batch, const T* in, T* out) {                        \
        orc_real_ctx_##SUF c;                                                                              \
        c.n = n;                                                                                           \
        c.m = (n % 2 == 0) ? n / 2 : n;                                                                    \
        c.sign = inverse ? 1 : -1;                                                                         \
        c.nr = orc_radices(c.m, c.radices);                                                                \
        orc_tables_##SUF(c.m, c.sign, c.radices, c.nr, &c.dft, &c.tw);                                     \
        c.rtw = orc_real_twiddles_##SUF(n, n / 2 + 1, c.sign);                                             \
        c.in = in;                                                                                         \
        c.out = out;                                                                                       \
        orc_for_rows(batch, sizeof(T) * 4 * (size_t)c.m, orc_r2c_row_##SUF, &c);                           \
        free(c.dft);                                                                                       \
        free(c.tw);                                                                                        \
        free(c.rtw);                                                                                       \
        return 0;                                                                                          \
    }                                                                                                      \
    /* c2r.cpp:23-110: even N pre-process + unpack x2, odd N Hermitian expand + real part. */             \
    static void orc_c2r_row_##SUF(void* vctx, int64_t row, void* scratch) {                               \
        orc_real_ctx_##SUF* c = (orc_real_ctx_##SUF*)vctx;                                                 \
        const int64_t n = c->n, m = c->m, h = n / 2 + 1;                                                   \
        T* ws0 = (T*)scratch;                                                                              \
        T* ws1 = ws0 + 2 * m;                                                                              \
        const T* x = c->in + 2 * row * h;                                                                  \
        T* out = c->out + row * n;                                                                         \
        if (n % 2 == 1) {                                                                                  \
            for (int64_t k = 0; k < n; ++k) {                                                              \
                if (k < h) {                                                                               \
                    ws0[2 * k] = x[2 * k];                                                                 \
                    ws0[2 * k + 1] = x[2 * k + 1];                                                         \
                } else {                                                                                   \
                    ws0[2 * k] = x[2 * (n - k)];                                                           \
                    ws0[2 * k + 1] = -x[2 * (n - k) + 1];                                                  \
                }                                                                                          \
            }                                                                                              \
        } else {                                                                                           \
            for (int64_t k = 0; k < m; ++k) {                                                              \
                if (k == 0) {                                                                              \
                    const T dc = x[0], ny = x[2 * m];                                                      \
                    ws0[0] = (T)0.5 * (dc + ny);                                                           \
                    ws0[1] = (T)0.5 * (dc - ny);                                                           \
                    continue;                                                                              \
                }                                                                                          \
                const T ar = x[2 * k], ai = x[2 * k + 1];                                                  \
                const T br = x[2 * (m - k)], bi = -x[2 * (m - k) + 1];                                     \
                const T er = (T)0.5 * (ar + br), ei = (T)0.5 * (ai + bi);                                  \
                const T dr = (T)0.5 * (ar - br), di = (T)0.5 * (ai - bi);                                  \
                const T wr = c->rtw[2 * k], wi = c->rtw[2 * k + 1];                                        \
                const T oddr = wr * dr - wi * di, oddi = wr * di + wi * dr;                                \
                ws0[2 * k] = er - oddi;                                                                    \
                ws0[2 * k + 1] = ei + oddr;                                                                \
            }                                                                                              \
        }                                                                                                  \
        T* z;                                                                                              \
        orc_stockham_row_##SUF(m, c->sign, c->radices, c->nr, c->dft, c->tw, ws0, ws1, &z);                \
        if (n % 2 == 1) {                                                                                  \
            for (int64_t i = 0; i < n; ++i) out[i] = z[2 * i];                                             \
        } else {                                                                                           \
            for (int64_t i = 0; i < n; ++i) out[i] = (T)2 * z[i];                                          \
        }                                                                                                  \
    }                                                                                                      \
    /* irfft(norm="forward") (inverse) or hfft (forward) of n/2+1 bins -> n reals per row. */             \
    int orc_c2r_##SUF(int64_t n, int inverse, int64_t batch, const T* in, T* out) {                        \
        orc_real_ctx_##SUF c;                                                                              \
        c.n = n;                                                                                           \
        c.m = (n % 2 == 0) ? n / 2 : n;                                                                    \
        c.sign = inverse ? 1 : -1;                                                                         \
        c.nr = orc_radices(c.m, c.radices);                                                                \
        orc_tables_##SUF(c.m, c.sign, c.radices, c.nr, &c.dft, &c.tw);                                     \
        c.rtw = orc_real_twiddles_##SUF(n, c.m, c.sign);                                                   \
        c.in = in;                                                                                         \
        c.out = out;                                                                                       \
        orc_for_rows(batch, sizeof(T) * 4 * (size_t)c.m, orc_c2r_row_##SUF, &c);                           \
        free(c.dft);                                                                                       \
        free(c.tw);                                                                                        \
        free(c.rtw);                                                                                       \
        return 0;                                                                                          \
    }

ORC_DEFINE_REAL(float, f32)
ORC_DEFINE_REAL(double, f64)
