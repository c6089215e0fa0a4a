/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for packed-b200.
 *
 * A plain-C restatement of the reference library's FFT / correlation path
 * (Dooez/packed), computed in double precision.  Only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it; the product never does.
 * It is pinned against outputs of the reference itself (fixtures under
 * tests/golden/, generated from the reference headers compiled by
 * oracle/Makefile into oracle/_ref/).
 *
 * What it restates, with the reference file:line each part follows:
 *  - packed split-complex layout, pidx<P>: vector.hpp:373-381,
 *    element_access.hpp:8-11; P = 1 interleaved: types.hpp:119-148.
 *  - forward DFT X[k] = sum_n x[n] e^{-2 pi i n k / N}, no scale:
 *    fft.hpp:728-750 (radix-2 decimation in time as in the reference's own
 *    test oracle tests/test_fft.cpp:66-99; twiddles wnk fft.hpp:77-87).
 *  - inverse with 1/N when normalised: fft.hpp:689-721, 828-915.
 *  - orders (fft.hpp:540-544): bit_reversed = bit reversal of normal order;
 *    unordered keeps at position p the frequency bitrev(sigma(p)), sigma
 *    moving bits (0,1,2,3) of p to (2,1,3,0) (established by running the
 *    reference, tests/golden/make_golden.py).
 *  - zero extension of short sources: fft.hpp:671-681, 1759-1795.
 *  - overlap-save correlation: fxcorr.hpp:62-136, with the block offset taken
 *    as an element index (pidx) and whole elements copied back;
 *    ground truth y[n] = sum_{j<K} x[n+j] conj(g[j]) as in
 *    tests/test_fxcorr.cpp:15-32.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static const double PI = 3.14159265358979323846264338327950288;

static size_t log2z(size_t n) {
    size_t l = 0;
    while ((n >> l) > 1) ++l;
    return l;
}

static size_t brev(size_t k, size_t bits) {
    size_t r = 0;
    for (size_t i = 0; i < bits; ++i) r |= ((k >> i) & 1u) << (bits - 1 - i);
    return r;
}

/* Position that holds frequency k (order 0 normal, 1 bit_reversed, 2 unordered). */
size_t orc_order_pos(size_t k, int order, size_t n) {
    size_t bits = log2z(n);
    if (order == 0) return k;
    size_t q = brev(k, bits);
    if (order == 1) return q;
    /* sigma^-1: bits (0,1,2,3) of q go to (3,1,0,2) */
    return (q & ~(size_t)15) | ((q >> 2) & 1u) | (q & 2u) | (((q >> 3) & 1u) << 2) | ((q & 1u) << 3);
}

/* In-place radix-2 DIT FFT of interleaved complex double data.
 * sign -1: forward (no scale); +1: inverse kernel (no scale). */
void orc_fft_c128(double* z, size_t n, int inverse) {
    size_t bits = log2z(n);
    for (size_t i = 0; i < n; ++i) {
        size_t j = brev(i, bits);
        if (i < j) {
            double tr = z[2 * i], ti = z[2 * i + 1];
            z[2 * i]         = z[2 * j];
            z[2 * i + 1]     = z[2 * j + 1];
            z[2 * j]         = tr;
            z[2 * j + 1]     = ti;
        }
    }
    const double sgn = inverse ? 1.0 : -1.0;
    for (size_t len = 2; len <= n; len <<= 1) {
        size_t half = len >> 1;
        for (size_t k = 0; k < half; ++k) {
            /* wnk(len, k) evaluated in double (fft.hpp:77-87 evaluates it in T) */
            double a  = sgn * 2.0 * PI * (double)k / (double)len;
            double wr = cos(a), wi = sin(a);
            if (4 * k == len) { wr = 0.0; wi = sgn; }
            for (size_t s = 0; s < n; s += len) {
                double* p = z + 2 * (s + k);
                double* q = z + 2 * (s + k + half);
                double  xr = q[0] * wr - q[1] * wi;
                double  xi = q[0] * wi + q[1] * wr;
                q[0]       = p[0] - xr;
                q[1]       = p[1] - xi;
                p[0] += xr;
                p[1] += xi;
            }
        }
    }
}

/* Direct DFT (O(n^2), long double accumulation) for pinning small sizes. */
void orc_dft_c128(const double* x, double* X, size_t n, int inverse) {
    const long double sgn = inverse ? 1.0L : -1.0L;
    for (size_t k = 0; k < n; ++k) {
        long double sr = 0, si = 0;
        for (size_t j = 0; j < n; ++j) {
            size_t      e = (j * k) % n;
            long double a = sgn * 2.0L * (long double)PI * (long double)e / (long double)n;
            long double c = cosl(a), s = sinl(a);
            sr += x[2 * j] * c - x[2 * j + 1] * s;
            si += x[2 * j] * s + x[2 * j + 1] * c;
        }
        X[2 * k]     = (double)sr;
        X[2 * k + 1] = (double)si;
    }
}

static size_t pk_re(size_t i, size_t p) { return (i / p) * 2 * p + (i % p); }

/* Reals needed to hold n elements at pack width p (vector.hpp:373-381). */
size_t orc_real_size(size_t n, size_t p) { return (n + p - 1) / p * 2 * p; }

#define ORC_PACK_FNS(T, SUF)                                                                       \
    void orc_unpack_##SUF(const T* src, size_t n, size_t p, double* z) {                           \
        for (size_t i = 0; i < n; ++i) {                                                           \
            z[2 * i]     = (double)src[pk_re(i, p)];                                               \
            z[2 * i + 1] = (double)src[pk_re(i, p) + p];                                           \
        }                                                                                          \
    }                                                                                              \
    void orc_pack_##SUF(const double* z, size_t n, size_t p, T* dst) {                             \
        for (size_t i = 0; i < n; ++i) {                                                           \
            dst[pk_re(i, p)]     = (T)z[2 * i];                                                    \
            dst[pk_re(i, p) + p] = (T)z[2 * i + 1];                                                \
        }                                                                                          \
    }                                                                                              \
    /* Reference-semantics transform of one row (see header).  dir 0 forward    \
     * (natural input, output in `order`), 1 inverse (input in `order`).  */     \
    int orc_fft_packed_##SUF(T* dst, const T* src, size_t n, size_t src_len, size_t pd, size_t ps,  \
                             int order, int dir, int norm) {                                       \
        double* a = (double*)calloc(2 * n, sizeof(double));                                        \
        double* b = (double*)calloc(2 * n, sizeof(double));                                        \
        if (!a || !b) { free(a); free(b); return 1; }                                              \
        if (src_len == 0 || src_len > n) src_len = n;                                              \
        orc_unpack_##SUF(src, src_len, ps, a);                                                     \
        if (dir == 0) {                                                                            \
            orc_fft_c128(a, n, 0);                                                                 \
            for (size_t k = 0; k < n; ++k) {                                                       \
                size_t q     = orc_order_pos(k, order, n);                                         \
                b[2 * q]     = a[2 * k];                                                           \
                b[2 * q + 1] = a[2 * k + 1];                                                       \
            }                                                                                      \
        } else {                                                                                   \
            for (size_t k = 0; k < n; ++k) {                                                       \
                size_t q     = orc_order_pos(k, order, n);                                         \
                b[2 * k]     = a[2 * q];                                                           \
                b[2 * k + 1] = a[2 * q + 1];                                                       \
            }                                                                                      \
            orc_fft_c128(b, n, 1);                                                                 \
            if (norm) {                                                                            \
                for (size_t i = 0; i < 2 * n; ++i) b[i] /= (double)n;                              \
            }                                                                                      \
        }                                                                                          \
        orc_pack_##SUF(b, n, pd, dst);                                                             \
        free(a);                                                                                   \
        free(b);                                                                                   \
        return 0;                                                                                  \
    }

ORC_PACK_FNS(float, f32)
ORC_PACK_FNS(double, f64)

/* y[i] = sum_{j<k, i+j<s} x[i+j] conj(g[j]); interleaved complex double. */
void orc_xcorr_direct(const double* x, size_t s, const double* g, size_t k, double* y) {
    for (size_t i = 0; i < s; ++i) {
        long double yr = 0, yi = 0;
        for (size_t j = 0; j < k && i + j < s; ++j) {
            double xr = x[2 * (i + j)], xi = x[2 * (i + j) + 1];
            double gr = g[2 * j], gi = -g[2 * j + 1];
            yr += xr * gr - xi * gi;
            yi += xr * gi + xi * gr;
        }
        y[2 * i]     = (double)yr;
        y[2 * i + 1] = (double)yi;
    }
}

/* Overlap-save as in fxcorr.hpp:102-136 (corrected offsets), in double.
 * step = floor((n_fft - (k-1)) / p) * p with p the signal's pack width. */
int orc_xcorr_ols(const double* x, size_t s, const double* g, size_t k, size_t n_fft, size_t p, double* y) {
    if (k == 0 || k > n_fft) return 1;
    size_t step = (n_fft - (k - 1)) / p * p;
    if (step == 0) return 1;
    double* kern = (double*)calloc(2 * n_fft, sizeof(double));
    double* tmp  = (double*)calloc(2 * n_fft, sizeof(double));
    if (!kern || !tmp) { free(kern); free(tmp); return 1; }
    memcpy(kern, g, 2 * k * sizeof(double));
    orc_fft_c128(kern, n_fft, 0);
    for (size_t off = 0; off < s; off += step) {
        size_t avail = s - off < n_fft ? s - off : n_fft;
        memset(tmp, 0, 2 * n_fft * sizeof(double));
        memcpy(tmp, x + 2 * off, 2 * avail * sizeof(double));
        orc_fft_c128(tmp, n_fft, 0);
        for (size_t i = 0; i < n_fft; ++i) {
            double ar = tmp[2 * i], ai = tmp[2 * i + 1];
            double br = kern[2 * i] / (double)n_fft, bi = -kern[2 * i + 1] / (double)n_fft;
            tmp[2 * i]     = ar * br - ai * bi;
            tmp[2 * i + 1] = ar * bi + ai * br;
        }
        orc_fft_c128(tmp, n_fft, 1);
        size_t l = s - off < step ? s - off : step;
        memcpy(y + 2 * off, tmp, 2 * l * sizeof(double));
    }
    free(kern);
    free(tmp);
    return 0;
}

/* Adjoint of orc_xcorr_direct for a real loss with cotangent gy
 * (d/dRe + i d/dIm convention): gx[m] = sum_j g[j] gy[m-j] (convolution),
 * gg[j] = sum_i x[i+j] conj(gy[i]) (correlation of gy with x). */
void orc_xcorr_vjp_direct(const double* x, size_t s, const double* g, size_t k, const double* gy, double* gx,
                          double* gg) {
    for (size_t m = 0; m < s; ++m) {
        long double r = 0, im = 0;
        for (size_t j = 0; j < k && j <= m; ++j) {
            double gr = g[2 * j], gi = g[2 * j + 1];
            double yr = gy[2 * (m - j)], yi = gy[2 * (m - j) + 1];
            r += gr * yr - gi * yi;
            im += gr * yi + gi * yr;
        }
        gx[2 * m]     = (double)r;
        gx[2 * m + 1] = (double)im;
    }
    if (!gg) return;
    for (size_t j = 0; j < k; ++j) {
        long double r = 0, im = 0;
        for (size_t i = 0; i + j < s; ++i) {
            double xr = x[2 * (i + j)], xi = x[2 * (i + j) + 1];
            double yr = gy[2 * i], yi = -gy[2 * i + 1];
            r += xr * yr - xi * yi;
            im += xr * yi + xi * yr;
        }
        gg[2 * j]     = (double)r;
        gg[2 * j + 1] = (double)im;
    }
}
