/*
 * Test infrastructure (oracle), not product code.
 *
 * A small FP64 implementation of the FFTW3 calls that empi's workspace makes
 * (inc/fftw.hpp:33,43,112,125,137,152 in the reference), so that the
 * reference's own sources (src/*.cpp) can be built here without FFTW.  empi
 * only ever plans power-of-two lengths (inc/fftw.hpp:161-168, fftwRound), so
 * this is the iterative radix-2 Cooley-Tukey method with a per-plan twiddle
 * table computed in long double.  A real-to-complex transform of length n runs
 * as one complex transform of length n/2 on the even/odd packed input followed
 * by the usual split step.  Forward sign is -1 as in FFTW, outputs are
 * unnormalised, the r2c output holds n/2+1 bins.
 *
 * Plans are independent: fftw_execute on distinct plans may run concurrently
 * (empi executes one plan per OpenMP thread, src/gabor.cpp:77-82,198-208).
 */
#include "fftw3.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct empi_shim_plan {
    int kind;          /* 0 = c2c, 1 = r2c */
    int n;             /* logical transform length */
    int m;             /* complex FFT length actually run */
    int sign;
    double* in;
    double* out;       /* interleaved complex */
    double* tw;        /* m/2 twiddles for the length-m FFT (interleaved) */
    double* split;     /* n/2 twiddles W_n^k for the r2c split step */
    double* work;      /* m complex scratch */
    int* rev;          /* bit reversal of length m */
};

void* fftw_malloc(size_t n) {
    void* p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    return p;
}

void fftw_free(void* p) { free(p); }

static void fill_twiddles(double* dst, int len, int count, int sign) {
    /* dst[2k], dst[2k+1] = exp(sign * 2 pi i k / len), k < count */
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k < count; ++k) {
        long double a = two_pi * (long double)k / (long double)len;
        dst[2 * k] = (double)cosl(a);
        dst[2 * k + 1] = (double)(sign * sinl(a));
    }
}

static int* make_rev(int m) {
    int* rev = (int*)malloc(sizeof(int) * (size_t)(m > 0 ? m : 1));
    int bits = 0;
    while ((1 << bits) < m) ++bits;
    for (int i = 0; i < m; ++i) {
        int r = 0;
        for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
        rev[i] = r;
    }
    return rev;
}

/* In-place iterative radix-2 DIT on a bit-reversed array of m complex values. */
static void fft_inplace(double* a, int m, const double* tw) {
    for (int len = 2; len <= m; len <<= 1) {
        int half = len >> 1;
        int step = m / len;
        for (int base = 0; base < m; base += len) {
            for (int j = 0; j < half; ++j) {
                double wr = tw[2 * (j * step)], wi = tw[2 * (j * step) + 1];
                double* p = a + 2 * (base + j);
                double* q = a + 2 * (base + j + half);
                double xr = q[0] * wr - q[1] * wi;
                double xi = q[0] * wi + q[1] * wr;
                q[0] = p[0] - xr;
                q[1] = p[1] - xi;
                p[0] += xr;
                p[1] += xi;
            }
        }
    }
}

static fftw_plan new_plan(int kind, int n, int m, int sign, double* in, double* out) {
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    if (!p) return NULL;
    p->kind = kind;
    p->n = n;
    p->m = m;
    p->sign = sign;
    p->in = in;
    p->out = out;
    p->tw = (double*)malloc(sizeof(double) * 2 * (size_t)(m / 2 + 1));
    p->work = (double*)malloc(sizeof(double) * 2 * (size_t)(m > 0 ? m : 1));
    p->rev = make_rev(m);
    fill_twiddles(p->tw, m, m / 2 + 1, sign);
    if (kind == 1) {
        p->split = (double*)malloc(sizeof(double) * 2 * (size_t)(n / 2 + 1));
        fill_twiddles(p->split, n, n / 2 + 1, -1);
    }
    return p;
}

fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags) {
    (void)flags;
    if (n < 1 || (n & (n - 1))) return NULL;
    return new_plan(0, n, n, sign < 0 ? -1 : +1, (double*)in, (double*)out);
}

fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags) {
    (void)flags;
    if (n < 2 || (n & (n - 1))) return NULL;
    return new_plan(1, n, n / 2, -1, in, (double*)out);
}

void fftw_execute(const fftw_plan p) {
    if (!p) return;
    const int m = p->m;
    double* w = p->work;
    if (p->kind == 0) {
        for (int i = 0; i < m; ++i) {
            w[2 * p->rev[i]] = p->in[2 * i];
            w[2 * p->rev[i] + 1] = p->in[2 * i + 1];
        }
        fft_inplace(w, m, p->tw);
        memcpy(p->out, w, sizeof(double) * 2 * (size_t)m);
        return;
    }
    /* r2c: z[j] = x[2j] + i x[2j+1], Z = FFT_m(z), then split. */
    for (int i = 0; i < m; ++i) {
        w[2 * p->rev[i]] = p->in[2 * i];
        w[2 * p->rev[i] + 1] = p->in[2 * i + 1];
    }
    fft_inplace(w, m, p->tw);
    double* X = p->out;
    for (int k = 0; k <= m; ++k) {
        int k1 = k % m, k2 = (m - k) % m;
        double ar = w[2 * k1], ai = w[2 * k1 + 1];
        double br = w[2 * k2], bi = -w[2 * k2 + 1];          /* conj(Z[m-k]) */
        double er = 0.5 * (ar + br), ei = 0.5 * (ai + bi);   /* even part */
        double dr = 0.5 * (ar - br), di = 0.5 * (ai - bi);   /* (A-B)/2 */
        /* odd part = (A-B)/(2i) = -i (A-B)/2 */
        double orr = di, oi = -dr;
        double wr = p->split[2 * k], wi = p->split[2 * k + 1];
        X[2 * k] = er + (orr * wr - oi * wi);
        X[2 * k + 1] = ei + (orr * wi + oi * wr);
    }
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->tw);
    free(p->work);
    free(p->rev);
    free(p->split);
    free(p);
}
