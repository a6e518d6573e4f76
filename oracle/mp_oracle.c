/*
 * Test infrastructure (oracle), not product code.
 *
 * Plain-C FP64 restatement of empi's Matching Pursuit decomposition loop, the
 * CPU checker for the CUDA engine.  Each function names the reference code it
 * restates (paths relative to the reference project).  It is pinned against
 * the reference's own sources built by oracle/Makefile (_ref/libempiref.so),
 * through tests/test_oracle.py and the fixtures in tests/golden/.
 *
 * Differences from the reference that do not change results:
 *   - maps hold one FP64 energy per (scale, t, f) instead of C complex values
 *     plus an indexed heap (inc/heap.hpp); the winner's complex values are
 *     recomputed from its window when needed;
 *   - the argmax is a linear scan over per-window maxima; ties keep the first
 *     entry in (scale, t, f) order, where the reference's heap/OpenMP order is
 *     arbitrary (src/gabor.cpp:85-107);
 *   - the FFT is this file's radix-2 FP64 transform, not FFTW.
 * The loop also reports, per iteration, the chosen (scale, t, f) indices and
 * the relative margin between the best and second-best energy, so parity
 * checks can exempt near-ties.
 */
#ifndef _GNU_SOURCE
#define _GNU_SOURCE
#endif
#include "mp_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_SQRT2
#define M_SQRT2 1.41421356237309504880
#endif

/* src/gabor.cpp:14,19 */
static const double GAUSS_HALF_WIDTH = 3.0;
static const double MIN_SCALE_IN_SAMPLES = 2.0;

/* inc/fftw.hpp:161-168 */
static long pow2_round(long x) {
    long y = 2;
    while (y < x) y *= 2;
    return y;
}

/* ---------------------------------------------------------------- geometry */

/* GaborWorkspaceBuilder::prepareWorkspace, src/gabor.cpp:213-252 */
int or_geometry(double fs, int N, double energyError, double scaleMin, double scaleMax,
                double freqMax, int cap, or_scale* out) {
    double smin = fmax(scaleMin, MIN_SCALE_IN_SAMPLES / fs);
    double smax = fmin(scaleMax, N / fs);
    double root = sqrt(-2.0 / M_PI * log(1.0 - energyError));
    double aDenomSqrt = 1.0 - energyError;
    double aNominPart = energyError * (2.0 - energyError) * (energyError * energyError - 2 * energyError + 2);
    double a = (1.0 + sqrt(aNominPart)) / (aDenomSqrt * aDenomSqrt);
    double dl = log(a);
    const double tMax = (N - 1) / fs;
    const double lMin = log(smin);
    const double lMax = log(smax);
    long lCount = lrint((lMax - lMin) / dl + 0.5) + 1;
    for (long i = 0; i < lCount; ++i) {
        const double s = exp(lMin + i * (lMax - lMin) / (lCount - 1));
        const double dt = root * s;
        const double df = root / s;
        const double hw = GAUSS_HALF_WIDTH * s;
        const long Ngauss = 2 * lrint(hw * fs - 0.5) + 1;
        long want = lrint(fs / df + 0.5);
        const long Nfft = pow2_round(Ngauss > want ? Ngauss : want);
        const long tCount = lrint(tMax / dt + 0.5) + 1;
        if ((Nfft > tCount ? Nfft : tCount) > 2147483647L) return -2; /* signalFileIsTooLongForThisDecomposition */
        long fCount = Nfft / 2 + 1;
        if (isfinite(freqMax) && freqMax > 0) {
            long fc = lrint(freqMax / fs * Nfft + 0.5) + 1;
            if (fc < fCount) fCount = fc;
        }
        if (i < cap) {
            out[i].s = s;
            out[i].nfft = (int)Nfft;
            out[i].fcount = (int)fCount;
            out[i].tcount = (int)tCount;
        }
    }
    return (int)lCount;
}

/* --------------------------------------------------------------------- FFT */

typedef struct {
    int n;
    double* tw;
    int* rev;
} fftplan;

static void fft_make(fftplan* p, int n) {
    p->n = n;
    p->tw = (double*)malloc(sizeof(double) * 2 * (size_t)(n / 2 + 1));
    p->rev = (int*)malloc(sizeof(int) * (size_t)n);
    const long double two_pi = 6.283185307179586476925286766559005768L;
    for (int k = 0; k <= n / 2; ++k) {
        long double ang = two_pi * (long double)k / (long double)n;
        p->tw[2 * k] = (double)cosl(ang);
        p->tw[2 * k + 1] = (double)(-sinl(ang));
    }
    int bits = 0;
    while ((1 << bits) < n) ++bits;
    for (int i = 0; i < n; ++i) {
        int r = 0;
        for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
        p->rev[i] = r;
    }
}

static void fft_free(fftplan* p) {
    free(p->tw);
    free(p->rev);
}

/* forward complex DFT (sign -1), in[] real of length n, out interleaved */
static void fft_real_input(const fftplan* p, const double* in, double* out) {
    const int n = p->n;
    for (int i = 0; i < n; ++i) {
        out[2 * p->rev[i]] = in[i];
        out[2 * p->rev[i] + 1] = 0.0;
    }
    for (int len = 2; len <= n; len <<= 1) {
        int half = len >> 1, step = n / len;
        for (int base = 0; base < n; base += len)
            for (int j = 0; j < half; ++j) {
                double wr = p->tw[2 * j * step], wi = p->tw[2 * j * step + 1];
                double* a = out + 2 * (base + j);
                double* b = out + 2 * (base + j + half);
                double xr = b[0] * wr - b[1] * wi, xi = b[0] * wi + b[1] * wr;
                b[0] = a[0] - xr;
                b[1] = a[1] - xi;
                a[0] += xr;
                a[1] += xi;
            }
    }
}

/* ------------------------------------------------------------------- maps */

typedef struct {
    or_scale g;
    double fs, tMax;
    int N;
} mapctx;

/* gaussize, src/gabor.cpp:31-40 */
static void gaussize(double* buffer, int n, double step, double center, double width) {
    const double w = sqrt(M_PI) / width;
    const double a = w * step;
    const double b = w * center;
    for (int i = 0; i < n; ++i) {
        const double xw = a * i - b;
        buffer[i] *= exp(-xw * xw);
    }
}

static double map_t(const mapctx* m, int ti) { return ti * m->tMax / (m->g.tcount - 1); } /* src/gabor.cpp:262-264 */
static double map_f(const mapctx* m, int fi) { return fi * m->fs / m->g.nfft; }         /* src/gabor.cpp:265-267 */

/* GaborWorkspaceMap::compute(SingleSignal, c, t), src/gabor.cpp:279-303.
 * work: 3*nfft doubles. values: fcount complex (interleaved). */
static void window_values(const mapctx* m, const fftplan* plan, const double* x, int ti,
                          double* work, double* values) {
    const long N = m->N;
    const double t0 = map_t(m, ti);
    const double hw = GAUSS_HALF_WIDTH * m->g.s;
    long l = lrint((t0 - hw) * m->fs), r = lrint((t0 + hw) * m->fs);
    int iL = (int)(l > 0 ? l : 0);
    int iR = (int)(r < N - 1 ? r : N - 1);
    const double t0fixed = t0 - iL / m->fs;
    double* in = work;
    double* out = work + m->g.nfft;
    memset(in, 0, sizeof(double) * (size_t)m->g.nfft);
    for (int i = iL; i <= iR; ++i) in[i - iL] = x[i];
    gaussize(in, iR - iL + 1, 1.0 / m->fs, t0fixed, m->g.s);
    fft_real_input(plan, in, out);
    const double norm = 1.0 / m->fs;
    const double mult = 2 * M_PI * t0fixed;
    for (int fi = 0; fi < m->g.fcount; ++fi) {
        double ang = map_f(m, fi) * mult;
        double cr = cos(ang), ci = sin(ang);
        double xr = norm * out[2 * fi], xi = norm * out[2 * fi + 1];
        values[2 * fi] = xr * cr - xi * ci;
        values[2 * fi + 1] = xr * ci + xi * cr;
    }
}

/* Mmp1Decomposition::constraint, src/mmp.cpp:9-21 */
static void mmp1_constraint(int C, double* v) {
    double dr = 0.0, di = 0.0;
    for (int c = 0; c < C; ++c) {
        double a = v[2 * c], b = v[2 * c + 1];
        dr += a * a - b * b;
        di += 2 * a * b;
    }
    double angle = 0.5 * atan2(di, dr);
    for (int c = 0; c < C; ++c) {
        double mag = hypot(v[2 * c], v[2 * c + 1]);
        double ph = atan2(v[2 * c + 1], v[2 * c]);
        double rho = mag * cos(ph - angle);
        v[2 * c] = rho * cos(angle);
        v[2 * c + 1] = rho * sin(angle);
    }
}

typedef struct {
    double normComplex, freqNyquist, f, f4Norm, expFactor;
    int isHighFreq;
} computer;

/* GaborComputer ctor, src/gabor.cpp:44-52 */
static computer make_computer(const mapctx* m, int fi) {
    computer k;
    k.normComplex = sqrt(M_SQRT2 / m->g.s);
    k.freqNyquist = 0.5 * m->fs;
    k.f = map_f(m, fi);
    k.isHighFreq = k.f > 0.5 * k.freqNyquist;
    k.f4Norm = k.isHighFreq ? (k.freqNyquist - k.f) : k.f;
    k.expFactor = exp(-2 * M_PI * m->g.s * m->g.s * k.f4Norm * k.f4Norm);
    return k;
}

/* GaborComputer::compute, src/gabor.cpp:54-71 (v modified by the constraint) */
static double compute_energy(const mapctx* m, const computer* k, double t, int C, double* v, int mmp1) {
    if (mmp1 && !k->isHighFreq) mmp1_constraint(C, v);
    double square = 0.0;
    for (int c = 0; c < C; ++c) {
        double phase = atan2(v[2 * c + 1], v[2 * c]);
        double phase4Norm = k->isHighFreq ? (2 * M_PI * k->freqNyquist * t - phase) : phase;
        double normReal = M_SQRT2 * k->normComplex / sqrt(1.0 + cos(2 * phase4Norm) * k->expFactor);
        double moduli = hypot(v[2 * c], v[2 * c + 1]) * normReal * sqrt(m->fs);
        square += moduli * moduli;
    }
    return square;
}

/* one scale's state: energies [t][f], per-window top-2 */
typedef struct {
    mapctx m;
    fftplan plan;
    double* E;
    double* best1;
    double* best2;
    int* arg1;
} mapstate;

static void refresh_window(mapstate* st, int C, const double* const* x, int ti, double* work,
                           double* vals, double* vc, int mmp1) {
    const mapctx* m = &st->m;
    const int F = m->g.fcount;
    for (int c = 0; c < C; ++c) window_values(m, &st->plan, x[c], ti, work, vals + (size_t)c * 2 * F);
    double t = map_t(m, ti);
    double b1 = -1.0, b2 = -1.0;
    int a1 = 0;
    for (int fi = 0; fi < F; ++fi) {
        computer k = make_computer(m, fi);
        for (int c = 0; c < C; ++c) {
            vc[2 * c] = vals[(size_t)c * 2 * F + 2 * fi];
            vc[2 * c + 1] = vals[(size_t)c * 2 * F + 2 * fi + 1];
        }
        double e = compute_energy(m, &k, t, C, vc, mmp1);
        st->E[(size_t)ti * F + fi] = e;
        if (e > b1) {
            b2 = b1;
            b1 = e;
            a1 = fi;
        } else if (e > b2) {
            b2 = e;
        }
    }
    st->best1[ti] = b1;
    st->best2[ti] = b2;
    st->arg1[ti] = a1;
}

/* SingleSignal::computeEnergy, inc/base.hpp:39-46 */
static double channel_energy(const double* x, int N, double fs) {
    double sum = 0.0;
    for (int i = 0; i < N; ++i) sum += x[i] * x[i];
    return sum / fs;
}

/* MultiSignal::computeEnergy, inc/base.hpp:52-58 */
static double multi_energy(double* const* x, int C, int N, double fs) {
    double sum = 0.0;
    for (int c = 0; c < C; ++c) sum += channel_energy(x[c], N, fs);
    return sum;
}

/* ------------------------------------------------------------ subtraction */

/* GaborWorkspace::subtractAtomFromSignal, src/gabor.cpp:143-187 */
void or_subtract_atom(double* params, double* samples, int Nint, double fs, int fit) {
    const double sA = params[3] / fs;
    const double fA = params[4] * fs / 2.0;
    const double tA = params[2] / fs;
    const double amplitude = fit ? 1.0 : params[1];
    const double omega = 2.0 * M_PI * fA;
    const double phase = params[5];
    const long N = Nint;
    const double hw = GAUSS_HALF_WIDTH * sA;
    long l = lrint((tA - hw) * fs), r = lrint((tA + hw) * fs);
    int iL = (int)(l > 0 ? l : 0);
    int iR = (int)(r < N - 1 ? r : N - 1);
    const int Nw = 1 + iR - iL;
    if (Nw <= 0) return;
    double* w = (double*)malloc(sizeof(double) * (size_t)Nw);
    for (int i = 0; i < Nw; ++i) {
        double t = (i + iL) / fs - tA;
        w[i] = amplitude * cos(omega * t + phase);
    }
    gaussize(w, Nw, 1.0 / fs, tA - iL / fs, sA);
    if (fit) {
        double norm2 = 0.0;
        for (int i = 0; i < Nw; ++i) norm2 += w[i] * w[i];
        double norm = sqrt(norm2);
        for (int i = 0; i < Nw; ++i) w[i] /= norm;
        double modulus = 0.0;
        for (int i = 0; i < Nw; ++i) modulus += w[i] * samples[iL + i];
        for (int i = 0; i < Nw; ++i) w[i] *= modulus;
        params[0] = modulus;
        params[1] = modulus / norm;
    }
    for (int i = 0; i < Nw; ++i) samples[iL + i] -= w[i];
    free(w);
}

/* ------------------------------------------------------------- the loop */

typedef struct {
    int nscales;
    mapstate* maps;
    double fs;
    int N;
} workspace;

static int ws_build(workspace* ws, double fs, int N, double eps, double smin, double smax, double fmax) {
    int n = or_geometry(fs, N, eps, smin, smax, fmax, 0, NULL);
    if (n <= 0) return -1;
    or_scale* g = (or_scale*)malloc(sizeof(or_scale) * (size_t)n);
    or_geometry(fs, N, eps, smin, smax, fmax, n, g);
    ws->nscales = n;
    ws->fs = fs;
    ws->N = N;
    ws->maps = (mapstate*)calloc((size_t)n, sizeof(mapstate));
    for (int j = 0; j < n; ++j) {
        mapstate* st = &ws->maps[j];
        st->m.g = g[j];
        st->m.fs = fs;
        st->m.tMax = (N - 1) / fs;
        st->m.N = N;
        fft_make(&st->plan, g[j].nfft);
        st->E = (double*)malloc(sizeof(double) * (size_t)g[j].fcount * g[j].tcount);
        st->best1 = (double*)malloc(sizeof(double) * (size_t)g[j].tcount);
        st->best2 = (double*)malloc(sizeof(double) * (size_t)g[j].tcount);
        st->arg1 = (int*)malloc(sizeof(int) * (size_t)g[j].tcount);
    }
    free(g);
    return 0;
}

static void ws_free(workspace* ws) {
    for (int j = 0; j < ws->nscales; ++j) {
        mapstate* st = &ws->maps[j];
        fft_free(&st->plan);
        free(st->E);
        free(st->best1);
        free(st->best2);
        free(st->arg1);
    }
    free(ws->maps);
}

/* refresh windows of every scale with |t - tA| <= 3 (s + sA), or all (tA NaN) */
static void ws_refresh(workspace* ws, int C, double* const* x, double tA, double sA, int mmp1) {
    int n = ws->nscales;
#pragma omp parallel
    {
        int maxnfft = 2, maxF = 1;
        for (int j = 0; j < n; ++j) {
            if (ws->maps[j].m.g.nfft > maxnfft) maxnfft = ws->maps[j].m.g.nfft;
            if (ws->maps[j].m.g.fcount > maxF) maxF = ws->maps[j].m.g.fcount;
        }
        double* work = (double*)malloc(sizeof(double) * 3 * (size_t)maxnfft);
        double* vals = (double*)malloc(sizeof(double) * 2 * (size_t)maxF * C);
        double* vc = (double*)malloc(sizeof(double) * 2 * (size_t)C);
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < n; ++j) {
            mapstate* st = &ws->maps[j];
            for (int ti = 0; ti < st->m.g.tcount; ++ti) {
                /* src/gabor.cpp:203-207 */
                if (isnan(tA) || fabs(map_t(&st->m, ti) - tA) <= (st->m.g.s + sA) * GAUSS_HALF_WIDTH)
                    refresh_window(st, C, (const double* const*)x, ti, work, vals, vc, mmp1);
            }
        }
        free(work);
        free(vals);
        free(vc);
    }
}

/* argmax + runner-up over all values (findBestMatch's reduction,
 * src/gabor.cpp:85-110); returns 0, or -1 when nothing beats 0 */
static int ws_best(const workspace* ws, int* bj, int* bt, int* bf, double* bval, double* second) {
    double b1 = 0.0, b2 = 0.0;
    int j1 = -1, t1 = 0, f1 = 0;
    for (int j = 0; j < ws->nscales; ++j) {
        const mapstate* st = &ws->maps[j];
        for (int ti = 0; ti < st->m.g.tcount; ++ti) {
            double v = st->best1[ti];
            if (v > b1) {
                b2 = b1;
                b1 = v;
                j1 = j;
                t1 = ti;
                f1 = st->arg1[ti];
                if (st->best2[ti] > b2) b2 = st->best2[ti];
            } else {
                if (v > b2) b2 = v;
            }
        }
    }
    if (j1 < 0) return -1;
    /* the winner window's runner-up may have been shadowed by an earlier b2 */
    if (ws->maps[j1].best2[t1] > b2) b2 = ws->maps[j1].best2[t1];
    *bj = j1;
    *bt = t1;
    *bf = f1;
    *bval = b1;
    *second = b2;
    return 0;
}

/* atom parameters of the winner, src/gabor.cpp:111-131 */
static void ws_atoms(workspace* ws, int C, double* const* x, int j, int ti, int fi, int mmp1,
                     double* params /* C*6 */) {
    mapstate* st = &ws->maps[j];
    const mapctx* m = &st->m;
    const int F = m->g.fcount;
    double* work = (double*)malloc(sizeof(double) * 3 * (size_t)m->g.nfft);
    double* vals = (double*)malloc(sizeof(double) * 2 * (size_t)F);
    double* vc = (double*)malloc(sizeof(double) * 2 * (size_t)C);
    for (int c = 0; c < C; ++c) {
        window_values(m, &st->plan, x[c], ti, work, vals);
        vc[2 * c] = vals[2 * fi];
        vc[2 * c + 1] = vals[2 * fi + 1];
    }
    computer k = make_computer(m, fi);
    double t = map_t(m, ti);
    compute_energy(m, &k, t, C, vc, mmp1);
    for (int c = 0; c < C; ++c) {
        double phase = atan2(vc[2 * c + 1], vc[2 * c]);
        double phase4Norm = k.isHighFreq ? (2 * M_PI * k.freqNyquist * t - phase) : phase;
        double normReal = M_SQRT2 * k.normComplex / sqrt(1.0 + cos(2 * phase4Norm) * k.expFactor);
        double mag = hypot(vc[2 * c], vc[2 * c + 1]);
        double* p = params + 6 * c;
        p[0] = mag * normReal * sqrt(ws->fs);
        p[1] = mag * normReal * normReal;
        p[2] = t * ws->fs;
        p[3] = m->g.s * ws->fs;
        p[4] = k.f * 2.0 / ws->fs;
        p[5] = phase;
    }
    free(work);
    free(vals);
    free(vc);
}

typedef struct {
    int maxAtoms;
    double* atoms;    /* [c][a][6] of the caller, c offset applied by caller */
    int* natoms;      /* one count (all channels share it in the loop) */
    double* energies; /* [a] */
    int* indices;     /* [a][3] */
    double* margins;  /* [a] */
    int atomsStride;  /* distance between channels in atoms, in atoms */
} sink;

/* Decomposition::compute, src/classes.cpp:26-73, on Cw channels held in x
 * (residual updated in place) */
static int mp_loop(workspace* ws, int Cw, double** x, int iterationMax, double residualEnergy,
                   int mmp1, sink* out, char* err, int errlen) {
    const int N = ws->N;
    const double fs = ws->fs;
    ws_refresh(ws, Cw, x, NAN, 0.0, mmp1);
    const double totalEnergy = multi_energy(x, Cw, N, fs);
    if (totalEnergy == 0) {
        snprintf(err, (size_t)errlen, "signalIsEmpty");
        return -1;
    }
    double* params = (double*)malloc(sizeof(double) * 6 * (size_t)Cw);
    int count = 0;
    for (int iteration = 1; iteration <= iterationMax; ++iteration) {
        int bj, bt, bf;
        double bval, second;
        if (ws_best(ws, &bj, &bt, &bf, &bval, &second) != 0) {
            snprintf(err, (size_t)errlen, "energyMapIsEmpty");
            free(params);
            return -1;
        }
        ws_atoms(ws, Cw, x, bj, bt, bf, mmp1, params);
        int a = count++;
        if (a < out->maxAtoms) {
            for (int c = 0; c < Cw; ++c)
                memcpy(out->atoms + ((size_t)c * out->atomsStride + a) * 6, params + 6 * c, sizeof(double) * 6);
            if (out->indices) {
                out->indices[3 * a] = bj;
                out->indices[3 * a + 1] = bt;
                out->indices[3 * a + 2] = bf;
            }
            if (out->margins) out->margins[a] = (bval - second) / bval;
            if (out->energies) out->energies[a] = NAN;
        }
        if (iteration == iterationMax) break;
        for (int c = 0; c < Cw; ++c) or_subtract_atom(params + 6 * c, x[c], N, fs, 0);
        double sA = params[3] / fs, tA = params[2] / fs;
        ws_refresh(ws, Cw, x, tA, sA, mmp1);
        double residueEnergy = multi_energy(x, Cw, N, fs);
        if (a < out->maxAtoms && out->energies) out->energies[a] = residueEnergy;
        if (residueEnergy / totalEnergy <= residualEnergy) break;
    }
    *out->natoms = count;
    free(params);
    return 0;
}

int or_decompose(int variant, double fs, int C, int N, double energyError, double scaleMin,
                 double scaleMax, double freqMax, int iterationMax, double residualEnergy,
                 const double* samples, int maxAtoms, double* atoms, int* natoms, double* energies,
                 int* indices, double* margins, char* err, int errlen) {
    char dummy[64];
    if (!err || errlen <= 0) {
        err = dummy;
        errlen = sizeof dummy;
    }
    err[0] = 0;
    if (C == 1) variant = OR_SMP; /* src/empi.cpp:118 */
    workspace ws;
    if (ws_build(&ws, fs, N, energyError, scaleMin, scaleMax, freqMax) != 0) {
        snprintf(err, (size_t)errlen, "invalidGeometry");
        return -1;
    }
    int rc = 0;
    if (variant == OR_SMP) {
        /* SmpDecomposition::compute, src/classes.cpp:77-87 */
        double* x = (double*)malloc(sizeof(double) * (size_t)N);
        for (int c = 0; c < C && rc == 0; ++c) {
            memcpy(x, samples + (size_t)c * N, sizeof(double) * (size_t)N);
            sink s = {maxAtoms,
                      atoms + (size_t)c * maxAtoms * 6,
                      natoms + c,
                      energies ? energies + (size_t)c * maxAtoms : NULL,
                      indices ? indices + (size_t)c * maxAtoms * 3 : NULL,
                      margins ? margins + (size_t)c * maxAtoms : NULL,
                      maxAtoms};
            rc = mp_loop(&ws, 1, &x, iterationMax, residualEnergy, 0, &s, err, errlen);
        }
        free(x);
    } else if (variant == OR_MMP2) {
        /* Mmp2Decomposition::compute, src/mmp.cpp:23-45 */
        double* sum = (double*)malloc(sizeof(double) * (size_t)N);
        memcpy(sum, samples, sizeof(double) * (size_t)N);
        for (int c = 1; c < C; ++c)
            for (int i = 0; i < N; ++i) sum[i] += samples[(size_t)c * N + i];
        int n = 0;
        sink s = {maxAtoms, atoms, &n, energies, indices, margins, maxAtoms};
        rc = mp_loop(&ws, 1, &sum, iterationMax, residualEnergy, 0, &s, err, errlen);
        if (rc == 0) {
            int na = n < maxAtoms ? n : maxAtoms;
            double* r = (double*)malloc(sizeof(double) * (size_t)N);
            double* sumAtoms = (double*)malloc(sizeof(double) * 6 * (size_t)(na > 0 ? na : 1));
            memcpy(sumAtoms, atoms, sizeof(double) * 6 * (size_t)na);
            for (int c = 0; c < C; ++c) {
                memcpy(r, samples + (size_t)c * N, sizeof(double) * (size_t)N);
                for (int a = 0; a < na; ++a) {
                    double p[6];
                    memcpy(p, sumAtoms + 6 * a, sizeof p);
                    or_subtract_atom(p, r, N, fs, 1);
                    memcpy(atoms + ((size_t)c * maxAtoms + a) * 6, p, sizeof p);
                }
                natoms[c] = n;
            }
            free(r);
            free(sumAtoms);
        }
        free(sum);
    } else {
        /* MMP1 (constraint) / MMP3: one C-channel workspace, src/mmp.hpp:11-31 */
        double** x = (double**)malloc(sizeof(double*) * (size_t)C);
        for (int c = 0; c < C; ++c) {
            x[c] = (double*)malloc(sizeof(double) * (size_t)N);
            memcpy(x[c], samples + (size_t)c * N, sizeof(double) * (size_t)N);
        }
        int n = 0;
        sink s = {maxAtoms, atoms, &n, energies, indices, margins, maxAtoms};
        rc = mp_loop(&ws, C, x, iterationMax, residualEnergy, variant == OR_MMP1, &s, err, errlen);
        for (int c = 0; c < C; ++c) {
            natoms[c] = n;
            free(x[c]);
        }
        free(x);
    }
    ws_free(&ws);
    return rc;
}

/* window values of one scale, for the map-level parity checks */
int or_window_values(double fs, int N, double s, int nfft, int fcount, int tcount, const double* x,
                     int ti, double* values) {
    mapctx m;
    m.g.s = s;
    m.g.nfft = nfft;
    m.g.fcount = fcount;
    m.g.tcount = tcount;
    m.fs = fs;
    m.N = N;
    m.tMax = (N - 1) / fs;
    fftplan p;
    fft_make(&p, nfft);
    double* work = (double*)malloc(sizeof(double) * 3 * (size_t)nfft);
    window_values(&m, &p, x, ti, work, values);
    free(work);
    fft_free(&p);
    return 0;
}

/* full energy map of one scale, [f][t] like the reference's TimeFreqMap;
 * values (optional) [c][f][t][2] */
int or_energy_map(double fs, int C, int N, double energyError, double scaleMin, double scaleMax,
                  double freqMax, int mmp1, const double* samples, int scale, double* energy,
                  double* values) {
    int n = or_geometry(fs, N, energyError, scaleMin, scaleMax, freqMax, 0, NULL);
    if (n <= 0 || scale < 0 || scale >= n) return -1;
    or_scale* g = (or_scale*)malloc(sizeof(or_scale) * (size_t)n);
    or_geometry(fs, N, energyError, scaleMin, scaleMax, freqMax, n, g);
    mapctx m;
    m.g = g[scale];
    m.fs = fs;
    m.N = N;
    m.tMax = (N - 1) / fs;
    free(g);
    const int F = m.g.fcount, T = m.g.tcount;
#pragma omp parallel
    {
        fftplan p;
        fft_make(&p, m.g.nfft);
        double* work = (double*)malloc(sizeof(double) * 3 * (size_t)m.g.nfft);
        double* vals = (double*)malloc(sizeof(double) * 2 * (size_t)F * C);
        double* vc = (double*)malloc(sizeof(double) * 2 * (size_t)C);
#pragma omp for schedule(dynamic, 4)
        for (int ti = 0; ti < T; ++ti) {
            for (int c = 0; c < C; ++c) window_values(&m, &p, samples + (size_t)c * N, ti, work, vals + (size_t)c * 2 * F);
            double t = map_t(&m, ti);
            for (int fi = 0; fi < F; ++fi) {
                computer k = make_computer(&m, fi);
                for (int c = 0; c < C; ++c) {
                    vc[2 * c] = vals[(size_t)c * 2 * F + 2 * fi];
                    vc[2 * c + 1] = vals[(size_t)c * 2 * F + 2 * fi + 1];
                    if (values) {
                        size_t o = (((size_t)c * F + fi) * T + ti) * 2;
                        values[o] = vc[2 * c];
                        values[o + 1] = vc[2 * c + 1];
                    }
                }
                energy[(size_t)fi * T + ti] = compute_energy(&m, &k, t, C, vc, mmp1);
            }
        }
        free(work);
        free(vals);
        free(vc);
        fft_free(&p);
    }
    return 0;
}
