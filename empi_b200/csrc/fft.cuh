// Batched shared-memory FFT for sm_100a (FP32, power-of-two sizes 1..4096).
//
// A CTA holds a batch of equal-size complex FFTs in one padded shared buffer
// and runs Stockham autosort passes: each job reads R points strided by L/R,
// applies the twiddles of its stage (W^k from the table, then its powers by
// rotation), runs an R-point DFT in registers and writes R points back at
// stride Ns.  Every thread carries VPT points through
// a pass (VPT = CTA capacity / threads), so registers stay fixed whatever the
// radix.  The first pass takes the odd radix (2, 4 or 8), then radix-16
// passes follow.  One float2 of padding every 16 keeps the stride-R stores of
// the early passes free of bank conflicts.
#pragma once

#include <cuda_runtime.h>

namespace empi {

__device__ __forceinline__ int pad16(int i) { return i + (i >> 4); }

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmulc(float2 a, float2 b) {  // a * conj(b)
    return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// exp(-2 pi i e / R) for the in-register DFT, e < R/2, R <= 16
template <int R>
__device__ __forceinline__ float2 unit_root(int e) {
    // cos / sin of 2 pi m / 16, m = 0..7
    constexpr float c16[8] = {1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f,
                              0.0f, -0.38268343236508977f, -0.70710678118654752f, -0.92387953251128674f};
    constexpr float s16[8] = {0.0f, 0.38268343236508977f, 0.70710678118654752f, 0.92387953251128674f,
                              1.0f, 0.92387953251128674f, 0.70710678118654752f, 0.38268343236508977f};
    const int m = e * (16 / R);
    return make_float2(c16[m], -s16[m]);
}

template <int R>
__device__ __forceinline__ constexpr int bitrev(int i) {
    int r = 0;
    for (int b = 1, o = R >> 1; b < R; b <<= 1, o >>= 1)
        if (i & b) r |= o;
    return r;
}

// In-register forward DFT of R points (natural order in and out).
template <int R>
__device__ __forceinline__ void dft(float2 (&v)[R]) {
#pragma unroll
    for (int h = R / 2; h >= 1; h >>= 1) {
#pragma unroll
        for (int i = 0; i < R; ++i) {
            if ((i & h) == 0) {
                const int j = i + h;
                float2 a = v[i], b = v[j];
                v[i] = cadd(a, b);
                float2 d = csub(a, b);
                const int e = (i & (h - 1)) * (R / (2 * h));
                if (e == 0) {
                    v[j] = d;
                } else if (4 * e == R) {
                    v[j] = make_float2(d.y, -d.x);  // * (-i)
                } else {
                    v[j] = cmul(d, unit_root<R>(e));
                }
            }
        }
    }
    float2 t[R];
#pragma unroll
    for (int i = 0; i < R; ++i) t[i] = v[bitrev<R>(i)];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = t[i];
}

// One Stockham pass of radix R over `points` (a multiple of L) in buf.
// tw: exp(-2 pi i m / TW_N), m < TW_N, with TW_N >= 2 * L.
template <int R, int VPT, int TW_N>
__device__ __forceinline__ void fft_pass(float2* buf, int logL, int logNs, int points,
                                         const float2* __restrict__ tw) {
    constexpr int JPT = VPT / R;
    constexpr int logR = R == 2 ? 1 : R == 4 ? 2 : R == 8 ? 3 : 4;
    const int Ns = 1 << logNs;
    const int logQ = logL - logR;
    const int Q = 1 << logQ;  // L / R
    const int jobs = points >> logR;
    const int twShift = TW_N >> (logNs + logR);
    float2 v[JPT][R];
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) {
        const int job = threadIdx.x + jj * blockDim.x;
        if (job < jobs) {
            const int j = job & (Q - 1);
            const int base = (job >> logQ) << logL;
            if (Q % 16 == 0) {
                // stride Q a multiple of 16: the padding adds Q / 16 per step
                const float2* src = buf + pad16(base + j);
#pragma unroll
                for (int r = 0; r < R; ++r) v[jj][r] = src[r * (Q + (Q >> 4))];
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) v[jj][r] = buf[pad16(base + j + r * Q)];
            }
            const int k = j & (Ns - 1);
            if (Ns > 1) {
                // W^(k r) by repeated multiplication with W^k from the table:
                // one load instead of R - 1 (the loads, not the arithmetic,
                // bounded these passes); 14 products add ~1e-6 relative error
                const float2 w1 = __ldg(tw + k * twShift);
                float2 w = w1;
#pragma unroll
                for (int r = 1; r < R; ++r) {
                    v[jj][r] = cmul(v[jj][r], w);
                    if (r + 1 < R) w = cmul(w, w1);
                }
            }
            dft<R>(v[jj]);
        }
    }
    __syncthreads();
#pragma unroll
    for (int jj = 0; jj < JPT; ++jj) {
        const int job = threadIdx.x + jj * blockDim.x;
        if (job < jobs) {
            const int j = job & (Q - 1);
            const int k = j & (Ns - 1);
            const int ob = ((job >> logQ) << logL) + (j - k) * R + k;
            // ob mod 16 plus any step r Ns mod 16 stays below 16, so the padding
            // of ob + r Ns is that of ob plus (r Ns) / 16
            float2* dst = buf + pad16(ob);
#pragma unroll
            for (int r = 0; r < R; ++r) dst[r * Ns + ((r * Ns) >> 4)] = v[jj][r];
        }
    }
    __syncthreads();
}

// Forward FFT of size L = 2^LOGL on `points` consecutive values (a batch of
// points / L transforms) held padded in buf: the odd radix (2, 4 or 8) first,
// then radix-16 passes.  Starts and ends with the data in shared memory;
// callers synchronise before the call.
template <int VPT, int TW_N, int LOGL>
__device__ __forceinline__ void fft_batch_t(float2* buf, int points, const float2* __restrict__ tw) {
    constexpr int first = LOGL & 3;
    if constexpr (first == 1) fft_pass<2, VPT, TW_N>(buf, LOGL, 0, points, tw);
    if constexpr (first == 2) fft_pass<4, VPT, TW_N>(buf, LOGL, 0, points, tw);
    if constexpr (first == 3) fft_pass<8, VPT, TW_N>(buf, LOGL, 0, points, tw);
#pragma unroll
    for (int logNs = first; logNs < LOGL; logNs += 4) fft_pass<16, VPT, TW_N>(buf, LOGL, logNs, points, tw);
}

// The radix-16 passes that follow an odd first pass done by the caller.
template <int VPT, int TW_N, int LOGL>
__device__ __forceinline__ void fft_batch_rest(float2* buf, int points, const float2* __restrict__ tw) {
    constexpr int first = LOGL & 3;
#pragma unroll
    for (int logNs = first; logNs < LOGL; logNs += 4) fft_pass<16, VPT, TW_N>(buf, LOGL, logNs, points, tw);
}

}  // namespace empi
