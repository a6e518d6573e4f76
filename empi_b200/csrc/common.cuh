// Types, counters and inline device helpers shared by the MP-loop kernels
// (kernels.cuh) and the refresh kernels (refresh.cuh), which are compiled in
// separate translation units (one per variant mode for the refresh).
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

#include "fft.cuh"
#include "plan.hpp"

namespace empi {

enum Mode { MODE_SINGLE = 0, MODE_MMP1 = 1, MODE_MMP3 = 3 };

enum Counter {
    CTR_UNITS = 0,       // refresh work-queue head
    CTR_TREE = 1,        // tree work-queue head
    CTR_CSLOTS = 2,      // candidate slots emitted
    CTR_CSLOT_Q = 3,     // candidate-slot work-queue head
    CTR_CBINS = 4,       // candidate bins emitted
    CTR_RESCORE_Q = 5,   // rescore work-queue head
    CTR_TOTAL_UNITS = 6,
    CTR_TOTAL_CHUNKS = 7,
    CTR_ACTIVE = 8,      // instances still running after the last schedule
    CTR_STAT_UNITS = 9,  // running totals for statistics
    CTR_STAT_SLOTS = 10,
    CTR_STAT_BINS = 11,
    CTR_STALLED = 12,    // instances stalled by a candidate overflow since the last regrowth
    CTR_CHECK = 13,      // (EMPI_CHECK builds) largest code of a failed bounds check
    CTR_PROP_ITERS = 14, // block proposal: iterations that used it
    CTR_PROP_HITS = 15,  // ... and whose atom lay in a proposed block
    CTR_PACTIVE = 16,    // persistent kernel: instances still running, by iteration parity (two words)
    CTR_COUNT = 18
};

// Block proposal geometry: 16 scale bands (scale j of n falls in band
// 16 j / n) x 32 time tiles (window t of tcount in tile 32 t / tcount).
constexpr int kPropBands = 16;
constexpr int kPropTiles = 32;
constexpr int kProposalBlocks = kPropBands * kPropTiles;

// Bounds self-checks of the data-dependent indices, compiled in with
// -DEMPI_CHECK (a diagnostic build, not the product): a failed check records
// its code in ctr[CTR_CHECK] and the access is skipped instead of made.
#ifdef EMPI_CHECK
#define EMPI_BAD(cond, code) ((cond) ? (atomicMax(b.ctr + CTR_CHECK, (code)), true) : false)
#else
#define EMPI_BAD(cond, code) false
#endif

// ST_STALLED: the candidate buffers overflowed in this iteration; the
// instance took no step and resumes once the host has grown the buffers
enum Status { ST_RUNNING = 0, ST_DONE = 1, ST_ERROR = 2, ST_STALLED = 3 };
enum ErrCode { ERR_NONE = 0, ERR_SIGNAL_EMPTY = 4, ERR_MAP_EMPTY = 5, ERR_CAND_OVERFLOW = 7 };

struct InstPlan {
    int dict, C, epoch, chan0;     // chan0: input channel (SMP) / -1 all / -2 sum (MMP2)
    int ij_off, cen_off, pad0, pad1;
    long long res_off, slot_off, chunk_off, out_off, in_off;
    int in_channels, pad2;
};

struct InstState {
    int status, it, err, nbins;
    double etotal, eres;
    unsigned long long best32;  // tree root: upper-bound bits << 32 | slot
    float bnorm;                // channel norm of max |residual| (the error bound's B)
    unsigned tstar;             // certified lower bound of the best exact energy (float bits)
    unsigned lround;            // block proposal: the tree root's lower bound between the rounds
    int pad_;
};

struct CandSlot {
    int inst, j, t, g;
};

struct CandBin {
    int inst, j, t, k;
    float e32;
    int pad;
    double e64;
};

// Grid barrier of the persistent kernel: arrivals of the current generation,
// the generation, and the error record (0, or 1 + the phase whose wait ran out).
struct GridSync {
    unsigned count;
    unsigned gen;
    int err;
    int pad_;
};

struct BatchDev {
    const ScalePlan* scales;
    const DictPlan* dicts;
    const InstPlan* insts;
    const int2* blk_ic;   // (instance, channel) of each per-channel block
    const float2* tw;     // exp(-2 pi i m / kTwN), then exp(-2 pi i m / 2^26), m < kTwN
    const float* input;   // all epochs, float32 interleaved
    int ninst, nblk_ic, cmax, iter_max, mode;
    double residual_energy;
    float band;
    int cslot_cap, cbin_cap, inst_bin_cap;
    double* residual;
    float* residual32;    // FP32 copy of the residual read by the refresh loads
    const float* etab;    // per-scale expFactor of the phase-dependent bins
    const int4* wtab;     // per-window (iL, W, ci, cf bits), WinGeom
    const float* whf;     // per-window fs t0 modulo 1 in [-0.5, 0.5)
    int4* units;          // refresh work units, one list per sub-FFT size: (inst, j | g << 16, t0, nwin)
    const int* loff;      // per size: offset of its list in units
    const int* lcap;      // per size: capacity of its list
    int* lcount;          // per size: units appended this round (reset before the schedule)
    int* lhead;           // per size: work-queue head (reset before the schedule)
    InstState* state;
    unsigned long long* slots;
    unsigned long long* chunks;
    unsigned* chunk_l;    // per leaf chunk: the largest certified lower bound of its slots (float bits)
    int2* dirty;        // per (i, j): t range [x, y]
    int* ij_units;      // per (i, j): exclusive unit prefix within instance (nscales + 1 per inst)
    int* ij_chunks;     // per (i, j): exclusive dirty-chunk prefix (nscales + 1 per inst)
    int2* ij_crange;    // per (i, j): first dirty chunk, count
    int* inst_units;    // exclusive prefix over instances (ninst + 1)
    int* inst_chunks;   // exclusive prefix over instances (ninst + 1)
    int* ctr;
    CandSlot* cslots;
    CandBin* cbins;
    double2* cbin_v;    // cbin_cap x cmax
    int* inst_bins;     // ninst x inst_bin_cap bin ids
    double* atoms;      // per instance: iter_max x C x 6
    double* energies;   // ninst x iter_max
    int4* indices;      // ninst x iter_max: (scale, t, f, -)
    double* chan_energy;  // per (instance, channel)
    float* chan_xmax;     // per (instance, channel): max |FP32 residual|
    double* stats;        // [0] reference-equivalent FFT flops, [1] algorithmic bytes, [2] slots
    float* dump;          // optional energy-map dump [f][t] of one scale
    // proposal-ceiling probe (null unless enabled): per slot, the upper bound
    // propagated through the last subtraction without recomputing it; totals
    // [0] dirty slots, [1] slots whose propagated bound reaches the next
    // certified best, [2] / [3] their reference-equivalent FFT work
    float* prop;
    double* probe;
    // block proposal (null unless enabled): per instance the scores of the
    // kProposalBlocks (scale band, time tile) blocks; per (instance, scale)
    // the proposed t-range (hull of the top-k blocks' tiles in the scale's
    // band) and the range the second, certified round must refresh
    float* pscores;
    int2* prange;
    int2* qrange;
    int prop_k;
    unsigned char* stale;  // block proposal: per slot, 1 while its key holds propagated bounds
    unsigned char* qmark;  // block proposal: on a unit block's first slot, 1 when round 2 must refresh the block
    unsigned char* chunk_stale;  // block proposal: per leaf chunk, 1 when it holds a stale slot (set by the tree)
    // persistent kernel (persist.cuh): its grid barrier, the time limit of a
    // wait in nanoseconds, and extra arrivals a barrier waits for (0; 1 only
    // in the test that makes every wait run out)
    GridSync* gsync;
    long long wait_ns;
    int wait_extra;
};


// ------------------------------------------------------------ helpers

// Loads of data that a persistent launch rewrites between its iterations (the
// FP32 residual, the refresh unit lists, the schedule's prefix sums).  Across
// separate kernels they take the read-only path (__ldg, __restrict__); inside
// the persistent kernel (translation units defining EMPI_PHASES_ONLY) they
// must be ordinary loads, which the grid barrier's fences order -- the
// read-only path is outside the memory model and could return a line another
// SM has rewritten since.
#ifdef EMPI_PHASES_ONLY
#define EMPI_RESTRICT_MUT
template <class T>
__device__ __forceinline__ T ld_mut(const T* p) {
    return *p;
}
#else
#define EMPI_RESTRICT_MUT __restrict__
template <class T>
__device__ __forceinline__ T ld_mut(const T* p) {
    return __ldg(p);
}
#endif


__device__ __forceinline__ unsigned long long pack_key(float e, unsigned low) {
    if (!(e >= 0.0f && e <= 3.0e38f)) e = 0.0f;
    return ((unsigned long long)__float_as_uint(e) << 32) | (unsigned long long)low;
}

// t grid, src/gabor.cpp:262-264 (t = ti * tMax / (tCount - 1))
__device__ __forceinline__ double grid_t(int ti, double tMax, int tcount) {
    return __ddiv_rn(__dmul_rn((double)ti, tMax), (double)(tcount - 1));
}

// window bounds, src/gabor.cpp:284-286
__device__ __forceinline__ void window_bounds(double t0, double hw, double fs, int N, int& iL, int& iR,
                                              double& t0fixed) {
    long long l = __double2ll_rn(__dmul_rn(__dsub_rn(t0, hw), fs));
    long long r = __double2ll_rn(__dmul_rn(__dadd_rn(t0, hw), fs));
    iL = (int)(l > 0 ? l : 0);
    iR = (int)(r < (long long)N - 1 ? r : (long long)N - 1);
    t0fixed = __dsub_rn(t0, __ddiv_rn((double)iL, fs));
}

// refresh rule |t - tA| <= (s + sA) * 3, src/gabor.cpp:204
__device__ __forceinline__ bool touches(int ti, double tMax, int tcount, double tA, double lim) {
    return fabs(__dsub_rn(grid_t(ti, tMax, tcount), tA)) <= lim;
}

__device__ __forceinline__ void dirty_range(const ScalePlan& sp, double tMax, double tA, double sA, int& lo,
                                            int& hi) {
    const double lim = __dmul_rn(__dadd_rn(sp.s, sA), 3.0);
    const int tc = sp.tcount;
    const double dt = tMax / (tc - 1);
    double a = floor((tA - lim) / dt) - 2.0, c = ceil((tA + lim) / dt) + 2.0;
    int g0 = (int)fmax(0.0, fmin((double)(tc - 1), a));
    int g1 = (int)fmax(0.0, fmin((double)(tc - 1), c));
    lo = g0;
    while (lo > 0 && touches(lo - 1, tMax, tc, tA, lim)) --lo;
    while (lo <= g1 && !touches(lo, tMax, tc, tA, lim)) ++lo;
    hi = g1;
    while (hi < tc - 1 && touches(hi + 1, tMax, tc, tA, lim)) ++hi;
    while (hi >= lo && !touches(hi, tMax, tc, tA, lim)) --hi;
    if (lo > hi) {
        lo = 0;
        hi = -1;
    }
}

__device__ __forceinline__ int group_units(int n, int g, const ScalePlan& sp) {
    const int B = g >= 2 ? sp.B2 : sp.B1;
    return (n + B - 1) / B;
}

__device__ __forceinline__ int upper_index(const int* prefix, int n, int u) {
    // largest i in [0, n) with prefix[i] <= u (prefix non-decreasing, prefix[0] = 0)
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (ld_mut(prefix + mid) <= u) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// exp(-2 pi i m / n) for n a power of two and m < n.  The twiddle buffer holds
// the coarse table W_kTwN^i followed by the fine table W_(2^26)^i (i < kTwN),
// both rounded from exact values on the host.  n <= kTwN: one coarse entry;
// n <= 2^26: W_kTwN^(m >> sh) * W_n^(m mod 2^sh) with sh = log2 n - 13, the
// second factor a fine entry; larger n: sincospif.
__device__ __forceinline__ float2 twiddle_pow2(unsigned m, unsigned n, const float2* __restrict__ tw) {
    if (n <= (unsigned)kTwN) return __ldg(tw + m * ((unsigned)kTwN / n));
    if (n <= (1u << kTwFineLog)) {
        const int sh = 31 - __clz(n) - kTwLog;
        const float2 hi = __ldg(tw + (m >> sh));
        const float2 lo = __ldg(tw + kTwN + ((m & ((1u << sh) - 1u)) << (kTwFineLog - kTwLog - sh)));
        return cmul(hi, lo);
    }
    float s, c;
    sincospif(-2.0f * (float)m / (float)n, &s, &c);
    return make_float2(c, s);
}

// (scale, window, group) of an instance's slot (slots are laid out scale by scale)
__device__ __forceinline__ void slot_to_jtg(const BatchDev& b, const DictPlan& dp, long long slot, int& j, int& t,
                                            int& g) {
    int lo = 0, hi = dp.nscales - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (b.scales[dp.scale0 + mid].slot_base <= slot) lo = mid;
        else hi = mid - 1;
    }
    j = lo;
    const ScalePlan sp = b.scales[dp.scale0 + j];
    const long long rel = slot - sp.slot_base;
    t = (int)(rel / sp.G);
    g = (int)(rel - (long long)t * sp.G);
}

// max over a CTA of 64-bit keys (valid in thread 0); red holds 32 words
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v, unsigned long long* red) {
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        unsigned long long o = __shfl_down_sync(0xffffffffu, v, off);
        v = o > v ? o : v;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0ull;
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            unsigned long long o = __shfl_down_sync(0xffffffffu, v, off);
            v = o > v ? o : v;
        }
    }
    __syncthreads();
    return v;
}

// max over a CTA of non-negative floats (ordered as their bit patterns);
// valid in every thread; red holds 32 words
__device__ __forceinline__ float block_max_nonneg(float v, unsigned* red) {
    unsigned x = __reduce_max_sync(0xffffffffu, __float_as_uint(fmaxf(v, 0.0f)));
    if (threadIdx.x < 32) red[threadIdx.x] = 0u;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) atomicMax(red, x);
    __syncthreads();
    x = red[0];
    __syncthreads();
    return __uint_as_float(x);
}


}  // namespace empi
