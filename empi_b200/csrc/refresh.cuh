// Refresh kernel: windowed pruned FFT + closed-form energies + slot maxima.
//
// One CTA takes a work unit: up to kUnitPoints complex FFT points of one
// (instance, scale, residue group), i.e. a batch of consecutive t-windows.
// The unit body is compiled per sub-FFT size L = 2^LOGL, so index math, padded
// strides and the radix sequence are compile-time.  Per channel:
//   (1) load: Gaussian-windowed FP32 residual samples packed two per complex
//       point, folded and twisted into the residue's sub-sequence;
//   (2) batched shared-memory Stockham FFT (fft.cuh);
//   (3) spectrum: X[k] from Z[k] and Z[Nh-k] for kBinsPerTask consecutive q
//       per thread, energy in closed form, max kept in registers, then over the
//       lanes of the window.
// Window geometry (iL, length, centre) comes from host tables computed in FP64
// with the reference's expressions, so the device does no per-window FP64.
#pragma once

#include "common.cuh"
#include "refresh_kernels.hpp"

namespace empi {

constexpr int kVPT = kUnitPoints / kUnitThreads;
constexpr int kBufFloat2 = kUnitPoints + kUnitPoints / 16 + 16;
constexpr int kBinsPerTask = 8;  // consecutive q per thread in the spectrum stage
constexpr int kEtabSmem = 512;   // expFactor entries of one scale staged in shared memory

// W_2L = exp(-i pi / L) for L = 2^0 .. 2^13 (cos and -sin of pi / L, rounded to
// float): the step of the spectrum stage's twiddle W_2L^q from bin q to q + 1.
struct Rot {
    float x, y;
};
constexpr Rot kW2L[14] = {
    {-1.0f, 0.0f},
    {0.0f, -1.0f},
    {0.70710678118654752f, -0.70710678118654752f},
    {0.92387953251128674f, -0.38268343236508977f},
    {0.98078528040323043f, -0.19509032201612825f},
    {0.99518472667219689f, -0.098017140329560602f},
    {0.99879545620517241f, -0.049067674327418015f},
    {0.99969881869620425f, -0.024541228522912288f},
    {0.99992470183914454f, -0.012271538285719925f},
    {0.99998117528260111f, -0.0061358846491544753f},
    {0.99999529380957619f, -0.0030679567629659761f},
    {0.99999882345170188f, -0.0015339801862847656f},
    {0.99999970586288223f, -0.00076699031874270449f},
    {0.99999992646571785f, -0.00038349518757139556f},
};

// shared-memory layout of a refresh CTA for sub-FFT size 2^LOGL: the window
// tables hold at most NW windows (a unit of kUnitPoints points holds
// kUnitPoints / L windows), so large transforms leave the rest of the SM's
// on-chip memory to the L1 cache that serves the residual loads
template <int LOGL>
struct RefreshSmem {
    static constexpr int NW = (kUnitPoints >> LOGL) < kMaxWindowsPerUnit ? (kUnitPoints >> LOGL) : kMaxWindowsPerUnit;
    static constexpr size_t buf = 0;
    static constexpr size_t win = buf + sizeof(float2) * kBufFloat2;  // int4 (iL, W, ci, cf bits)
    static constexpr size_t rot = win + sizeof(int4) * NW;            // float4 (hrot, step)
    static constexpr size_t key = rot + sizeof(float4) * NW;          // u32 max over non-phase bins
    static constexpr size_t keyp = key + sizeof(unsigned) * NW;       // u32 max over phase-dependent bins
    static constexpr size_t etab = keyp + sizeof(unsigned) * NW;      // float, kEtabSmem
    static constexpr size_t acc = etab + sizeof(float) * kEtabSmem;   // (MMP) per-bin channel sums
};

// (MMP1) per-window certified upper / lower bounds of the constrained
// phase-dependent bins, after the channel sums
template <int MODE, int LOGL>
constexpr size_t refresh_bnd_offset() {
    return RefreshSmem<LOGL>::acc + (MODE == MODE_SINGLE ? 0
                                                       : sizeof(float) * (kUnitPoints + RefreshSmem<LOGL>::NW) *
                                                             (MODE == MODE_MMP1 ? 3 : 1));
}

template <int MODE, int LOGL>
constexpr size_t refresh_smem_bytes() {
    return refresh_bnd_offset<MODE, LOGL>() + (MODE == MODE_MMP1 ? 2 * sizeof(unsigned) * RefreshSmem<LOGL>::NW : 0);
}

// e^{i psi} with psi = 2 theta_kk = 2 pi (2 kk c / Nfft), c = ci + cf the
// window centre in samples (the phase correction of src/gabor.cpp:296-298,
// doubled): the exact integer part through the table (or sincospif of an
// exact fraction), the fractional part through sincospif.
__device__ __forceinline__ float2 centre_rot(unsigned kk, int ci, float cf, unsigned nf,
                                             const float2* __restrict__ tw) {
    const unsigned m = (unsigned)(((unsigned long long)(2u * kk) * (unsigned)ci) & (nf - 1u));
    const float2 t = twiddle_pow2(m, nf, tw);
    const float2 a = make_float2(t.x, -t.y);
    float s, c;
    sincospif(2.0f * (2.0f * (float)kk * cf / (float)nf), &s, &c);
    return cmul(a, make_float2(c, s));
}

// fs |v|^2 normReal^2 of one channel (GaborComputer::compute,
// src/gabor.cpp:54-71) in closed form K |X|^4 / (|X|^2 + e Re(X^2 e^{i psi}));
// rot = e^{i psi}.
__device__ __forceinline__ float energy_phase(float2 X, float e, float2 rot, float Kc) {
    const float p = X.x * X.x + X.y * X.y;
    const float re = (X.x * X.x - X.y * X.y) * rot.x - 2.0f * X.x * X.y * rot.y;
    const float D = p + e * re;
    return (D > 0.0f && p > 0.0f) ? Kc * p * (p / D) : 0.0f;
}

// MMP1 closed form from P = sum |X_c|^2 and S = sum X_c^2 (constraint of
// src/mmp.cpp:9-21 folded into the normalisation); low-frequency bins.
__device__ __forceinline__ float energy_mmp1(float P, float2 S, bool phase, float e, float2 rot, float K1) {
    const float as = sqrtf(S.x * S.x + S.y * S.y);
    if (!phase) return K1 * (P + as);
    if (as == 0.0f) return K1 * P / (1.0f + e);
    const float re = S.x * rot.x - S.y * rot.y;
    const float D = as + e * re;
    return D > 0.0f ? K1 * (P + as) * (as / D) : 0.0f;
}

__device__ __forceinline__ void emit_candidate(const BatchDev& b, int inst, int j, int t, int k, float e) {
    if (EMPI_BAD(inst < 0 || inst >= b.ninst || k < 0, 4)) return;
    const int slot = atomicAdd(b.ctr + CTR_CBINS, 1);
    if (slot >= b.cbin_cap) {
        b.state[inst].err = ERR_CAND_OVERFLOW;
        return;
    }
    // every counted record is written, even when the instance's own list is
    // full: k_rescore re-scores all of them
    CandBin cb;
    cb.inst = inst;
    cb.j = j;
    cb.t = t;
    cb.k = k;
    cb.e32 = e;
    cb.pad = 0;
    cb.e64 = 0.0;
    b.cbins[slot] = cb;
    const int li = atomicAdd(&b.state[inst].nbins, 1);
    if (li < b.inst_bin_cap) b.inst_bins[(long long)inst * b.inst_bin_cap + li] = slot;
    else b.state[inst].err = ERR_CAND_OVERFLOW;
}

// ------------------------------------------------------------ error bound
//
// For every bin of a window |X32_k - X_k| <= dlt = bnd_d * B (B = channel norm
// of max |residual|, geometry.cpp's set_error_bound), and sqrt(energy) is a
// norm of X, so the exact (FP64) energy E of a bin whose FP32 energy is e
// satisfies
//   (sqrt(e (1 - tau)) - d)^2 <= E <= (sqrt(e (1 + tau)) + d)^2
// with d = sqrt(Kc) dlt (times sqrt(bnd_rho) for phase-dependent bins) and tau
// the relative error of the energy formula.  Both ends grow with e, so a
// window needs only the largest e of each class (non-phase, phase-dependent).
// The slot key stores the upper bound U (high word, ranked by the tree) and
// the lower bound L (low word).  Margins of 8-16 u cover the FP32 evaluation
// of the bounds themselves.
constexpr float kU = 5.9604645e-8f;  // 2^-24

struct BoundTerms {
    float d_np, d_ph, tau_np, tau_ph;
};

__device__ __forceinline__ BoundTerms bound_terms(const ScalePlan& sp, float bnorm, int C) {
    BoundTerms t;
    const float dlt = sp.bnd_d * bnorm * (1.0f + 8.0f * kU);
    t.d_np = sp.sKc * dlt;
    t.d_ph = t.d_np * sp.bnd_srho;
    const float tc = (float)(2 * (C + 4)) * kU;  // channel sums (MMP1 / MMP3)
    t.tau_np = 8.0f * kU + tc;
    t.tau_ph = sp.bnd_tph + tc;
    return t;
}

// upper and lower bound of the exact energy of a bin class whose largest FP32
// energy has code `code` (float bits + 1; 0: no bin of this class)
__device__ __forceinline__ void class_bounds(unsigned code, float d, float tau, float& U, float& L) {
    if (!code) {
        U = 0.0f;
        L = 0.0f;
        return;
    }
    const float e = __uint_as_float(code - 1u);
    const float su = sqrtf(e * (1.0f + tau)) * (1.0f + 8.0f * kU) + d;
    U = su * su * (1.0f + 16.0f * kU);
    const float sl = sqrtf(e * fmaxf(0.0f, 1.0f - tau)) * (1.0f - 8.0f * kU) - d;
    L = sl > 0.0f ? sl * sl * (1.0f - 16.0f * kU) : 0.0f;
}

// smallest FP32 energy of a class whose upper bound can reach tstar
__device__ __forceinline__ unsigned class_threshold(float tstar, float d, float tau) {
    const float r = sqrtf(tstar) * (1.0f - 8.0f * kU) - d;
    if (r <= 0.0f) return 0u;
    return __float_as_uint(r * r / (1.0f + tau) * (1.0f - 16.0f * kU));
}

// MMP1, constrained phase-dependent bin (k < klo, src/mmp.cpp:9-21 then
// src/gabor.cpp:54-71): E = Kc Q / (1 + e cos a) with Q = (P + |S|) / 2 the
// best common-phase projection energy (a squared seminorm of the channel
// values) and a = arg S + psi.  Q moves like a norm; the angle a moves by at
// most asin(|dS| / |S|) plus the rotation's angle error, and the factor is
// bounded over that interval (or by 1 / (1 -+ e) when |dS| >= |S|).
// At k = 0 the values are real, exactly and in FP32 (X = Re Z + Im Z), so S
// is real and non-negative, a = 0 and the factor is 1 / (1 + e) with e = 1.
__device__ __forceinline__ void mmp1_phase_bounds(float P, float2 S, float e, float2 rot, float Kc, float dlt,
                                                  int C, bool dc, float& U, float& L) {
    const float tq = (float)(2 * (C + 4)) * kU;
    const float as = sqrtf(S.x * S.x + S.y * S.y);
    const float Q = 0.5f * (P + as);
    const float su = sqrtf(Q * (1.0f + tq)) * (1.0f + 8.0f * kU) + dlt;
    const float sl = sqrtf(Q * (1.0f - tq)) * (1.0f - 8.0f * kU) - dlt;
    const float dS = 2.0f * sqrtf(P) * dlt + dlt * dlt + tq * P;
    float fup = 1.0f / (1.0f - e), flo = 1.0f / (1.0f + e);
    if (dc) {
        fup = flo;
    } else if (dS < as) {
        const float ca = fminf(1.0f, fmaxf(-1.0f, (S.x * rot.x - S.y * rot.y) / as));
        const float a = acosf(ca);
        const float da = asinf(dS / as) * (1.0f + 1e-5f) + 2e-5f;
        fup = 1.0f / (1.0f + e * cosf(fminf(3.14159265f, a + da)) - 1e-6f);
        flo = 1.0f / (1.0f + e * cosf(fmaxf(0.0f, a - da)) + 1e-6f);
        fup = fminf(fup, 1.0f / (1.0f - e));
        flo = fmaxf(flo, 1.0f / (1.0f + e));
    }
    const float rho = dc ? 1.0f : 1.0f / (1.0f - e);
    U = Kc * su * su * fup * (1.0f + (76.0f * rho + 24.0f) * kU);
    L = sl > 0.0f ? Kc * sl * sl * flo * (1.0f - (76.0f * rho + 24.0f) * kU) : 0.0f;
}

// What the spectrum stage does with a bin's final energy.  Refresh: keep the
// largest energy of each class (non-phase / phase-dependent bins) as float
// bits + 1 (0: no bin); negative, NaN and infinite energies count as 0.
// Collect: emit the bins whose upper bound reaches the instance's certified
// lower bound tstar, i.e. whose energy is at least its class threshold.
template <bool COLLECT>
struct BinSink {
    const BatchDev& b;
    int inst, j, t, tcount;
    unsigned thr_np, thr_ph;
    unsigned best_np, best_ph;
    __device__ __forceinline__ void put(int k, float e, bool ph) {
        if (COLLECT) {
            if (__float_as_uint(e) >= (ph ? thr_ph : thr_np) && e <= 3.0e38f) emit_candidate(b, inst, j, t, k, e);
        } else {
            if (b.dump) b.dump[(long long)k * tcount + t] = e;
            const unsigned v = __float_as_uint(e >= 0.0f && e <= 3.0e38f ? e : 0.0f) + 1u;
            if (ph) best_ph = max(best_ph, v);
            else best_np = max(best_np, v);
        }
    }
    // a bin with explicit bounds (MMP1's constrained phase-dependent bins)
    __device__ __forceinline__ void put_bounded(int k, float e, float U, float L, float tstar, unsigned* s_ub,
                                                unsigned* s_lb, int w) {
        if (COLLECT) {
            if (U >= tstar) emit_candidate(b, inst, j, t, k, e);
        } else {
            if (b.dump) b.dump[(long long)k * tcount + t] = e;
            atomicMax(s_ub + w, __float_as_uint(U));
            atomicMax(s_lb + w, __float_as_uint(L));
        }
    }
};

// Max of one window's class maxima over the lanes holding its tasks (TPW
// consecutive, aligned lanes) into the window's shared keys.
template <int TPW>
__device__ __forceinline__ void sink_reduce(unsigned best, unsigned* s_key, int w, bool valid, int tid) {
    if (TPW >= 32) {
        best = __reduce_max_sync(0xffffffffu, best);
        if ((tid & 31) == 0 && valid && best) atomicMax(s_key + w, best);
    } else {
#pragma unroll
        for (int off = TPW / 2; off; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
        if ((tid & (TPW - 1)) == 0 && valid && best) atomicMax(s_key + w, best);
    }
}

template <int LOGL, int MODE, bool COLLECT>
__device__ __forceinline__ void unit_body(const BatchDev& b, unsigned char* smem, int inst, int j, int g, int t_start,
                                          int nwin, float tstar) {
    constexpr int L = 1 << LOGL;
    constexpr int CH = L < kBinsPerTask ? L : kBinsPerTask;  // q values per task
    constexpr int TPW = L / CH;                                // tasks per window
    float2* buf = reinterpret_cast<float2*>(smem + RefreshSmem<LOGL>::buf);
    int4* s_win = reinterpret_cast<int4*>(smem + RefreshSmem<LOGL>::win);
    float4* s_rot = reinterpret_cast<float4*>(smem + RefreshSmem<LOGL>::rot);
    float* s_etab = reinterpret_cast<float*>(smem + RefreshSmem<LOGL>::etab);
    unsigned* s_key = reinterpret_cast<unsigned*>(smem + RefreshSmem<LOGL>::key);
    unsigned* s_keyp = reinterpret_cast<unsigned*>(smem + RefreshSmem<LOGL>::keyp);
    float* acc = reinterpret_cast<float*>(smem + RefreshSmem<LOGL>::acc);
    unsigned* s_ub = reinterpret_cast<unsigned*>(smem + refresh_bnd_offset<MODE, LOGL>());
    unsigned* s_lb = s_ub + RefreshSmem<LOGL>::NW;

    if (EMPI_BAD(inst < 0 || inst >= b.ninst, 10)) return;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    if (EMPI_BAD(j < 0 || j >= dp.nscales, 10)) return;
    const ScalePlan sp = b.scales[dp.scale0 + j];
    if (EMPI_BAD(sp.logL != LOGL || g < 0 || g >= sp.G || t_start < 0 || nwin < 1 ||
                     t_start + nwin > sp.tcount || nwin > RefreshSmem<LOGL>::NW, 10))
        return;
    if (EMPI_BAD(MODE != MODE_SINGLE && nwin * (g == 0 ? (1 << LOGL) + 1 : (g >= 2 ? 2 << LOGL : 1 << LOGL)) >
                                            kUnitPoints + RefreshSmem<LOGL>::NW, 8))
        return;
    const int M = sp.M, F = sp.F;
    const int Nh = sp.nfft >> 1;
    const unsigned nfu = (unsigned)sp.nfft;
    const bool pair = g >= 2;
    const int nf = pair ? 2 : 1;
    const int nb = g == 0 ? L + 1 : (pair ? 2 * L : L);  // bins per window (accumulator stride)
    const int r = g == 0 ? 0 : (g == 1 ? M / 2 : g - 1);
    const int rho0 = r, rho1 = M - r;                       // residues of the group's FFTs
    const int tid = threadIdx.x, T = blockDim.x;
    const float2* __restrict__ tw = b.tw;
    const float aG2 = sp.aG2, Kc = sp.Kc;
    // certified error bound of this unit's bins (see "error bound" above)
    const float bnorm = b.state[inst].bnorm;
    const BoundTerms bt = bound_terms(sp, bnorm, ip.C);
    const float dlt = sp.bnd_d * bnorm * (1.0f + 8.0f * kU);
    const unsigned thr_np = COLLECT ? class_threshold(tstar, bt.d_np, bt.tau_np) : 0u;
    const unsigned thr_ph = COLLECT ? class_threshold(tstar, bt.d_ph, bt.tau_ph) : 0u;

    // Per window: geometry, and for the phase-dependent bins e^{-2 pi i fs t0}
    // (high bins) and the step of psi from q to q + 1; the scale's expFactor
    // table when it fits.  Read by the spectrum stage instead of global loads
    // and transcendentals inside its tasks.
    const int ecount = sp.klo + (sp.fcount - 1 - sp.khi);
    const bool etab_smem = ecount <= kEtabSmem;
    {
        const long long w0 = sp.win_base + t_start;
        for (int w = tid; w < nwin; w += T) {
            int4 m = __ldg(b.wtab + w0 + w);
            if (EMPI_BAD(m.x < 0 || m.y < 1 || m.x + m.y > dp.N, 11)) m.y = 0;
            s_win[w] = m;
            float sh, ch;
            sincospif(-2.0f * __ldg(b.whf + w0 + w), &sh, &ch);
            const float2 st = centre_rot((unsigned)sp.M, m.z, __int_as_float(m.w), (unsigned)sp.nfft, b.tw);
            s_rot[w] = make_float4(ch, sh, st.x, st.y);
            s_key[w] = 0u;
            s_keyp[w] = 0u;
            if (MODE == MODE_MMP1) {
                s_ub[w] = 0u;
                s_lb[w] = 0u;
            }
        }
        if (etab_smem)
            for (int i = tid; i < ecount; i += T) s_etab[i] = __ldg(b.etab + sp.eoff + i);
    }
    const float* __restrict__ etv = etab_smem ? s_etab : b.etab + sp.eoff;
    // expFactor of a phase-dependent bin (k < klo or k > khi), src/gabor.cpp:51
    auto efac = [&](int k) { return etv[k < sp.klo ? k : sp.klo + (k - sp.khi - 1)]; };
    float2 wr0 = make_float2(1.f, 0.f), wr1 = make_float2(1.f, 0.f);  // W_Nfft^rho
    if (g >= 1) {
        float s0, c0;
        sincospif(-2.0f * (float)rho0 / (float)sp.nfft, &s0, &c0);
        wr0 = make_float2(c0, s0);
        sincospif(-2.0f * (float)rho1 / (float)sp.nfft, &s0, &c0);
        wr1 = make_float2(c0, s0);
    }
    if (MODE != MODE_SINGLE) {
        for (int i = tid; i < nwin * nb * (MODE == MODE_MMP1 ? 3 : 1); i += T) acc[i] = 0.0f;
    }
    __syncthreads();

    const int ntasks = nwin * TPW;
    // tasks with phase-dependent bins: tau < tlo (kmin < klo) and tau >= thi
    // (kmax > khi); kmin and kmax grow with tau, so both ends are found by
    // bisection (the q0 = 0 task of group 0, which also holds the Nyquist
    // bin, has kmin = 0 < klo)
    int tlo = 0, thi = TPW;
    {
        const int rmin = pair ? min(rho0, rho1) : (g == 1 ? rho0 : 0);
        const int rmax = pair ? max(rho0, rho1) : (g == 1 ? rho0 : 0);
        int lo = 0, hi = TPW;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (M * mid * CH + rmin >= sp.klo) hi = mid;
            else lo = mid + 1;
        }
        tlo = lo;
        lo = 0;
        hi = TPW;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (M * (mid * CH + CH - 1) + rmax > sp.khi) hi = mid;
            else lo = mid + 1;
        }
        thi = max(lo, tlo);
    }
    const int nph = tlo + (TPW - thi);
    // Twiddles of the load, per unit: the twist of residue group g at input
    // index n is W_Nh^{r n} (a pair's two residues r, M - r use it and its
    // conjugate) or W_2L^n (g = 1, residue M/2); a pair's second FFT input is
    // also multiplied by W_L^n.  A thread's points step through n by fixed
    // strides, so one table lookup per window or job is followed by
    // rotations.
    for (int c = 0; c < ip.C; ++c) {
        const float* EMPI_RESTRICT_MUT x = b.residual32 + ip.res_off + (long long)c * dp.N;
        const float2 one = make_float2(1.f, 0.f);
        auto twist = [&](int n) -> float2 {
            if (g == 1) return __ldg(tw + ((n & (2 * L - 1)) << (12 - LOGL)));
            const unsigned rn = ((unsigned)r * (unsigned)n) & (unsigned)(Nh - 1);
            return twiddle_pow2(rn, (unsigned)Nh, tw);
        };
        auto pfac = [&](int n) -> float2 { return __ldg(tw + ((n & (L - 1)) << (13 - LOGL))); };
        // step from fold m to m + 1 (n + L): W_2L^L = -1, or W_Nh^{r L}
        const float2 fold = g == 0 ? one : (g == 1 ? make_float2(-1.f, 0.f) : twist(L));
        constexpr int FIRST = LOGL & 3;  // log2 of the odd first radix; 0: radix-16 passes only
        constexpr int R0 = 1 << FIRST;
        constexpr int LQ = LOGL - FIRST;  // log2 of L / R0
        // fused first pass: a job's points are jq + rr L / R0
        // A pair's second FFT input is z conj(W_Nh^{r n}) W_L^n = z conj(t2) with
        // t2 = W_Nh^{r n} conj(W_L^n), rotated like t.
        const float2 jstep = (FIRST != 0 && g >= 1) ? twist(1 << LQ) : one;
        const float2 j2step = (FIRST != 0 && pair) ? cmulc(jstep, pfac(1 << LQ)) : one;
        // other sizes: a thread's points are np0 + i T within a window
        const int np0 = tid & (L - 1);
        const float2 t0 = (FIRST == 0 && g >= 1) ? twist(np0) : one;
        const float2 t20 = (FIRST == 0 && pair) ? cmulc(t0, pfac(np0)) : one;
        const float2 tstep = (FIRST == 0 && g >= 1 && L > kUnitThreads) ? twist(kUnitThreads) : one;
        const float2 t2step = (FIRST == 0 && pair && L > kUnitThreads) ? cmulc(tstep, pfac(kUnitThreads)) : one;
        // (1) load: y_r[n'] = sum_m z[n' + mL] W_Nh^{r (n' + mL)}; for the second
        // FFT of a pair the sum is conjugate-twisted and multiplied by W_L^{n'}.
        // t, t2 = the twists at n = np.
        auto load_point = [&](const int4& m, float cf, int np, float2 t, float2 t2, float2& a1, float2& a2) {
            const float* EMPI_RESTRICT_MUT xs = x + m.x;
            a1 = make_float2(0.f, 0.f);
            a2 = make_float2(0.f, 0.f);
            if (F == 1) {
                // one fold (every scale whose longest window fits its sub-FFT):
                // no loop and no rotation of the twist to a next fold
                const int i0 = 2 * np;
                if (i0 < m.y) {
                    const float x0 = ld_mut(xs + i0);
                    const float x1 = (i0 + 1 < m.y) ? ld_mut(xs + i0 + 1) : 0.0f;
                    const float d0 = (float)(i0 - m.z) - cf;
                    const float y0 = d0 * aG2, y1 = (d0 + 1.0f) * aG2;
                    const float2 z = make_float2(x0 * exp2f(-y0 * y0), x1 * exp2f(-y1 * y1));
                    if (g == 0) {
                        a1 = z;
                    } else {
                        a1 = cmul(z, t);
                        if (g >= 2) a2 = cmulc(z, t2);
                    }
                }
                return;
            }
            const float2 pf = cmulc(t, t2);  // W_L^{np}
            int n = np;
            for (int mm = 0; mm < F; ++mm, n += L) {
                const int i0 = 2 * n;
                if (i0 >= m.y) break;
                const float x0 = ld_mut(xs + i0);
                const float x1 = (i0 + 1 < m.y) ? ld_mut(xs + i0 + 1) : 0.0f;
                const float d0 = (float)(i0 - m.z) - cf;
                const float y0 = d0 * aG2, y1 = (d0 + 1.0f) * aG2;
                const float2 z = make_float2(x0 * exp2f(-y0 * y0), x1 * exp2f(-y1 * y1));
                if (g == 0) {
                    a1 = cadd(a1, z);
                } else if (g == 1) {
                    a1 = cadd(a1, cmul(z, t));
                    t = make_float2(-t.x, -t.y);
                } else {
                    a1 = cadd(a1, cmul(z, t));
                    a2 = cadd(a2, cmulc(z, t));
                    t = cmul(t, fold);
                }
            }
            if (g >= 2) a2 = cmul(a2, pf);
        };
        if constexpr (FIRST != 0) {
            // the first Stockham pass (radix 2^FIRST, no twiddles) fused into the load
            for (int job = tid; job < (nwin << LQ); job += T) {
                const int w = job >> LQ;
                const int jq = job & ((1 << LQ) - 1);
                const int4 m = s_win[w];
                const float cf = __int_as_float(m.w);
                float2 t = g >= 1 ? twist(jq) : one;
                float2 t2 = pair ? cmulc(t, pfac(jq)) : one;
                float2 v1[R0], v2[R0];
#pragma unroll
                for (int rr = 0; rr < R0; ++rr) {
                    load_point(m, cf, jq + (rr << LQ), t, t2, v1[rr], v2[rr]);
                    if (rr + 1 < R0) {
                        t = cmul(t, jstep);
                        if (pair) t2 = cmul(t2, j2step);
                    }
                }
                // o mod 16 is a multiple of R0, so o + rr keeps o's padding
                float2* po = buf + pad16(((w * nf) << LOGL) + jq * R0);
                dft<R0>(v1);
#pragma unroll
                for (int rr = 0; rr < R0; ++rr) po[rr] = v1[rr];
                if (pair) {
                    dft<R0>(v2);
#pragma unroll
                    for (int rr = 0; rr < R0; ++rr) po[L + L / 16 + rr] = v2[rr];
                }
            }
            __syncthreads();
            fft_batch_rest<kVPT, kTwN, LOGL>(buf, (nwin * nf) << LOGL, tw);
        } else {
            if constexpr (L > kUnitThreads) {
                // a window at a time: its geometry read once, the twist rotated
                // from point to point (np0 + i T)
                for (int w = 0; w < nwin; ++w) {
                    const int4 m = s_win[w];
                    const float cf = __int_as_float(m.w);
                    // points np0 + i T: padded offsets step by T + T / 16
                    float2* pp = buf + pad16(((w * nf) << LOGL) + np0);
                    float2 t = t0, t2 = t20;
#pragma unroll 4
                    for (int np = np0; np < L; np += kUnitThreads, pp += kUnitThreads + kUnitThreads / 16) {
                        float2 a1, a2;
                        load_point(m, cf, np, t, t2, a1, a2);
                        pp[0] = a1;
                        if (pair) pp[L + L / 16] = a2;
                        t = cmul(t, tstep);
                        if (pair) t2 = cmul(t2, t2step);
                    }
                }
            } else {
                for (int idx = tid; idx < (nwin << LOGL); idx += T) {
                    const int w = idx >> LOGL;
                    const int np = idx & (L - 1);
                    const int4 m = s_win[w];
                    float2 a1, a2;
                    load_point(m, __int_as_float(m.w), np, t0, t20, a1, a2);
                    const int o = (w * nf) << LOGL;
                    buf[pad16(o + np)] = a1;
                    if (pair) buf[pad16(o + L + np)] = a2;
                }
            }
            __syncthreads();
            // (2) FFT of every sub-sequence in the unit
            fft_batch_t<kVPT, kTwN, LOGL>(buf, (nwin * nf) << LOGL, tw);
        }
        // (3) spectrum, energies, maxima
        const bool last = (c == ip.C - 1);
        // Two passes (3a, 3b) for L >= 64 (from L = 1024 on, where a unit holds
        // at most eight windows, the second takes its bins one per thread).  Small transforms (L <= 32) are almost all
        // phase-dependent bins, and MMP1 folds the phase into its channel sums:
        // those keep the single pass.
        constexpr bool kSplit = MODE != MODE_MMP1 && LOGL >= 6;
        if constexpr (!kSplit && LOGL >= 3 && MODE == MODE_SINGLE) {
            // (8 <= L <= 32.)  Mirrored pairs: bins k and Nh - k read the same two values
            // (Z[k], Z[Nh - k]) with A and B exchanged, so one pair of loads
            // gives both.  A task takes q0 .. q0 + nq - 1 and their mirrors: the
            // partner residue's L - 1 - q (pairs, g = 1) or L - q (g = 0, where
            // q = 0 also gives the Nyquist bin and the last task adds q = L/2).
            constexpr int QH = CH / 2;
            for (int base = 0; base < ntasks; base += T) {
                const int task = base + tid;
                const bool valid = task < ntasks;
                const int w = valid ? task / TPW : 0;
                const int tau = task - w * TPW;
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                if (valid) {
                    const int4 m = s_win[w];
                    const float cf = __int_as_float(m.w);
                    const int nq = pair ? CH : QH;
                    const int q0 = tau * nq;
                    const int kmin = M * q0 + rho0, kmax = M * (q0 + nq - 1) + rho0;
                    const bool phase = kmin < sp.klo || kmax > sp.khi || Nh - kmax < sp.klo || Nh - kmin > sp.khi;
                    float2 hrot = make_float2(1.f, 0.f), step = make_float2(1.f, 0.f), ew = make_float2(1.f, 0.f);
                    float2 rot = make_float2(1.f, 0.f);
                    if (phase) {
                        const float4 hr = s_rot[w];
                        hrot = make_float2(hr.x, hr.y);
                        step = make_float2(hr.z, hr.w);
                        float se, ce;
                        sincospif(2.0f * cf, &se, &ce);  // e^{i 2 pi c}: e^{i psi(Nh - k)} = e^{i 2 pi c} conj(e^{i psi(k)})
                        ew = make_float2(ce, se);
                        rot = centre_rot((unsigned)kmin, m.z, cf, nfu, tw);
                    }
                    const int o0 = (w * nf) << LOGL;
                    const int ob = pair ? o0 + L : o0;  // the partner residue's FFT
                    // q0 .. q0 + nq - 1 and L - 1 - q stay inside one 16-block each
                    const float2* pA = buf + pad16(o0 + q0);
                    const float2* pB = buf + pad16(ob + L - 1 - q0);
                    // W_Nfft^k = W_Nfft^rho0 W_2L^q, rotated by W_2L from bin to bin; the
                    // mirror's twiddle is -conj(W_Nfft^k) (W_Nfft^M = W_2L and rho1 =
                    // M - rho0), so with E = (A + conj B) / 2 and D = (A - conj B) / 2i:
                    // X[k] = E + W D and X[Nh - k] = conj(E - W D)
                    float2 wk = __ldg(tw + (q0 << (12 - LOGL)));  // W_2L^q
                    if (g != 0) wk = cmul(wr0, wk);
#pragma unroll 2
                    for (int qq = 0; qq < nq; ++qq) {
                        const int q = q0 + qq;
                        const int k = M * q + rho0;
                        const int km = Nh - k;
                        const float2 A = pA[qq];
                        const float2 Bq = (g == 0) ? buf[pad16(o0 + ((L - q) & (L - 1)))] : pB[-qq];
                        const float ex = 0.5f * (A.x + Bq.x), ey = 0.5f * (A.y - Bq.y);
                        const float dx = 0.5f * (A.x - Bq.x), dy = 0.5f * (A.y + Bq.y);
                        const float u = wk.x * dy + wk.y * dx, v = wk.y * dy - wk.x * dx;
                        const float2 X = make_float2(ex + u, ey + v);
                        const float2 Xm = make_float2(ex - u, v - ey);
                        if (k < sp.fcount) {
                            const bool pk = phase && (k < sp.klo || k > sp.khi);
                            const float e = pk ? energy_phase(X, efac(k), k >= sp.khf ? cmul(rot, hrot) : rot, Kc)
                                               : Kc * (X.x * X.x + X.y * X.y);
                            sink.put(k, e, pk);
                        }
                        if (km < sp.fcount) {
                            const bool pk = phase && (km < sp.klo || km > sp.khi);
                            float e;
                            if (pk) {
                                const float2 rotm = cmulc(ew, rot);  // e^{i 2 pi c} conj(rot)
                                e = energy_phase(Xm, efac(km), km >= sp.khf ? cmul(rotm, hrot) : rotm, Kc);
                            } else {
                                e = Kc * (Xm.x * Xm.x + Xm.y * Xm.y);
                            }
                            sink.put(km, e, pk);
                        }
                        if (phase) rot = cmul(rot, step);
                        wk = cmul(wk, make_float2(kW2L[LOGL].x, kW2L[LOGL].y));
                    }
                    if (g == 0 && tau == TPW - 1) {
                        // q = L/2, its own mirror; wk = W_2L^{L/2}
                        const int q = L / 2;
                        const int k = M * q;
                        const float2 A = buf[pad16(o0 + q)];
                        const float ex = A.x, dy = A.y;
                        const float2 X = make_float2(ex + wk.x * dy, wk.y * dy);
                        if (k < sp.fcount) {
                            const bool pk = k < sp.klo || k > sp.khi;
                            float e;
                            if (pk) {
                                const float2 rk = centre_rot((unsigned)k, m.z, cf, nfu, tw);
                                const float4 hr = s_rot[w];
                                e = energy_phase(X, efac(k), k >= sp.khf ? cmul(rk, make_float2(hr.x, hr.y)) : rk, Kc);
                            } else {
                                e = Kc * (X.x * X.x + X.y * X.y);
                            }
                            sink.put(k, e, pk);
                        }
                    }
                }
                if (!COLLECT) {
                    sink_reduce<TPW>(sink.best_np, s_key, w, valid, tid);
                    sink_reduce<TPW>(sink.best_ph, s_keyp, w, valid, tid);
                }
            }
        } else if constexpr (!kSplit) {
            for (int base = 0; base < ntasks; base += T) {
                const int task = base + tid;
                const bool valid = task < ntasks;
                const int w = valid ? task / TPW : 0;
                const int q0 = (task - w * TPW) * CH;
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                if (valid) {
                    const int4 m = s_win[w];
                    const float cf = __int_as_float(m.w);
                    const int kmin = M * q0 + (pair ? min(rho0, rho1) : (g == 1 ? rho0 : 0));
                    const int kmax = (g == 0 && q0 == 0) ? Nh
                                                         : M * (q0 + CH - 1) + (pair ? max(rho0, rho1) : (g == 1 ? rho0 : 0));
                    const bool phase = kmin < sp.klo || kmax > sp.khi;
                    float2 hrot = make_float2(1.f, 0.f), step = make_float2(1.f, 0.f);
                    if (phase) {
                        const float4 hr = s_rot[w];
                        hrot = make_float2(hr.x, hr.y);  // e^{-2 pi i fs t0} for high bins
                        step = make_float2(hr.z, hr.w);  // psi increment from q to q + 1
                    }
                    const int o0 = (w * nf) << LOGL;
                    const int o1 = o0 + L;
    #pragma unroll 1
                    for (int h = 0; h < nf; ++h) {
                        const int rho = h ? rho1 : rho0;
                        const float2 wr = h ? wr1 : wr0;
                        const int oa = h ? o1 : o0;                // A = Y_h[q]
                        const int ob = pair ? (h ? o0 : o1) : o0;  // B = partner FFT
                        float2 rot = make_float2(1.f, 0.f);
                        if (phase) rot = centre_rot((unsigned)(M * q0 + rho), m.z, cf, nfu, tw);
                        const int pa = pad16(oa + q0);
                        // partner L - 1 - q for g >= 1: a descending run inside one
                        // 16-block, since (L - 1 - q0) mod 16 is 15 or 7
                        const int pb = pad16(ob + L - 1 - q0);
                        // W_Nfft^k = W_Nfft^rho W_2L^q: the table entry at q0, then one
                        // rotation by W_2L per bin
                        float2 wk = __ldg(tw + (q0 << (12 - LOGL)));
                        if (g != 0) wk = cmul(wr, wk);
    #pragma unroll 2
                        for (int qq = 0; qq < CH; ++qq) {
                            const int q = q0 + qq;
                            const int k = M * q + rho;
                            const float2 A = buf[pa + qq];
                            const float2 Bq = (g == 0) ? buf[pad16(ob + ((L - q) & (L - 1)))] : buf[pb - qq];
                            const float ex = 0.5f * (A.x + Bq.x), ey = 0.5f * (A.y - Bq.y);
                            const float dx = 0.5f * (A.x - Bq.x), dy = 0.5f * (A.y + Bq.y);
                            const float2 X = make_float2(ex + wk.x * dy + wk.y * dx, ey + wk.y * dy - wk.x * dx);
                            if (k < sp.fcount) {
                                const bool pk = phase && (k < sp.klo || k > sp.khi);
                                const int ai = w * nb + q + h * L;
                                if (MODE == MODE_SINGLE || MODE == MODE_MMP3 || k >= sp.khf) {
                                    float e;
                                    if (pk) e = energy_phase(X, efac(k),
                                                             k >= sp.khf ? cmul(rot, hrot) : rot, Kc);
                                    else e = Kc * (X.x * X.x + X.y * X.y);
                                    if (MODE == MODE_SINGLE) sink.put(k, e, pk);
                                    else acc[ai] += e;
                                } else {
                                    acc[ai] += X.x * X.x + X.y * X.y;
                                    acc[nwin * nb + ai] += X.x * X.x - X.y * X.y;
                                    acc[2 * nwin * nb + ai] += 2.0f * X.x * X.y;
                                }
                            }
                            if (phase) rot = cmul(rot, step);
                            wk = cmul(wk, make_float2(kW2L[LOGL].x, kW2L[LOGL].y));
                        }
                    }
                    if (g == 0 && q0 == 0 && Nh < sp.fcount) {
                        // Nyquist bin k = Nh (a high-frequency bin): X = Re Z[0] - Im Z[0]
                        const float2 Z0 = buf[pad16(o0)];
                        const float2 X = make_float2(Z0.x - Z0.y, 0.0f);
                        const bool pk = Nh < sp.klo || Nh > sp.khi;
                        const float e = pk ? energy_phase(X, efac(Nh),
                                                          cmul(centre_rot((unsigned)Nh, m.z, cf, nfu, tw), hrot), Kc)
                                           : Kc * X.x * X.x;
                        if (MODE == MODE_SINGLE) sink.put(Nh, e, pk);
                        else acc[w * nb + L] += e;
                    }
                    if (MODE != MODE_SINGLE && last) {
                        // energies of the accumulated channels
                        const int nq = (g == 0 && q0 == 0) ? CH + 1 : CH;
    #pragma unroll 1
                        for (int h = 0; h < nf; ++h) {
                            const int rho = h ? rho1 : rho0;
                            float2 rot = make_float2(1.f, 0.f);
                            if (phase && MODE == MODE_MMP1) rot = centre_rot((unsigned)(M * q0 + rho), m.z, cf, nfu, tw);
    #pragma unroll 1
                            for (int qq = 0; qq < nq; ++qq) {
                                const bool nyq = qq == CH;
                                const int q = nyq ? L : q0 + qq;
                                const int k = nyq ? Nh : M * q + rho;
                                if (k < sp.fcount && !(nyq && h == 1)) {
                                    const int ai = w * nb + q + h * L;
                                    if (MODE == MODE_MMP3 || k >= sp.khf) {
                                        sink.put(k, acc[ai], k < sp.klo || k > sp.khi);
                                    } else {
                                        const bool pk = k < sp.klo;
                                        const float P = acc[ai];
                                        const float2 S = make_float2(acc[nwin * nb + ai], acc[2 * nwin * nb + ai]);
                                        const float e = energy_mmp1(P, S, pk, pk ? efac(k) : 0.0f, rot, sp.K1);
                                        if (pk) {
                                            float Ub, Lb;
                                            mmp1_phase_bounds(P, S, efac(k), rot, Kc, dlt, ip.C, k == 0, Ub, Lb);
                                            sink.put_bounded(k, e, Ub, Lb, tstar, s_ub, s_lb, w);
                                        } else {
                                            sink.put(k, e, false);
                                        }
                                    }
                                }
                                if (phase && MODE == MODE_MMP1 && !nyq) rot = cmul(rot, step);
                            }
                        }
                    }
                }
                if (!COLLECT && (MODE == MODE_SINGLE || last)) {
                    // class maxima over the lanes of this window
                    sink_reduce<TPW>(sink.best_np, s_key, w, valid, tid);
                    sink_reduce<TPW>(sink.best_ph, s_keyp, w, valid, tid);
                }
            }
        } else {
            // (3a) every bin whose energy has no phase term.  A task is q0 .. q0 +
            // CH - 1 of one window; the tasks holding phase-dependent bins (k < klo
            // or k > khi) are the first tlo and those from thi on, the same in every
            // window, and only their phase-dependent bins are left to (3b).
            static_assert(MODE == MODE_SINGLE || MODE == MODE_MMP3, "the split spectrum serves SMP and MMP3");
            {
                // bins k and Nh - k from one pair of loads, as for 8 <= L <= 32 (the
                // phase-dependent ones, whichever task holds them, are (3b)'s);
                // MMP3 adds each channel's energy to the bin's sum instead
                constexpr int QH = CH / 2;
                for (int base = 0; base < ntasks; base += T) {
                    const int task = base + tid;
                    const bool valid = task < ntasks;
                    const int w = valid ? task / TPW : 0;
                    const int tau = task - w * TPW;
                    BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                    if (valid) {
                        const int nq = pair ? CH : QH;
                        const int q0 = tau * nq;
                        const int o0 = (w * nf) << LOGL;
                        const int ob = pair ? o0 + L : o0;
                        const float2* pA = buf + pad16(o0 + q0);
                        const float2* pB = buf + pad16(ob + L - 1 - q0);
                        // W_Nfft^k = W_Nfft^rho0 W_2L^q, rotated by W_2L from bin to bin.
                        // The mirror's twiddle is -conj(W_Nfft^k) (W_Nfft^M = W_2L and
                        // rho1 = M - rho0), so with E = (A + conj B) / 2 and
                        // D = (A - conj B) / 2i: X[k] = E + W D, X[Nh-k] = conj(E - W D).
                        float2 wk = __ldg(tw + (q0 << (12 - LOGL)));  // W_2L^q
                        if (g != 0) wk = cmul(wr0, wk);
#pragma unroll 8
                        for (int qq = 0; qq < nq; ++qq) {
                            const int q = q0 + qq;
                            const int k = M * q + rho0;
                            const int km = Nh - k;
                            const float2 A = pA[qq];
                            const float2 Bq = (g == 0) ? buf[pad16(o0 + ((L - q) & (L - 1)))] : pB[-qq];
                            const float ex = 0.5f * (A.x + Bq.x), ey = 0.5f * (A.y - Bq.y);
                            const float dx = 0.5f * (A.x - Bq.x), dy = 0.5f * (A.y + Bq.y);
                            const float u = wk.x * dy + wk.y * dx, v = wk.y * dy - wk.x * dx;
                            if (k < sp.fcount && k >= sp.klo && k <= sp.khi) {
                                const float2 X = make_float2(ex + u, ey + v);
                                const float e = Kc * (X.x * X.x + X.y * X.y);
                                if (MODE == MODE_SINGLE) sink.put(k, e, false);
                                else acc[w * nb + q] += e;
                            }
                            if (km < sp.fcount && km >= sp.klo && km <= sp.khi) {
                                const float2 Xm = make_float2(ex - u, v - ey);
                                const float e = Kc * (Xm.x * Xm.x + Xm.y * Xm.y);
                                if (MODE == MODE_SINGLE) sink.put(km, e, false);
                                else acc[w * nb + (pair ? 2 * L - 1 - q : (g == 0 ? L - q : L - 1 - q))] += e;
                            }
                            wk = cmul(wk, make_float2(kW2L[LOGL].x, kW2L[LOGL].y));
                        }
                        if (g == 0 && tau == TPW - 1) {
                            // q = L/2, its own mirror; wk = W_2L^{L/2}
                            const int k = M * (L / 2);
                            if (k < sp.fcount && k >= sp.klo && k <= sp.khi) {
                                const float2 A = buf[pad16(o0 + L / 2)];
                                const float2 X = make_float2(A.x + wk.x * A.y, wk.y * A.y);
                                const float e = Kc * (X.x * X.x + X.y * X.y);
                                if (MODE == MODE_SINGLE) sink.put(k, e, false);
                                else acc[w * nb + L / 2] += e;
                            }
                        }
                    }
                    if (!COLLECT && MODE == MODE_SINGLE) sink_reduce<TPW>(sink.best_np, s_key, w, valid, tid);
                }
            }
            if constexpr (LOGL >= 10 && (MODE == MODE_SINGLE || MODE == MODE_MMP3)) {
                // (3b) for L >= 1024: the phase-dependent bins one per thread (a
                // unit holds at most eight windows, so task-sized items would leave
                // a few warps doing all of them).  Per half h they are q < ql and
                // qh <= q < qe (k < klo, k > khi, k < fcount), plus the Nyquist bin.
                int ql[2] = {0, 0}, qh[2] = {0, 0}, cnt[2] = {0, 0};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    if (h < nf) {
                        const int rho = h ? rho1 : rho0;
                        const int qe = max(0, min(L, (sp.fcount - rho + M - 1) / M));
                        const int lo = sp.klo - rho;
                        ql[h] = min(qe, lo > 0 ? (lo + M - 1) / M : 0);
                        const int hi = sp.khi - rho;
                        qh[h] = max(ql[h], min(qe, hi >= 0 ? hi / M + 1 : 0));
                        cnt[h] = ql[h] + (qe - qh[h]);
                    }
                }
                const int nyq = (g == 0 && Nh < sp.fcount) ? 1 : 0;
                const int nper = cnt[0] + cnt[1] + nyq;
                for (int i = tid; i < nwin * nper; i += T) {
                    const int w = i / nper;
                    int jx = i - w * nper;
                    const int4 m = s_win[w];
                    const float cf = __int_as_float(m.w);
                    const float4 hr = s_rot[w];
                    const float2 hrot = make_float2(hr.x, hr.y);
                    const int o0 = (w * nf) << LOGL;
                    float2 X;
                    int k, aq;
                    if (jx == cnt[0] + cnt[1]) {
                        // Nyquist bin k = Nh (g = 0): X = Re Z[0] - Im Z[0]
                        const float2 Z0 = buf[pad16(o0)];
                        X = make_float2(Z0.x - Z0.y, 0.0f);
                        k = Nh;
                        aq = L;
                    } else {
                        const int h = jx < cnt[0] ? 0 : 1;
                        if (h) jx -= cnt[0];
                        const int q = jx < ql[h] ? jx : qh[h] + (jx - ql[h]);
                        const int rho = h ? rho1 : rho0;
                        const float2 wr = h ? wr1 : wr0;
                        const int oa = h ? o0 + L : o0;
                        const int ob = pair ? (h ? o0 : o0 + L) : o0;
                        const float2 A = buf[pad16(oa + q)];
                        const float2 Bq = (g == 0) ? buf[pad16(ob + ((L - q) & (L - 1)))] : buf[pad16(ob + L - 1 - q)];
                        const float2 t = __ldg(tw + (q << (12 - LOGL)));
                        const float2 wk = (g == 0) ? t : cmul(wr, t);
                        const float ex = 0.5f * (A.x + Bq.x), ey = 0.5f * (A.y - Bq.y);
                        const float dx = 0.5f * (A.x - Bq.x), dy = 0.5f * (A.y + Bq.y);
                        X = make_float2(ex + wk.x * dy + wk.y * dx, ey + wk.y * dy - wk.x * dx);
                        k = M * q + rho;
                        aq = q + h * L;
                    }
                    const float2 rot = centre_rot((unsigned)k, m.z, cf, nfu, tw);
                    const float e = energy_phase(X, efac(k), k >= sp.khf ? cmul(rot, hrot) : rot, Kc);
                    if constexpr (MODE == MODE_SINGLE) {
                        BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                        sink.put(k, e, true);
                        if (!COLLECT) atomicMax(s_keyp + w, sink.best_ph);
                    } else {
                        acc[w * nb + aq] += e;
                    }
                }
            } else
            // (3b) the phase-dependent bins (and the Nyquist bin), task by task as in
            // (3a) but spread over all threads: nph such tasks per window
            for (int i = tid; i < nwin * nph; i += T) {
                const int w = i / nph;
                const int jx = i - w * nph;
                const int q0 = (jx < tlo ? jx : thi + (jx - tlo)) * CH;
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                const int4 m = s_win[w];
                const float cf = __int_as_float(m.w);
                const float4 hr = s_rot[w];
                const float2 hrot = make_float2(hr.x, hr.y);  // e^{-2 pi i fs t0} for high bins
                const float2 step = make_float2(hr.z, hr.w);  // psi increment from q to q + 1
                const int o0 = (w * nf) << LOGL;
                const int o1 = o0 + L;
#pragma unroll 1
                for (int h = 0; h < nf; ++h) {
                    const int rho = h ? rho1 : rho0;
                    const float2 wr = h ? wr1 : wr0;
                    const int oa = h ? o1 : o0;
                    const int ob = pair ? (h ? o0 : o1) : o0;
                    float2 rot = centre_rot((unsigned)(M * q0 + rho), m.z, cf, nfu, tw);
                    const int pa = pad16(oa + q0);
                    const int pb = pad16(ob + L - 1 - q0);
                    // W_Nfft^k = W_Nfft^rho W_2L^q, rotated by W_2L from bin to bin
                    float2 wk = __ldg(tw + (q0 << (12 - LOGL)));
                    if (g != 0) wk = cmul(wr, wk);
#pragma unroll 2
                    for (int qq = 0; qq < CH; ++qq, wk = cmul(wk, make_float2(kW2L[LOGL].x, kW2L[LOGL].y))) {
                        const int q = q0 + qq;
                        const int k = M * q + rho;
                        const float2 A = buf[pa + qq];
                        const float2 Bq = (g == 0) ? buf[pad16(ob + ((L - q) & (L - 1)))] : buf[pb - qq];
                        if (k < sp.fcount && (k < sp.klo || k > sp.khi)) {
                            const float ex = 0.5f * (A.x + Bq.x), ey = 0.5f * (A.y - Bq.y);
                            const float dx = 0.5f * (A.x - Bq.x), dy = 0.5f * (A.y + Bq.y);
                            const float2 X = make_float2(ex + wk.x * dy + wk.y * dx, ey + wk.y * dy - wk.x * dx);
                            const float e = energy_phase(X, efac(k), k >= sp.khf ? cmul(rot, hrot) : rot, Kc);
                            if (MODE == MODE_SINGLE) sink.put(k, e, true);
                            else acc[w * nb + q + h * L] += e;
                        }
                        rot = cmul(rot, step);
                    }
                }
                if (g == 0 && q0 == 0 && Nh < sp.fcount) {
                    // Nyquist bin k = Nh (a high-frequency bin): X = Re Z[0] - Im Z[0]
                    const float2 Z0 = buf[pad16(o0)];
                    const float2 X = make_float2(Z0.x - Z0.y, 0.0f);
                    const bool pk = Nh < sp.klo || Nh > sp.khi;
                    const float e = pk ? energy_phase(X, efac(Nh),
                                                      cmul(centre_rot((unsigned)Nh, m.z, cf, nfu, tw), hrot), Kc)
                                       : Kc * X.x * X.x;
                    if (MODE == MODE_SINGLE) sink.put(Nh, e, pk);
                    else acc[w * nb + L] += e;
                }
                if (!COLLECT && MODE == MODE_SINGLE) {
                    if (sink.best_ph) atomicMax(s_keyp + w, sink.best_ph);
                    if (sink.best_np) atomicMax(s_key + w, sink.best_np);
                }
            }
            if (MODE == MODE_MMP3 && last) {
                // energies of the accumulated channels
                __syncthreads();
                for (int base = 0; base < ntasks; base += T) {
                    const int task = base + tid;
                    const bool valid = task < ntasks;
                    const int w = valid ? task / TPW : 0;
                    const int q0 = (task - w * TPW) * CH;
                    BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_np, thr_ph, 0u, 0u};
                    if (valid) {
                        const int nq = (g == 0 && q0 == 0) ? CH + 1 : CH;
#pragma unroll 1
                        for (int h = 0; h < nf; ++h) {
                            const int rho = h ? rho1 : rho0;
#pragma unroll 1
                            for (int qq = 0; qq < nq; ++qq) {
                                const bool nyq = qq == CH;
                                const int q = nyq ? L : q0 + qq;
                                const int k = nyq ? Nh : M * q + rho;
                                if (k < sp.fcount && !(nyq && h == 1))
                                    sink.put(k, acc[w * nb + q + h * L], k < sp.klo || k > sp.khi);
                            }
                        }
                    }
                    if (!COLLECT) {
                        sink_reduce<TPW>(sink.best_np, s_key, w, valid, tid);
                        sink_reduce<TPW>(sink.best_ph, s_keyp, w, valid, tid);
                    }
                }
            }
        }
        __syncthreads();
    }

    if (!COLLECT) {
        // slot key: certified upper bound (high word) and lower bound (low word)
        // of the exact energies of the slot's bins
        unsigned long long* out = b.slots + ip.slot_off + sp.slot_base;
        for (int w = tid; w < nwin; w += T) {
            float Un, Ln, Up, Lp;
            class_bounds(s_key[w], bt.d_np, bt.tau_np, Un, Ln);
            class_bounds(s_keyp[w], bt.d_ph, bt.tau_ph, Up, Lp);
            float U = fmaxf(Un, Up), Lo = fmaxf(Ln, Lp);
            if (MODE == MODE_MMP1) {
                U = fmaxf(U, __uint_as_float(s_ub[w]));
                Lo = fmaxf(Lo, __uint_as_float(s_lb[w]));
            }
            if (!(U <= 3.0e38f)) U = 3.0e38f;  // NaN / inf inputs: keep the slot competitive
            out[(long long)(t_start + w) * sp.G + g] =
                ((unsigned long long)__float_as_uint(U) << 32) | (unsigned long long)__float_as_uint(Lo);
            if (b.stale) b.stale[ip.slot_off + sp.slot_base + (long long)(t_start + w) * sp.G + g] = 0;
        }
    }
    __syncthreads();
}

// One size of the candidate path's runtime dispatch (inlined: the call
// boundary of an out-of-line body cost more than the larger kernel).
template <int LOGL, int MODE>
__device__ __forceinline__ void collect_body(const BatchDev& b, unsigned char* smem, int inst, int j, int g, int t,
                                             float tstar) {
    unit_body<LOGL, MODE, true>(b, smem, inst, j, g, t, 1, tstar);
}

// Refresh of one sub-FFT size: CTAs pull (instance, scale, group, t-batch)
// units from that size's list, which the schedule filled.  MINB = 2: two
// CTAs per SM at 64 registers a thread (the default); MINB = 1: one CTA per SM
// at 128 registers, without spills (the "wide" variant the autotuner may pick
// per size).
template <int LOGL, int MODE>
__device__ __forceinline__ void refresh_queue(const BatchDev& b, unsigned char* smem, int* s_unit) {
    const int total = min(b.lcount[LOGL], b.lcap[LOGL]);
    const int4* EMPI_RESTRICT_MUT list = b.units + b.loff[LOGL];
    for (;;) {
        if (threadIdx.x == 0) *s_unit = atomicAdd(b.lhead + LOGL, 1);
        __syncthreads();
        const int u = *s_unit;
        __syncthreads();
        if (u >= total) break;
        const int4 un = list[u];  // (instance, scale | group << 16, t_start, nwin)
        unit_body<LOGL, MODE, false>(b, smem, un.x, un.y & 0xffff, un.y >> 16, un.z, un.w, 0.0f);
    }
}

template <int MODE, int LOGL, int MINB>
__global__ void __launch_bounds__(kUnitThreads, MINB) k_refresh(BatchDev b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    refresh_queue<LOGL, MODE>(b, smem, &s_unit);
}

// Every sub-FFT size's list in one pass, largest transforms first (the
// persistent kernel's refresh phase); smem holds the largest layout.
template <int MODE>
__device__ __forceinline__ void refresh_all_sizes(const BatchDev& b, unsigned char* smem, int* s_unit) {
#define EMPI_REFRESH_SIZE(LG) \
    if (b.lcount[LG] > 0) refresh_queue<LG, MODE>(b, smem, s_unit);
    EMPI_REFRESH_SIZE(12)
    EMPI_REFRESH_SIZE(11)
    EMPI_REFRESH_SIZE(10)
    EMPI_REFRESH_SIZE(9)
    EMPI_REFRESH_SIZE(8)
    EMPI_REFRESH_SIZE(7)
    EMPI_REFRESH_SIZE(6)
    EMPI_REFRESH_SIZE(5)
    EMPI_REFRESH_SIZE(4)
    EMPI_REFRESH_SIZE(3)
    EMPI_REFRESH_SIZE(2)
    EMPI_REFRESH_SIZE(1)
    EMPI_REFRESH_SIZE(0)
#undef EMPI_REFRESH_SIZE
}

// FP32 recompute of the candidate slots (one window each), emitting every bin
// whose certified upper bound reaches the instance's lower bound tstar.
template <int MODE>
__device__ __forceinline__ void collect_queue(const BatchDev& b, unsigned char* smem, int* s_unit_p) {
    int& s_unit = *s_unit_p;
    const int total = min(b.ctr[CTR_CSLOTS], b.cslot_cap);
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(b.ctr + CTR_CSLOT_Q, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= total) break;
        const CandSlot cs = b.cslots[u];
        if (EMPI_BAD(cs.inst < 0 || cs.inst >= b.ninst, 2)) continue;
        const float tstar = __uint_as_float(b.state[cs.inst].tstar);
        const InstPlan ip = b.insts[cs.inst];
        if (EMPI_BAD(cs.j < 0 || cs.j >= b.dicts[ip.dict].nscales, 2)) continue;
        const ScalePlan& sp = b.scales[b.dicts[ip.dict].scale0 + cs.j];
        if (EMPI_BAD(cs.t < 0 || cs.t >= sp.tcount || cs.g < 0 || cs.g >= sp.G, 3)) continue;
        // slots below the refined threshold hold no candidate bin
        const unsigned long long key = b.slots[ip.slot_off + sp.slot_base + (long long)cs.t * sp.G + cs.g];
        if (__uint_as_float((unsigned)(key >> 32)) < tstar) continue;
        switch (sp.logL) {
#define EMPI_COLLECT_CASE(LG) \
    case LG: collect_body<LG, MODE>(b, smem, cs.inst, cs.j, cs.g, cs.t, tstar); break;
            EMPI_COLLECT_CASE(0)
            EMPI_COLLECT_CASE(1)
            EMPI_COLLECT_CASE(2)
            EMPI_COLLECT_CASE(3)
            EMPI_COLLECT_CASE(4)
            EMPI_COLLECT_CASE(5)
            EMPI_COLLECT_CASE(6)
            EMPI_COLLECT_CASE(7)
            EMPI_COLLECT_CASE(8)
            EMPI_COLLECT_CASE(9)
            EMPI_COLLECT_CASE(10)
            EMPI_COLLECT_CASE(11)
            EMPI_COLLECT_CASE(12)
#undef EMPI_COLLECT_CASE
            default: break;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kUnitThreads, 1) k_collect(BatchDev b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    collect_queue<MODE>(b, smem, &s_unit);
}

// The refresh and collect kernels of one variant mode, with their shared
// memory, for the engine (filled in that mode's translation unit).
template <int MODE, int LG>
void fill_refresh_size(RefreshKernels& rk) {
    rk.refresh[LG][0] = (void*)k_refresh<MODE, LG, 2>;
    rk.refresh[LG][1] = (void*)k_refresh<MODE, LG, 1>;
    rk.smem[LG] = refresh_smem_bytes<MODE, LG>();
}

template <int MODE>
void fill_refresh_kernels(RefreshKernels& rk) {
    fill_refresh_size<MODE, 0>(rk);
    fill_refresh_size<MODE, 1>(rk);
    fill_refresh_size<MODE, 2>(rk);
    fill_refresh_size<MODE, 3>(rk);
    fill_refresh_size<MODE, 4>(rk);
    fill_refresh_size<MODE, 5>(rk);
    fill_refresh_size<MODE, 6>(rk);
    fill_refresh_size<MODE, 7>(rk);
    fill_refresh_size<MODE, 8>(rk);
    fill_refresh_size<MODE, 9>(rk);
    fill_refresh_size<MODE, 10>(rk);
    fill_refresh_size<MODE, 11>(rk);
    fill_refresh_size<MODE, 12>(rk);
    rk.collect = (void*)k_collect<MODE>;
    size_t most = 0;
    for (int lg = 0; lg < kRefreshSizes; ++lg) most = rk.smem[lg] > most ? rk.smem[lg] : most;
    rk.collect_smem = most;
}

}  // namespace empi
