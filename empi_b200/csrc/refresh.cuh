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
// Included from kernels.cuh.
#pragma once

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
    static constexpr size_t key = rot + sizeof(float4) * NW;          // u32 energy bits
    static constexpr size_t etab = key + sizeof(unsigned) * NW;       // float, kEtabSmem
    static constexpr size_t acc = etab + sizeof(float) * kEtabSmem;   // (MMP) per-bin channel sums
};

template <int MODE, int LOGL>
constexpr size_t refresh_smem_bytes() {
    return RefreshSmem<LOGL>::acc + (MODE == MODE_SINGLE ? 0
                                                       : sizeof(float) * (kUnitPoints + RefreshSmem<LOGL>::NW) *
                                                             (MODE == MODE_MMP1 ? 3 : 1));
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
    const int slot = atomicAdd(b.ctr + CTR_CBINS, 1);
    if (slot < b.cbin_cap) {
        const int li = atomicAdd(&b.state[inst].nbins, 1);
        if (li < b.inst_bin_cap) {
            CandBin cb;
            cb.inst = inst;
            cb.j = j;
            cb.t = t;
            cb.k = k;
            cb.e32 = e;
            cb.pad = 0;
            cb.e64 = 0.0;
            b.cbins[slot] = cb;
            b.inst_bins[(long long)inst * b.inst_bin_cap + li] = slot;
            return;
        }
    }
    b.state[inst].err = ERR_CAND_OVERFLOW;
}

// What the spectrum stage does with a bin's final energy.  The slot keeps only
// its maximum energy (the tree keys slots by index); negative, NaN and
// infinite energies count as 0, as in pack_key.
template <bool COLLECT>
struct BinSink {
    const BatchDev& b;
    int inst, j, t, tcount;
    unsigned thr_bits;
    float best;
    __device__ __forceinline__ void put(int k, float e) {
        if (COLLECT) {
            if (__float_as_uint(e) >= thr_bits) emit_candidate(b, inst, j, t, k, e);
        } else {
            if (b.dump) b.dump[(long long)k * tcount + t] = e;
            best = fmaxf(best, e <= 3.0e38f ? e : 0.0f);
        }
    }
};

// Max of one window's bins over the lanes holding its tasks (TPW consecutive,
// aligned lanes) into the window's shared key; non-negative floats order as
// their bit patterns.
template <int TPW>
__device__ __forceinline__ void sink_reduce(float bestf, unsigned* s_key, int w, bool valid, int tid) {
    unsigned best = __float_as_uint(bestf);
    if (TPW >= 32) {
        best = __reduce_max_sync(0xffffffffu, best);
        if ((tid & 31) == 0 && valid) atomicMax(s_key + w, best);
    } else {
#pragma unroll
        for (int off = TPW / 2; off; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
        if ((tid & (TPW - 1)) == 0 && valid) atomicMax(s_key + w, best);
    }
}

template <int LOGL, int MODE, bool COLLECT>
__device__ __forceinline__ void unit_body(const BatchDev& b, unsigned char* smem, int inst, int j, int g, int t_start,
                                          int nwin, unsigned thr_bits) {
    constexpr int L = 1 << LOGL;
    constexpr int CH = L < kBinsPerTask ? L : kBinsPerTask;  // q values per task
    constexpr int TPW = L / CH;                                // tasks per window
    float2* buf = reinterpret_cast<float2*>(smem + RefreshSmem<LOGL>::buf);
    int4* s_win = reinterpret_cast<int4*>(smem + RefreshSmem<LOGL>::win);
    float4* s_rot = reinterpret_cast<float4*>(smem + RefreshSmem<LOGL>::rot);
    float* s_etab = reinterpret_cast<float*>(smem + RefreshSmem<LOGL>::etab);
    unsigned* s_key = reinterpret_cast<unsigned*>(smem + RefreshSmem<LOGL>::key);
    float* acc = reinterpret_cast<float*>(smem + RefreshSmem<LOGL>::acc);

    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const ScalePlan sp = b.scales[dp.scale0 + j];
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

    // Per window: geometry, and for the phase-dependent bins e^{-2 pi i fs t0}
    // (high bins) and the step of psi from q to q + 1; the scale's expFactor
    // table when it fits.  Read by the spectrum stage instead of global loads
    // and transcendentals inside its tasks.
    const int ecount = sp.klo + (sp.fcount - 1 - sp.khi);
    const bool etab_smem = ecount <= kEtabSmem;
    {
        const long long w0 = sp.win_base + t_start;
        for (int w = tid; w < nwin; w += T) {
            const int4 m = __ldg(b.wtab + w0 + w);
            s_win[w] = m;
            float sh, ch;
            sincospif(-2.0f * __ldg(b.whf + w0 + w), &sh, &ch);
            const float2 st = centre_rot((unsigned)sp.M, m.z, __int_as_float(m.w), (unsigned)sp.nfft, b.tw);
            s_rot[w] = make_float4(ch, sh, st.x, st.y);
            s_key[w] = 0u;
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
        const float* __restrict__ x = b.residual32 + ip.res_off + (long long)c * dp.N;
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
            const float* __restrict__ xs = x + m.x;
            a1 = make_float2(0.f, 0.f);
            a2 = make_float2(0.f, 0.f);
            if (F == 1) {
                // one fold (every scale whose longest window fits its sub-FFT):
                // no loop and no rotation of the twist to a next fold
                const int i0 = 2 * np;
                if (i0 < m.y) {
                    const float x0 = __ldg(xs + i0);
                    const float x1 = (i0 + 1 < m.y) ? __ldg(xs + i0 + 1) : 0.0f;
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
                const float x0 = __ldg(xs + i0);
                const float x1 = (i0 + 1 < m.y) ? __ldg(xs + i0 + 1) : 0.0f;
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
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
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
                            sink.put(k, e);
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
                            sink.put(km, e);
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
                            sink.put(k, e);
                        }
                    }
                }
                if (!COLLECT) sink_reduce<TPW>(sink.best, s_key, w, valid, tid);
            }
        } else if constexpr (!kSplit) {
            for (int base = 0; base < ntasks; base += T) {
                const int task = base + tid;
                const bool valid = task < ntasks;
                const int w = valid ? task / TPW : 0;
                const int q0 = (task - w * TPW) * CH;
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
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
                                    if (MODE == MODE_SINGLE) sink.put(k, e);
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
                        if (MODE == MODE_SINGLE) sink.put(Nh, e);
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
                                    float e;
                                    if (MODE == MODE_MMP3 || k >= sp.khf) {
                                        e = acc[ai];
                                    } else {
                                        const bool pk = k < sp.klo;
                                        e = energy_mmp1(acc[ai], make_float2(acc[nwin * nb + ai], acc[2 * nwin * nb + ai]),
                                                        pk, pk ? efac(k) : 0.0f, rot, sp.K1);
                                    }
                                    sink.put(k, e);
                                }
                                if (phase && MODE == MODE_MMP1 && !nyq) rot = cmul(rot, step);
                            }
                        }
                    }
                }
                if (!COLLECT && (MODE == MODE_SINGLE || last)) {
                    // max over the lanes of this window (TPW consecutive, aligned lanes);
                    // non-negative floats order as their bit patterns
                    unsigned best = __float_as_uint(sink.best);
                    if (TPW >= 32) {
                        best = __reduce_max_sync(0xffffffffu, best);
                        if ((tid & 31) == 0 && valid) atomicMax(s_key + w, best);
                    } else {
    #pragma unroll
                        for (int off = TPW / 2; off; off >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, off));
                        if ((tid & (TPW - 1)) == 0 && valid) s_key[w] = best;
                    }
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
                    BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
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
                                if (MODE == MODE_SINGLE) sink.put(k, e);
                                else acc[w * nb + q] += e;
                            }
                            if (km < sp.fcount && km >= sp.klo && km <= sp.khi) {
                                const float2 Xm = make_float2(ex - u, v - ey);
                                const float e = Kc * (Xm.x * Xm.x + Xm.y * Xm.y);
                                if (MODE == MODE_SINGLE) sink.put(km, e);
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
                                if (MODE == MODE_SINGLE) sink.put(k, e);
                                else acc[w * nb + L / 2] += e;
                            }
                        }
                    }
                    if (!COLLECT && MODE == MODE_SINGLE) sink_reduce<TPW>(sink.best, s_key, w, valid, tid);
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
                        BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
                        sink.put(k, e);
                        if (!COLLECT) atomicMax(s_key + w, __float_as_uint(sink.best));
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
                BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
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
                            if (MODE == MODE_SINGLE) sink.put(k, e);
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
                    if (MODE == MODE_SINGLE) sink.put(Nh, e);
                    else acc[w * nb + L] += e;
                }
                if (!COLLECT && MODE == MODE_SINGLE) atomicMax(s_key + w, __float_as_uint(sink.best));
            }
            if (MODE == MODE_MMP3 && last) {
                // energies of the accumulated channels
                __syncthreads();
                for (int base = 0; base < ntasks; base += T) {
                    const int task = base + tid;
                    const bool valid = task < ntasks;
                    const int w = valid ? task / TPW : 0;
                    const int q0 = (task - w * TPW) * CH;
                    BinSink<COLLECT> sink{b, inst, j, t_start + w, sp.tcount, thr_bits, 0.0f};
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
                                if (k < sp.fcount && !(nyq && h == 1)) sink.put(k, acc[w * nb + q + h * L]);
                            }
                        }
                    }
                    if (!COLLECT) sink_reduce<TPW>(sink.best, s_key, w, valid, tid);
                }
            }
        }
        __syncthreads();
    }

    if (!COLLECT) {
        unsigned long long* out = b.slots + ip.slot_off + sp.slot_base;
        for (int w = tid; w < nwin; w += T) out[(long long)(t_start + w) * sp.G + g] = (unsigned long long)s_key[w] << 32;
    }
    __syncthreads();
}

// One size of the candidate path's runtime dispatch (inlined: the call
// boundary of an out-of-line body cost more than the larger kernel).
template <int LOGL, int MODE>
__device__ __forceinline__ void collect_body(const BatchDev& b, unsigned char* smem, int inst, int j, int g, int t,
                                          unsigned thr_bits) {
    unit_body<LOGL, MODE, true>(b, smem, inst, j, g, t, 1, thr_bits);
}

#ifndef EMPI_REFRESH_MIN_BLOCKS
#define EMPI_REFRESH_MIN_BLOCKS 2
#endif

// Refresh of one sub-FFT size: CTAs pull (instance, scale, group, t-batch)
// units from that size's list, which the schedule filled.
template <int MODE, int LOGL>
__global__ void __launch_bounds__(kUnitThreads, EMPI_REFRESH_MIN_BLOCKS) k_refresh(BatchDev b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    const int total = min(b.lcount[LOGL], b.lcap[LOGL]);
    const int4* __restrict__ list = b.units + b.loff[LOGL];
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(b.lhead + LOGL, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= total) break;
        const int4 un = list[u];  // (instance, scale | group << 16, t_start, nwin)
        unit_body<LOGL, MODE, false>(b, smem, un.x, un.y & 0xffff, un.y >> 16, un.z, un.w, 0u);
    }
}

// FP32 recompute of the candidate slots (one window each), emitting every bin
// within the band of the instance's best.
template <int MODE>
__global__ void __launch_bounds__(kUnitThreads, 1) k_collect(BatchDev b) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    const int total = min(b.ctr[CTR_CSLOTS], b.cslot_cap);
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(b.ctr + CTR_CSLOT_Q, 1);
        __syncthreads();
        const int u = s_unit;
        __syncthreads();
        if (u >= total) break;
        const CandSlot cs = b.cslots[u];
        const unsigned best = (unsigned)(b.state[cs.inst].best32 >> 32);
        const unsigned thr = __float_as_uint(__uint_as_float(best) * (1.0f - b.band));
        const InstPlan ip = b.insts[cs.inst];
        switch (b.scales[b.dicts[ip.dict].scale0 + cs.j].logL) {
#define EMPI_COLLECT_CASE(LG) \
    case LG: collect_body<LG, MODE>(b, smem, cs.inst, cs.j, cs.g, cs.t, thr); break;
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
