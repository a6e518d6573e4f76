// sm_100a kernels of the Matching Pursuit loop.
//
// Per MP iteration the device runs (all launches captured in a CUDA graph):
//   k_cand_slots  the instance's best over its chunk maxima (the tree's root),
//                 then the slots whose FP32 max lies within the candidate band
//   k_refresh<COLLECT>  FP32 recompute of those slots, emitting every bin in
//                 the band
//   k_rescore     FP64 direct DFT of each candidate bin, per channel
//   k_select      FP64 energy (the reference formula) -> argmax -> atom params
//   k_subtract    FP64 atom subtraction on the residual + channel energies
//   k_sched_a/b   stop test, dirty t-range per scale, work-unit prefix sums
//   k_refresh     windowed FFT + energies + per-slot max over the dirty range
//   k_tree        leaf-chunk maxima for the chunks the refresh touched
// In this multi-kernel form nothing spins: ordering comes from kernel
// boundaries.  The same per-iteration steps run as phases of one persistent
// kernel for small batches (persist.cuh), separated by a bounded grid barrier;
// each kernel here is a thin wrapper around its phase body.
#pragma once

#include "common.cuh"

// A translation unit that includes this file for the phase bodies only (the
// persistent kernel's) gets its own internal copies of the wrapper kernels.
#ifdef EMPI_PHASES_ONLY
#define EMPI_GLOBAL static __global__
#else
#define EMPI_GLOBAL __global__
#endif

namespace empi {

// ------------------------------------------------------------ schedule

enum SchedMode { SCHED_ITERATE = 0, SCHED_INIT = 1, SCHED_ATOM = 2 };

// statistics of refreshing windows lo..hi of a scale: reference-equivalent
// FFT flops (2.5 Nfft log2 Nfft per window and channel) and compulsory bytes
// (the FP32 residual span read once per channel, one 8-byte slot write per
// (window, group))
__device__ __forceinline__ void refresh_stats(const DictPlan& dp, const ScalePlan& sp, int C, int lo, int hi,
                                              double& flops, double& bytes, double& slots) {
    const int n = hi - lo + 1;
    int iL0, iR0, iL1, iR1;
    double tf;
    window_bounds(grid_t(lo, dp.tMax, sp.tcount), sp.hw, dp.fs, dp.N, iL0, iR0, tf);
    window_bounds(grid_t(hi, dp.tMax, sp.tcount), sp.hw, dp.fs, dp.N, iL1, iR1, tf);
    const double lg = log2((double)sp.nfft);
    flops += (double)n * C * 2.5 * sp.nfft * lg;
    bytes += 4.0 * C * (double)(iR1 - iL0 + 1) + 8.0 * (double)n * sp.G;
    slots += (double)n * sp.G;
}

// One CTA per instance.  SCHED_INIT: every window dirty (only_scale >= 0
// restricts it to one scale).  SCHED_ITERATE: stop test on the residual energy
// of the previous subtraction (src/classes.cpp:67-70), then the dirty range of
// every scale from the subtracted atom (src/gabor.cpp:197-208).  SCHED_ATOM:
// dirty ranges of the atom (tA, sA) given by the caller.
__device__ __forceinline__ void sched_a_inst(const BatchDev& b, int inst, int mode, int only_scale, double tA_in,
                                             double sA_in) {
    const int init = mode == SCHED_INIT;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    __shared__ int s_active;
    __shared__ double s_tA, s_sA;
    if (threadIdx.x == 0) {
        InstState& st = b.state[inst];
        int active = st.status == ST_RUNNING;
        if (mode == SCHED_ATOM) {
            s_tA = tA_in;
            s_sA = sA_in;
        } else if (active && init) {
            double e = 0.0;
            for (int c = 0; c < ip.C; ++c) e += b.chan_energy[ip.cen_off + c];
            st.etotal = e;
            st.eres = e;
            if (e == 0.0) {
                st.status = ST_ERROR;
                st.err = ERR_SIGNAL_EMPTY;
                active = 0;
            }
        } else if (active) {
            double e = 0.0;
            for (int c = 0; c < ip.C; ++c) e += b.chan_energy[ip.cen_off + c];
            st.eres = e;
            b.energies[(long long)inst * b.iter_max + st.it - 1] = e;
            if (e / st.etotal <= b.residual_energy) {
                st.status = ST_DONE;
                active = 0;
            } else if (EMPI_BAD(st.it < 1, 13)) {
                active = 0;
            } else {
                const double* p = b.atoms + ip.out_off + (long long)(st.it - 1) * ip.C * 6;
                s_tA = p[2] / dp.fs;
                s_sA = p[3] / dp.fs;
            }
        }
        s_active = active;
    }
    __syncthreads();
    if (mode == SCHED_ATOM) {
        // the caller changed a channel's residual (the workspace seam): its
        // largest |sample| anew
        __shared__ unsigned redm[32];
        for (int c = 0; c < ip.C; ++c) {
            const float* x32 = b.residual32 + ip.res_off + (long long)c * dp.N;
            float xm = 0.0f;
            for (int i = threadIdx.x; i < dp.N; i += blockDim.x) xm = fmaxf(xm, fabsf(x32[i]));
            xm = block_max_nonneg(xm, redm);
            if (threadIdx.x == 0) b.chan_xmax[ip.cen_off + c] = xm;
        }
    }
    if (threadIdx.x == 0) {
        // B of the refresh's error bound: the channel norm of max |residual|
        double q = 0.0;
        for (int c = 0; c < ip.C; ++c) {
            const double xm = (double)b.chan_xmax[ip.cen_off + c];
            q += xm * xm;
        }
        b.state[inst].bnorm = __double2float_ru(sqrt(q));
    }
    int* units = b.ij_units + ip.ij_off + inst;
    int* chunks = b.ij_chunks + ip.ij_off + inst;
    double st_flops = 0.0, st_bytes = 0.0, st_slots = 0.0;  // statistics, one atomic each per CTA
    // per-scale unit and chunk counts, scanned across the CTA a blockDim-sized
    // batch of scales at a time into units[j + 1], chunks[j + 1] (inclusive
    // prefix sums; units[0] = chunks[0] = 0)
    __shared__ int s_wu[32], s_wc[32], s_carry[2];
    if (threadIdx.x == 0) {
        s_carry[0] = 0;
        s_carry[1] = 0;
        units[0] = 0;
        chunks[0] = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < dp.nscales; base += blockDim.x) {
        const int j = base + threadIdx.x;
        int nu = 0, nc = 0;
        if (j < dp.nscales) {
            const ScalePlan sp = b.scales[dp.scale0 + j];
            int lo = 0, hi = -1;
            if (s_active) {
                if (init) {
                    if (only_scale < 0 || only_scale == j) {
                        lo = 0;
                        hi = sp.tcount - 1;
                    }
                } else {
                    dirty_range(sp, dp.tMax, s_tA, s_sA, lo, hi);
                }
            }
            b.dirty[ip.ij_off + j] = make_int2(lo, hi);
            int c0 = 0;
            if (hi >= lo) {
                // the windows refreshed now: the dirty range, or with a block
                // proposal only its proposed part (the rest get propagated
                // bounds and a certified second round, k_round2_sched)
                int ulo = lo, uhi = hi;
                if (b.prange && mode == SCHED_ITERATE) {
                    const int2 pr = b.prange[ip.ij_off + j];
                    ulo = max(lo, pr.x);
                    uhi = min(hi, pr.y);
                }
                if (uhi >= ulo) {
                    const int n = uhi - ulo + 1;
                    for (int g = 0; g < sp.G; ++g) nu += group_units(n, g, sp);
                    // this scale's units go to the list of its sub-FFT size
                    int at = atomicAdd(b.lcount + sp.logL, nu);
                    const int cap = b.lcap[sp.logL];
                    int4* list = b.units + b.loff[sp.logL];
                    for (int g = 0; g < sp.G; ++g) {
                        const int B = g >= 2 ? sp.B2 : sp.B1;
                        for (int t0 = ulo; t0 <= uhi; t0 += B, ++at)
                            if (at < cap) list[at] = make_int4(inst, j | (g << 16), t0, min(B, uhi - t0 + 1));
                    }
                    refresh_stats(dp, sp, ip.C, ulo, uhi, st_flops, st_bytes, st_slots);
                }
                const long long s0 = sp.slot_base + (long long)lo * sp.G;
                const long long s1 = sp.slot_base + (long long)(hi + 1) * sp.G - 1;
                c0 = (int)(s0 / kChunk);
                nc = (int)(s1 / kChunk) - c0 + 1;
            }
            b.ij_crange[ip.ij_off + j] = make_int2(c0, nc);
        }
        int iu = nu, ic = nc;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int yu = __shfl_up_sync(0xffffffffu, iu, off), yc = __shfl_up_sync(0xffffffffu, ic, off);
            if (lane >= off) {
                iu += yu;
                ic += yc;
            }
        }
        if (lane == 31) {
            s_wu[warp] = iu;
            s_wc[warp] = ic;
        }
        __syncthreads();
        int pu = s_carry[0], pc = s_carry[1];
        for (int wp = 0; wp < warp; ++wp) {
            pu += s_wu[wp];
            pc += s_wc[wp];
        }
        if (j < dp.nscales) {
            units[j + 1] = pu + iu;
            chunks[j + 1] = pc + ic;
        }
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) {
            s_carry[0] = pu + iu;
            s_carry[1] = pc + ic;
        }
        __syncthreads();
    }
    {
        __shared__ double s_st[3][32];
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            st_flops += __shfl_down_sync(0xffffffffu, st_flops, off);
            st_bytes += __shfl_down_sync(0xffffffffu, st_bytes, off);
            st_slots += __shfl_down_sync(0xffffffffu, st_slots, off);
        }
        if ((threadIdx.x & 31) == 0) {
            s_st[0][threadIdx.x >> 5] = st_flops;
            s_st[1][threadIdx.x >> 5] = st_bytes;
            s_st[2][threadIdx.x >> 5] = st_slots;
        }
        __syncthreads();
        if (threadIdx.x < 3) {
            double v = 0.0;
            for (int wp = 0; wp < (int)(blockDim.x >> 5); ++wp) v += s_st[threadIdx.x][wp];
            if (v != 0.0) atomicAdd(b.stats + threadIdx.x, v);
        }
    }
}

EMPI_GLOBAL void k_sched_a(BatchDev b, int mode, int only_scale, double tA_in, double sA_in) {
    sched_a_inst(b, blockIdx.x, mode, only_scale, tA_in, sA_in);
}

// Single CTA (any size up to 1024 threads): exclusive scan of per-instance
// unit and chunk totals; resets the work queues and candidate lists.
__device__ __forceinline__ void sched_b_block(const BatchDev& b) {
    __shared__ int s_u[1024], s_c[1024], s_a[1024];
    const int T = blockDim.x, tid = threadIdx.x;
    const int per = (b.ninst + T - 1) / T;
    const int i0 = tid * per, i1 = min(b.ninst, i0 + per);
    int su = 0, sc = 0, sa = 0;
    for (int i = i0; i < i1; ++i) {
        const InstPlan ip = b.insts[i];
        const int ns = b.dicts[ip.dict].nscales;
        su += b.ij_units[ip.ij_off + i + ns];
        sc += b.ij_chunks[ip.ij_off + i + ns];
        sa += b.state[i].status == ST_RUNNING;
    }
    s_u[tid] = su;
    s_c[tid] = sc;
    s_a[tid] = sa;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        int vu = tid >= off ? s_u[tid - off] : 0;
        int vc = tid >= off ? s_c[tid - off] : 0;
        int va = tid >= off ? s_a[tid - off] : 0;
        __syncthreads();
        s_u[tid] += vu;
        s_c[tid] += vc;
        s_a[tid] += va;
        __syncthreads();
    }
    int pu = tid ? s_u[tid - 1] : 0, pc = tid ? s_c[tid - 1] : 0;
    for (int i = i0; i < i1; ++i) {
        const InstPlan ip = b.insts[i];
        const int ns = b.dicts[ip.dict].nscales;
        b.inst_units[i] = pu;
        b.inst_chunks[i] = pc;
        pu += b.ij_units[ip.ij_off + i + ns];
        pc += b.ij_chunks[ip.ij_off + i + ns];
    }
    if (tid == T - 1) {
        b.inst_units[b.ninst] = s_u[T - 1];
        b.inst_chunks[b.ninst] = s_c[T - 1];
        b.ctr[CTR_TOTAL_UNITS] = s_u[T - 1];
        b.ctr[CTR_TOTAL_CHUNKS] = s_c[T - 1];
        b.ctr[CTR_ACTIVE] = s_a[T - 1];
        b.ctr[CTR_STAT_UNITS] += s_u[T - 1];
        b.ctr[CTR_UNITS] = 0;
        b.ctr[CTR_TREE] = 0;
        b.ctr[CTR_CSLOTS] = 0;
        b.ctr[CTR_CSLOT_Q] = 0;
        b.ctr[CTR_CBINS] = 0;
        b.ctr[CTR_RESCORE_Q] = 0;
    }
}

EMPI_GLOBAL void k_sched_b(BatchDev b) { sched_b_block(b); }

// ------------------------------------------------------------ tournament tree

// Leaf chunks: max over kChunk slot keys, re-keyed by slot index.  One warp:
// the leaf chunk holding dirty chunk `rem` of instance inst (its scales' dirty
// chunk ranges in order, prefix sums ij_chunks).
__device__ __forceinline__ void tree_chunk(const BatchDev& b, int inst, int rem, int lane) {
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const int j = upper_index(b.ij_chunks + ip.ij_off + inst, dp.nscales, rem);
    rem -= ld_mut(b.ij_chunks + ip.ij_off + inst + j);
    const int chunk = b.ij_crange[ip.ij_off + j].x + rem;
    if (EMPI_BAD(chunk < 0 || chunk >= dp.chunks, 12)) return;
    const long long s0 = (long long)chunk * kChunk;
    const long long s1 = min(s0 + kChunk, dp.slots);
    const unsigned long long* sl = b.slots + ip.slot_off;
    unsigned long long best = 0;
    unsigned bestl = 0;
    for (long long s = s0 + lane; s < s1; s += 32) {
        const unsigned long long v = sl[s];
        const unsigned long long key = (v & 0xffffffff00000000ull) | (unsigned long long)(s);
        best = key > best ? key : best;
        bestl = max(bestl, (unsigned)(v & 0xffffffffull));
    }
    if (b.chunk_stale) {
        // with a block proposal: does the chunk hold a stale slot (k_qualify's filter)
        int any = 0;
        for (long long s = s0 + lane; s < s1; s += 32) any |= b.stale[ip.slot_off + s];
        any = __any_sync(0xffffffffu, any);
        if (lane == 0) b.chunk_stale[ip.chunk_off + chunk] = (unsigned char)(any != 0);
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        unsigned long long o = __shfl_down_sync(0xffffffffu, best, off);
        best = o > best ? o : best;
    }
    bestl = __reduce_max_sync(0xffffffffu, bestl);
    if (lane == 0) {
        b.chunks[ip.chunk_off + chunk] = best;
        b.chunk_l[ip.chunk_off + chunk] = bestl;
    }
}

// (blocks bid of nb: a fixed chunk per warp and stride, no work-queue atomic
// per chunk)
__device__ __forceinline__ void tree_body(const BatchDev& b, int bid, int nb) {
    const int lane = threadIdx.x & 31;
    const int total = b.ctr[CTR_TOTAL_CHUNKS];
    const int nwarps = (int)((nb * blockDim.x) >> 5);
    for (int item = (int)((bid * blockDim.x + threadIdx.x) >> 5); item < total; item += nwarps) {
        const int inst = upper_index(b.inst_chunks, b.ninst, item);
        tree_chunk(b, inst, item - ld_mut(b.inst_chunks + inst), lane);
    }
}

// The dirty leaf chunks of one instance, by the warps of one CTA (the
// persistent kernel's tree step).
__device__ __forceinline__ void tree_inst(const BatchDev& b, int inst) {
    const InstPlan ip = b.insts[inst];
    const int total = ld_mut(b.ij_chunks + ip.ij_off + inst + b.dicts[ip.dict].nscales);
    for (int item = (int)(threadIdx.x >> 5); item < total; item += (int)(blockDim.x >> 5))
        tree_chunk(b, inst, item, threadIdx.x & 31);
}

EMPI_GLOBAL void k_tree(BatchDev b) { tree_body(b, blockIdx.x, gridDim.x); }

// ------------------------------------------------------------ proposal-ceiling probe
//
// A block proposal may skip refreshing a window only if a bound certifies that
// the window cannot hold the next atom.  Subtracting a * atom changes a
// window's value X_k by at most |a| sum_n g_atom(n) g_window(n) (the atom's
// envelope times the window's Gaussian, whatever the frequency), and
// sqrt(energy) is a norm of X, so sqrt(U) grows by at most
// sqrt(Kc rho) |a| (fs sA s / sqrt(sA^2 + s^2) exp(-pi (t - tA)^2 / (sA^2 + s^2)) + 1)
// (the Gaussian product's integral plus one sample).  k_propagate keeps that
// propagated bound for every window the plain rule refreshes; k_probe, after
// the next iteration's candidate step, counts those whose propagated bound
// still reaches the certified lower bound of the best value: no exact
// proposal scheme can skip them, so their share of the refresh work bounds
// what any proposal can save (for one step; stale bounds only grow).

// per dirty slot of scale j, visited through the dirty leaf chunks like k_tree
template <typename F>
__device__ __forceinline__ void for_dirty_slots(const BatchDev& b, F&& f) {
    const int lane = threadIdx.x & 31;
    const int total = b.ctr[CTR_TOTAL_CHUNKS];
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int item = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); item < total; item += nwarps) {
        const int inst = upper_index(b.inst_chunks, b.ninst, item);
        int rem = item - b.inst_chunks[inst];
        const InstPlan ip = b.insts[inst];
        const DictPlan dp = b.dicts[ip.dict];
        const int j = upper_index(b.ij_chunks + ip.ij_off + inst, dp.nscales, rem);
        rem -= b.ij_chunks[ip.ij_off + inst + j];
        const int chunk = b.ij_crange[ip.ij_off + j].x + rem;
        const ScalePlan sp = b.scales[dp.scale0 + j];
        const int2 dr = b.dirty[ip.ij_off + j];
        const long long s0 = max((long long)chunk * kChunk, sp.slot_base + (long long)dr.x * sp.G);
        const long long s1 = min((long long)(chunk + 1) * kChunk, sp.slot_base + (long long)(dr.y + 1) * sp.G);
        for (long long s = s0 + lane; s < s1; s += 32) f(inst, ip, dp, sp, j, s);
    }
}

EMPI_GLOBAL void k_propagate(BatchDev b) {
    for_dirty_slots(b, [&](int inst, const InstPlan& ip, const DictPlan& dp, const ScalePlan& sp, int, long long s) {
        const InstState& st = b.state[inst];
        if (st.it < 1) return;
        const double* p = b.atoms + ip.out_off + (long long)(st.it - 1) * ip.C * 6;
        double a2 = 0.0;
        for (int c = 0; c < ip.C; ++c) a2 += p[c * 6 + 1] * p[c * 6 + 1];
        const double tA = p[2] / dp.fs, sA = p[3] / dp.fs;
        const int t = (int)((s - sp.slot_base) / sp.G);
        const double dt = grid_t(t, dp.tMax, sp.tcount) - tA;
        const double w2 = sA * sA + sp.s * sp.s;
        const double ov = dp.fs * sA * sp.s / sqrt(w2) * exp(-CUDART_PI * dt * dt / w2) + 1.0;
        const double d = sqrt((double)sp.Kc * (double)fmaxf(1.0f, sp.bnd_rho)) * sqrt(a2) * ov * (1.0 + 1e-6);
        const double u = sqrt((double)__uint_as_float((unsigned)(b.slots[ip.slot_off + s] >> 32))) + d;
        b.prop[ip.slot_off + s] = (float)fmin(u * u, 3.0e38);
    });
}

EMPI_GLOBAL void k_probe(BatchDev b) {
    __shared__ double red[4][32];
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for_dirty_slots(b, [&](int inst, const InstPlan& ip, const DictPlan& dp, const ScalePlan& sp, int, long long s) {
        const InstState& st = b.state[inst];
        if (st.status != ST_RUNNING || st.it < 1) return;
        const double work = 2.5 * sp.nfft * log2((double)sp.nfft) * (ip.chan0 == -1 ? ip.C : 1) / sp.G;
        acc[0] += 1.0;
        acc[2] += work;
        if (b.prop[ip.slot_off + s] >= __uint_as_float(st.tstar)) {
            acc[1] += 1.0;
            acc[3] += work;
        }
    });
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = acc[k];
#pragma unroll
        for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) red[k][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += red[threadIdx.x][w];
        if (v != 0.0) atomicAdd(b.probe + threadIdx.x, v);
    }
}

// ------------------------------------------------------------ block proposal
//
// With a proposal, an iteration's dirty windows (the reference's refresh rule)
// are handled in two rounds.  Round 1 refreshes exactly the dirty windows in
// the proposed blocks (k_topk_ranges -> k_sched_a).  Every other dirty slot
// gets its bounds propagated through the subtraction without recomputing
// (k_propagate_stale, the increment of k_propagate).  Round 2 refreshes the
// dirty windows of every slot whose upper bound still reaches the tree root's
// lower bound (k_root, k_qualify, k_round2_sched).  What stays stale has an
// upper bound below a certified value and cannot be the argmax; later
// candidate steps recompute any stale slot they consider, so the atoms are
// the plain decomposition's.

// Heuristic proposer (a baseline for the learned one): the blocks nearest, in
// (band, tile) steps, to the block of the atom just subtracted.
EMPI_GLOBAL void k_scores_last_atom(BatchDev b) {
    const int inst = blockIdx.x;
    const InstState& st = b.state[inst];
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    int band = 0, tile = 0;
    if (st.it >= 1) {
        const int4 a = b.indices[(long long)inst * b.iter_max + st.it - 1];
        const ScalePlan sp = b.scales[dp.scale0 + a.x];
        band = a.x * kPropBands / dp.nscales;
        tile = (int)((long long)kPropTiles * a.y / sp.tcount);
    }
    for (int i = threadIdx.x; i < kProposalBlocks; i += blockDim.x)
        b.pscores[(long long)inst * kProposalBlocks + i] =
            -(float)(abs(i / kPropTiles - band) + abs(i % kPropTiles - tile));
}

// per instance: the top prop_k blocks of the scores, then per scale the hull of
// the selected tiles of its band as a t-range
EMPI_GLOBAL void k_topk_ranges(BatchDev b) {
    __shared__ float s_sc[kProposalBlocks];
    __shared__ unsigned s_sel[kPropBands];
    __shared__ unsigned long long red[32];
    const int inst = blockIdx.x;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    for (int i = threadIdx.x; i < kProposalBlocks; i += blockDim.x) {
        const float v = b.pscores[(long long)inst * kProposalBlocks + i];
        s_sc[i] = v == v ? v : -3.0e38f;
    }
    if (threadIdx.x < kPropBands) s_sel[threadIdx.x] = 0u;
    __syncthreads();
    for (int r = 0; r < b.prop_k; ++r) {
        // largest score, ties to the lowest block: order-preserving key
        unsigned long long key = 0ull;
        for (int i = threadIdx.x; i < kProposalBlocks; i += blockDim.x) {
            const unsigned u = __float_as_uint(s_sc[i]);
            const unsigned o = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
            const unsigned long long k = ((unsigned long long)o << 32) | (unsigned)(kProposalBlocks - 1 - i);
            key = k > key ? k : key;
        }
        key = block_max_u64(key, red);
        __shared__ int s_pick;
        if (threadIdx.x == 0) {
            s_pick = kProposalBlocks - 1 - (int)(key & 0xffffffffull);
            s_sel[s_pick / kPropTiles] |= 1u << (s_pick % kPropTiles);
            s_sc[s_pick] = -3.4e38f;
        }
        __syncthreads();
    }
    for (int j = threadIdx.x; j < dp.nscales; j += blockDim.x) {
        const ScalePlan sp = b.scales[dp.scale0 + j];
        const unsigned m = s_sel[j * kPropBands / dp.nscales];
        int2 pr = make_int2(0, -1);
        if (m) {
            const long long tc = sp.tcount;
            const int lo = __ffs(m) - 1, hi = 31 - __clz(m);
            // window t lies in tile 32 t / tcount
            pr.x = (int)((lo * tc + kPropTiles - 1) / kPropTiles);
            pr.y = (int)(((hi + 1) * tc + kPropTiles - 1) / kPropTiles) - 1;
        }
        b.prange[ip.ij_off + j] = pr;
    }
}

// The last atom of an instance, for the bound increment of its windows:
// its amplitude over channels |a| = sqrt(sum_c a_c^2), centre and scale in
// seconds; one warp, lanes over channels (any count).
struct LastAtom {
    double a, tA, sA;
};

__device__ __forceinline__ LastAtom last_atom_warp(const BatchDev& b, const InstPlan& ip, const DictPlan& dp,
                                                  const InstState& st, int lane) {
    const double* p = b.atoms + ip.out_off + (long long)(st.it - 1) * ip.C * 6;
    double a2 = 0.0;
    for (int c = lane; c < ip.C; c += 32) a2 += p[c * 6 + 1] * p[c * 6 + 1];
#pragma unroll
    for (int off = 16; off; off >>= 1) a2 += __shfl_xor_sync(0xffffffffu, a2, off);
    return LastAtom{sqrt(a2), p[2] / dp.fs, p[3] / dp.fs};
}

// the bound increment of a window of scale sp at t from the instance's last
// atom: |delta X| <= sqrt(Kc rho) |a| (fs sA s / sqrt(sA^2 + s^2)
// exp(-pi dt^2 / (sA^2 + s^2)) + 1) (Gaussian overlap of atom and window)
__device__ __forceinline__ double atom_increment(const DictPlan& dp, const ScalePlan& sp, const LastAtom& la, int t) {
    const double dt = grid_t(t, dp.tMax, sp.tcount) - la.tA;
    const double w2 = la.sA * la.sA + sp.s * sp.s;
    const double ov = dp.fs * la.sA * sp.s / sqrt(w2) * exp(-CUDART_PI * dt * dt / w2) + 1.0;
    return sqrt((double)sp.Kc * (double)fmaxf(1.0f, sp.bnd_rho)) * la.a * ov * (1.0 + 1e-6);
}

__device__ __forceinline__ bool in_range(int2 r, int t) { return t >= r.x && t <= r.y; }

// Every dirty slot outside the proposed range gets bounds propagated through
// the subtraction and is marked stale (warp per dirty leaf chunk, the atom's
// terms once per warp).
EMPI_GLOBAL void k_propagate_stale(BatchDev b) {
    const int lane = threadIdx.x & 31;
    const int total = b.ctr[CTR_TOTAL_CHUNKS];
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int item = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); item < total; item += nwarps) {
        const int inst = upper_index(b.inst_chunks, b.ninst, item);
        const InstState& st = b.state[inst];
        if (st.it < 1) continue;
        int rem = item - b.inst_chunks[inst];
        const InstPlan ip = b.insts[inst];
        const DictPlan dp = b.dicts[ip.dict];
        const int j = upper_index(b.ij_chunks + ip.ij_off + inst, dp.nscales, rem);
        rem -= b.ij_chunks[ip.ij_off + inst + j];
        const int chunk = b.ij_crange[ip.ij_off + j].x + rem;
        const ScalePlan sp = b.scales[dp.scale0 + j];
        const int2 dr = b.dirty[ip.ij_off + j];
        const int2 pr = b.prange[ip.ij_off + j];
        const LastAtom la = last_atom_warp(b, ip, dp, st, lane);
        const long long s0 = max((long long)chunk * kChunk, sp.slot_base + (long long)dr.x * sp.G);
        const long long s1 = min((long long)(chunk + 1) * kChunk, sp.slot_base + (long long)(dr.y + 1) * sp.G);
        if (s0 >= s1) continue;
        // a lane per window of the chunk: the increment once per window, then
        // the window's residue-group slots that lie in the chunk
        const int t0 = (int)((s0 - sp.slot_base) / sp.G), t1 = (int)((s1 - 1 - sp.slot_base) / sp.G);
        for (int t = t0 + lane; t <= t1; t += 32) {
            if (in_range(pr, t)) continue;  // refreshed in round 1
            const double d = atom_increment(dp, sp, la, t);
            const long long sw = sp.slot_base + (long long)t * sp.G;
            for (int g = 0; g < sp.G; ++g) {
                const long long s = sw + g;
                if (s < s0 || s >= s1) continue;
                const unsigned long long key = b.slots[ip.slot_off + s];
                const double u = sqrt((double)__uint_as_float((unsigned)(key >> 32))) + d;
                const double l = sqrt((double)__uint_as_float((unsigned)(key & 0xffffffffull))) - d;
                const float U = __double2float_ru(fmin(u * u, 3.0e38));
                const float L = l > 0.0 ? __double2float_rd(l * l) : 0.0f;
                b.slots[ip.slot_off + s] = ((unsigned long long)__float_as_uint(U) << 32) | __float_as_uint(L);
                b.stale[ip.slot_off + s] = 1;
            }
        }
    }
}

// per instance: the largest certified lower bound of any slot after round 1
EMPI_GLOBAL void k_root(BatchDev b) {
    __shared__ unsigned long long red[32];
    const int inst = blockIdx.x;
    InstState& st = b.state[inst];
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    unsigned lmax = 0;
    for (int c = threadIdx.x; c < dp.chunks; c += blockDim.x) lmax = max(lmax, b.chunk_l[ip.chunk_off + c]);
    const unsigned long long l = block_max_u64((unsigned long long)lmax, red);
    if (threadIdx.x == 0) st.lround = (unsigned)l;
}

// Every stale slot (propagated bounds, from this iteration's dirty set or left
// from earlier ones) whose upper bound reaches its instance's largest
// certified lower bound: a warp per leaf chunk over all instances' chunks,
// skipping chunks whose maximum is below it.  Qualifying windows widen their
// scale's round-2 range.
EMPI_GLOBAL void k_qualify(BatchDev b, int total_chunks) {
    const int lane = threadIdx.x & 31;
    const int nwarps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int item = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); item < total_chunks; item += nwarps) {
        // the instance owning global chunk `item` (chunk_off is a prefix over instances)
        int lo = 0, hi = b.ninst - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (b.insts[mid].chunk_off <= item) lo = mid;
            else hi = mid - 1;
        }
        const int inst = lo;
        const InstState& st = b.state[inst];
        if (st.status != ST_RUNNING || st.it < 1) continue;
        const InstPlan ip = b.insts[inst];
        const unsigned lb = st.lround;
        const int c = item - (int)ip.chunk_off;
        if (!b.chunk_stale[item] || (unsigned)(b.chunks[item] >> 32) < lb) continue;
        const DictPlan dp = b.dicts[ip.dict];
        const long long s0 = (long long)c * kChunk;
        const long long s1 = min(s0 + kChunk, dp.slots);
        // the chunk's slots, kScanBatch stale flags and keys per lane in
        // flight; the loop runs the same trips in every lane (warp collectives
        // below), slots past the chunk's end do not qualify
        constexpr int kScanBatch = 8;
        // the scale of the chunk's first slot; later slots of the chunk step
        // forward from it (a chunk spans few scales)
        int jc, tfirst, gfirst;
        slot_to_jtg(b, dp, s0, jc, tfirst, gfirst);
        for (long long base = s0; base < s1; base += 32 * kScanBatch) {
            unsigned char sv[kScanBatch];
            unsigned long long kv[kScanBatch];
#pragma unroll
            for (int i = 0; i < kScanBatch; ++i) {
                const long long s = base + lane + 32 * i;
                sv[i] = s < s1 ? b.stale[ip.slot_off + s] : 0;
                kv[i] = s < s1 ? b.slots[ip.slot_off + s] : 0ull;
            }
#pragma unroll
            for (int i = 0; i < kScanBatch; ++i) {
                const long long s = base + lane + 32 * i;
                const bool q = sv[i] && (unsigned)(kv[i] >> 32) >= lb;
                if (!__any_sync(0xffffffffu, q)) continue;
                int j = -1, t = 0;
                if (q) {
                    j = jc;
                    while (j + 1 < dp.nscales && b.scales[dp.scale0 + j + 1].slot_base <= s) ++j;
                    const ScalePlan& sp = b.scales[dp.scale0 + j];
                    const int rel = (int)(s - sp.slot_base);
                    t = rel / sp.G;
                    const int g = rel - t * sp.G;
                    // mark the group's unit block holding t (on the block's first slot)
                    const int B = g >= 2 ? sp.B2 : sp.B1;
                    b.qmark[ip.slot_off + sp.slot_base + (long long)(t / B) * B * sp.G + g] = 1;
                }
                // the scale's t range: one atomic pair per scale present in the
                // warp's qualifying slots, not one per slot
                const unsigned grp = __match_any_sync(0xffffffffu, j);
                if (q) {
                    const int tmin = __reduce_min_sync(grp, t), tmax = __reduce_max_sync(grp, t);
                    if (lane == __ffs(grp) - 1) {
                        atomicMin(&b.qrange[ip.ij_off + j].x, tmin);
                        atomicMax(&b.qrange[ip.ij_off + j].y, tmax);
                    }
                }
            }
        }
    }
}

// refresh_stats for one residue group's slots of windows lo..hi: its share of
// the window's transform work (1 or 2 of the M residues), its slot writes
__device__ __forceinline__ void refresh_stats_group(const DictPlan& dp, const ScalePlan& sp, int C, int g, int lo,
                                                    int hi, double& flops, double& bytes, double& slots) {
    double f = 0.0, by = 0.0, sl = 0.0;
    refresh_stats(dp, sp, C, lo, hi, f, by, sl);
    const int n = hi - lo + 1;
    flops += f * (sp.M == 1 ? 1.0 : (g >= 2 ? 2.0 : 1.0) / sp.M);
    bytes += by - 8.0 * n * (sp.G - 1);
    slots += n;
}

// per instance: round 2's units, exactly the unit blocks (per scale and
// residue group, B windows aligned to B) that hold a qualifying slot; the
// marks are cleared as the units are emitted
EMPI_GLOBAL void k_round2_sched(BatchDev b) {
    const int inst = blockIdx.x;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    double st_flops = 0.0, st_bytes = 0.0, st_slots = 0.0;
    // a warp per scale, its lanes over 32 consecutive unit blocks at a time
    // (the marks of a wide range are read in parallel, and a warp takes its
    // units' list places with one atomic per round)
    for (int j = threadIdx.x >> 5; j < dp.nscales; j += nw) {
        const int2 q = b.qrange[ip.ij_off + j];
        __syncwarp();
        if (lane == 0) b.qrange[ip.ij_off + j] = make_int2(0x7fffffff, -1);
        if (q.y < q.x) continue;
        const ScalePlan sp = b.scales[dp.scale0 + j];
        const int cap = b.lcap[sp.logL];
        int4* list = b.units + b.loff[sp.logL];
        int tmin = 0x7fffffff, tmax = -1;
        for (int g = 0; g < sp.G; ++g) {
            const int B = g >= 2 ? sp.B2 : sp.B1;
            for (int first = (q.x / B) * B; first <= q.y; first += 32 * B) {
                const int t0 = first + lane * B;
                bool emit = false;
                if (t0 <= q.y) {
                    unsigned char* mk = b.qmark + ip.slot_off + sp.slot_base + (long long)t0 * sp.G + g;
                    emit = *mk != 0;
                    if (emit) *mk = 0;
                }
                const unsigned em = __ballot_sync(0xffffffffu, emit);
                if (!em) continue;
                int at = 0;
                if (lane == 0) at = atomicAdd(b.lcount + sp.logL, __popc(em));
                at = __shfl_sync(0xffffffffu, at, 0) + __popc(em & ((1u << lane) - 1u));
                if (emit) {
                    const int n = min(B, sp.tcount - t0);
                    if (at < cap) list[at] = make_int4(inst, j | (g << 16), t0, n);
                    refresh_stats_group(dp, sp, ip.C, g, t0, t0 + n - 1, st_flops, st_bytes, st_slots);
                    tmin = min(tmin, t0);
                    tmax = max(tmax, t0 + n - 1);
                }
            }
        }
        tmin = __reduce_min_sync(0xffffffffu, tmin);
        tmax = __reduce_max_sync(0xffffffffu, tmax);
        if (tmax < tmin || lane != 0) continue;
        // the leaf chunks the tree re-reduces after round 2: the dirty range's
        // and the refreshed blocks' (stale slots of earlier iterations lie
        // outside the dirty range), as one covering range
        int c0 = (int)((sp.slot_base + (long long)tmin * sp.G) / kChunk);
        int c1 = (int)((sp.slot_base + (long long)(tmax + 1) * sp.G - 1) / kChunk);
        const int2 cr = b.ij_crange[ip.ij_off + j];
        if (cr.y > 0) {
            c0 = min(c0, cr.x);
            c1 = max(c1, cr.x + cr.y - 1);
        }
        b.ij_crange[ip.ij_off + j] = make_int2(c0, c1 - c0 + 1);
    }
    // the work statistics: summed over the warp, one set of atomics per warp
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        st_flops += __shfl_down_sync(0xffffffffu, st_flops, off);
        st_bytes += __shfl_down_sync(0xffffffffu, st_bytes, off);
        st_slots += __shfl_down_sync(0xffffffffu, st_slots, off);
    }
    if (lane == 0 && st_flops != 0.0) {
        atomicAdd(b.stats + 0, st_flops);
        atomicAdd(b.stats + 1, st_bytes);
        atomicAdd(b.stats + 2, st_slots);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the instance's chunk prefix over scales (k_tree's index)
        int* chunks = b.ij_chunks + ip.ij_off + inst;
        int acc = 0;
        for (int j = 0; j < dp.nscales; ++j) {
            acc += b.ij_crange[ip.ij_off + j].y;
            chunks[j + 1] = acc;
        }
    }
}

// Single CTA: the chunk prefix over instances after round 2 widened their
// chunk ranges (the chunk part of k_sched_b).
EMPI_GLOBAL void k_chunk_prefix(BatchDev b) {
    __shared__ int s_c[1024];
    const int T = blockDim.x, tid = threadIdx.x;
    const int per = (b.ninst + T - 1) / T;
    const int i0 = tid * per, i1 = min(b.ninst, i0 + per);
    int sc = 0;
    for (int i = i0; i < i1; ++i) {
        const InstPlan ip = b.insts[i];
        sc += b.ij_chunks[ip.ij_off + i + b.dicts[ip.dict].nscales];
    }
    s_c[tid] = sc;
    __syncthreads();
    for (int off = 1; off < T; off <<= 1) {
        const int v = tid >= off ? s_c[tid - off] : 0;
        __syncthreads();
        s_c[tid] += v;
        __syncthreads();
    }
    int pc = tid ? s_c[tid - 1] : 0;
    for (int i = i0; i < i1; ++i) {
        const InstPlan ip = b.insts[i];
        b.inst_chunks[i] = pc;
        pc += b.ij_chunks[ip.ij_off + i + b.dicts[ip.dict].nscales];
    }
    if (tid == T - 1) {
        b.inst_chunks[b.ninst] = s_c[T - 1];
        b.ctr[CTR_TOTAL_CHUNKS] = s_c[T - 1];
    }
}


// ------------------------------------------------------------ candidates


// One CTA per instance: the root of the tournament tree (the slot with the
// largest certified upper bound U) and the largest certified lower bound L of
// any slot (per leaf chunk in chunk_l), a lower bound of the best exact
// energy; every slot whose U reaches it is a candidate (a warp per qualifying
// leaf chunk), and the largest L among the candidates becomes the instance's
// threshold tstar for the bins (k_collect).  No slot
// outside the candidates can hold the exact maximum, whatever the FP32 error.
__device__ __forceinline__ void cand_slots_inst(const BatchDev& b, int inst) {
    __shared__ unsigned long long red[32];
    __shared__ unsigned long long s_root;
    __shared__ unsigned s_tstar;
    InstState& st = b.state[inst];
    if (st.status != ST_RUNNING) return;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    unsigned long long root = 0;
    unsigned lmax = 0;
    for (int c = threadIdx.x; c < dp.chunks; c += blockDim.x) {
        const unsigned long long v = b.chunks[ip.chunk_off + c];
        root = v > root ? v : root;
        lmax = max(lmax, b.chunk_l[ip.chunk_off + c]);
    }
    root = block_max_u64(root, red);  // valid in thread 0
    // the largest certified lower bound of any slot: a lower bound of the best
    const unsigned long long lkey = block_max_u64((unsigned long long)lmax, red);
    if (threadIdx.x == 0) {
        st.best32 = root;
        st.nbins = 0;
        s_root = root;
        s_tstar = (unsigned)lkey;
    }
    __syncthreads();
    if ((unsigned)(s_root >> 32) == 0u) {  // nothing beats 0: src/gabor.cpp:108-110
        if (threadIdx.x == 0) {
            st.status = ST_ERROR;
            st.err = ERR_MAP_EMPTY;
        }
        return;
    }
    const float lroot = __uint_as_float(s_tstar);
    const unsigned tbits = __float_as_uint(lroot * (1.0f - b.band));
    const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5;
    for (int c = threadIdx.x >> 5; c < dp.chunks; c += nwarps) {
        if ((unsigned)(b.chunks[ip.chunk_off + c] >> 32) < tbits) continue;
        const long long s0 = (long long)c * kChunk;
        const long long s1 = min(s0 + kChunk, dp.slots);
        // a lane's kChunk / 32 slots in batches of kScanBatch independent loads:
        // the warp scans a chunk in a few L2 round trips, not one per slot
        constexpr int kScanBatch = 8;
        for (long long sb = s0 + lane; sb < s1; sb += 32 * kScanBatch) {
            unsigned long long v[kScanBatch];
#pragma unroll
            for (int i = 0; i < kScanBatch; ++i) {
                const long long s = sb + 32 * i;
                v[i] = s < s1 ? b.slots[ip.slot_off + s] : 0ull;
            }
#pragma unroll
            for (int i = 0; i < kScanBatch; ++i) {
                if (sb + 32 * i < s1 && (unsigned)(v[i] >> 32) >= tbits) {
                    atomicMax(&s_tstar, (unsigned)(v[i] & 0xffffffffull));
                    const int at = atomicAdd(b.ctr + CTR_CSLOTS, 1);
                    if (at < b.cslot_cap) {
                        CandSlot cs;
                        cs.inst = inst;
                        slot_to_jtg(b, dp, sb + 32 * i, cs.j, cs.t, cs.g);
                        b.cslots[at] = cs;
                    } else {
                        st.err = ERR_CAND_OVERFLOW;
                    }
                }
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) st.tstar = __float_as_uint(__uint_as_float(s_tstar) * (1.0f - b.band));
}

EMPI_GLOBAL void k_cand_slots(BatchDev b) { cand_slots_inst(b, blockIdx.x); }

// FP64 value of one candidate bin and channel by direct DFT over its window
// (GaborWorkspaceMap::compute, src/gabor.cpp:279-299, in FP64).
__device__ __forceinline__ void rescore_body(const BatchDev& b) {
    __shared__ double2 red[32];
    __shared__ int s_item;
    const int nb = min(b.ctr[CTR_CBINS], b.cbin_cap);
    const int total = nb * b.cmax;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(b.ctr + CTR_RESCORE_Q, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= total) break;
        const int bin = item / b.cmax, c = item - bin * b.cmax;
        if (EMPI_BAD(bin >= b.cbin_cap, 5)) continue;
        const CandBin cb = b.cbins[bin];
        if (EMPI_BAD(cb.inst < 0 || cb.inst >= b.ninst, 5)) continue;
        const InstPlan ip = b.insts[cb.inst];
        if (c >= ip.C) continue;
        const DictPlan dp = b.dicts[ip.dict];
        const ScalePlan sp = b.scales[dp.scale0 + cb.j];
        const double fs = dp.fs;
        const double t0 = grid_t(cb.t, dp.tMax, sp.tcount);
        int iL, iR;
        double t0fixed;
        window_bounds(t0, sp.hw, fs, dp.N, iL, iR, t0fixed);
        const int W = iR - iL + 1;
        if (EMPI_BAD(iL < 0 || iR >= dp.N || cb.j < 0 || cb.j >= dp.nscales || cb.t < 0 || cb.t >= sp.tcount, 5))
            continue;
        // gaussize, src/gabor.cpp:31-40
        const double wg = sqrt(CUDART_PI) / sp.s;
        const double ga = wg * (1.0 / fs);
        const double gb = wg * t0fixed;
        const double* x = b.residual + ip.res_off + (long long)c * dp.N + iL;
        const long long nfft = sp.nfft;
        const int T = blockDim.x;
        const int chunk = (W + T - 1) / T;
        const int n0 = threadIdx.x * chunk, n1 = min(W, n0 + chunk);
        double sr = 0.0, si = 0.0;
        if (n0 < n1) {
            double ws, wc, ss, sc;
            sincospi(-2.0 * (double)(((long long)cb.k * n0) & (nfft - 1)) / (double)nfft, &ws, &wc);
            sincospi(-2.0 * (double)cb.k / (double)nfft, &ss, &sc);
            for (int n = n0; n < n1; ++n) {
                const double xw = __dsub_rn(__dmul_rn(ga, (double)n), gb);
                const double v = x[n] * exp(-xw * xw);
                sr += v * wc;
                si += v * ws;
                const double nc = wc * sc - ws * ss;
                ws = wc * ss + ws * sc;
                wc = nc;
            }
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            sr += __shfl_down_sync(0xffffffffu, sr, off);
            si += __shfl_down_sync(0xffffffffu, si, off);
        }
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = make_double2(sr, si);
        __syncthreads();
        if (threadIdx.x == 0) {
            double tr = 0.0, tim = 0.0;
            for (int w = 0; w < (T >> 5); ++w) {
                tr += red[w].x;
                tim += red[w].y;
            }
            // value = (1/fs) X polar(1, f * 2 pi t0fixed), src/gabor.cpp:295-299
            const double norm = 1.0 / fs;
            const double f = (double)cb.k * fs / (double)nfft;
            const double ang = f * (2 * CUDART_PI * t0fixed);
            double sa, ca;
            sincos(ang, &sa, &ca);
            const double xr = norm * tr, xi = norm * tim;
            b.cbin_v[(long long)bin * b.cmax + c] = make_double2(xr * ca - xi * sa, xr * sa + xi * ca);
        }
        __syncthreads();
    }
}

EMPI_GLOBAL void k_rescore(BatchDev b) { rescore_body(b); }

// GaborComputer for one bin in FP64 (src/gabor.cpp:44-71), constraint first
// for MMP1 at low frequency (src/mmp.cpp:9-21).  v is modified in place.
struct Computer64 {
    double normComplex, freqNyquist, f, f4Norm, expFactor, t;
    bool isHighFreq;
};

__device__ __forceinline__ Computer64 make_computer64(const ScalePlan& sp, const DictPlan& dp, int k, int ti) {
    Computer64 q;
    q.normComplex = sqrt(1.41421356237309504880 / sp.s);
    q.freqNyquist = 0.5 * dp.fs;
    q.f = (double)k * dp.fs / (double)sp.nfft;
    q.isHighFreq = q.f > 0.5 * q.freqNyquist;
    q.f4Norm = q.isHighFreq ? (q.freqNyquist - q.f) : q.f;
    q.expFactor = exp(-2 * CUDART_PI * sp.s * sp.s * q.f4Norm * q.f4Norm);
    q.t = grid_t(ti, dp.tMax, sp.tcount);
    return q;
}

// Mmp1Decomposition::constraint (src/mmp.cpp:9-21) in two passes over the
// channel values of one bin (stride 1 in global memory), so any channel count
// works: the common angle from sum v_c^2, then each channel's projection.
__device__ __forceinline__ double mmp1_angle64(const double2* v, int C) {
    double dr = 0.0, di = 0.0;
    for (int c = 0; c < C; ++c) {
        const double2 w = v[c];
        dr += w.x * w.x - w.y * w.y;
        di += 2.0 * w.x * w.y;
    }
    return 0.5 * atan2(di, dr);
}

__device__ __forceinline__ double2 mmp1_project64(double2 w, double angle, double sa, double ca) {
    const double rho = hypot(w.x, w.y) * cos(atan2(w.y, w.x) - angle);
    return make_double2(rho * ca, rho * sa);
}

__device__ __forceinline__ double norm_real(const Computer64& q, double phase) {
    const double p4 = q.isHighFreq ? (2 * CUDART_PI * q.freqNyquist * q.t - phase) : phase;
    return 1.41421356237309504880 * q.normComplex / sqrt(1.0 + cos(2 * p4) * q.expFactor);
}

// One CTA per instance: FP64 energies of its candidate bins, argmax (ties to
// the lowest (scale, t, f)), atom parameters (src/gabor.cpp:111-131).
// (energy, key, bin) of the better candidate: larger energy, ties to the
// lower (scale, t, f) key
__device__ __forceinline__ void better_bin(double& e, unsigned long long& k, int& bin, double oe,
                                           unsigned long long ok, int obin) {
    if (oe > e || (oe == e && ok < k)) {
        e = oe;
        k = ok;
        bin = obin;
    }
}

// (any block size up to 1024 threads)
__device__ __forceinline__ void select_inst(const BatchDev& b, int inst) {
    __shared__ double s_e[32];
    __shared__ unsigned long long s_key[32];
    __shared__ int s_bin[32];
    __shared__ double s_angle;
    InstState& st = b.state[inst];
    if (st.status != ST_RUNNING) return;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const int C = ip.C;
    const int nbins = min(st.nbins, b.inst_bin_cap);
    if (st.err == ERR_CAND_OVERFLOW) {
        // some candidate did not fit: take no step; the host grows the
        // buffers and resumes the instance (k_unstall)
        if (threadIdx.x == 0) {
            st.status = ST_STALLED;
            atomicAdd(b.ctr + CTR_STALLED, 1);
        }
        return;
    }
    if (nbins == 0) {
        if (threadIdx.x == 0) {
            st.status = ST_ERROR;
            st.err = ERR_MAP_EMPTY;
        }
        return;
    }
    double be = -1.0;
    unsigned long long bk = ~0ull;
    int bbin = -1;
    for (int i = threadIdx.x; i < nbins; i += blockDim.x) {
        const int bin = b.inst_bins[(long long)inst * b.inst_bin_cap + i];
        if (EMPI_BAD(bin < 0 || bin >= b.cbin_cap, 6)) continue;
        const CandBin cb = b.cbins[bin];
        const ScalePlan sp = b.scales[dp.scale0 + cb.j];
        const Computer64 q = make_computer64(sp, dp, cb.k, cb.t);
        const double2* v = b.cbin_v + (long long)bin * b.cmax;
        const bool constrain = b.mode == MODE_MMP1 && !q.isHighFreq;
        double angle = 0.0, sa = 0.0, ca = 1.0;
        if (constrain) {
            angle = mmp1_angle64(v, C);
            sincos(angle, &sa, &ca);
        }
        double square = 0.0;
        for (int c = 0; c < C; ++c) {
            const double2 w = constrain ? mmp1_project64(v[c], angle, sa, ca) : v[c];
            const double phase = atan2(w.y, w.x);
            const double nr = norm_real(q, phase);
            const double mod = hypot(w.x, w.y) * nr * sqrt(dp.fs);
            square += mod * mod;
        }
        b.cbins[bin].e64 = square;
        const unsigned long long key =
            ((unsigned long long)cb.j << 48) | ((unsigned long long)cb.t << 20) | (unsigned long long)cb.k;
        if (square > be || (square == be && key < bk)) {
            be = square;
            bk = key;
            bbin = bin;
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1)
        better_bin(be, bk, bbin, __shfl_down_sync(0xffffffffu, be, off), __shfl_down_sync(0xffffffffu, bk, off),
                   __shfl_down_sync(0xffffffffu, bbin, off));
    if ((threadIdx.x & 31) == 0) {
        s_e[threadIdx.x >> 5] = be;
        s_key[threadIdx.x >> 5] = bk;
        s_bin[threadIdx.x >> 5] = bbin;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); ++w) better_bin(be, bk, bbin, s_e[w], s_key[w], s_bin[w]);
        s_bin[0] = bbin;
    }
    __syncthreads();
    const int win = s_bin[0];
    if (EMPI_BAD(win < 0 || win >= b.cbin_cap, 7)) return;
    const CandBin cb = b.cbins[win];
    const ScalePlan sp = b.scales[dp.scale0 + cb.j];
    const Computer64 q = make_computer64(sp, dp, cb.k, cb.t);
    const double2* v = b.cbin_v + (long long)win * b.cmax;
    const bool constrain = b.mode == MODE_MMP1 && !q.isHighFreq;
    if (threadIdx.x == 0) s_angle = constrain ? mmp1_angle64(v, C) : 0.0;
    __syncthreads();
    double sa = 0.0, ca = 1.0;
    if (constrain) sincos(s_angle, &sa, &ca);
    const int it = st.it;
    for (int c = threadIdx.x; c < C; c += blockDim.x) {
        const double2 vc = constrain ? mmp1_project64(v[c], s_angle, sa, ca) : v[c];
        const double phase = atan2(vc.y, vc.x);
        const double nr = norm_real(q, phase);
        const double mag = hypot(vc.x, vc.y);
        double* p = b.atoms + ip.out_off + ((long long)it * C + c) * 6;
        p[0] = mag * nr * sqrt(dp.fs);
        p[1] = mag * nr * nr;
        p[2] = q.t * dp.fs;
        p[3] = sp.s * dp.fs;
        p[4] = q.f * 2.0 / dp.fs;
        p[5] = phase;
    }
    if (threadIdx.x == 0) {
        if (b.prange && it >= 1) {
            // block proposal: did the atom lie in a proposed block?
            atomicAdd(b.ctr + CTR_PROP_ITERS, 1);
            if (in_range(b.prange[ip.ij_off + cb.j], cb.t)) atomicAdd(b.ctr + CTR_PROP_HITS, 1);
        }
        b.indices[(long long)inst * b.iter_max + it] = make_int4(cb.j, cb.t, cb.k, nbins);
        st.it = it + 1;
        if (st.it >= b.iter_max) st.status = ST_DONE;  // src/classes.cpp:57-59
        atomicAdd(b.ctr + CTR_STAT_BINS, nbins);
    }
}

EMPI_GLOBAL void k_select(BatchDev b) { select_inst(b, blockIdx.x); }

// ------------------------------------------------------------ residual

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int off = 16; off; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
        red[32] = t;
    }
    __syncthreads();
    t = red[32];
    __syncthreads();
    return t;
}

// Gabor waveform sample i of an atom window, subtractAtomFromSignal
// (src/gabor.cpp:143-163).
struct AtomWindow {
    double sA, fA, tA, amplitude, omega, phase, ga, gb;
    int iL, iR;
};

__device__ __forceinline__ AtomWindow atom_window(const double* params, double fs, int N, bool fit) {
    AtomWindow a;
    a.sA = params[3] / fs;
    a.fA = params[4] * fs / 2.0;
    a.tA = params[2] / fs;
    a.amplitude = fit ? 1.0 : params[1];
    a.omega = 2.0 * CUDART_PI * a.fA;
    a.phase = params[5];
    const double hw = 3.0 * a.sA;
    long long l = __double2ll_rn(__dmul_rn(__dsub_rn(a.tA, hw), fs));
    long long r = __double2ll_rn(__dmul_rn(__dadd_rn(a.tA, hw), fs));
    a.iL = (int)(l > 0 ? l : 0);
    a.iR = (int)(r < (long long)N - 1 ? r : (long long)N - 1);
    const double wg = sqrt(CUDART_PI) / a.sA;
    a.ga = wg * (1.0 / fs);
    a.gb = wg * __dsub_rn(a.tA, __ddiv_rn((double)a.iL, fs));
    return a;
}

__device__ __forceinline__ double atom_sample(const AtomWindow& a, int i, double fs) {
    const double t = __dsub_rn(__ddiv_rn((double)(i + a.iL), fs), a.tA);
    const double w = a.amplitude * cos(__dadd_rn(__dmul_rn(a.omega, t), a.phase));
    const double xw = __dsub_rn(__dmul_rn(a.ga, (double)i), a.gb);
    return w * exp(-xw * xw);
}

// One CTA per (instance, channel): residual -= atom (fit = false), then the
// channel's energy sum(x^2)/fs (SingleSignal::computeEnergy, inc/base.hpp:39-46).
__device__ __forceinline__ void subtract_ic(const BatchDev& b, int inst, int c) {
    __shared__ double red[33];
    const InstState& st = b.state[inst];
    if (st.status != ST_RUNNING) return;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const double fs = dp.fs;
    double* x = b.residual + ip.res_off + (long long)c * dp.N;
    const double* p = b.atoms + ip.out_off + ((long long)(st.it - 1) * ip.C + c) * 6;
    const AtomWindow a = atom_window(p, fs, dp.N, false);
    const int Nw = a.iR - a.iL + 1;
    float* x32 = b.residual32 + ip.res_off + (long long)c * dp.N;
    for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
        const double v = x[a.iL + i] - atom_sample(a, i, fs);
        x[a.iL + i] = v;
        x32[a.iL + i] = (float)v;
    }
    __syncthreads();
    double s = 0.0;
    float xm = 0.0f;
    for (int i = threadIdx.x; i < dp.N; i += blockDim.x) {
        s += x[i] * x[i];
        xm = fmaxf(xm, fabsf(x32[i]));
    }
    s = block_sum(s, red);
    __shared__ unsigned redm[32];
    xm = block_max_nonneg(xm, redm);
    if (threadIdx.x == 0) {
        b.chan_energy[ip.cen_off + c] = s / fs;
        b.chan_xmax[ip.cen_off + c] = xm;
    }
}

__device__ __forceinline__ void subtract_blk(const BatchDev& b, int blk) {
    const int2 ic = b.blk_ic[blk];
    subtract_ic(b, ic.x, ic.y);
}

EMPI_GLOBAL void k_subtract(BatchDev b) { subtract_blk(b, blockIdx.x); }

// One CTA per (instance, channel): residual from the float32 input
// (src/io.cpp:33 converts to double; MMP2 sums channels, src/mmp.cpp:24-32)
// unless the caller wrote the residual itself, its energy, and the instance
// state.
EMPI_GLOBAL void k_init(BatchDev b, int from_input) {
    __shared__ double red[33];
    const int2 ic = b.blk_ic[blockIdx.x];
    const int inst = ic.x, c = ic.y;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const float* in = b.input + ip.in_off;
    const int Cin = ip.in_channels;
    double* x = b.residual + ip.res_off + (long long)c * dp.N;
    double s = 0.0;
    float xm = 0.0f;
    for (int i = threadIdx.x; i < dp.N; i += blockDim.x) {
        double v;
        if (!from_input) {
            v = x[i];
        } else if (ip.chan0 == -2) {
            v = (double)in[(long long)i * Cin];
            for (int k = 1; k < Cin; ++k) v += (double)in[(long long)i * Cin + k];
        } else if (ip.chan0 >= 0) {
            v = (double)in[(long long)i * Cin + ip.chan0];
        } else {
            v = (double)in[(long long)i * Cin + c];
        }
        if (from_input) x[i] = v;
        b.residual32[ip.res_off + (long long)c * dp.N + i] = (float)v;
        s += v * v;
        xm = fmaxf(xm, fabsf((float)v));
    }
    s = block_sum(s, red);
    __shared__ unsigned redm[32];
    xm = block_max_nonneg(xm, redm);
    if (threadIdx.x == 0) {
        b.chan_energy[ip.cen_off + c] = s / dp.fs;
        b.chan_xmax[ip.cen_off + c] = xm;
        if (c == 0) {
            InstState& st = b.state[inst];
            st.status = ST_RUNNING;
            st.it = 0;
            st.err = ERR_NONE;
            st.nbins = 0;
            st.best32 = 0;
            st.bnorm = 0.0f;
            st.tstar = 0u;
        }
    }
}

// Resumes the instances a candidate overflow stalled, once the host has
// grown the candidate buffers.
EMPI_GLOBAL void k_unstall(BatchDev b) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < b.ninst; i += gridDim.x * blockDim.x) {
        InstState& st = b.state[i];
        if (st.status == ST_STALLED) {
            st.status = ST_RUNNING;
            st.err = ERR_NONE;
            st.nbins = 0;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) b.ctr[CTR_STALLED] = 0;
}

// Workspace::subtractAtomFromSignal on one FP64 signal (src/gabor.cpp:143-187),
// fit or not; a single CTA.  params (6) are updated in place when fitting.
EMPI_GLOBAL void k_subtract_signal(double* x, float* x32, int N, double fs, double* params, int fit) {
    __shared__ double red[33];
    double p[6];
    for (int k = 0; k < 6; ++k) p[k] = params[k];
    const AtomWindow w = atom_window(p, fs, N, fit != 0);
    const int Nw = w.iR - w.iL + 1;
    if (Nw <= 0) return;
    double norm = 1.0, dot = 1.0;
    if (fit) {
        double n2 = 0.0, d = 0.0;
        for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
            const double v = atom_sample(w, i, fs);
            n2 += v * v;
        }
        n2 = block_sum(n2, red);
        norm = sqrt(n2);
        for (int i = threadIdx.x; i < Nw; i += blockDim.x) d += (atom_sample(w, i, fs) / norm) * x[w.iL + i];
        dot = block_sum(d, red);
    }
    for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
        const double v = atom_sample(w, i, fs);
        x[w.iL + i] -= fit ? (v / norm) * dot : v;
        if (x32) x32[w.iL + i] = (float)x[w.iL + i];
    }
    if (fit && threadIdx.x == 0) {
        params[0] = dot;
        params[1] = dot / norm;
    }
}

// MMP2 per-channel fit (src/mmp.cpp:36-43 with subtractAtomFromSignal's fit
// branch, src/gabor.cpp:165-183): one CTA per (epoch, channel), atoms in
// order, each projected on the channel's residual in FP64.
EMPI_GLOBAL void k_mmp2_fit(BatchDev b, const int2* fit_map, double* fit_atoms, int fit_cap) {
    __shared__ double red[33];
    const int2 ec = fit_map[blockIdx.x];  // (instance of the channel sum, input channel)
    const int inst = ec.x, c = ec.y;
    const InstPlan ip = b.insts[inst];
    const DictPlan dp = b.dicts[ip.dict];
    const InstState& st = b.state[inst];
    const double fs = dp.fs;
    const float* in = b.input + ip.in_off;
    const int Cin = ip.in_channels;
    extern __shared__ double xs[];
    for (int i = threadIdx.x; i < dp.N; i += blockDim.x) xs[i] = (double)in[(long long)i * Cin + c];
    __syncthreads();
    const int n = min(st.it, fit_cap);
    for (int a = 0; a < n; ++a) {
        const double* p0 = b.atoms + ip.out_off + (long long)a * 6;
        double* po = fit_atoms + ((long long)blockIdx.x * fit_cap + a) * 6;
        double p[6];
        for (int k = 0; k < 6; ++k) p[k] = p0[k];
        const AtomWindow w = atom_window(p, fs, dp.N, true);
        const int Nw = w.iR - w.iL + 1;
        double n2 = 0.0, dot = 0.0;
        for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
            const double v = atom_sample(w, i, fs);
            n2 += v * v;
        }
        n2 = block_sum(n2, red);
        const double norm = sqrt(n2);
        for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
            const double v = atom_sample(w, i, fs) / norm;
            dot += v * xs[w.iL + i];
        }
        dot = block_sum(dot, red);
        for (int i = threadIdx.x; i < Nw; i += blockDim.x) {
            const double v = atom_sample(w, i, fs) / norm;
            xs[w.iL + i] -= v * dot;
        }
        if (threadIdx.x == 0) {
            po[0] = dot;
            po[1] = dot / norm;
            for (int k = 2; k < 6; ++k) po[k] = p[k];
        }
        __syncthreads();
    }
}

}  // namespace empi
