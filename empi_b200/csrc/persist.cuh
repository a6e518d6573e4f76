// Persistent kernel of the MP loop for small batches.
//
// With few, short instances an MP iteration is a dozen dependent launches of
// a few microseconds' work each: the multi-kernel CUDA graph is then bound by
// launch and drain latency, not by the work.  Here one cooperative launch runs
// a chunk of iterations (one 512-thread CTA per SM, all co-resident: the
// launch is cooperative); the kernels of kernels.cuh and refresh.cuh become
// phases separated by grid barriers, and the steps that touch one instance
// only run back to back in the CTA that owns it (k_persist below).
//
// Every barrier wait is bounded in time (BatchDev::wait_ns): a CTA whose wait
// runs out records the phase in GridSync::err and returns, and every other CTA
// returns at its next barrier, so the kernel always ends and the host reports
// deviceWaitTimeout.  Each instance goes through the graph's steps in the
// graph's order, so the atoms are the same.
#pragma once

#include "kernels.cuh"
#include "refresh.cuh"

namespace empi {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned atom_add_acq_rel_gpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void st_release_gpu(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// All CTAs of the grid (plus wait_extra that never come) arrive; true in every
// thread of the CTA when all did, false when this CTA's wait ran out or
// another CTA's had.  Writes before the barrier are visible after it: the
// CTA's threads meet thread 0 at __syncthreads, thread 0 arrives with a
// release and leaves with an acquire of the generation word (2.0 us per
// barrier over 148 CTAs on a B200, against 2.8 us with full fences).
__device__ __forceinline__ bool grid_barrier(const BatchDev& b, int phase) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        GridSync* g = b.gsync;
        volatile GridSync* vg = g;
        int ok = 1;
        const unsigned gen = ld_acquire_gpu(&g->gen);  // read before arriving: it moves only once all have
        if (vg->err) {
            ok = 0;
        } else {
            const unsigned target = gridDim.x + (unsigned)b.wait_extra;
            if (atom_add_acq_rel_gpu(&g->count, 1u) + 1u == target) {
                g->count = 0u;  // ordered before the release below
                st_release_gpu(&g->gen, gen + 1u);
            } else {
                const unsigned long long t0 = global_ns();
                // a backstop on the iteration count too (each takes well over 8 ns)
                const unsigned long long max_spins = (unsigned long long)b.wait_ns / 8ull + 1024ull;
                for (unsigned long long spins = 0; ld_acquire_gpu(&g->gen) == gen; ++spins) {
                    if (vg->err) {
                        ok = 0;
                        break;
                    }
                    if (((spins & 31ull) == 0ull && global_ns() - t0 > (unsigned long long)b.wait_ns) ||
                        spins > max_spins) {
                        atomicCAS(&g->err, 0, 1 + phase);
                        ok = 0;
                        break;
                    }
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Every sub-FFT size's refresh units from one queue (head CTR_UNITS), the
// largest transforms first: unit u of the concatenated lists, found by the
// per-size counts the schedule left in lcount.
template <int MODE>
__device__ __forceinline__ void refresh_combined(const BatchDev& b, unsigned char* smem) {
    __shared__ int s_cnt[kRefreshSizes];
    __shared__ int s_unit;
    if (threadIdx.x < kRefreshSizes) s_cnt[threadIdx.x] = min(b.lcount[threadIdx.x], b.lcap[threadIdx.x]);
    __syncthreads();
    for (;;) {
        if (threadIdx.x == 0) s_unit = atomicAdd(b.ctr + CTR_UNITS, 1);
        __syncthreads();
        int u = s_unit;
        __syncthreads();
        int lg = kRefreshSizes - 1;
        for (; lg >= 0 && u >= s_cnt[lg]; --lg) u -= s_cnt[lg];
        if (lg < 0) break;
        const int4 un = ld_mut(b.units + b.loff[lg] + u);  // (instance, scale | group << 16, t_start, nwin)
        const int inst = un.x, j = un.y & 0xffff, g = un.y >> 16;
        switch (lg) {
#define EMPI_PERSIST_UNIT(LG) \
    case LG: unit_body<LG, MODE, false>(b, smem, inst, j, g, un.z, un.w, 0.0f); break;
            EMPI_PERSIST_UNIT(0)
            EMPI_PERSIST_UNIT(1)
            EMPI_PERSIST_UNIT(2)
            EMPI_PERSIST_UNIT(3)
            EMPI_PERSIST_UNIT(4)
            EMPI_PERSIST_UNIT(5)
            EMPI_PERSIST_UNIT(6)
            EMPI_PERSIST_UNIT(7)
            EMPI_PERSIST_UNIT(8)
            EMPI_PERSIST_UNIT(9)
            EMPI_PERSIST_UNIT(10)
            EMPI_PERSIST_UNIT(11)
            EMPI_PERSIST_UNIT(12)
#undef EMPI_PERSIST_UNIT
            default: break;
        }
    }
}

// `iterations` MP iterations of every instance of the batch (a chunk; the
// host loop around it is the graph path's).  Five phases per iteration, each
// ended by a grid barrier; the steps that need only one instance's state run
// back to back in the CTA that owns the instance:
//
//   A  per instance: tree over its dirty chunks (the last refresh's), then
//      the root and candidate slots (k_tree + k_cand_slots)
//   B  candidate recompute, work queue (k_collect)
//   C  FP64 re-scoring, work queue (k_rescore)
//   D  per instance: select, subtract every channel, schedule its next
//      refresh (k_select + k_subtract + k_sched_a); count the running ones
//   E  refresh of every size from one queue (the refresh fork)
//
// Counters are reset by CTA 0 in a phase where nothing reads or writes them:
// the refresh lists (lcount, lhead), the refresh queue's head and the running
// count of this iteration's parity in B, the candidate and queue counters in E.
template <int MODE>
__global__ void __launch_bounds__(kUnitThreads, 1) k_persist(BatchDev b, int iterations) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    const int bid = blockIdx.x, nb = gridDim.x;
    for (int k = 0; k < iterations; ++k) {
        int* active = b.ctr + CTR_PACTIVE + (k & 1);
        for (int i = bid; i < b.ninst; i += nb) {
            tree_inst(b, i);
            __syncthreads();
            cand_slots_inst(b, i);
            __syncthreads();
        }
        if (!grid_barrier(b, 1)) return;
        if (bid == 0 && threadIdx.x < 32) b.lcount[threadIdx.x] = 0;  // lcount and lhead (2 x 16 ints)
        if (bid == 0 && threadIdx.x == 0) {
            *active = 0;
            b.ctr[CTR_UNITS] = 0;  // the refresh queue's head (phase E)
        }
        collect_queue<MODE>(b, smem, &s_unit);
        if (!grid_barrier(b, 2)) return;
        rescore_body(b);
        if (!grid_barrier(b, 3)) return;
        for (int i = bid; i < b.ninst; i += nb) {
            select_inst(b, i);
            __syncthreads();
            const int C = b.insts[i].C;
            for (int c = 0; c < C; ++c) {
                subtract_ic(b, i, c);
                __syncthreads();
            }
            sched_a_inst(b, i, SCHED_ITERATE, -1, 0.0, 0.0);
            __syncthreads();
            if (threadIdx.x == 0) {
                const InstPlan ip = b.insts[i];
                atomicAdd(b.ctr + CTR_STAT_UNITS, ld_mut(b.ij_units + ip.ij_off + i + b.dicts[ip.dict].nscales));
                if (b.state[i].status == ST_RUNNING) atomicAdd(active, 1);
            }
        }
        if (!grid_barrier(b, 4)) return;
        // the candidate counters for the next phase A (before any return: a
        // chunk that ends here is followed by one that starts with phase A)
        if (bid == 0 && threadIdx.x == 0) {
            b.ctr[CTR_CSLOTS] = 0;
            b.ctr[CTR_CSLOT_Q] = 0;
            b.ctr[CTR_CBINS] = 0;
            b.ctr[CTR_RESCORE_Q] = 0;
        }
        // every instance stopped or stalled: the rest of the chunk would do
        // nothing (the same value in every CTA, read after the barrier)
        const int running = ld_mut(active);
        if (bid == 0 && threadIdx.x == 0) b.ctr[CTR_ACTIVE] = running;
        if (running == 0) return;
        refresh_combined<MODE>(b, smem);
        if (!grid_barrier(b, 5)) return;
    }
}

}  // namespace empi
