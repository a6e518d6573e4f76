// Persistent kernel of the MP loop for small batches.
//
// With few, short instances an MP iteration is a dozen dependent launches of
// a few microseconds' work each: the multi-kernel CUDA graph is then bound by
// launch and drain latency, not by the work.  Here one cooperative launch runs
// a chunk of iterations; the kernels of kernels.cuh and refresh.cuh become
// phases of one grid (one 512-thread CTA per SM, all co-resident: the launch
// is cooperative), separated by a grid barrier:
//
//   candidates (tree root, candidate slots)   per instance
//   collect (FP32 recompute of the slots)     work queue
//   rescore (FP64 direct DFT)                 work queue
//   select (FP64 energy, argmax, atom)        per instance
//   subtract (FP64)                           per (instance, channel)
//   schedule: dirty ranges, units             per instance, then one CTA
//   refresh of every sub-FFT size             work queues, largest first
//   tree                                      warp per dirty leaf chunk
//
// Every barrier wait is bounded in time (BatchDev::wait_ns): a CTA whose wait
// runs out records the phase in GridSync::err and returns, and every other CTA
// returns at its next barrier, so the kernel always ends and the host reports
// deviceWaitTimeout.  The steps and their order are the graph's, so the atoms
// are the same.
#pragma once

#include "kernels.cuh"
#include "refresh.cuh"

namespace empi {

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// All CTAs of the grid (plus wait_extra that never come) arrive; true in every
// thread of the CTA when all did, false when this CTA's wait ran out or
// another CTA's had.  Writes before the barrier are visible after it.
__device__ __forceinline__ bool grid_barrier(const BatchDev& b, int phase) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        GridSync* g = b.gsync;
        volatile GridSync* vg = g;
        int ok = 1;
        const unsigned gen = vg->gen;  // read before arriving: it moves only once all have
        if (vg->err) {
            ok = 0;
        } else {
            __threadfence();
            const unsigned target = gridDim.x + (unsigned)b.wait_extra;
            if (atomicAdd(&g->count, 1u) + 1u == target) {
                atomicExch(&g->count, 0u);
                __threadfence();
                atomicAdd(&g->gen, 1u);
            } else {
                const unsigned long long t0 = global_ns();
                // a backstop on the iteration count too (each takes well over 8 ns)
                const unsigned long long max_spins = (unsigned long long)b.wait_ns / 8ull + 1024ull;
                for (unsigned long long spins = 0; vg->gen == gen; ++spins) {
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
                    __nanosleep(32);
                }
            }
            __threadfence();
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// `iterations` MP iterations of every instance of the batch (a chunk; the
// host loop around it is the graph path's).
template <int MODE>
__global__ void __launch_bounds__(kUnitThreads, 1) k_persist(BatchDev b, int iterations) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_unit;
    const int bid = blockIdx.x, nb = gridDim.x;
    for (int k = 0; k < iterations; ++k) {
        for (int i = bid; i < b.ninst; i += nb) {
            cand_slots_inst(b, i);
            __syncthreads();
        }
        if (!grid_barrier(b, 1)) return;
        collect_queue<MODE>(b, smem, &s_unit);
        if (!grid_barrier(b, 2)) return;
        rescore_body(b);
        if (!grid_barrier(b, 3)) return;
        for (int i = bid; i < b.ninst; i += nb) {
            select_inst(b, i);
            __syncthreads();
        }
        // the refresh lists' counts and heads (lcount, lhead: 2 x 16 ints)
        // for the schedule two phases on; the last refresh ended long before
        if (bid == 0 && threadIdx.x < 32) b.lcount[threadIdx.x] = 0;
        if (!grid_barrier(b, 4)) return;
        for (int i = bid; i < b.nblk_ic; i += nb) {
            subtract_blk(b, i);
            __syncthreads();
        }
        if (!grid_barrier(b, 5)) return;
        for (int i = bid; i < b.ninst; i += nb) {
            sched_a_inst(b, i, SCHED_ITERATE, -1, 0.0, 0.0);
            __syncthreads();
        }
        if (!grid_barrier(b, 6)) return;
        if (bid == 0) sched_b_block(b);
        if (!grid_barrier(b, 7)) return;
        // every instance stopped or stalled: the rest of the chunk would do
        // nothing (the same value in every CTA, read after the barrier)
        if (b.ctr[CTR_ACTIVE] == 0) return;
        refresh_all_sizes<MODE>(b, smem, &s_unit);
        if (!grid_barrier(b, 8)) return;
        tree_body(b, bid, nb);
        if (!grid_barrier(b, 9)) return;
    }
}

}  // namespace empi
