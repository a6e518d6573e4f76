// Host view of the refresh kernels: each variant mode's kernels are compiled
// in their own translation units (refresh_single.cu, refresh_mmp1.cu,
// refresh_mmp3.cu, and persist_*.cu for the persistent kernel) and handed to
// the engine through this table.
#pragma once

#include <cstddef>

namespace empi {

constexpr int kRefreshSizes = 13;  // sub-FFT sizes 2^0 .. 2^12

struct RefreshKernels {
    void* refresh[kRefreshSizes][2];  // [log2 L][0: two CTAs per SM, 1: one 128-register CTA per SM]
    size_t smem[kRefreshSizes];       // dynamic shared memory per size
    void* collect;                    // candidate recompute (any size)
    size_t collect_smem;
    void* persist;                    // persistent MP loop for small batches (persist.cuh), or null
    size_t persist_smem;              // its dynamic shared memory (the largest refresh layout)
};

void refresh_kernels_single(RefreshKernels& rk);  // SMP and MMP2's channel sum
void refresh_kernels_mmp1(RefreshKernels& rk);
void refresh_kernels_mmp3(RefreshKernels& rk);
// the persistent kernel of each mode, compiled in persist_*.cu
void persist_kernel_single(RefreshKernels& rk);
void persist_kernel_mmp1(RefreshKernels& rk);
void persist_kernel_mmp3(RefreshKernels& rk);

}  // namespace empi
