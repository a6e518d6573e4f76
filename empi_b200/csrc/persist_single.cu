// Persistent MP-loop kernel of the SMP and MMP2's channel sum mode (persist.cuh), in a
// translation unit of its own so the modes compile in parallel.
#define EMPI_PHASES_ONLY
#include "persist.cuh"
#include "refresh_kernels.hpp"

namespace empi {

void persist_kernel_single(RefreshKernels& rk) {
    rk.persist = (void*)k_persist<MODE_SINGLE>;
    rk.persist_smem = rk.collect_smem;
}

}  // namespace empi
