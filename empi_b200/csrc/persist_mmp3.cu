// Persistent MP-loop kernel of the MMP3 mode (persist.cuh), in a
// translation unit of its own so the modes compile in parallel.
#define EMPI_PHASES_ONLY
#include "persist.cuh"
#include "refresh_kernels.hpp"

namespace empi {

void persist_kernel_mmp3(RefreshKernels& rk) {
    rk.persist = (void*)k_persist<MODE_MMP3>;
    rk.persist_smem = rk.collect_smem;
}

}  // namespace empi
