// Refresh and collect kernels of the mmp3 variant mode (refresh.cuh), in a
// translation unit of their own so the three modes compile in parallel.
#include "refresh.cuh"
#include "refresh_kernels.hpp"

namespace empi {

void refresh_kernels_mmp3(RefreshKernels& rk) { fill_refresh_kernels<MODE_MMP3>(rk); }

}  // namespace empi
