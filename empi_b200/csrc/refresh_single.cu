// Refresh and collect kernels of the single variant mode (refresh.cuh), in a
// translation unit of their own so the three modes compile in parallel.
#include "refresh.cuh"
#include "refresh_kernels.hpp"

namespace empi {

void refresh_kernels_single(RefreshKernels& rk) { fill_refresh_kernels<MODE_SINGLE>(rk); }

}  // namespace empi
