// Internal helpers shared by the engine and the host surface.
#pragma once

#include <string>

#include "../../include/empi_b200.h"

namespace empi {

empi_status fail(empi_status st, const std::string& msg);
empi_status ok();
empi_status batch_load_device(empi_batch* b, const float* const* device_data);

}  // namespace empi
