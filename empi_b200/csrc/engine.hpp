// Internal helpers shared by the engine and the host surface.
#pragma once

#include <functional>
#include <string>

#include "../../include/empi_b200.h"

namespace empi {

empi_status fail(empi_status st, const std::string& msg);
empi_status ok();
empi_status batch_load_device(empi_batch* b, const float* const* device_data);

// empi_batch_run with a hook called after every CUDA-graph chunk (K MP
// iterations of every instance), with the engine's stream idle.
empi_status batch_run_hooked(empi_batch* b, const std::function<void()>& after_chunk);

// Progress of one MP loop of an epoch (loop = channel for SMP, 0 otherwise):
// atoms found so far, whether it is still running, its total energy and the
// residual energy after each of its first `it` iterations (energies holds
// the iteration cap).
empi_status batch_loop_progress(empi_batch* b, int epoch, int loop, int* it, int* running, double* etotal,
                                double* energies);

// Copies the next batch's epochs (same shapes) to the batch's spare input
// buffer on a separate copy stream, so the copy overlaps a run in progress;
// the next run waits for it and decomposes those epochs.
empi_status batch_stage(empi_batch* b, const empi_epoch* epochs);

}  // namespace empi
