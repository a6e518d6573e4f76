// Tuned launch shapes read from the autotuner's cache file (tune.cpp).
#pragma once

#include <string>

namespace empi {

struct TuneKey {
    int mode;        // 0 single-channel MP loops (SMP, MMP2's channel sum), 1 MMP1, 3 MMP3
    int channels;    // channels per MP loop
    double fs;
    int samples;
    double energy_error;
};

struct TuneParams {
    int transform_cap = 0;         // 0: keep the engine's
    int iterations_per_graph = 0;  // 0: keep the engine's
    int wide_mask = 0;             // bit lg: one 128-register CTA per SM for sub-FFT size 2^lg
    int persistent = -1;           // 1 / 0: the persistent kernel on / off; -1: the engine's choice
};

// Looks `key` up in the cache file; false with a camelCase reason in err when
// the file is unreadable or malformed ("invalidTuneCache") or holds no entry
// for the key ("noTunedEntry").
bool tune_lookup(const char* path, const TuneKey& key, TuneParams& out, std::string& err);

}  // namespace empi
