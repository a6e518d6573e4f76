// Adapter from empi's Workspace seam (empi's inc/classes.hpp:63-80) to the
// empi_b200 C ABI: the class a maintainer adds to empi so that its own
// Decomposition / Smp / Mmp1 / Mmp2 / Mmp3 loops (src/classes.cpp:26-87,
// src/mmp.cpp:23-45) run on the B200 engine unchanged.  Compile it with
// empi's inc/ and this repository's include/ on the include path and link
// empi_b200/libempi_b200.so; gpu_workspace.cpp routes the static
// Workspace::subtractAtomFromSignal (which src/classes.cpp:15-22 dispatches to
// GaborWorkspace) to the GPU as well.
#pragma once

#include <cstdint>
#include <vector>

#include "classes.hpp"
#include "empi_b200.h"

namespace empi_gpu {

// empi's errors are Exception(camelCaseMessage); the C ABI's messages use the
// same texts (signalIsEmpty, energyMapIsEmpty, ...)
inline void check(empi_status st) {
    if (st != EMPI_OK) throw Exception(empi_last_error());
}

// The process's engine: created on first use on device EMPI_DEVICE (default 0).
empi_engine* engine();

// Workspace::subtractAtomFromSignal(atom, signal, fit) on the GPU
// (GaborWorkspace::subtractAtomFromSignal, src/gabor.cpp:143-187).
void subtract_atom_from_signal(Atom& atom, SingleSignal& signal, bool fit);

class GpuWorkspace : public Workspace {
    empi_workspace* ws_ = nullptr;
    int C_, N_;

public:
    GpuWorkspace(const empi_dictionary& d, double fs, int channels, int samples, bool mmp1)
        : C_(channels), N_(samples) {
        check(empi_workspace_create(engine(), &d, fs, channels, samples, mmp1 ? EMPI_MMP1 : EMPI_MMP3, &ws_));
    }
    ~GpuWorkspace() override { empi_workspace_destroy(ws_); }
    GpuWorkspace(const GpuWorkspace&) = delete;
    GpuWorkspace& operator=(const GpuWorkspace&) = delete;

    // Workspace::compute (src/gabor.cpp:75-83): all maps of a signal
    void compute(const MultiSignal& signal) override {
        std::vector<double> x;
        x.reserve((size_t)C_ * N_);
        for (const SingleSignal& ch : signal.channels) x.insert(x.end(), ch.samples.begin(), ch.samples.end());
        check(empi_workspace_compute(ws_, x.data()));
    }

    // Workspace::findBestMatch (src/gabor.cpp:85-133): one atom per channel
    Atoms findBestMatch() const override {
        std::vector<double> p((size_t)6 * C_);
        check(empi_workspace_find_best(ws_, p.data(), nullptr));
        Atoms atoms((size_t)C_);
        for (int c = 0; c < C_; ++c) {
            atoms[c].type = ATOM_GABOR;
            atoms[c].params.assign(p.begin() + 6 * c, p.begin() + 6 * (c + 1));
        }
        return atoms;
    }

    // Workspace::getAtomCount (src/gabor.cpp:135-141)
    size_t getAtomCount() const override {
        uint64_t n = 0;
        check(empi_workspace_atom_count(ws_, &n));
        return (size_t)n;
    }

    // Workspace::subtractAtom (src/gabor.cpp:189-209): the atom off one
    // channel, then the refresh of the maps it touches
    void subtractAtom(const Atom& atom, SingleSignal& signal, int channel) override {
        check(empi_workspace_subtract_atom(ws_, atom.params.data(), signal.samples.data(), channel));
    }
};

// WorkspaceBuilder (GaborWorkspaceBuilder, src/gabor.cpp:213-252): only MMP1
// passes a constraint (src/mmp.cpp:9-21), which selects the constrained maps.
class GpuWorkspaceBuilder : public WorkspaceBuilder {
    empi_dictionary d_;

public:
    GpuWorkspaceBuilder(double energyError, double scaleMin, double scaleMax, double freqMax)
        : d_{energyError, scaleMin, scaleMax, freqMax} {}
    Workspace* prepareWorkspace(double freqSampling, int channelCount, int sampleCount,
                                MultichannelConstraint constraint) const override {
        return new GpuWorkspace(d_, freqSampling, channelCount, sampleCount, constraint != nullptr);
    }
};

}  // namespace empi_gpu
