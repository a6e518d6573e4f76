// Engine and static subtraction of the empi adapter (gpu_workspace.hpp).
// empi's src/classes.cpp:15-22 dispatches Workspace::subtractAtomFromSignal
// to GaborWorkspace::subtractAtomFromSignal; with this file linked in place
// of src/gabor.cpp that call runs on the GPU too (MMP2's per-channel fit,
// src/mmp.cpp:36-43).
#include "gpu_workspace.hpp"

#include <cstdlib>
#include <memory>
#include <mutex>

#include "gabor.hpp"

namespace empi_gpu {

empi_engine* engine() {
    static std::once_flag once;
    static empi_engine* eng = nullptr;
    std::call_once(once, [] {
        empi_engine_opts o;
        empi_engine_opts_default(&o);
        if (const char* d = std::getenv("EMPI_DEVICE")) o.device = std::atoi(d);
        check(empi_engine_create(&o, &eng));
    });
    return eng;
}

void subtract_atom_from_signal(Atom& atom, SingleSignal& signal, bool fit) {
    check(empi_subtract_atom_from_signal(engine(), atom.params.data(), signal.samples.data(),
                                         (int)signal.samples.size(), signal.freqSampling, fit ? 1 : 0));
}

}  // namespace empi_gpu

void GaborWorkspace::subtractAtomFromSignal(Atom& atom, SingleSignal& signal, bool fit) {
    empi_gpu::subtract_atom_from_signal(atom, signal, fit);
}
