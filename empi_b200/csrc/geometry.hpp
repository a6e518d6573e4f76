#pragma once

#include <string>
#include <vector>

#include "plan.hpp"

namespace empi {

// Appends the scales of one dictionary (fs, N, energyError, scale/frequency
// limits) to `scales`, their expFactor tables to `etab` and (when given) the
// per-window geometry to `wgeom` / `whf` (fs * t0 modulo 1), and fills `dict`.
// Returns false with a camelCase message in `err` on invalid input.
bool build_dictionary(double fs, int N, double energyError, double scaleMin, double scaleMax,
                      double freqMax, int lcap, DictPlan& dict, std::vector<ScalePlan>& scales,
                      std::vector<float>& etab, std::vector<WinGeom>* wgeom, std::vector<float>* whf,
                      std::string& err);

}  // namespace empi
