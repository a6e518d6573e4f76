/*
 * Test infrastructure (oracle), not product code.
 *
 * The reference's own decomposition loops (empi's src/classes.cpp and
 * src/mmp.cpp, compiled unmodified) running on the GPU workspace through the
 * adapter a maintainer would add (empi_b200/adapter/gpu_workspace.hpp): the
 * proof that the C ABI is a drop-in for empi's Workspace seam
 * (inc/classes.hpp:63-80).  Variant selection and the channel count of the
 * workspace follow src/empi.cpp:114-130.
 *
 *   seam <smp|mmp1|mmp2|mmp3> <fs> <channels> <samples> <energyError>
 *        <iterations> <energyPercent> <scaleMin> <scaleMax> <freqMax> <in> <out>
 *
 * in: channels x samples doubles, channel-major.  out: per channel, the atom
 * count (one double) then count x 6 params.  0 for a limit means none.
 */
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "classes.hpp"
#include "gpu_workspace.hpp"
#include "mmp.hpp"

int main(int argc, char** argv) {
    if (argc != 13) {
        fprintf(stderr, "usage: seam variant fs channels samples energyError iterations energyPercent "
                        "scaleMin scaleMax freqMax in out\n");
        return 2;
    }
    const std::string variant = argv[1];
    const double fs = atof(argv[2]);
    const int C = atoi(argv[3]), N = atoi(argv[4]);
    const double eps = atof(argv[5]);
    const int iters = atoi(argv[6]);
    const double pct = atof(argv[7]);
    double smin = atof(argv[8]), smax = atof(argv[9]), fmax = atof(argv[10]);
    if (!(smax > 0)) smax = INFINITY;
    if (!(fmax > 0)) fmax = INFINITY;
    std::vector<double> x((size_t)C * N);
    FILE* f = fopen(argv[11], "rb");
    if (!f || fread(x.data(), sizeof(double), x.size(), f) != x.size()) {
        fprintf(stderr, "cannot read %s\n", argv[11]);
        return 2;
    }
    fclose(f);
    MultiSignal signal;
    signal.channels.resize(C);
    for (int c = 0; c < C; ++c) {
        signal.channels[c].freqSampling = fs;
        signal.channels[c].samples.assign(x.begin() + (size_t)c * N, x.begin() + (size_t)(c + 1) * N);
    }
    std::unique_ptr<Decomposition> dec;
    int workspaceChannels = C;
    if (C == 1 || variant == "smp") {
        dec.reset(new SmpDecomposition);
        workspaceChannels = 1;
    } else if (variant == "mmp1") {
        dec.reset(new Mmp1Decomposition);
    } else if (variant == "mmp2") {
        dec.reset(new Mmp2Decomposition);
        workspaceChannels = 1;
    } else {
        dec.reset(new Mmp3Decomposition);
    }
    try {
        empi_gpu::GpuWorkspaceBuilder builder(eps, smin, smax, fmax);
        std::unique_ptr<Workspace> ws(builder.prepareWorkspace(fs, workspaceChannels, N, dec->constraint));
        DecompositionSettings settings{iters, 1.0 - 0.01 * pct};
        MultiChannelResult res = dec->compute(settings, ws.get(), signal);
        FILE* o = fopen(argv[12], "wb");
        for (const Atoms& ch : res) {
            const double n = (double)ch.size();
            fwrite(&n, sizeof(double), 1, o);
            for (const Atom& a : ch) fwrite(a.params.data(), sizeof(double), 6, o);
        }
        fclose(o);
    } catch (const std::exception& e) {
        fprintf(stderr, "ERROR\t%s\n", e.what());
        return 1;
    }
    return 0;
}
