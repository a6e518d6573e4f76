/*
 * Test infrastructure (oracle), not product code.
 *
 * extern "C" access to the reference's OWN workspace and decomposition classes
 * (compiled unmodified from the reference's src/gabor.cpp, src/classes.cpp,
 * src/mmp.cpp together with fftw_shim.c), used to pin the C restatement
 * (mp_oracle.c) and to generate the golden vectors under tests/golden/.
 *
 *   empiref_geometry   GaborWorkspaceBuilder::prepareWorkspace   src/gabor.cpp:213-252
 *   empiref_map        GaborWorkspaceMap::compute + GaborComputer src/gabor.cpp:44-71,270-303
 *   empiref_decompose  Decomposition / Smp / Mmp1 / Mmp2 / Mmp3   src/classes.cpp:26-87, src/mmp.cpp:9-45
 *
 * The reference keeps the per-scale maps private; they are read through the
 * standard explicit-instantiation access idiom below rather than by editing
 * the reference headers.
 */
#include <algorithm>
#include <cmath>
#include <complex>
#include <iostream>
#include <limits>
#include <memory>
#include <sstream>
#include <streambuf>
#include <vector>

#include "classes.hpp"
#include "gabor.hpp"
#include "mmp.hpp"

namespace {

template <typename Tag, typename Tag::type M>
struct Access {
    friend typename Tag::type member_of(Tag) { return M; }
};

struct MapsTag {
    typedef std::vector<std::shared_ptr<GaborWorkspaceMap>> GaborWorkspace::*type;
    friend type member_of(MapsTag);
};
template struct Access<MapsTag, &GaborWorkspace::maps>;

struct NfftTag {
    typedef const int GaborWorkspaceMap::*type;
    friend type member_of(NfftTag);
};
template struct Access<NfftTag, &GaborWorkspaceMap::Nfft>;

class NullBuf : public std::streambuf {
protected:
    int overflow(int c) override { return c; }
};

struct Silence {
    NullBuf null;
    std::streambuf* old;
    Silence() : old(std::cout.rdbuf(&null)) {}
    ~Silence() { std::cout.rdbuf(old); }
};

MultiSignal make_signal(double fs, int C, int N, const double* samples) {
    MultiSignal sig;
    sig.channels.resize(C);
    for (int c = 0; c < C; ++c) {
        sig.channels[c].freqSampling = fs;
        sig.channels[c].samples.assign(samples + (size_t)c * N, samples + (size_t)(c + 1) * N);
    }
    return sig;
}

std::unique_ptr<Decomposition> make_decomposition(int variant) {
    switch (variant) {
        case 0: return std::unique_ptr<Decomposition>(new SmpDecomposition);
        case 1: return std::unique_ptr<Decomposition>(new Mmp1Decomposition);
        case 2: return std::unique_ptr<Decomposition>(new Mmp2Decomposition);
        case 3: return std::unique_ptr<Decomposition>(new Mmp3Decomposition);
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

/* Dictionary geometry as the reference builds it. Returns the scale count,
 * or -1 on error; arrays are filled up to cap entries. */
int empiref_geometry(double fs, int N, double energyError, double scaleMin, double scaleMax,
                     double freqMax, int cap, double* s, int* nfft, int* fcount, int* tcount) {
    try {
        GaborWorkspaceBuilder builder(energyError, scaleMin, scaleMax, freqMax);
        std::unique_ptr<Workspace> ws(builder.prepareWorkspace(fs, 1, N, nullptr));
        GaborWorkspace* gw = static_cast<GaborWorkspace*>(ws.get());
        auto& maps = gw->*member_of(MapsTag());
        int n = (int)maps.size();
        for (int i = 0; i < n && i < cap; ++i) {
            s[i] = maps[i]->s;
            nfft[i] = (*maps[i]).*member_of(NfftTag());
            fcount[i] = maps[i]->fCount;
            tcount[i] = maps[i]->tCount;
        }
        return n;
    } catch (...) {
        return -1;
    }
}

/* Full energy map (and optionally complex values) of one scale after
 * Workspace::compute.  energy is laid out [f][t]; values [c][f][t][re,im]. */
int empiref_map(double fs, int C, int N, double energyError, double scaleMin, double scaleMax,
                double freqMax, int mmp1, const double* samples, int scale, double* energy,
                double* values) {
    try {
        GaborWorkspaceBuilder builder(energyError, scaleMin, scaleMax, freqMax);
        Mmp1Decomposition mmp1dec;
        MultichannelConstraint constraint = mmp1 ? static_cast<Decomposition&>(mmp1dec).constraint : nullptr;
        std::unique_ptr<Workspace> ws(builder.prepareWorkspace(fs, C, N, constraint));
        MultiSignal sig = make_signal(fs, C, N, samples);
        ws->compute(sig);
        GaborWorkspace* gw = static_cast<GaborWorkspace*>(ws.get());
        auto& maps = gw->*member_of(MapsTag());
        if (scale < 0 || scale >= (int)maps.size()) return -2;
        GaborWorkspaceMap* map = maps[scale].get();
        std::vector<complex> buffer(C);
        for (int f = 0; f < map->fCount; ++f) {
            GaborComputer comp(map, f);
            for (int t = 0; t < map->tCount; ++t) {
                energy[(size_t)f * map->tCount + t] = comp.compute(t, buffer);
            }
        }
        if (values) {
            for (int c = 0; c < C; ++c)
                for (int f = 0; f < map->fCount; ++f)
                    for (int t = 0; t < map->tCount; ++t) {
                        size_t o = (((size_t)c * map->fCount + f) * map->tCount + t) * 2;
                        complex v = map->value(c, f, t);
                        values[o] = v.real();
                        values[o + 1] = v.imag();
                    }
        }
        return 0;
    } catch (...) {
        return -1;
    }
}

/* Runs the reference decomposition (variant 0 SMP, 1 MMP1, 2 MMP2, 3 MMP3) on
 * one epoch held in memory.  atoms: [c][iteration][6]; natoms: per channel.
 * energies: residual energy after each iteration (first channel's residual for
 * SMP runs per channel, so it is [c][iteration]); for MMP2 the energies are
 * those of the channel-sum signal that drives the loop.  The residual path
 * replays Workspace::subtractAtomFromSignal exactly as Decomposition::compute
 * does (src/classes.cpp:57-70). Returns 0 or a negative error. */
int empiref_decompose(int variant, double fs, int C, int N, double energyError, double scaleMin,
                      double scaleMax, double freqMax, int iterationMax, double residualEnergy,
                      const double* samples, int maxAtoms, double* atoms, int* natoms,
                      double* energies, char* err, int errlen) {
    try {
        Silence quiet;
        if (C == 1) variant = 0; /* one channel always runs SMP, src/empi.cpp:118 */
        std::unique_ptr<Decomposition> dec = make_decomposition(variant);
        if (!dec) return -3;
        int builderChannels = (variant == 0 || variant == 2 || C == 1) ? 1 : C;
        GaborWorkspaceBuilder builder(energyError, scaleMin, scaleMax, freqMax);
        std::unique_ptr<Workspace> ws(builder.prepareWorkspace(fs, builderChannels, N, dec->constraint));
        MultiSignal sig = make_signal(fs, C, N, samples);
        DecompositionSettings settings{iterationMax, residualEnergy};
        MultiChannelResult res = dec->compute(settings, ws.get(), sig);
        for (int c = 0; c < C; ++c) {
            int n = (int)res[c].size();
            natoms[c] = n;
            for (int a = 0; a < n && a < maxAtoms; ++a)
                for (int p = 0; p < 6; ++p)
                    atoms[((size_t)c * maxAtoms + a) * 6 + p] = res[c][a].params[p];
        }
        if (energies) {
            /* residual-energy trajectory (replayed with the reference's own subtraction) */
            if (variant == 0 || C == 1) {
                for (int c = 0; c < C; ++c) {
                    SingleSignal r = sig.channels[c];
                    for (int a = 0; a < natoms[c] && a < maxAtoms; ++a) {
                        if (a + 1 == iterationMax) { energies[(size_t)c * maxAtoms + a] = NAN; continue; }
                        Atom atom = res[c][a];
                        Workspace::subtractAtomFromSignal(atom, r, false);
                        energies[(size_t)c * maxAtoms + a] = r.computeEnergy();
                    }
                }
            } else if (variant == 2) {
                SingleSignal sum = sig.channels[0];
                for (int c = 1; c < C; ++c)
                    for (int i = 0; i < N; ++i) sum.samples[i] += sig.channels[c].samples[i];
                /* the sum atoms: params 2..5 are shared; amplitude of the sum loop is not kept
                 * by the reference, so the trajectory is replayed by re-running the loop */
                GaborWorkspaceBuilder b2(energyError, scaleMin, scaleMax, freqMax);
                std::unique_ptr<Workspace> ws2(b2.prepareWorkspace(fs, 1, N, nullptr));
                MultiSignal s1;
                s1.channels.push_back(sum);
                SmpDecomposition smp;
                MultiChannelResult r1 = smp.compute(settings, ws2.get(), s1);
                SingleSignal r = sum;
                for (int a = 0; a < (int)r1[0].size() && a < maxAtoms; ++a) {
                    if (a + 1 == iterationMax) { energies[a] = NAN; break; }
                    Atom atom = r1[0][a];
                    Workspace::subtractAtomFromSignal(atom, r, false);
                    energies[a] = r.computeEnergy();
                }
            } else {
                MultiSignal r = sig;
                for (int a = 0; a < natoms[0] && a < maxAtoms; ++a) {
                    if (a + 1 == iterationMax) { energies[a] = NAN; break; }
                    for (int c = 0; c < C; ++c) {
                        Atom atom = res[c][a];
                        Workspace::subtractAtomFromSignal(atom, r.channels[c], false);
                    }
                    energies[a] = r.computeEnergy();
                }
            }
        }
        return 0;
    } catch (const std::exception& e) {
        if (err && errlen > 0) {
            std::string m = e.what();
            size_t n = std::min((size_t)errlen - 1, m.size());
            std::copy(m.begin(), m.begin() + n, err);
            err[n] = 0;
        }
        return -1;
    }
}

}  // extern "C"
