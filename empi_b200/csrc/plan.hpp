// Dictionary geometry and the per-scale launch plan, shared by host and device.
//
// The geometry (scales, FFT lengths, grid sizes) is computed on the host in
// FP64 with the same expressions and rounding as the reference's
// GaborWorkspaceBuilder::prepareWorkspace (src/gabor.cpp:213-252) and
// GaborWorkspaceMap's grids (src/gabor.cpp:256-268), so every (scale, t, f)
// index means what it means in the reference.
//
// On top of it each scale gets a transform plan for the device:
//   * a window of W <= Wmax real samples is packed two-per-complex (z[n] =
//     x[2n] + i x[2n+1]) into a length-Nh = Nfft/2 complex sequence whose
//     nonzero part is ceil(Wmax/2) long;
//   * that sequence is split by residue: Z[M q + r] = FFT_L(y_r)[q] with
//     y_r[n'] = sum_m z[n' + m L] W_Nh^{r (n' + m L)}, L = Nh / M, so every
//     shared-memory FFT is at most `lcap` points long whatever Nfft is
//     (fold factor F = ceil(ceil(Wmax/2) / L) input points per y value);
//   * the real spectrum needs Z[k] and Z[Nh - k]; those live in residues r and
//     M - r, so residues are processed in "groups": {0}, {M/2}, {r, M - r}.
// A (window, group) pair owns one "slot": the max energy over its bins.
#pragma once

#include <cstdint>

namespace empi {

constexpr int kChunk = 1024;          // slots per tournament-tree leaf chunk
constexpr int kTwN = 8192;            // length of the FP32 twiddle table
constexpr int kTwLog = 13;            // log2 kTwN
constexpr int kTwFineLog = 26;        // the fine table holds W_2^26^i, i < kTwN
constexpr int kUnitPoints = 8192;     // complex points per CTA work unit
constexpr int kUnitThreads = 512;     // threads per refresh CTA
constexpr int kMaxWindowsPerUnit = 1024;

struct ScalePlan {
    double s;          // scale in seconds
    double hw;         // 3 s (GAUSS_HALF_WIDTH * s)
    int nfft, fcount, tcount;
    int logL, L, M, F, G;  // sub-FFT size, residue count, fold factor, groups
    int B1, B2;        // windows per unit for single-residue groups / pairs
    int klo, khi;      // bins k < klo or k > khi carry the phase-dependent norm term
    int khf;           // first bin with f > fs/4 (isHighFreq)
    int wmax;          // longest window (samples)
    long long slot_base;  // first slot of this scale within an instance
    long long win_base;   // first entry of this scale in the window tables
    float aG;          // sqrt(pi) / (s fs): Gaussian exponent per sample
    float Kc;          // 2 sqrt(2) / (s fs): single-channel energy factor
    float K1;          // sqrt(2) / (s fs): MMP1 energy factor
    float aG2;         // aG sqrt(log2 e): Gaussian as exp2(-(d aG2)^2)
    int eoff;          // offset of this scale's expFactor table (bins k < klo, then k > khi)
    // Certified FP32 error bound of the refresh (see refresh.cuh, "error
    // bound"): |X32_k - X_k| <= bnd_d * B for every bin of a window, B the
    // instance's channel norm of max |residual|; phase-dependent bins scale
    // it by sqrt(bnd_rho) and carry the relative formula error bnd_tph.
    float bnd_d;       // eta (s fs + 1 + wmax 2^-20): FFT error per unit of max |x|
    float bnd_rho;     // 1 / (1 - expFactor) of the worst phase-dependent bin (1 if none)
    float bnd_srho;    // sqrt(bnd_rho)
    float bnd_tph;     // relative error of a phase-dependent bin's energy formula
    float sKc;         // sqrt(Kc)
    int pad_;
};

// Window geometry of one (scale, t): first sample, length, and the window
// centre c = t0fixed * fs split into integer and fraction (src/gabor.cpp:279-286).
struct WinGeom {
    int iL, W, ci;
    float cf;
};

struct DictPlan {
    double fs, tMax;
    int N, scale0, nscales, chunks;
    long long slots;
    unsigned long long values;  // sum fCount * tCount (getAtomCount)
};

}  // namespace empi
