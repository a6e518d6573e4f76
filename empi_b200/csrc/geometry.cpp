// Host-side dictionary geometry and per-scale transform plans.
#include "geometry.hpp"

#include <algorithm>
#include <cmath>
#include <limits>

namespace empi {

namespace {

const double kGaussHalfWidth = 3.0;     // src/gabor.cpp:14
const double kMinScaleInSamples = 2.0;  // src/gabor.cpp:19

long pow2_round(long x) {  // inc/fftw.hpp:161-168
    long y = 2;
    while (y < x) y *= 2;
    return y;
}

int ilog2(long x) {
    int l = 0;
    while ((1L << l) < x) ++l;
    return l;
}

// Worst-case FP32 error of the refresh's window values, as constants per
// scale (unit roundoff u = 2^-24; every count below rounds up).
//
// Each computed value X32_k is a linear function of the window's packed
// samples z_n = x_{2n} g_{2n} + i x_{2n+1} g_{2n+1}.  Along the computation
// (fold, twist, Stockham passes, unpacking) every intermediate value is a
// unit-modulus-weighted sum of a subset of the z_n, so its modulus is at most
// A = sum_n |x_n| g_n, and a rounding error made at one stage reaches X_k
// through unit-modulus factors.  Summing the worst relative error of each
// stage therefore gives |X32_k - X_k| <= eta A with, in units of u:
//   residual rounded to FP32                          1
//   Gaussian exp2f (approximate) and its argument     6
//   sample product                                    2
//   twist W_Nh^{rn}: table product plus up to 8
//     rotations, and its complex product              40
//   each fold: sum plus fold rotation                 4 per fold (F)
//   each Stockham pass: W^k rotated up to 15 times
//     and the in-register radix-16 DFT                64 per pass (P)
// counted twice (X_k = E + W D combines Z[k] and Z[Nh - k]), plus the
// unpacking and the W_2L rotation of up to 8 bins   40.
// A <= max|x| (sum_n g_n + W 2^-20), and sum_n g_n <= s fs + 1 for a
// Gaussian of width s fs >= 2 samples (Poisson summation); the 2^-20 per
// sample covers the exp2f absolute error where g is tiny.
//
// The energy is a norm of X: for a single channel fs |v|^2 normReal^2 =
// Kc |X|^2 / (1 + e cos 2phi'), the maximum over phases of a quadratic form
// whose eigenvalues lie in [Kc / (1 + e), Kc / (1 - e)] (e = expFactor), so
// sqrt(E) moves by at most sqrt(Kc / (1 - e)) |X32 - X| (summed over channels
// by Minkowski's inequality for MMP3, and for MMP1's constrained sums).
// Phase-dependent bins (k != 0, Nh; bins 0 and Nh are real) have
// e <= e1 = exp(-2 pi (s fs / Nfft)^2), bnd_rho = 1 / (1 - e1).  Their
// closed-form energy Kc p^2 / (p + e Re(X^2 e^{i psi})) divides by
// D >= p (1 - e): rounding in D (8 u) and the magnitude error of the
// rotated e^{i psi} (60 u) are amplified by bnd_rho, its angle error (180 u)
// by at most e / sqrt(1 - e^2) <= sqrt(bnd_rho); the rest adds 7 u.
void set_error_bound(ScalePlan& p, double fs) {
    const double u = std::ldexp(1.0, -24);
    const int first = p.logL & 3;
    const int passes = (first ? 1 : 0) + (p.logL - first) / 4;
    const double eta = u * (2.0 * (1 + 6 + 2 + 40 + 4.0 * p.F + 64.0 * passes) + 40);
    const double width = p.s * fs + 1.0 + p.wmax * std::ldexp(1.0, -20);
    p.bnd_d = (float)(eta * width * (1.0 + 1e-6));
    const long Nh = p.nfft / 2;
    // any phase-dependent bin other than k = 0 and k = Nh
    const bool low = p.klo > 1, high = p.khi < p.fcount - 1 && std::min<long>(p.fcount - 1, Nh - 1) > p.khi;
    double rho = 1.0;
    if (low || high) {
        const double x = p.s * fs / p.nfft;
        const double e1 = std::exp(-2.0 * M_PI * x * x);
        rho = 1.0 / (1.0 - e1);
    }
    p.bnd_rho = (float)(rho * (1.0 + 1e-6));
    p.bnd_srho = (float)(std::sqrt(rho) * (1.0 + 1e-6));
    p.bnd_tph = (float)(u * (7.0 + rho * (8.0 + 60.0) + 2.0 * std::sqrt(rho) * 180.0));
    p.sKc = (float)(std::sqrt(2.0 * M_SQRT2 / (p.s * fs)) * (1.0 + 1e-6));
}

}  // namespace

bool build_dictionary(double fs, int N, double energyError, double scaleMin, double scaleMax,
                      double freqMax, int lcap, DictPlan& dict, std::vector<ScalePlan>& scales,
                      std::vector<float>& etab, std::vector<WinGeom>* wgeom, std::vector<float>* whf,
                      std::string& err) {
    if (!(fs > 0.0) || !std::isfinite(fs)) {
        err = "invalidSamplingFrequency";
        return false;
    }
    if (!(energyError > 0.0 && energyError < 1.0)) {
        err = "invalidEnergyErrorValue";
        return false;
    }
    if (N < 4) {
        err = "signalIsTooShortForThisDecomposition";
        return false;
    }
    if (lcap < 16 || lcap > kUnitPoints / 2 || (lcap & (lcap - 1))) {
        err = "invalidTransformCap";
        return false;
    }
    // GaborWorkspaceBuilder::prepareWorkspace, src/gabor.cpp:213-252
    const double smin = std::max(scaleMin, kMinScaleInSamples / fs);
    const double smax = std::min(scaleMax, N / fs);
    const double root = std::sqrt(-2.0 / M_PI * std::log(1.0 - energyError));
    const double aDenomSqrt = 1.0 - energyError;
    const double aNominPart =
        energyError * (2.0 - energyError) * (energyError * energyError - 2 * energyError + 2);
    const double a = (1.0 + std::sqrt(aNominPart)) / (aDenomSqrt * aDenomSqrt);
    const double dl = std::log(a);
    const double tMax = (N - 1) / fs;
    const double lMin = std::log(smin);
    const double lMax = std::log(smax);
    const long lCount = std::lrint((lMax - lMin) / dl + 0.5) + 1;
    if (lCount < 2 || !(smax >= smin)) {
        err = "invalidDictionary";
        return false;
    }
    dict = DictPlan{};
    dict.fs = fs;
    dict.tMax = tMax;
    dict.N = N;
    dict.scale0 = (int)scales.size();
    dict.nscales = (int)lCount;
    long long slots = 0;
    unsigned long long values = 0;
    for (long i = 0; i < lCount; ++i) {
        ScalePlan p{};
        const double s = std::exp(lMin + i * (lMax - lMin) / (lCount - 1));
        const double dt = root * s;
        const double df = root / s;
        const double hw = kGaussHalfWidth * s;
        const long Ngauss = 2 * std::lrint(hw * fs - 0.5) + 1;
        const long Nfft = pow2_round(std::max(Ngauss, std::lrint(fs / df + 0.5)));
        const long tCount = std::lrint(tMax / dt + 0.5) + 1;
        if (std::max(Nfft, tCount) > static_cast<long>(std::numeric_limits<int>::max())) {
            err = "signalFileIsTooLongForThisDecomposition";
            return false;
        }
        long fCount = Nfft / 2 + 1;
        if (std::isfinite(freqMax) && freqMax > 0) {
            fCount = std::min(fCount, std::lrint(freqMax / fs * Nfft + 0.5) + 1);
        }
        if (!std::isfinite(s) || tCount < 2 || fCount < 1) {
            err = "invalidDictionary";
            return false;
        }
        p.s = s;
        p.hw = hw;
        p.nfft = (int)Nfft;
        p.fcount = (int)fCount;
        p.tcount = (int)tCount;

        // window of every t (src/gabor.cpp:279-292) and the longest one
        int wmax = 1;
        p.win_base = wgeom ? (long long)wgeom->size() : 0;
        for (long ti = 0; ti < tCount; ++ti) {
            const double t0 = ti * tMax / (tCount - 1);
            long l = std::lrint((t0 - hw) * fs), r = std::lrint((t0 + hw) * fs);
            long iL = std::max(0L, l), iR = std::min((long)N - 1, r);
            wmax = std::max(wmax, (int)(iR - iL + 1));
            if (wgeom) {
                const double t0fixed = t0 - iL / fs;
                const double c = t0fixed * fs;
                const double cfl = std::floor(c);
                wgeom->push_back(WinGeom{(int)iL, (int)(iR - iL + 1), (int)cfl, (float)(c - cfl)});
                const double ft = fs * t0;
                whf->push_back((float)(ft - std::rint(ft)));
            }
        }
        if (wmax > Nfft) {
            // the reference would write past its FFT buffer here
            err = "windowLongerThanTransform";
            return false;
        }
        p.wmax = wmax;

        const long Nh = Nfft / 2;
        const long zlen = (wmax + 1) / 2;
        long L = std::min(Nh, pow2_round(std::max(zlen, 1L)));
        if (Nh == 1) L = 1;
        L = std::min(L, (long)lcap);
        p.L = (int)L;
        p.logL = ilog2(L);
        p.M = (int)(Nh / L);
        p.F = (int)((zlen + L - 1) / L);
        if (p.F < 1) p.F = 1;
        p.G = p.M == 1 ? 1 : (p.M == 2 ? 2 : p.M / 2 + 1);
        p.B1 = std::min(kMaxWindowsPerUnit, (int)(kUnitPoints / L));
        p.B2 = std::max(1, std::min(kMaxWindowsPerUnit, (int)(kUnitPoints / (2 * L))));

        // bins whose normalisation depends on the phase (expFactor >= 2^-30),
        // and the first "high frequency" bin (src/gabor.cpp:44-52)
        const double thr = std::ldexp(1.0, -30);
        const double nyq = 0.5 * fs;
        int khf = (int)fCount;
        for (long k = 0; k < fCount; ++k) {
            double f = k * fs / Nfft;
            if (f > 0.5 * nyq) {
                khf = (int)k;
                break;
            }
        }
        auto need = [&](long k) {
            double f = k * fs / Nfft;
            bool high = f > 0.5 * nyq;
            double f4 = high ? (nyq - f) : f;
            double e = std::exp(-2 * M_PI * s * s * f4 * f4);
            return e >= thr;
        };
        int klo = 0;
        while (klo < khf && need(klo)) ++klo;
        int khi = (int)fCount - 1;
        while (khi >= khf && need(khi)) --khi;
        p.klo = klo;
        p.khi = khi;
        p.khf = khf;
        // expFactor (src/gabor.cpp:51) of the phase-dependent bins, FP64 -> FP32
        p.eoff = (int)etab.size();
        auto efac = [&](long k) {
            double f = k * fs / Nfft;
            bool high = f > 0.5 * nyq;
            double f4 = high ? (nyq - f) : f;
            return (float)std::exp(-2 * M_PI * s * s * f4 * f4);
        };
        for (long k = 0; k < klo; ++k) etab.push_back(efac(k));
        for (long k = khi + 1; k < fCount; ++k) etab.push_back(efac(k));
        p.slot_base = slots;
        p.aG = (float)(std::sqrt(M_PI) / (s * fs));
        p.Kc = (float)(2.0 * M_SQRT2 / (s * fs));
        p.K1 = (float)(M_SQRT2 / (s * fs));
        p.aG2 = (float)(std::sqrt(M_PI) / (s * fs) * std::sqrt(1.0 / std::log(2.0)));
        set_error_bound(p, fs);
        slots += (long long)tCount * p.G;
        values += (unsigned long long)fCount * (unsigned long long)tCount;
        scales.push_back(p);
    }
    dict.slots = slots;
    dict.chunks = (int)((slots + kChunk - 1) / kChunk);
    dict.values = values;
    return true;
}

}  // namespace empi
